/*
 * cueva_oracle.h -- CPU restatement of the CUEVA (ByMar09/MHD-KH-instability)
 * per-step hot path, used ONLY as test infrastructure: the checker that the
 * B200 kernels are compared against in tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py.  Nothing in the product links this library.
 *
 * Parity status: UNPINNED against the reference itself.  The reference is
 * Fortran 95 and no Fortran compiler exists on either machine, and the
 * reference ships no golden vectors or known-answer tests.  The restatement
 * follows the Fortran line by line (each routine cites the file:line it
 * mirrors) and is pinned by analytic/structural tests (polynomial exactness
 * of MP5/7/9, odd symmetry, HLL consistency, con2prim round trips, uniform
 * state preservation, periodic conservation, tableau sums, 1-thread vs
 * N-thread bit identity) plus regression fixtures under tests/golden/.
 *
 * Arithmetic follows the Fortran evaluation order (left to right, integer
 * powers expanded as gfortran's powi does: x**2 = x*x, x**3 = (x*x)*x,
 * x**4 = (x*x)*(x*x)) and must be compiled with -ffp-contract=off.
 */
#ifndef CUEVA_ORACLE_H
#define CUEVA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_params {
  int32_t imax, jmax;      /* grid points 0..imax x 0..jmax (parameters.f95:110-111) */
  int32_t order;           /* IMEX tableau: 1,2,3,4,5,6,8 (imex_scheme.f95) */
  int32_t flux_solver;     /* 1 Lax-Friedrichs+MC (15_lax_flow.f95), 2 HLL+MC (16_hll_flow_mcl.f95),
                              3 HLLE+MC (16_hlle_flow_mcl.f95), 4 HLLC+MC (16_hllc_flow_mcl.f95),
                              5 HLL+MPX, 6 HLLE+MPX, 7 HLLC+MPX (main_cueva_code.f95:247-273) */
  int32_t rec_mp;          /* 0 MP5, 1 MP7, 2 MP9 (parameters.f95:33) */
  int32_t c2p;             /* 1 Cardano, 0 Newton-Raphson (parameters.f95:37) */
  int32_t bc_x, bc_y;      /* 0 copy, 1 periodic (04_boundary.f95 BOUND 1/2/6) */
  int32_t intsum_reset;    /* 0: intsum zeroed once per step (07_clean_var.f95, main_cueva_code.f95:184),
                              as the reference; 1: zeroed before every stage (textbook IMEX-RK) */
  int32_t primitive_rec;   /* 1: reconstruct the primitives at the start of every step
                              (05_reconstruct.f95, main_cueva_code.f95:170-175) */
  double lx, ly, lz;       /* Longx, Longy, Longz */
  double cfl, sigma, gamma;
  double dt;               /* <= 0: CFL*min(Delx,Dely,Delz) (parameters.f95:312) */
} oracle_params;

/* carried primitive fields, interior (imax+1)*(jmax+1), i fastest */
enum {
  OR_RHO = 0, OR_P, OR_VX, OR_VY, OR_VZ, OR_PSI, OR_PHI,
  OR_EX, OR_EY, OR_EZ, OR_BX, OR_BY, OR_BZ, OR_Q, OR_NPRIM
};

void*   oracle_create(const oracle_params* p);
void    oracle_destroy(void* h);
void    oracle_set_threads(int32_t n);
/* 0 (default): deterministic Cardano seed shared with the kernels; 1: C-library acos/cos/pow */
void    oracle_set_libm_seed(int32_t on);
void    oracle_chebyshev_roots(double y, double* out3);
double  oracle_cbrt(double x);
double  oracle_dt(void* h);
void    oracle_set_prims(void* h, const double* const* prims14);
void    oracle_get_prims(void* h, double* const* prims14);
/* one full time step h of main_cueva_code.f95:47-356; returns status (0 ok) */
int32_t oracle_step(void* h, int32_t nsteps);
/* runs boundary+startconvar+cleanvarint and RK stages 1..upto only */
int32_t oracle_run_stages(void* h, int32_t upto);
/* interior copy of a named internal array ("psiflux", "Exastsour", "Exlaxpsi",
 * "Exint", "Jxint", "D", "tau", ...); l selects the stage for per-stage arrays */
int32_t oracle_get_named(void* h, const char* name, int32_t l, double* out);
/* the whole ghosted array, (jmax+13) x (imax+13), element (i, j) at (i+6) + (j+6)*(imax+13) */
int32_t oracle_get_named_full(void* h, const char* name, int32_t l, double* out);
void    oracle_counters(void* h, int64_t* out3);

/* KH initial data in the reference orientation (x_ref = problem y, copy;
 * y_ref = problem x, periodic), conventions of 03_init_var_primitive.f95:2297-2336 */
void    oracle_kh_init(int32_t imax, int32_t jmax, double lx, double ly,
                       double v0, double a, double amp, double width,
                       double kpert, double phase, double bshear,
                       double rho0, double p0, double* const* prims14);

/* unit entry points for the pins */
void    oracle_mp_line(int32_t rec_mp, int32_t n, const double* u /* n+13, starts at -6 */,
                       int32_t posfix, double* up, double* um /* n+13 */);
double  oracle_hllc_vel(double a, double b, double c, double rt);
/* Cardano con2prim of one point (12_varprimitive.f95:48-813, l_swap=1);
 * in: D tau Sx Sy Sz Ex Ey Ez Bx By Bz vx0 vy0 vz0 rho0 p0 ; out: vx vy vz rho p W */
int32_t oracle_c2p_cardano(const double* in16, double gamma, double eps1, double* out6);
int32_t oracle_c2p_nr(const double* in16, double gamma, double* out6);
int32_t oracle_tableau(int32_t order, double* wb8, double* wbt8, double* ab64, double* abt64);
/* run diagnostics of the writer, 22_writer.f95:821-1019 (lector, DIM == 2),
 * on the current state in its loop order; 45 slots in the order of cueva.h's
 * cueva_diag_slot.  d_from_startconvar != 0 first recomputes D and tau from
 * the primitives (a step-boundary state); otherwise D and tau are varfin's
 * values left by oracle_step, as at the writer's call.  abs45 (nullable)
 * receives sum |term| of each of the 35 sums. */
void    oracle_lector(void* h, double b0, double lr, double ly, double delta_rec, int32_t d_from_startconvar,
                      double* out45, double* abs45);

#ifdef __cplusplus
}
#endif
#endif
