/*
 * cueva.h -- C-ABI of the B200 (sm_100a) implementation of the CUEVA per-step
 * hot path (ByMar09/MHD-KH-instability, directory cueva_2D_base/).
 *
 * The reference is Fortran 95 whose hot routines take no arguments and read
 * and write module arrays dimensioned (-6:imax+6, -6:jmax+6[, 1:kmax, 1:lmax])
 * (threevectors.f95:12-81, fourvectors.f95:12-170).  A Fortran caller keeps
 * those arrays and binds them here once with c_loc(array(-6,-6,1[,1]))
 * (see fortran/cueva_gpu.f90); this library mirrors them on
 * the GPU and replaces the routines listed next to each entry point.
 *
 * Conventions: every entry point returns 0 (CUEVA_OK) or a positive error
 * class; the message of the last failure on the calling thread is in
 * cueva_last_error().  A context is bound to one CUDA device and one stream,
 * is not re-entrant, and must be driven from one host thread (the reference
 * calls its routines from the serial driver, main_cueva_code.f95:202-328).
 * Where the reference prints and STOPs (non-physical states), the kernels set
 * bits of a device status word instead; cueva_step() and the routine mirrors
 * report them as CUEVA_ERR_PHYSICS at the next synchronisation.
 */
#ifndef CUEVA_H
#define CUEVA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUEVA_OK 0
#define CUEVA_ERR_ARG 1       /* invalid argument or unsupported configuration */
#define CUEVA_ERR_CUDA 2      /* CUDA runtime failure (no device, out of memory, ...) */
#define CUEVA_ERR_UNBOUND 3   /* a field the call needs was never bound */
#define CUEVA_ERR_PHYSICS 4   /* a kernel hit a reference STOP condition, see cueva_status */

/* status bits reported by cueva_status (reference STOP sites) */
#define CUEVA_ST_C2P_FAIL 1u        /* 12_varprimitive.f95:382-428,485 */
#define CUEVA_ST_SUPERLUMINAL 2u    /* 12_varprimitive.f95:678,691; 12_varprimitive_nr.f95:217 */
#define CUEVA_ST_HLLC_NOCONV 4u     /* funciones.f95:240-245 */
#define CUEVA_ST_HLLC_VSTAR 8u      /* 16_hllc_flow_mpx.f95:4294,4605 */
#define CUEVA_ST_NONFINITE 16u      /* con2prim returned NaN/Inf (the reference continues silently) */
#define CUEVA_ST_HLLE_SPEED 32u     /* 16_hlle_flow_mpx.f95:2796-2803, 2974-2981 (NaN wave bounds) */
#define CUEVA_ST_TC_TIMEOUT 64u     /* a bounded tensor-core (tcgen05) wait ran out; no reference counterpart */
#define CUEVA_ST_TC_TEARDOWN 128u   /* after such a time-out the teardown's bounded wait ran out too: TMEM was
                                       released while an MMA may still write it; destroy the context */
#define CUEVA_ST_COPY_TIMEOUT 256u  /* a bounded wait for the stage kernel's bulk copies of stencil rows ran
                                       out; the state of that step is incomplete; no reference counterpart */

typedef struct cueva_ctx cueva_ctx;

/* Run configuration: the compile-time constants of parameters.f95 that the
 * hot path reads, as runtime values. */
typedef struct cueva_params {
  int32_t imax, jmax;   /* grid points 0..imax x 0..jmax (parameters.f95:110-111), both >= 6 */
  int32_t order;        /* IMEX tableau (parameters.f95:10): 1, 2 SSP2(2,2,2), 3 SSP2(3,3,2), 4 SSP3(4,3,3), 5, 6, 8 */
  int32_t flux_solver;  /* 1 Lax-Friedrichs with MC slopes (15_lax_flow.f95); 2 HLL, 3 HLLE, 4 HLLC with
                           the second-order MC reconstruction (16_hll/hlle/hllc_flow_mcl.f95) -- rec_mp
                           does not apply to 1-4 --; 5 HLL+MPX, 6 HLLE+MPX, 7 HLLC+MPX
                           (main_cueva_code.f95:247-273) */
  int32_t rec_mp;       /* 0 MP5, 1 MP7, 2 MP9 (parameters.f95:33) */
  int32_t c2p;          /* 1 Cardano, 0 Newton-Raphson (parameters.f95:37), 2 learned seed + Newton */
  int32_t bc_x, bc_y;   /* per-axis ghost rule: 0 copy, 1 periodic (BOUND 1 / 2 / 6 of 04_boundary.f95) */
  int32_t precision;    /* 0 FP64 throughout; 1 FP32 reconstruction + Riemann, FP64 elsewhere
                           (flux_solver 1, 2, 4..7: psi, phi, E, B reconstructed as differences
                           from a cell value and their fluxes kept in FP64) */
  int32_t device;       /* CUDA device ordinal */
  int32_t intsum_reset; /* 0: the stage sums are zeroed once per step and accumulate over the stages
                           (07_clean_var.f95 via main_cueva_code.f95:184, the reference); 1: zeroed
                           before every stage (textbook IMEX-RK; the reference's SSP3(4,3,3) marked
                           "NO" in imex_scheme.f95:278 is only stable this way) */
  int32_t primitive_rec;/* 1: reconstruct the primitives at the start of every step
                           (primitive_rec of parameters.f95:26, 05_reconstruct.f95:525-746,
                           main_cueva_code.f95:170-175); 0 (default): no reconstruction */
  double lx, ly, lz;    /* Longx, Longy, Longz (Delx = lx/imax, Dely = ly/jmax, Delz = lz) */
  double cfl, sigma, gamma;
  double dt;            /* <= 0 selects CFL*min(Delx,Dely,Delz) (parameters.f95:312) */
} cueva_params;

/* Field ids for cueva_bind_field.  Base = address of element (-6,-6) of the
 * Fortran array (and stage 1 for the stage arrays); layout column-major with
 * leading dimension imax+13, second dimension jmax+13, stage stride
 * (imax+13)*(jmax+13). */
enum cueva_field {
  /* carried primitives (threevectors.f95:32-64) */
  CUEVA_RHO = 0, CUEVA_P, CUEVA_VX, CUEVA_VY, CUEVA_VZ, CUEVA_PSI, CUEVA_PHI,
  CUEVA_EX, CUEVA_EY, CUEVA_EZ, CUEVA_BX, CUEVA_BY, CUEVA_BZ, CUEVA_Q,
  /* startconvar outputs at time n (threevectors.f95:38,64) */
  CUEVA_D, CUEVA_TAU, CUEVA_SX, CUEVA_SY, CUEVA_SZ, CUEVA_W,
  /* stage state, (.., 1:lmax) arrays of fourvectors.f95:18-50 */
  CUEVA_PSIINT, CUEVA_PHIINT, CUEVA_EXINT, CUEVA_EYINT, CUEVA_EZINT,
  CUEVA_BXINT, CUEVA_BYINT, CUEVA_BZINT, CUEVA_QINT, CUEVA_DDINT, CUEVA_TAUINT,
  CUEVA_SXINT, CUEVA_SYINT, CUEVA_SZINT, CUEVA_JXINT, CUEVA_JYINT, CUEVA_JZINT,
  CUEVA_EXAST, CUEVA_EYAST, CUEVA_EZAST,
  /* stage right-hand sides, fourvectors.f95:140-145 */
  CUEVA_PSIFLUX, CUEVA_PHIFLUX, CUEVA_EXASTFLUX, CUEVA_EYASTFLUX, CUEVA_EZASTFLUX,
  CUEVA_BXFLUX, CUEVA_BYFLUX, CUEVA_BZFLUX, CUEVA_QFLUX, CUEVA_DFLUX, CUEVA_TAUFLUX,
  CUEVA_SXFLUX, CUEVA_SYFLUX, CUEVA_SZFLUX, CUEVA_EXASTSOUR, CUEVA_EYASTSOUR, CUEVA_EZASTSOUR,
  /* stage interface fluxes, (.., 1:lmax) arrays of fourvectors.f95: the outputs of the
   * flux routines (15_lax_flow.f95, 16_*_flow_mcl.f95, 16_*_flow_mpx.f95) that
   * 17_fluxandsource.f95 reads.  X(i,j) of an x array is the flux through i+1/2, of a y
   * array the flux through j+1/2 */
  CUEVA_EXLAXPSI, CUEVA_EYLAXPSI, CUEVA_BXLAXPHI, CUEVA_BYLAXPHI, CUEVA_PHILAXBX, CUEVA_EZLAXBX,
  CUEVA_EZLAXBY, CUEVA_PHILAXBY, CUEVA_EYLAXBZ, CUEVA_EXLAXBZ, CUEVA_PSILAXEX, CUEVA_BZLAXEX,
  CUEVA_BZLAXEY, CUEVA_PSILAXEY, CUEVA_BYLAXEZ, CUEVA_BXLAXEZ, CUEVA_JXLAX, CUEVA_JYLAX,
  CUEVA_FDXLAX, CUEVA_FDYLAX, CUEVA_FTAUXLAX, CUEVA_FTAUYLAX, CUEVA_FSXXLAX, CUEVA_FSXYLAX,
  CUEVA_FSXZLAX, CUEVA_FSYXLAX, CUEVA_FSYYLAX, CUEVA_FSYZLAX,
  /* final stage sums (threevectors.f95), the increments of varfin / electricfield */
  CUEVA_PSIFINSUM, CUEVA_PHIFINSUM, CUEVA_BXFINSUM, CUEVA_BYFINSUM, CUEVA_BZFINSUM, CUEVA_EXFINSUM,
  CUEVA_EYFINSUM, CUEVA_EZFINSUM, CUEVA_QFINSUM, CUEVA_DFINSUM, CUEVA_TAUFINSUM, CUEVA_SXFINSUM,
  CUEVA_SYFINSUM, CUEVA_SZFINSUM,
  CUEVA_NFIELDS
};

/* transfer groups for cueva_upload / cueva_download */
#define CUEVA_G_PRIMS 1u   /* the 14 carried primitives */
#define CUEVA_G_CONS 2u    /* D, tau, Sx, Sy, Sz, W */

/* ---- lifecycle ------------------------------------------------------- */
int32_t cueva_ctx_create(const cueva_params* p, cueva_ctx** out);
int32_t cueva_ctx_destroy(cueva_ctx* ctx);
const char* cueva_last_error(void);
int32_t cueva_set_stream(cueva_ctx* ctx, void* cuda_stream); /* NULL: the context's own stream */
double cueva_dt(const cueva_ctx* ctx);
int32_t cueva_tableau_stages(const cueva_ctx* ctx);

/* ---- fields and transfers -------------------------------------------- */
int32_t cueva_bind_field(cueva_ctx* ctx, int32_t field, double* base);
/* page-lock a host range (e.g. a bound Fortran array) so transfers run at full PCIe rate */
int32_t cueva_pin_host(void* ptr, uint64_t bytes);
int32_t cueva_unpin_host(void* ptr);
/* host -> device of the bound interior points; uploading CUEVA_G_PRIMS also
 * runs startconvar and prepares stage 1, so cueva_step can follow directly */
int32_t cueva_upload(cueva_ctx* ctx, uint32_t groups);
/* device -> host of the bound interior points (ghost cells are left to the
 * caller's boundary routine, as main_cueva_code.f95:328 does); synchronises
 * and reports kernel status */
int32_t cueva_download(cueva_ctx* ctx, uint32_t groups);
/* cueva_download without the wait: the copies run on a second stream, after
 * the work already queued on the context stream, one field after another.
 * The bound host arrays are being written until a call that waits for the
 * host returns: cueva_sync, cueva_download or cueva_status.  Until then the
 * caller must not read, modify, rebind or free them (later calls such as
 * cueva_step only order their device work after the copies; they do not
 * wait).  A following cueva_upload of the same arrays waits per field on the
 * device, so field f goes back up while field f+1 still comes down.  Kernel
 * status is reported by the next call that synchronises. */
int32_t cueva_download_async(cueva_ctx* ctx, uint32_t groups);

/* ---- the hot path ----------------------------------------------------- */
/* nsteps executions of the body of the time loop, main_cueva_code.f95:53-328
 * (boundary, recons_var_primitive when params.primitive_rec, startconvar,
 * cleanvarint, RK stages with sumint / varint /
 * electricvarint / flowinit / {hll,hllc}_flow_mpx / fluxandsource / sumfin,
 * varfin, electricfield, varprimitivecardano or varprimitive_nr), on the
 * device-resident state.  Asynchronous on the context stream. */
int32_t cueva_step(cueva_ctx* ctx, int32_t nsteps);
/* No counterpart in the reference (an implementation choice of the step).
 * fused = 1 runs each RK stage as one kernel (y faces, x faces and the point
 * update of a strip of the grid in one CTA, the y fluxes kept in shared
 * memory); fused = 0 as a y-face kernel and an x-face + update kernel that
 * pass the y fluxes through device memory.  Both give bit-identical results.
 * The default is 1 where the fused kernel exists (MP5 and the MC slopes of
 * flux routines 1-4); elsewhere 1 is refused with CUEVA_ERR_ARG. */
int32_t cueva_set_stage_kernel(cueva_ctx* ctx, int32_t fused);
/* bytes of the context's device field slab (state, stage sums, stored stage
 * right-hand sides, flux scratch); no counterpart in the reference */
int32_t cueva_device_bytes(const cueva_ctx* ctx, uint64_t* bytes);
int32_t cueva_get_stage_kernel(const cueva_ctx* ctx, int32_t* fused);
int32_t cueva_sync(cueva_ctx* ctx);
int32_t cueva_status(cueva_ctx* ctx, uint32_t* status_bits);
int32_t cueva_counters(cueva_ctx* ctx, int64_t out3[3]);   /* contador_r, contador_p, contador_v */
/* Status bits stay set (the reference stops at these sites) until cleared:
 * after restoring a good state (cueva_upload or cueva_checkpoint_load) a
 * caller that handles the error clears them and continues. */
int32_t cueva_clear_status(cueva_ctx* ctx);
/* nsteps steps launched one kernel at a time (no CUDA graph) with events
 * between the launches on the context stream; ms_out[k] receives the summed
 * device time of the y-face (k = 0) and the x-face + update (k = 1) kernels
 * (k = 2 is reserved, 0) and launches_out[k] their launch counts.
 * Synchronises.  No counterpart in the reference (it is instrumentation for
 * the per-kernel roofline). */
int32_t cueva_profile_steps(cueva_ctx* ctx, int32_t nsteps, double ms_out[3], int32_t launches_out[3]);

/* ---- routine mirrors (synchronous; bound host arrays in and out) ------- */
/* startconvar, 06_conserved_var.f95:79-140: prims -> D, tau, S, W */
int32_t cueva_startconvar(cueva_ctx* ctx);
/* electricvarint (IMEX), 11_elecvarint.f95:279-328, plus the current J of
 * flowinit, 14_flowinit.f95:280-302: Exast(l), Bxint(l).., qint(l), W, V ->
 * Exint(l).., Jxint(l).. */
int32_t cueva_electricvarint(cueva_ctx* ctx, int32_t l);
/* the flux routine selected by flux_solver (main_cueva_code.f95:247-279) +
 * fluxandsource for stage l:
 * psiint(l)..Szint(l), Exint(l).., Jxint(l).., V, p, rho, W ->
 * psiflux(l)..Szflux(l), Exastsour(l).. */
int32_t cueva_flux_rhs(cueva_ctx* ctx, int32_t l);
/* The same split at the reference's routine boundary.  cueva_flux_flow is the
 * flux routine alone (lax_flow, hll_flow, hlle_flow, hllc_flow, hll_flow_mpx,
 * hlle_flow_mpx or hllc_flow_mpx by flux_solver): same inputs as
 * cueva_flux_rhs -> the 28 interface flux arrays of stage l (Exlaxpsi(l) ..
 * FSyzlax(l)), each on the faces 17_fluxandsource.f95 reads: x arrays at
 * i = -1..imax, j = 0..jmax, y arrays at i = 0..imax, j = -1..jmax (the rest
 * of the arrays is left as it was).  cueva_fluxandsource is
 * 17_fluxandsource.f95:433-699: those fluxes, psiint(l)..Szint(l), Exint(l)..,
 * V, W -> psiflux(l)..Szflux(l), Exastsour(l)..  The two calls in a row give
 * the result of cueva_flux_rhs bit for bit. */
int32_t cueva_flux_flow(cueva_ctx* ctx, int32_t l);
int32_t cueva_fluxandsource(cueva_ctx* ctx, int32_t l);
/* varfin (19_varfin.f95:16-54): psi, phi, B, q, D, tau, S += Delt * their
 * final sums; electricfield (20_electricfield.f95:153-167, IMEX):
 * E += Delt * Exfinsum.. (the same update the fused step applies after its
 * last stage) */
int32_t cueva_varfin(cueva_ctx* ctx);
int32_t cueva_electricfield(cueva_ctx* ctx);
/* varprimitivecardano / varprimitive_nr with l_swap = 1: D, tau, S, E, B and
 * the seeds V, rho, p -> V, rho, p */
int32_t cueva_con2prim(cueva_ctx* ctx);

/* ---- learned con2prim seed (c2p = 2) ---------------------------------- */
/* No counterpart in the reference.  A 6 -> 64 -> 64 -> 64 -> 1 SiLU network
 * (bf16 weights, FP32 accumulation) predicts log p from the conserved state;
 * a Newton-Raphson solve of the ideal-gas pressure equation refines it to a
 * relative step of 1e-12, and the Cardano recovery (12_varprimitive.f95) is
 * the fall-back whenever the refinement fails.  Training runs on the GPU with
 * the library's own forward/backward kernels (minibatch Adam).
 * Conserved arrays (d_cons) are device SoA blocks of 11 x n doubles:
 * D, tau, Sx, Sy, Sz, Ex, Ey, Ez, Bx, By, Bz; primitive arrays 5 x n:
 * rho, p, vx, vy, vz. */
typedef struct cueva_mlp cueva_mlp;
#define CUEVA_MLP_NPARAM 8833   /* W1[64][6] b1 W2[64][64] b2 W3[64][64] b3 W4[64] b4 */
#define CUEVA_MLP_NNORM 14      /* feature mean[6], sd[6], target mean, sd */
int32_t cueva_mlp_create(int32_t device, uint64_t seed, cueva_mlp** out);
int32_t cueva_mlp_destroy(cueva_mlp* mlp);
/* n = CUEVA_MLP_NPARAM + CUEVA_MLP_NNORM floats: parameters then normalisation */
int32_t cueva_mlp_get_params(cueva_mlp* mlp, float* host, int32_t n);
int32_t cueva_mlp_set_params(cueva_mlp* mlp, const float* host, int32_t n);
/* n synthetic states (seeded, counter-based): rho log-uniform [1e-3,10],
 * p log-uniform [1e-4,10], W uniform [1,20], |B|^2/(rho h) log-uniform
 * [1e-3,10], isotropic v and B, E = -v x B + N(0,1e-3) */
int32_t cueva_mlp_synthetic_pairs(int32_t device, int64_t n, uint64_t seed, double gamma, double* d_cons,
                                  double* d_prims, void* stream);
/* feature / target mean and deviation over a training set (d_p: n pressures) */
int32_t cueva_mlp_fit_normalisation(cueva_mlp* mlp, const double* d_cons, const double* d_p, int64_t n);
/* `steps` Adam steps on minibatches of `batch` rows drawn with replacement,
 * cosine-decayed learning rate from lr; loss_out = last batch's MSE */
int32_t cueva_mlp_train(cueva_mlp* mlp, const double* d_cons, const double* d_p, int64_t n, int32_t steps,
                        int32_t batch, float lr, uint64_t seed, float* loss_out);
/* loss and gradient (CUEVA_MLP_NPARAM floats, host) of the MSE over the first
 * n rows, for checking the backward kernels */
int32_t cueva_mlp_gradients(cueva_mlp* mlp, const double* d_cons, const double* d_p, int32_t n, float* grads,
                            float* loss_out);
/* network pressure seeds of n states (device out): per thread in FP32
 * (tensor_cores = 0), warp-cooperative mma.sync with bf16 activations (1),
 * or tcgen05 MMA on tiles of 128 states with the accumulator in tensor
 * memory and bf16 activations (2, the form the step uses by default).
 * 3 is the self-test of the tcgen05 path's bounded waits: no MMA is issued,
 * the first wait gives up after a short limit, every CTA frees its tensor
 * memory, and the call returns CUEVA_ERR_PHYSICS (status 64) without
 * writing seeds; the device stays usable. */
int32_t cueva_mlp_predict(cueva_mlp* mlp, const double* d_cons, int64_t n, double* d_pseed, int32_t tensor_cores);
/* batch con2prim for comparisons: method 1 Cardano, 2 network seed + Newton,
 * 3 Newton from d_seed, 4 Newton from the network seed or the previous
 * pressure, whichever leaves the smaller residual (the seed choice of the
 * learned step); d_prev (5 x n: rho, p, vx, vy, vz) are the previous
 * primitives the Cardano path and method 4 seed from; d_iters (optional)
 * gets the Newton iterations (-1 = failed, then the Cardano result is
 * stored; 0 for method 1) */
int32_t cueva_c2p_batch(int32_t device, int32_t method, const cueva_mlp* mlp, double gamma, double eps1,
                        const double* d_cons, const double* d_prev, const double* d_seed, int64_t n, double* d_out,
                        int32_t* d_iters);
/* copy a trained network into ctx; con2prim uses it when params.c2p == 2:
 * Newton from the network's pressure or the previous pressure, whichever
 * leaves the smaller residual, Cardano where Newton fails */
int32_t cueva_attach_mlp(cueva_ctx* ctx, const cueva_mlp* mlp);
/* where the learned con2prim runs: 1 (set by cueva_attach_mlp) = a kernel of
 * its own after the last RK stage, network on the tcgen05 tensor cores in
 * tiles of 128 points, Newton in FP64, Cardano fall-back, then the next
 * step's startconvar; 0 = inside the last stage's update with warp mma.sync
 * inference (the earlier form, kept for comparison) */
int32_t cueva_set_learned_kernel(cueva_ctx* ctx, int32_t mode);
/* Newton iterations, points and Cardano fall-backs of the learned path so far */
int32_t cueva_learned_stats(cueva_ctx* ctx, int64_t out3[3]);

/* ---- ensembles ---------------------------------------------------------- */
/* No counterpart in the reference (it runs one grid per process).  n
 * independent grids -- each with its own size, sigma, boundaries, dt and c2p
 * method, sharing order, flux_solver, rec_mp, precision, intsum_reset and
 * device -- advanced together: each RK stage is one y-face and one x-face +
 * update launch over the tiles of all instances, and a step is one CUDA
 * graph.  Primitive blocks on the host are 14 x (imax+1) x (jmax+1) doubles,
 * field-major, i fastest, in cueva_field order (rho .. q). */
typedef struct cueva_ens cueva_ens;
int32_t cueva_ens_create(const cueva_params* params, int32_t n, cueva_ens** out);
int32_t cueva_ens_destroy(cueva_ens* ens);
int32_t cueva_ens_set_stream(cueva_ens* ens, void* cuda_stream);
int32_t cueva_ens_set_prims(cueva_ens* ens, int32_t k, const double* host_prims);
int32_t cueva_ens_get_prims(cueva_ens* ens, int32_t k, double* host_prims);
/* Kelvin-Helmholtz initial data for instance k (same conventions as cueva_kh_init) */
int32_t cueva_ens_kh_init(cueva_ens* ens, int32_t k, double v0, double a, double amp, double width, double kpert,
                          double phase, double bshear, double rho0, double p0);
/* nsteps ensemble steps (prepares stage 1 first if the state changed) */
int32_t cueva_ens_step(cueva_ens* ens, int32_t nsteps);
/* synchronise; status_out (optional, n words) gets each instance's status bits */
int32_t cueva_ens_sync(cueva_ens* ens, uint32_t* status_out);
/* launch shape: tile height rows (8 or 4) and CTAs per SM of a persistent
 * grid (0 = one tile per CTA) */
int32_t cueva_ens_set_shape(cueva_ens* ens, int32_t rows, int32_t ctas_per_sm);
/* times the candidate shapes on the current state, keeps the fastest and
 * restores the state; reports the choice and its ms per step */
int32_t cueva_ens_autotune(cueva_ens* ens, int32_t* rows, int32_t* ctas_per_sm, double* ms_per_step);
int32_t cueva_ens_attach_mlp(cueva_ens* ens, const cueva_mlp* mlp);
int32_t cueva_ens_set_learned_kernel(cueva_ens* ens, int32_t mode);   /* as cueva_set_learned_kernel */
int32_t cueva_ens_learned_stats(cueva_ens* ens, int64_t out3[3]);

/* ---- stage right-hand side without any device allocation -------------- */
/* No counterpart in the reference.  Computes the same stage right-hand side
 * as cueva_flux_rhs ({hll,hllc}_flow_mpx 2D + fluxandsource), but on device
 * arrays the caller already owns and without a context, so it never calls
 * cudaMalloc, cudaFree or anything else that allocates device memory.  It is
 * meant for callers that cannot allocate at this point: code running under a
 * fixed memory budget or a pre-sized arena whose free memory belongs to
 * another framework, and loops that must not pay the device-wide
 * synchronisation that cudaMalloc / cudaFree imply.
 *
 * Arrays (device memory, FP64, interior points only): point (i, j) of field
 * f of a group is at base[f * fstride + j * pitch + i], 0 <= i <= imax,
 * 0 <= j <= jmax, with pitch >= imax + 1 and fstride >= pitch * (jmax + 1):
 *   prim   the 14 primitives of time n in cueva_field order (rho .. q);
 *   W      the Lorentz factor of time n (one field);
 *   stage  the stage's 14 conserved (psi, phi, E, B, q, D, tau, S, in
 *          cueva_field order) followed by Jx, Jy, Jz (17 fields);
 *   rhs    out: psiflux .. Szflux, Exastsour .. Ezastsour (17 fields).
 * Only params' imax, jmax, flux_solver, rec_mp, bc_x, bc_y, precision,
 * device, lx, ly, lz, gamma and sigma are read.
 *
 * The interface-flux scratch is a fixed 32 MiB block of static device
 * memory inside the library (14 flux fields of (round32(imax + 2)) *
 * (jmax + 2) doubles plus a small header): grids that need more are
 * rejected with CUEVA_ERR_ARG and a message giving both sizes; 512 x 512
 * fits.  The first call on a device looks up the block's address and sets
 * the kernels' shared-memory limits there (no allocation), under a lock, so
 * host threads that make their first calls together set up once.  The call
 * uploads its kernel descriptor from host memory of the call itself and may
 * wait for the stream, so it returns CUEVA_ERR_ARG on a stream that is being
 * captured into a CUDA graph.  The status word in the block is zeroed by
 * every call.  The block is shared by all calls on a device, so calls that
 * overlap in time on the GPU (on different streams or host threads) race on
 * it; serialise them.
 *
 * Asynchronous on `stream` (0 = the legacy default stream).  If
 * status_bits is non-null the call waits for the stream and stores the
 * kernel status bits there; a non-zero status returns CUEVA_ERR_PHYSICS. */
int32_t cueva_flux_rhs_noalloc(const cueva_params* params, const double* prim, const double* W,
                               const double* stage, double* rhs, int32_t pitch, int64_t fstride, void* stream,
                               uint32_t* status_bits);

/* ---- run diagnostics (22_writer.f95:821-1001, subroutine lector) ------- */
/* Slots of a diagnostics record.  Slots 0..34 are the volume integrals
 * sum(x * Delx * Dely) over the points 0..imax x 0..jmax that the writer
 * prints to the Fortran units in brackets, with its expressions kept as
 * written: B2 leaves Bx out, and in eint_r and efluid_r only the p term is
 * multiplied by Delx * Dely.  D and tau are the conserved values of varfin
 * (con2prim does not write them back), as at the writer's call
 * (main_cueva_code.f95:332). */
enum cueva_diag_slot {
  CUEVA_DG_SUM_PSI = 0,   /* [80] psi */
  CUEVA_DG_SUM_PHI,       /* [81] phi */
  CUEVA_DG_SUM_EX,        /* [82] Ex^2 */
  CUEVA_DG_SUM_EY,        /* [83] Ey^2 */
  CUEVA_DG_SUM_EZ,        /* [84] Ez^2 */
  CUEVA_DG_SUM_EXEY,      /* [85] Ex Ey */
  CUEVA_DG_SUM_EXEZ,      /* [86] Ex Ez */
  CUEVA_DG_SUM_EYEZ,      /* [87] Ey Ez */
  CUEVA_DG_SUM_BX,        /* [88] Bx^2 */
  CUEVA_DG_SUM_BY,        /* [90] By^2 */
  CUEVA_DG_SUM_BZ,        /* [91] Bz^2 */
  CUEVA_DG_SUM_BXBY,      /* [92] Bx By */
  CUEVA_DG_SUM_BXBZ,      /* [93] Bx Bz */
  CUEVA_DG_SUM_BYBZ,      /* [94] By Bz */
  CUEVA_DG_SUM_VXVYVZ,    /* [95] v^2 */
  CUEVA_DG_SUM_BXBYBZ,    /* [96] B^2 */
  CUEVA_DG_SUM_VX,        /* [97] vx^2 */
  CUEVA_DG_SUM_VY,        /* [98] vy^2 */
  CUEVA_DG_SUM_VZ,        /* [99] vz^2 */
  CUEVA_DG_SUM_VXVY,      /* [200] vx vy */
  CUEVA_DG_SUM_VXVZ,      /* [201] vx vz */
  CUEVA_DG_SUM_VYVZ,      /* [202] vy vz */
  CUEVA_DG_SUM_Q,         /* [203] q */
  CUEVA_DG_SUM_P,         /* [204] p */
  CUEVA_DG_SUM_RHO,       /* [205] rho */
  CUEVA_DG_EKIN_C,        /* [206] rho v^2 / 2 */
  CUEVA_DG_EKIN_R,        /* [207] D (W - 1) */
  CUEVA_DG_ETOT,          /* [208] tau */
  CUEVA_DG_EFLUID_R,      /* [209] sum(rho h W^2 - p Delx Dely) */
  CUEVA_DG_EMAG,          /* [210] (E^2 + By^2 + Bz^2) / 2 */
  CUEVA_DG_EINT_C,        /* [211] rho eps */
  CUEVA_DG_EINT_R,        /* [212] sum(W^2 (rho eps + p) - p Delx Dely) */
  CUEVA_DG_LORENTZ,       /* [213] W */
  CUEVA_DG_SUM_D,         /* [214] D */
  CUEVA_DG_SUM_D_MED,     /* [215] D over i = floor(imax/4) .. floor(3 imax/4) */
  CUEVA_DG_MAX_BX,        /* [216] max Bx / B0 */
  CUEVA_DG_MAX_PHI,       /* [217] max phi */
  CUEVA_DG_DELTA_REC,     /* [67] B0 r tanh(Delx/delta_rec) delta_rec / By(imed+1, jmed+1) */
  CUEVA_DG_EZ_MED,        /* [68] Ez(imed, jmed), imed = floor(imax/2), jmed = floor(jmax/2) */
  CUEVA_DG_BY_MED,        /* By(imed+1, jmed+1), the denominator of [67] */
  /* Courant check (no counterpart in the reference, whose HLL-type fluxes use
   * the light-speed bounds -1, +1 and a fixed Delt): never changes Delt */
  CUEVA_DG_MAX_V,         /* max |v| */
  CUEVA_DG_MAX_W,         /* max W */
  CUEVA_DG_MAX_LAMBDA_X,  /* max |lambda| of the relativistic sound waves along x */
  CUEVA_DG_MAX_LAMBDA_Y,  /* ... along y */
  CUEVA_DG_COURANT,       /* Delt * max(max_lambda_x / Delx, max_lambda_y / Dely) */
  CUEVA_NDIAG
};

typedef struct cueva_diag_record {
  int64_t h;                /* step index h of the reference's time loop */
  double t;                 /* t_advance after that step */
  double v[CUEVA_NDIAG];
} cueva_diag_record;

typedef struct cueva_diag_config {
  int32_t hglb;        /* a record after step h when h == 1 or mod(h, hglb) == 0 (22_writer.f95:821) */
  int32_t capacity;    /* records kept on the device between cueva_diag_read calls */
  double b0;           /* B0 (parameters.f95:131) */
  double lr, ly;       /* Lr, Ly (parameters.f95:168,175) */
  double delta_rec;    /* delta_rec (parameters.f95:206) */
} cueva_diag_config;

/* Step clock of the context: h = index of the last completed step and
 * t = t_advance.  cueva_ctx_create starts at h = 0, t = 0 (hini = 1,
 * main_cueva_code.f95:45); each step adds 1 to h and Delt to t
 * (main_cueva_code.f95:161).  Set it when a run restarts from a backup. */
int32_t cueva_set_clock(cueva_ctx* ctx, int64_t h, double t);
int32_t cueva_get_clock(const cueva_ctx* ctx, int64_t* h, double* t);
/* Enables (cfg non-null) or disables the records and empties the record
 * buffer.  While enabled, cueva_step appends a record after each step whose
 * h is 1 or a multiple of hglb (the last stage of such a step also stores
 * varfin's D and tau for it). */
int32_t cueva_diag_enable(cueva_ctx* ctx, const cueva_diag_config* cfg);
/* Copies up to max_records of the records not yet read, oldest first, and
 * marks them read; when more than capacity records were appended since the
 * last read, the oldest were overwritten and are skipped.  *n_out = number
 * copied.  Synchronises the context's stream. */
int32_t cueva_diag_read(cueva_ctx* ctx, cueva_diag_record* out, int32_t max_records, int32_t* n_out);
/* One record of the state now on the device, with h and t of the clock;
 * D and tau here are startconvar's values of the current primitives.
 * Needs a config from cueva_diag_enable for B0, Lr, Ly and delta_rec. */
int32_t cueva_diag_now(cueva_ctx* ctx, cueva_diag_record* out);

/* ---- checkpoint / restart --------------------------------------------- */
/* Binary checkpoint of the device state at a step boundary: the 14 carried
 * primitives (all a step reads: startconvar rebuilds the rest) and the
 * clock, with the grid, the writing configuration and a checksum in the
 * header.  Loading needs a context of the same grid; it replaces the device
 * state and the clock, prepares stage 1 like cueva_upload, and leaves the
 * bound host arrays alone.  A run continued from a checkpoint is
 * bit-identical to the uninterrupted run.  No counterpart in the reference
 * (which restarts from its text backups, below). */
int32_t cueva_checkpoint_save(cueva_ctx* ctx, const char* path);
int32_t cueva_checkpoint_load(cueva_ctx* ctx, const char* path);
/* The reference's backup text files all_variables_NNNN.dat: written by the
 * writer every hloc steps (22_writer.f95:1134-1150), read by init_restart
 * (03_restart_primitive.f95:51-57).  One list-directed record per point,
 * i = -6..imax+6 outer, j = -6..jmax+6 inner, values psi phi Bx By Bz Vx Vy
 * Vz Ex Ey Ez q rho p, ghosts included.  fields[CUEVA_RHO .. CUEVA_Q] are
 * the 14 primitive host arrays in the Fortran layout (base = element
 * (-6,-6)).  The reader follows list-directed input (separators, repeat
 * counts, null values, slash, E/D/Q exponents and letter-less exponents such
 * as 1.0-100, records spanning lines); the writer prints 17 significant
 * digits, so a write-read round trip is exact, and like the reference it
 * refuses to replace an existing file unless overwrite != 0.  nthreads <= 0
 * uses every host core.  Host only: no GPU needed. */
int32_t cueva_read_all_variables(const char* path, int32_t imax, int32_t jmax, double* const* fields,
                                 int32_t nthreads);
int32_t cueva_write_all_variables(const char* path, int32_t imax, int32_t jmax, const double* const* fields,
                                  int32_t overwrite, int32_t nthreads);

/* ---- synthetic input ------------------------------------------------- */
/* Kelvin-Helmholtz initial data on the Fortran-layout prim arrays bound to
 * ctx (interior points; reference orientation: x = shear normal with copy
 * boundaries, y = periodic flow direction), conventions of
 * 03_init_var_primitive.f95:2297-2336:
 *   vy = v0 tanh(x/a), vx = amp sin(kpert y + phase) exp(-x^2/width),
 *   B = (0, bshear, 0), E = -v x B, rho = rho0, p = p0, psi = phi = q = 0,
 * with x = -lx/2 + i*Delx, y = -ly/2 + j*Dely. */
int32_t cueva_kh_init(cueva_ctx* ctx, double v0, double a, double amp, double width, double kpert,
                      double phase, double bshear, double rho0, double p0);

#ifdef __cplusplus
}
#endif
#endif /* CUEVA_H */
