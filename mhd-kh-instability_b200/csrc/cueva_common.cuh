// cueva_common.cuh -- shared definitions of the B200 CUEVA kernels.
//
// Device data layout (HBM): structure of arrays, one slab per field group,
// interior points only.  Point (i, j), 0 <= i <= imax, 0 <= j <= jmax, of
// field f lives at base + f * fstride + j * pitch + i, with pitch a multiple
// of 32 doubles (256 B rows) so every warp-wide row access is one aligned
// 256 B segment.  Ghost cells of the Fortran arrays are never stored: loads
// outside the interior go through the per-axis index map of the reference's
// boundary routines (copy = clamp to [0, N]; periodic = node duplicate,
// -k -> N-k and N+k -> k; 04_boundary.f95:1390-1533, 2867-3033).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cueva {

// ---- field groups --------------------------------------------------------
// carried primitive state, order of the C-ABI prims (include/cueva.h)
enum Prim { P_RHO = 0, P_P, P_VX, P_VY, P_VZ, P_PSI, P_PHI, P_EX, P_EY, P_EZ, P_BX, P_BY, P_BZ, P_Q, NPRIM };
// conserved D, tau, S and the Lorentz factor at time n (startconvar)
enum Aux { A_D = 0, A_TAU, A_SX, A_SY, A_SZ, A_W, NAUX };
// RK stage state: the 14 conserved of stage l (E already implicit) + J
enum Stage { Q_PSI = 0, Q_PHI, Q_EX, Q_EY, Q_EZ, Q_BX, Q_BY, Q_BZ, Q_Q, Q_D, Q_TAU, Q_SX, Q_SY, Q_SZ,
             Q_JX, Q_JY, Q_JZ, NSTAGE };
constexpr int NCONS = 14;   // first 14 stage fields are the conserved set
// stage right-hand side: F (14, same order as the conserved set) + E sources
enum Rhs { K_SEX = 14, K_SEY, K_SEZ, NRHS };

// ---- status bits (host maps them to C-ABI error codes) -------------------
enum StatusBits : uint32_t {
  ST_C2P_FAIL = 1u,        // Cardano "stop" branches, 12_varprimitive.f95:382-428,485
  ST_SUPERLUMINAL = 2u,    // 12_varprimitive.f95:678,691 ; 12_varprimitive_nr.f95:217
  ST_HLLC_NOCONV = 4u,     // funciones.f95:240-245
  ST_HLLC_VSTAR = 8u,      // 16_hllc_flow_mpx.f95:4294,4605
  ST_NONFINITE = 16u,      // con2prim returned NaN / Inf
  ST_HLLE_SPEED = 32u,     // 16_hlle_flow_mpx.f95:2796-2803, 2974-2981
  ST_TC_TIMEOUT = 64u,     // a bounded tensor-core wait ran out (no reference counterpart)
  ST_TC_TEARDOWN = 128u,   // after such a time-out the teardown's bounded wait for the MMAs still in
                           // flight ran out too: TMEM was released while an MMA may still write it, so
                           // the context is suspect and should not be reused
  ST_COPY_TIMEOUT = 256u,  // a bounded wait for the bulk copies of the stage kernel's stencil rows ran
                           // out (no reference counterpart); the CTA stopped
};

// ---- per-instance descriptor (one grid of the ensemble) -------------------
struct InstDesc {
  // device buffers
  double* prim[2];     // double-buffered NPRIM slabs
  double* aux[2];      // double-buffered NAUX slabs
  double* stage[2];    // double-buffered NSTAGE slabs
  double* intsum;      // NCONS slab (needed when the tableau has >= 3 stages)
  double* finsum;      // NCONS slab
  double* kbuf;        // nk * NRHS slabs of stored stage right-hand sides
  double* rhs_out;     // NRHS slab written in the store-rhs mode
  uint32_t* status;    // status word
  unsigned long long* counters;  // [3] fix-up counters (rho, p, v)
  // learned con2prim seed network (null unless c2p method 2)
  const void* mlp;
  // geometry
  int imax, jmax;      // interior points 0..imax, 0..jmax
  int pitch;           // doubles per row
  long long fstride;   // doubles per field slab
  int bc_x, bc_y;      // 0 copy, 1 periodic
  // scalars
  double delx, dely, dt, sigma, gamma, kappa_psi, kappa_phi;
  // 1/delx, 1/dely when the spacing is a power of two (then v * inv == v / del
  // exactly and the divisions of the flux divergence become multiplications);
  // 0 otherwise
  double inv_delx_pow2, inv_dely_pow2;
  double eps1_c2p;     // value of the Fortran module variable eps1 when con2prim runs
  int c2p;             // 1 Cardano, 0 NR, 2 learned seed + Newton (Cardano fallback)
  int primitive_rec;   // 1: the step starts with the primitive reconstruction (k_recons_begin),
                       // so the last stage does not prepare the next step's stage 1
  int c2p_tc;          // c2p 2 with a network: 1 = con2prim in k_c2p_step on the tcgen05 tensor
                       // cores after the last stage, 0 = inside the last stage (warp mma.sync)
  // interface flux scratch: Fx(i+1/2, j) at fx[(j) * fpitch + (i + 1)],
  // Fy(i, j+1/2) at fy[(j + 1) * fpitch + i], NFACE fields each
  double* fx;
  double* fy;
  int fpitch;
  long long ffs;       // doubles per flux field
  // work decomposition: tiles of each launch kind (x faces + update, y faces,
  // learned con2prim, fused stage)
  int block_begin[4];
  int block_count[4];
  int seg_rows;        // fused stage tiles: grid rows per tile (bands of the tile height, less one row)
};

// ---- tableau data of one stage launch (by value, kernel parameter space) -----
struct StageArgs {
  int l;               // 1-based RK stage being swept
  int s;               // number of stages
  int cur;             // which prim/aux buffer holds time n
  int qin;             // which stage buffer holds stage l
  double wb, wbt;      // wb(l), wbt(l)
  double ab_next[8];   // Ab(l+1, 1..l)
  double abt_next[8];  // Abt(l+1, 1..l)
  double abt_diag_next;// Abt(l+1, l+1)
  double abt_diag_first;// Abt(1,1) (next step's stage 1)
  int kslot[8];        // slot of stored K_m in kbuf, -1 if not stored
  int store_k_slot;    // slot to store K_l, -1 if not needed
  int store_k_src;     // K_l is only read through its E sources (every later row has Ab = 0 in
                       // column l): store the 3 sources, not the 14 fluxes
  int fin_load;        // the final sums of earlier stages are not all zero (some wb, wbt of m < l
                       // is non-zero): load them; else they start from zero
  int fin_store;       // the final sums after this stage are not identically zero: store them
  int need_intsum_load;  // stage l >= 2 and s >= 3: intsum_l is stored
  int need_intsum_store; // l + 1 < s
  int mode;            // 0 fused (next stage / final), 1 store rhs only, 2 also the x-face fluxes (I.fx)
  double* diag_cons;   // last stage: D and tau of varfin stored here (2 slabs) when non-null
};

// ---- small math helpers (Fortran semantics) ------------------------------
template <typename T> __device__ __forceinline__ T pw2(T x) { return x * x; }
template <typename T> __device__ __forceinline__ T pw3(T x) { return (x * x) * x; }
template <typename T> __device__ __forceinline__ T pw4(T x) { T t = x * x; return t * t; }
template <typename T> __device__ __forceinline__ T fmin2(T a, T b) { return (b < a) ? b : a; }
template <typename T> __device__ __forceinline__ T fmax2(T a, T b) { return (b > a) ? b : a; }
template <typename T> __device__ __forceinline__ T fsgn1(T b) { return copysign(T(1), b); }

// ghost index maps of the reference's boundary routines
__device__ __forceinline__ int map_idx(int i, int n, int periodic) {
  if (i < 0) return periodic ? i + n : 0;
  if (i > n) return periodic ? i - n : n;
  return i;
}

// launch geometry: 32 x ROWS threads per CTA for the face tiles (x tiles
// update 31 points per row; ROWS is 8 or 4), 256 threads for the pointwise
// kernels
constexpr int FACE_ROWS = 8;   // default tile height
constexpr int NFACE = 14;   // interface fluxes per face (the Riemann roles)
constexpr int POINT_THREADS = 256;
enum LaunchKind { LK_XUPD = 0, LK_YFACE = 1, LK_C2P = 2, LK_STAGE = 3 };

// launch shape of one RK stage: tile height, CTAs per launch kind and the
// tiles they loop over (grid == ntiles: one tile per CTA; smaller: persistent).
// fused: the stage runs as one k_stage launch (grid[LK_STAGE] CTAs over
// ntiles[LK_STAGE] tiles) instead of k_yface + k_xupd.
struct StageShape {
  int rows = FACE_ROWS;
  int grid[4] = {0, 0, 0, 0};
  int ntiles[4] = {0, 0, 0, 0};
  bool fused = false;
};

// tiles of one instance for a tile height (x tiles: 31 points by rows)
inline int xupd_tiles(int imax, int jmax, int rows) { return ((imax + 1 + 30) / 31) * ((jmax + 1 + rows - 1) / rows); }
inline int yface_tiles(int imax, int jmax, int rows) { return ((imax + 1 + 31) / 32) * ((jmax + 2 + rows - 1) / rows); }
// fused stage tiles: strips of 31 points by segments of seg_rows grid rows
inline int stage_tiles(int imax, int jmax, int seg_rows) {
  return ((imax + 1 + 30) / 31) * ((jmax + 1 + seg_rows - 1) / seg_rows);
}

// The mixed-precision flux routines keep the fluxes of the field roles psi,
// phi, Bn, Bt1, Bt2, En, Et1, Et2 (roles 0..7) in FP64: they carry the
// uniform background field (B ~ 0.1 in the KH runs), whose FP32 rounding
// (~4e-9) is not small against E itself, and the final IMEX combination
// passes that error into E(n+1) undamped.  All routines but HLLE-MC
// (flux_solver 3, whose field star states use the sound-speed bounds).
__host__ __device__ constexpr bool mixed_em_f64(int solver) { return solver >= 1 && solver <= 7 && solver != 3; }
// The mixed-precision MP routines HLL, HLLE and HLLC (flux_solver 5..7) also
// form the normal momentum flux in FP64: its pressure part, ~1 in the KH
// layer, is added to the FP32 rest there (see the split pressure of the
// stage kernels).
__host__ __device__ constexpr bool mixed_split_p(int solver) { return solver >= 5 && solver <= 7; }
constexpr int ROLE_SN = 11;   // the normal momentum flux (R_SN of the Riemann roles)

// Place of role r in the y-flux scratch (NFACE slabs of ffs doubles): f64
// tells the element type and off the slab's first element in units of that
// type.  FP64 kernels: double slab r.  Mixed kernels: FP32 slab r; with
// mixed_em_f64, double slabs 0..7 for roles 0..7, then FP32 slabs for roles
// 8..13 from byte offset 64 * ffs on; with mixed_split_p also, the normal
// momentum flux in double slab 8 and the other five FP32 slabs from byte
// offset 72 * ffs on.
struct FluxSlot {
  bool f64;
  long long off;
};
__host__ __device__ inline FluxSlot flux_slot(bool mixed, int solver, int r, long long ffs) {
  if (!mixed) return {true, r * ffs};
  if (!mixed_em_f64(solver)) return {false, r * ffs};
  if (r <= 7) return {true, r * ffs};
  if (mixed_split_p(solver)) {
    if (r == ROLE_SN) return {true, 8 * ffs};
    return {false, (18 + (r < ROLE_SN ? r - 8 : r - 9)) * ffs};
  }
  return {false, (16 + (r - 8)) * ffs};
}

}  // namespace cueva
