// cueva_abi.cu -- the C-ABI of include/cueva.h: contexts, Fortran-layout
// transfers, step orchestration with CUDA graphs, routine mirrors.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cueva.h"
#include "cueva_common.cuh"
#include "cueva_launch.h"
#include "cueva_mlp.cuh"

using namespace cueva;

namespace {

thread_local std::string g_err;

int32_t fail(int32_t code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace

int32_t cueva_fail(int32_t code, const std::string& msg) { return fail(code, msg); }

namespace {

#define CUDA_TRY(x)                                                                          \
  do {                                                                                       \
    cudaError_t e_ = (x);                                                                    \
    if (e_ != cudaSuccess) return fail(CUEVA_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// IMEX tableaux, imex_scheme.f95:13-507 (MIRK = 0)
struct Tableau { int s = 0; double wb[8] = {}, wbt[8] = {}, Ab[8][8] = {}, Abt[8][8] = {}; };

bool make_tableau(int order, Tableau& T) {
  T = Tableau();
  const double cst = 1.0 - 1.0 / std::sqrt(2.0);
  const double alpha1 = 0.24169426078821, beta1 = 0.06042356519705, etha1 = 0.12915286960590;
  switch (order) {
  case 1: T.s = 1; T.wb[0] = 1.0; T.Ab[0][0] = 1.0; return true;
  case 2:
    T.s = 2; T.wb[0] = T.wb[1] = 0.5; T.wbt[0] = T.wbt[1] = 0.5; T.Ab[1][0] = 1.0;
    T.Abt[0][0] = cst; T.Abt[1][0] = 1.0 - 2.0 * cst; T.Abt[1][1] = cst; return true;
  case 3:
    T.s = 3; for (int k = 0; k < 3; ++k) { T.wb[k] = 1.0 / 3.0; T.wbt[k] = 1.0 / 3.0; }
    T.Ab[1][0] = 0.5; T.Ab[2][0] = 0.5; T.Ab[2][1] = 0.5;
    T.Abt[0][0] = 1.0 / 5.0; T.Abt[1][0] = 1.0 / 10.0; T.Abt[1][1] = 1.0 / 5.0;
    T.Abt[2][0] = 1.0 / 3.0; T.Abt[2][1] = 1.0 / 3.0; T.Abt[2][2] = 1.0 / 3.0; return true;
  case 4:
    T.s = 4; T.wb[1] = 1.0 / 6.0; T.wb[2] = 1.0 / 6.0; T.wb[3] = 2.0 / 3.0;
    for (int k = 0; k < 4; ++k) T.wbt[k] = T.wb[k];
    T.Ab[2][1] = 1.0; T.Ab[3][1] = 0.25; T.Ab[3][2] = 0.25;
    T.Abt[0][0] = alpha1; T.Abt[1][0] = -1.0 * alpha1; T.Abt[1][1] = alpha1;
    T.Abt[2][1] = 1.0 - alpha1; T.Abt[2][2] = alpha1;
    T.Abt[3][0] = beta1; T.Abt[3][1] = etha1; T.Abt[3][2] = 0.5 - beta1 - etha1 - alpha1; T.Abt[3][3] = alpha1;
    return true;
  case 5: {
    T.s = 5;
    const double wb[5] = {1.0 / 4.0, 7.0 / 4.0, 3.0 / 4.0, -7.0 / 4.0, 0.0};
    const double wbt[5] = {0.0, 3.0 / 2.0, -3.0 / 2.0, 0.5, 0.5};
    const double A[5][5] = {{0, 0, 0, 0, 0}, {0.5, 0, 0, 0, 0}, {11.0 / 18.0, 1.0 / 18.0, 0, 0, 0},
                            {5.0 / 6.0, -5.0 / 6.0, 0.5, 0, 0}, {1.0 / 4.0, 7.0 / 4.0, 3.0 / 4.0, -7.0 / 4.0, 0}};
    const double At[5][5] = {{0, 0, 0, 0, 0}, {0, 0.5, 0, 0, 0}, {0, 1.0 / 6.0, 0.5, 0, 0},
                             {0, -0.5, 0.5, 0.5, 0}, {0, 3.0 / 2.0, -3.0 / 2.0, 0.5, 0.5}};
    for (int a = 0; a < 5; ++a) { T.wb[a] = wb[a]; T.wbt[a] = wbt[a];
      for (int b = 0; b < 5; ++b) { T.Ab[a][b] = A[a][b]; T.Abt[a][b] = At[a][b]; } }
    return true; }
  case 6: {
    T.s = 6;
    const double w[6] = {-0.035877095577305, 0.673080876788404, 0.149064711243777,
                         0.137173305022086, 0.150219587614740, -0.073661385091702};
    const double A[6][6] = {
      {0, 0, 0, 0, 0, 0}, {0.342975342284516, 0, 0, 0, 0, 0},
      {0.016193013787920, 0.309787886268879, 0, 0, 0, 0},
      {-0.135950059698287, 0.640189764616023, 0.342154021907072, 0, 0, 0},
      {-0.042056958294301, 0.660781723165128, -0.381308869908091, 1.001236515566727, 0, 0},
      {0.099109299514465, -0.466919631638661, 1.030492210860962, 0.564549736036252, -0.119257987827582, 0}};
    const double At[6][6] = {
      {0.449855695709406, 0, 0, 0, 0, 0}, {-0.295189486209790, 0.449855695709406, 0, 0, 0, 0},
      {0.879036496969614, -0.042071370873823, 0.449855695709406, 0, 0, 0},
      {0.751731896214317, -0.222508174774298, 0.220689305480633, 0.449855695709406, 0, 0},
      {-0.039570781554756, 0.788509712948086, 0.685131268735182, -0.144071924307435, 0.449855695709406, 0},
      {0.382760589609172, -0.196622622060158, 0.904049611197476, 0.680864149962184, 0.571862669923976,
       0.449855695709406}};
    for (int a = 0; a < 6; ++a) { T.wb[a] = w[a]; T.wbt[a] = w[a];
      for (int b = 0; b < 6; ++b) { T.Ab[a][b] = A[a][b]; T.Abt[a][b] = At[a][b]; } }
    return true; }
  case 8: {
    T.s = 8;
    const double w[8] = {0.0, 277.0 / 1720.0, 385.0 / 1314.0, 587.0 / 1885.0, 31.0 / 18247.0, 665.0 / 2906.0,
                         0.0, 23.0 / 5731.0};
    const double A[8][8] = {
      {0, 0, 0, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0}, {0, 966.0 / 2039.0, 0, 0, 0, 0, 0, 0},
      {0, 199.0 / 5291.0, 735.0 / 1709.0, 0, 0, 0, 0, 0},
      {0, 306.0 / 4373.0, 533.0 / 1060.0, 773.0 / 628.0, 0, 0, 0, 0},
      {0, 61.0 / 10399.0, 552.0 / 8267.0, 881.0 / 1054.0, 52.0 / 9395.0, 0, 0, 0},
      {184.0 / 2869.0, 141.0 / 3059.0, 826.0 / 1929.0, 1567.0 / 757.0, 1754.0 / 977.0, 161.0 / 599.0, 0, 0},
      {0, 27.0 / 359.0, 227.0 / 2338.0, 53.0 / 557.0, 569.0 / 4644.0, 859.0 / 1966.0, 0, 0}};
    const double g = 1026.0 / 3919.0;
    const double At[8][8] = {
      {g, 0, 0, 0, 0, 0, 0, 0}, {-1148.0 / 4385.0, g, 0, 0, 0, 0, 0, 0},
      {-1165.0 / 2683.0, 904.0 / 1399.0, g, 0, 0, 0, 0, 0},
      {1480.0 / 2439.0, -1469.0 / 4070.0, -121.0 / 3026.0, g, 0, 0, 0, 0},
      {-2788.0 / 397.0, 2069.0 / 294.0, 722.0 / 339.0, -411.0 / 682.0, g, 0, 0, 0},
      {-165.0 / 12667.0, 105.0 / 671.0, 133.0 / 500.0, 1307.0 / 5430.0, 55.0 / 26474.0, g, 0, 0},
      {837.0 / 1003.0, 629.0 / 1976.0, 1195.0 / 149.0, -5209.0 / 618.0, 1045.0 / 1459.0, 2767.0 / 911.0, g, 0},
      {-752.0 / 647.0, -771.0 / 2338.0, 3197.0 / 469.0, 2313.0 / 586.0, -2267.0 / 2341.0, -2128.0 / 275.0, 0, g}};
    for (int a = 0; a < 8; ++a) { T.wb[a] = w[a]; T.wbt[a] = w[a];
      for (int b = 0; b < 8; ++b) { T.Ab[a][b] = A[a][b]; T.Abt[a][b] = At[a][b]; } }
    return true; }
  default: return false;
  }
}

}  // namespace

namespace {

int32_t validate_params(const cueva_params* p) {
  if (p->imax < 6 || p->jmax < 6) return fail(CUEVA_ERR_ARG, "imax and jmax must be >= 6 (6 ghost cells)");
  if (p->flux_solver < 1 || p->flux_solver > 7)
    return fail(CUEVA_ERR_ARG, "flux_solver must be 1 (Lax+MC), 2 (HLL+MC), 3 (HLLE+MC), 4 (HLLC+MC), "
                               "5 (HLL+MPX), 6 (HLLE+MPX) or 7 (HLLC+MPX)");
  if (p->rec_mp < 0 || p->rec_mp > 2) return fail(CUEVA_ERR_ARG, "rec_mp must be 0, 1 or 2");
  if (p->c2p < 0 || p->c2p > 2) return fail(CUEVA_ERR_ARG, "c2p must be 0, 1 or 2");
  if ((p->bc_x != 0 && p->bc_x != 1) || (p->bc_y != 0 && p->bc_y != 1))
    return fail(CUEVA_ERR_ARG, "bc_x, bc_y must be 0 (copy) or 1 (periodic)");
  if (p->precision != 0 && p->precision != 1) return fail(CUEVA_ERR_ARG, "precision must be 0 or 1");
  if (p->intsum_reset != 0 && p->intsum_reset != 1) return fail(CUEVA_ERR_ARG, "intsum_reset must be 0 or 1");
  if (p->primitive_rec != 0 && p->primitive_rec != 1) return fail(CUEVA_ERR_ARG, "primitive_rec must be 0 or 1");
  return CUEVA_OK;
}

// K_m storage: needed when a row r >= m+2 of the tableau uses column m
int kslots(const Tableau& T, int (&kslot_of)[8]) {
  int n = 0;
  for (int m = 0; m < 8; ++m) kslot_of[m] = -1;
  for (int m = 0; m < T.s; ++m) {
    bool need = false;
    for (int r = m + 2; r < T.s; ++r) need = need || T.Ab[r][m] != 0.0 || T.Abt[r][m] != 0.0;
    if (need) kslot_of[m] = n++;
  }
  return n;
}

// geometry and device layout of one grid
struct InstGeom {
  int imax, jmax, nx, ny, pitch, fpitch;
  long long fstride, ffs, nslab;
  double delx, dely, delz, dt;
};

InstGeom inst_geom(const cueva_params* p, int nkslot) {
  InstGeom G{};
  G.imax = p->imax; G.jmax = p->jmax; G.nx = p->imax + 1; G.ny = p->jmax + 1;
  G.pitch = (G.nx + 31) / 32 * 32;
  G.fstride = (long long)G.pitch * G.ny;
  G.delx = p->lx / (double)p->imax;
  G.dely = p->ly / (double)p->jmax;
  G.delz = p->lz / 1.0;
  double mn = (G.dely < G.delx) ? G.dely : G.delx;
  mn = (G.delz < mn) ? G.delz : mn;
  G.dt = (p->dt > 0.0) ? p->dt : p->cfl * mn;
  // interface flux scratch: x faces -1/2 .. imax+1/2 (imax+2 per row) on
  // jmax+1 rows, y faces on jmax+2 rows of imax+1
  G.fpitch = (G.nx + 1 + 31) / 32 * 32;
  G.ffs = (long long)G.fpitch * (G.ny + 1);
  const long long nfields = 2LL * NPRIM + 2LL * NAUX + 2LL * NSTAGE + 2LL * NCONS + (long long)nkslot * NRHS + NRHS;
  G.nslab = nfields * G.fstride + 2LL * NFACE * G.ffs;
  return G;
}

// instance descriptor over a slab of G.nslab doubles (tile ranges not set)
void fill_desc(const cueva_params* p, const InstGeom& G, int nkslot, double* slab, uint32_t* status,
               unsigned long long* counters, InstDesc& I) {
  const long long fs = G.fstride;
  double* q = slab;
  I.prim[0] = q; q += NPRIM * fs; I.prim[1] = q; q += NPRIM * fs;
  I.aux[0] = q; q += NAUX * fs; I.aux[1] = q; q += NAUX * fs;
  I.stage[0] = q; q += NSTAGE * fs; I.stage[1] = q; q += NSTAGE * fs;
  I.intsum = q; q += NCONS * fs;
  I.finsum = q; q += NCONS * fs;
  I.kbuf = q; q += (long long)nkslot * NRHS * fs;
  I.rhs_out = q; q += NRHS * fs;
  I.fx = q; q += NFACE * G.ffs;
  I.fy = q; q += NFACE * G.ffs;
  I.fpitch = G.fpitch; I.ffs = G.ffs;
  I.status = status;
  I.counters = counters;
  I.mlp = nullptr;
  I.imax = G.imax; I.jmax = G.jmax; I.pitch = G.pitch; I.fstride = fs;
  I.bc_x = p->bc_x; I.bc_y = p->bc_y;
  I.delx = G.delx; I.dely = G.dely; I.dt = G.dt; I.sigma = p->sigma; I.gamma = p->gamma;
  auto inv_pow2 = [](double d) {
    int e = 0;
    return (std::frexp(d, &e) == 0.5 && std::isnormal(1.0 / d)) ? 1.0 / d : 0.0;
  };
  I.inv_delx_pow2 = inv_pow2(G.delx);
  I.inv_dely_pow2 = inv_pow2(G.dely);
  const double mn = (G.dely < G.delx) ? G.dely : G.delx;   // parameters.f95:329-334
  const double cp = std::sqrt(mn / 1.0);
  I.kappa_psi = 1.0 / (cp * cp);
  I.kappa_phi = 1.0 / (cp * cp);
  // the Fortran module variable eps1 keeps the value the flux routine stored last
  // (the Lax and MCL routines of flux_solver 1 and 2 never set it: zero-initialised)
  I.eps1_c2p = (p->flux_solver == 7) ? (double)1.0e-6f : (p->flux_solver <= 2 ? 0.0 : 1.0e-6);
  I.c2p = p->c2p;
  I.c2p_tc = 0;
  I.primitive_rec = p->primitive_rec;
  I.block_begin[LK_C2P] = 0;
  I.block_count[LK_C2P] = c2p_tiles(G.imax, G.jmax);
}

}  // namespace

struct cueva_ctx {
  cueva_params P{};
  Tableau T;
  int dev = 0;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  int imax = 0, jmax = 0, nx = 0, ny = 0, pitch = 0;
  long long fstride = 0;
  double delx = 0, dely = 0, delz = 0, dt = 0;
  // device memory
  double* slab = nullptr;
  uint32_t* d_status = nullptr;
  unsigned long long* d_counters = nullptr;
  InstDesc* d_inst = nullptr;
  InstDesc h_inst{};
  int nkslot = 0;
  int kslot_of[8];        // slot of K_m (0-based m) or -1
  StageShape shape;       // tile height, CTAs and tiles of the two stage launches
  int cur = 0, qin = 0;
  bool primed = false;
  double* bound[CUEVA_NFIELDS] = {};
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  MLPDevice* d_mlp = nullptr;                 // attached learned seed (c2p = 2)
  unsigned long long* d_mlp_stats = nullptr;  // Newton iterations, points, fall-backs
  // step clock (h, t_advance) and run diagnostics
  long long h = 0;
  double t = 0.0;
  bool diag_on = false;
  cueva_diag_config diag{};
  double* d_diag_cons = nullptr;          // varfin D, tau (2 slabs) of record steps
  double* d_diag_part = nullptr;          // per-CTA partial results
  cueva_diag_record* d_diag_rec = nullptr;// ring of diag.capacity records
  long long diag_written = 0, diag_read = 0;
  cudaGraphExec_t graph_diag[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  // cueva_download_async: copies on a second stream, one event per field
  // (14 prims, then the 6 conserved fields), so that the next upload of field
  // f waits only for field f's readback
  cudaStream_t xfer = nullptr;
  cudaEvent_t ev_ready = nullptr, ev_xfer_done = nullptr;
  cudaEvent_t ev_field[NPRIM + NAUX] = {};
  bool dl_pending = false;
  bool field_pending[NPRIM + NAUX] = {};
};

namespace {

// Orders the context stream after a pending cueva_download_async: its copies
// read device buffers that later work on the stream overwrites.
int32_t join_downloads(cueva_ctx* c) {
  if (!c->dl_pending) return CUEVA_OK;
  CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_xfer_done, 0));
  c->dl_pending = false;
  for (bool& b : c->field_pending) b = false;
  return CUEVA_OK;
}

// Every entry point starts here; join = false only where the caller orders
// itself per field (cueva_upload) or only reads host state.
int32_t check_ctx(cueva_ctx* c, bool join = true) {
  if (!c) return fail(CUEVA_ERR_ARG, "null context");
  if (join) return join_downloads(c);
  return CUEVA_OK;
}

size_t host_field_elems(const cueva_ctx* c) { return (size_t)(c->imax + 13) * (size_t)(c->jmax + 13); }
double* host_interior(const cueva_ctx* c, double* base, int l) {
  // element (0, 0) of stage l of a (-6:imax+6, -6:jmax+6, 1:lmax) array
  return base + (size_t)(l - 1) * host_field_elems(c) + 6 + (size_t)6 * (c->imax + 13);
}

int32_t h2d(cueva_ctx* c, double* dst, int field, int l) {
  if (!c->bound[field]) return fail(CUEVA_ERR_UNBOUND, "field " + std::to_string(field) + " not bound");
  CUDA_TRY(cudaMemcpy2DAsync(dst, (size_t)c->pitch * 8, host_interior(c, c->bound[field], l),
                             (size_t)(c->imax + 13) * 8, (size_t)c->nx * 8, (size_t)c->ny, cudaMemcpyHostToDevice,
                             c->stream));
  return CUEVA_OK;
}
int32_t d2h(cueva_ctx* c, const double* src, int field, int l) {
  if (!c->bound[field]) return fail(CUEVA_ERR_UNBOUND, "field " + std::to_string(field) + " not bound");
  CUDA_TRY(cudaMemcpy2DAsync(host_interior(c, c->bound[field], l), (size_t)(c->imax + 13) * 8, src,
                             (size_t)c->pitch * 8, (size_t)c->nx * 8, (size_t)c->ny, cudaMemcpyDeviceToHost,
                             c->stream));
  return CUEVA_OK;
}

double* prim_f(cueva_ctx* c, int buf, int f) { return c->h_inst.prim[buf] + (long long)f * c->fstride; }
double* aux_f(cueva_ctx* c, int buf, int f) { return c->h_inst.aux[buf] + (long long)f * c->fstride; }
double* stage_f(cueva_ctx* c, int buf, int f) { return c->h_inst.stage[buf] + (long long)f * c->fstride; }

int32_t read_status(cueva_ctx* c) {
  uint32_t st = 0;
  CUDA_TRY(cudaMemcpyAsync(&st, c->d_status, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (st) {
    char buf[160];
    snprintf(buf, sizeof buf, "kernel status 0x%x (1 con2prim, 2 superluminal, 4 hllc_vel, 8 v* not finite, 16 non-finite state, 32 HLLE wave speed, 64 tensor-core wait, 128 tensor-core teardown: context suspect, 256 stencil copy wait)", st);
    return fail(CUEVA_ERR_PHYSICS, buf);
  }
  return CUEVA_OK;
}

StageArgs stage_args_of(const Tableau& T, const int* kslot_of, int intsum_reset, int cur, int qin, int l,
                        int mode) {
  StageArgs sa{};
  sa.l = l; sa.s = T.s; sa.cur = cur; sa.qin = qin; sa.mode = mode;
  sa.wb = T.wb[l - 1]; sa.wbt = T.wbt[l - 1];
  for (int m = 0; m < 8; ++m) { sa.kslot[m] = -1; sa.ab_next[m] = 0.0; sa.abt_next[m] = 0.0; }
  if (l < T.s) {
    for (int m = 1; m <= l; ++m) { sa.ab_next[m - 1] = T.Ab[l][m - 1]; sa.abt_next[m - 1] = T.Abt[l][m - 1]; }
    sa.abt_diag_next = T.Abt[l][l];
  }
  sa.abt_diag_first = T.Abt[0][0];
  for (int m = 1; m < l; ++m) sa.kslot[m - 1] = kslot_of[m - 1];
  sa.store_k_slot = (l < T.s) ? kslot_of[l - 1] : -1;
  // K_l is read by rows r >= l+2 only through its E sources when every such
  // row has Ab(r, l) = 0 (SSP3(4,3,3): K_1, whose only later use is Abt(4,1))
  sa.store_k_src = 1;
  for (int r = l + 1; r < T.s; ++r) sa.store_k_src = sa.store_k_src && T.Ab[r][l - 1] == 0.0;
  // the final sums stay zero while every stage so far has zero weights
  // (SSP3(4,3,3): wb(1) = wbt(1) = 0)
  sa.fin_load = 0;
  for (int m = 1; m < l; ++m) sa.fin_load = sa.fin_load || T.wb[m - 1] != 0.0 || T.wbt[m - 1] != 0.0;
  sa.fin_store = sa.fin_load || T.wb[l - 1] != 0.0 || T.wbt[l - 1] != 0.0;
  // the reference zeroes the stage sums once per step, so stage l+1 starts
  // from the sums of stage l; with intsum_reset every stage starts from zero
  sa.need_intsum_load = (!intsum_reset && l >= 2 && l < T.s) ? 1 : 0;
  sa.need_intsum_store = (!intsum_reset && l + 1 < T.s) ? 1 : 0;
  return sa;
}

StageArgs stage_args(const cueva_ctx* c, int l, int mode) {
  return stage_args_of(c->T, c->kslot_of, c->P.intsum_reset, c->cur, c->qin, l, mode);
}

// Kelvin-Helmholtz initial data at one node (reference orientation: x the
// shear normal, y the flow direction; 03_init_var_primitive.f95:2297-2336)
struct KHParams { double v0, a, amp, width, kpert, phase, bshear, rho0, p0; };
void kh_point(const KHParams& k, double posx, double posy, double (&pv)[NPRIM]) {
  const double vx = k.amp * std::sin(k.kpert * posy + k.phase) * std::exp(-(posx * posx) / k.width);
  const double vy = k.v0 * std::tanh(posx / k.a);
  const double vz = 0.0;
  const double Bx = 0.0, By = k.bshear, Bz = 0.0;
  pv[P_RHO] = k.rho0; pv[P_P] = k.p0;
  pv[P_VX] = vx; pv[P_VY] = vy; pv[P_VZ] = vz;
  pv[P_PSI] = 0.0; pv[P_PHI] = 0.0; pv[P_Q] = 0.0;
  pv[P_BX] = Bx; pv[P_BY] = By; pv[P_BZ] = Bz;
  pv[P_EX] = -(vy * Bz - vz * By);
  pv[P_EY] = -(vz * Bx - vx * Bz);
  pv[P_EZ] = -(vx * By - vy * Bx);
}

int32_t run_begin_step(cueva_ctx* c) {
  CUDA_TRY(launch_begin_step((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur, c->qin, c->T.Abt[0][0]));
  c->primed = true;
  return CUEVA_OK;
}

bool learned_tc(const InstDesc& I, const MLPDevice* d_mlp) { return I.c2p == 2 && I.c2p_tc && d_mlp; }

int32_t enqueue_step(cueva_ctx* c, double* diag_cons = nullptr) {
  if (c->P.primitive_rec) {   // main_cueva_code.f95:170-184: reconstruction, then startconvar and stage 1
    CUDA_TRY(launch_recons_begin((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur, c->qin, c->T.Abt[0][0]));
    c->cur ^= 1;
  }
  for (int l = 1; l <= c->T.s; ++l) {
    StageArgs sa = stage_args(c, l, 0);
    if (l == c->T.s) sa.diag_cons = diag_cons;
    CUDA_TRY(launch_stage(c->P.rec_mp, c->P.flux_solver, c->P.precision, c->shape, c->stream, c->d_inst, 1, sa));
    c->qin ^= 1;
  }
  if (learned_tc(c->h_inst, c->d_mlp))   // con2prim of the learned method and the next stage 1
    CUDA_TRY(launch_c2p_step(c->stream, c->d_inst, 1, c->h_inst.block_count[LK_C2P], c->d_mlp, c->cur, c->qin,
                             c->T.Abt[0][0]));
  c->cur ^= 1;
  return CUEVA_OK;
}

void destroy_graphs(cueva_ctx* c) {
  for (auto& row : c->graph)
    for (auto& g : row)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  for (auto& row : c->graph_diag)
    for (auto& g : row)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

bool diag_step(const cueva_ctx* c, long long h) {
  return c->diag_on && (h == 1 || (c->diag.hglb > 0 && h % c->diag.hglb == 0));
}

void free_diag(cueva_ctx* c) {
  if (c->d_diag_cons) cudaFree(c->d_diag_cons);
  if (c->d_diag_part) cudaFree(c->d_diag_part);
  if (c->d_diag_rec) cudaFree(c->d_diag_rec);
  c->d_diag_cons = c->d_diag_part = nullptr;
  c->d_diag_rec = nullptr;
  c->diag_on = false;
}

}  // namespace

extern "C" {

const char* cueva_last_error(void) { return g_err.c_str(); }

int32_t cueva_ctx_create(const cueva_params* p, cueva_ctx** out) {
  if (!p || !out) return fail(CUEVA_ERR_ARG, "null argument");
  *out = nullptr;
  if (int32_t e = validate_params(p)) return e;
  cueva_ctx* c = new cueva_ctx();
  c->P = *p;
  if (!make_tableau(p->order, c->T)) { delete c; return fail(CUEVA_ERR_ARG, "unsupported IMEX order"); }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    delete c; cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, "no CUDA device available");
  }
  if (p->device < 0 || p->device >= ndev) { delete c; return fail(CUEVA_ERR_ARG, "device ordinal out of range"); }
  c->dev = p->device;
  if (cudaSetDevice(c->dev) != cudaSuccess) { delete c; return fail(CUEVA_ERR_CUDA, "cudaSetDevice failed"); }
  c->nkslot = kslots(c->T, c->kslot_of);
  const InstGeom G = inst_geom(p, c->nkslot);
  c->imax = G.imax; c->jmax = G.jmax; c->nx = G.nx; c->ny = G.ny; c->pitch = G.pitch; c->fstride = G.fstride;
  c->delx = G.delx; c->dely = G.dely; c->delz = G.delz; c->dt = G.dt;
  if (cudaMalloc(&c->slab, (size_t)G.nslab * sizeof(double)) != cudaSuccess) {
    delete c; cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, "cudaMalloc of the field slab failed");
  }
  cudaMemset(c->slab, 0, (size_t)G.nslab * sizeof(double));
  if (cudaMalloc(&c->d_status, 4) != cudaSuccess || cudaMalloc(&c->d_counters, 3 * 8) != cudaSuccess ||
      cudaMalloc(&c->d_inst, sizeof(InstDesc)) != cudaSuccess) {
    cueva_ctx_destroy(c); cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, "cudaMalloc of the context descriptors failed");
  }
  cudaMemset(c->d_status, 0, 4);
  cudaMemset(c->d_counters, 0, 24);
  InstDesc& I = c->h_inst;
  fill_desc(p, G, c->nkslot, c->slab, c->d_status, c->d_counters, I);
  // x tiles: 31 points (32 faces) x FACE_ROWS rows; y tiles: 32 columns x
  // FACE_ROWS face rows of j = -1..jmax
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev);
  I.block_count[LK_XUPD] = xupd_tiles(c->imax, c->jmax, FACE_ROWS);
  I.block_count[LK_YFACE] = yface_tiles(c->imax, c->jmax, FACE_ROWS);
  I.seg_rows = stage_seg_rows(c->imax, c->jmax, FACE_ROWS, 2 * nsm);
  I.block_count[LK_STAGE] = stage_tiles(c->imax, c->jmax, I.seg_rows);
  c->shape.rows = FACE_ROWS;
  for (int k : {LK_XUPD, LK_YFACE, LK_STAGE}) {
    I.block_begin[k] = 0;
    c->shape.grid[k] = c->shape.ntiles[k] = I.block_count[k];   // one tile per CTA
  }
  // the fused stage kernel where it exists (k_yface + k_xupd otherwise)
  c->shape.fused = stage_fused_available(p->rec_mp, p->flux_solver);
  if (prepare_stage(p->rec_mp, p->flux_solver, p->precision) != cudaSuccess ||
      cudaMemcpy(c->d_inst, &I, sizeof(InstDesc), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cueva_ctx_destroy(c); cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, "context set-up failed");
  }
  c->stream = c->own_stream;
  *out = c;
  return CUEVA_OK;
}

int32_t cueva_ctx_destroy(cueva_ctx* c) {
  if (!c) return CUEVA_OK;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  destroy_graphs(c);
  if (c->slab) cudaFree(c->slab);
  if (c->d_status) cudaFree(c->d_status);
  if (c->d_counters) cudaFree(c->d_counters);
  if (c->d_inst) cudaFree(c->d_inst);
  if (c->d_mlp) cudaFree(c->d_mlp);
  if (c->d_mlp_stats) cudaFree(c->d_mlp_stats);
  free_diag(c);
  if (c->xfer) {
    cudaStreamSynchronize(c->xfer);
    cudaStreamDestroy(c->xfer);
  }
  for (cudaEvent_t ev : c->ev_field) if (ev) cudaEventDestroy(ev);
  if (c->ev_ready) cudaEventDestroy(c->ev_ready);
  if (c->ev_xfer_done) cudaEventDestroy(c->ev_xfer_done);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return CUEVA_OK;
}

int32_t cueva_device_bytes(const cueva_ctx* c, uint64_t* bytes) {
  if (!c || !bytes) return fail(CUEVA_ERR_ARG, "null argument");
  const InstGeom G = inst_geom(&c->P, c->nkslot);
  *bytes = (uint64_t)G.nslab * sizeof(double);
  return CUEVA_OK;
}

int32_t cueva_set_stage_kernel(cueva_ctx* c, int32_t fused) {
  if (int32_t e = check_ctx(c)) return e;
  if (fused != 0 && fused != 1) return fail(CUEVA_ERR_ARG, "fused must be 0 (two kernels per stage) or 1 (one)");
  if (fused && !stage_fused_available(c->P.rec_mp, c->P.flux_solver))
    return fail(CUEVA_ERR_ARG, "no fused stage kernel for this reconstruction (MP5 and the MC slopes have one)");
  CUDA_TRY(cudaSetDevice(c->dev));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  destroy_graphs(c);
  c->shape.fused = fused != 0;
  return CUEVA_OK;
}

int32_t cueva_get_stage_kernel(const cueva_ctx* c, int32_t* fused) {
  if (!c || !fused) return fail(CUEVA_ERR_ARG, "null argument");
  *fused = c->shape.fused ? 1 : 0;
  return CUEVA_OK;
}

int32_t cueva_set_stream(cueva_ctx* c, void* s) {
  if (int32_t e = check_ctx(c, false)) return e;
  destroy_graphs(c);
  c->stream = s ? (cudaStream_t)s : c->own_stream;
  return join_downloads(c);   // the new stream also follows a pending readback
}

double cueva_dt(const cueva_ctx* c) { return c ? c->dt : 0.0; }
int32_t cueva_tableau_stages(const cueva_ctx* c) { return c ? c->T.s : 0; }

int32_t cueva_bind_field(cueva_ctx* c, int32_t field, double* base) {
  if (int32_t e = check_ctx(c)) return e;
  if (field < 0 || field >= CUEVA_NFIELDS) return fail(CUEVA_ERR_ARG, "field id out of range");
  c->bound[field] = base;
  return CUEVA_OK;
}

int32_t cueva_pin_host(void* ptr, uint64_t bytes) {
  CUDA_TRY(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
  return CUEVA_OK;
}
int32_t cueva_unpin_host(void* ptr) {
  CUDA_TRY(cudaHostUnregister(ptr));
  return CUEVA_OK;
}

}  // extern "C"

namespace {

const int kConsField[NAUX] = {CUEVA_D, CUEVA_TAU, CUEVA_SX, CUEVA_SY, CUEVA_SZ, CUEVA_W};

// The stream waits for a pending asynchronous readback of transfer slot k
// (0..13 prims, 14..19 conserved fields) before its next copy overwrites that
// field's host array or device buffer.
int32_t wait_field(cueva_ctx* c, int k) {
  if (!c->field_pending[k]) return CUEVA_OK;
  CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_field[k], 0));
  c->field_pending[k] = false;
  return CUEVA_OK;
}

}  // namespace

extern "C" {

int32_t cueva_upload(cueva_ctx* c, uint32_t groups) {
  if (int32_t e = check_ctx(c, false)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  if (groups & CUEVA_G_PRIMS) {
    for (int f = 0; f < NPRIM; ++f) {
      if (int32_t e = wait_field(c, f)) return e;
      if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
    }
  }
  if (groups & CUEVA_G_CONS) {
    for (int f = 0; f < NAUX; ++f) {
      if (int32_t e = wait_field(c, NPRIM + f)) return e;
      if (int32_t e = h2d(c, aux_f(c, c->cur, f), kConsField[f], 1)) return e;
    }
  }
  // the stage-1 preparation writes the conserved buffers: the whole readback
  // precedes it
  if (int32_t e = join_downloads(c)) return e;
  if (groups & CUEVA_G_PRIMS)
    if (int32_t e = run_begin_step(c)) return e;
  return CUEVA_OK;
}

int32_t cueva_download(cueva_ctx* c, uint32_t groups) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  if (groups & CUEVA_G_PRIMS)
    for (int f = 0; f < NPRIM; ++f)
      if (int32_t e = d2h(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  if (groups & CUEVA_G_CONS)
    for (int f = 0; f < NAUX; ++f)
      if (int32_t e = d2h(c, aux_f(c, c->cur, f), kConsField[f], 1)) return e;
  return read_status(c);
}

int32_t cueva_download_async(cueva_ctx* c, uint32_t groups) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int k = 0; k < NPRIM + NAUX; ++k) {
    int field = k < NPRIM ? CUEVA_RHO + k : kConsField[k - NPRIM];
    bool want = k < NPRIM ? (groups & CUEVA_G_PRIMS) : (groups & CUEVA_G_CONS);
    if (want && !c->bound[field]) return fail(CUEVA_ERR_UNBOUND, "field " + std::to_string(field) + " not bound");
  }
  if (!c->xfer) {
    // the transfer stream and its events come into use together or not at all
    cudaStream_t xs = nullptr;
    cudaEvent_t evs[NPRIM + NAUX + 2] = {};
    cudaError_t ce = cudaStreamCreateWithFlags(&xs, cudaStreamNonBlocking);
    for (cudaEvent_t& ev : evs)
      if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (ce != cudaSuccess) {
      for (cudaEvent_t ev : evs) if (ev) cudaEventDestroy(ev);
      if (xs) cudaStreamDestroy(xs);
      return fail(CUEVA_ERR_CUDA, std::string("transfer stream set-up: ") + cudaGetErrorString(ce));
    }
    c->xfer = xs;
    c->ev_ready = evs[NPRIM + NAUX];
    c->ev_xfer_done = evs[NPRIM + NAUX + 1];
    for (int k = 0; k < NPRIM + NAUX; ++k) c->ev_field[k] = evs[k];
  }
  CUDA_TRY(cudaEventRecord(c->ev_ready, c->stream));
  CUDA_TRY(cudaStreamWaitEvent(c->xfer, c->ev_ready, 0));
  for (int k = 0; k < NPRIM + NAUX; ++k) {
    bool prim = k < NPRIM;
    if (!(groups & (prim ? CUEVA_G_PRIMS : CUEVA_G_CONS))) continue;
    int field = prim ? CUEVA_RHO + k : kConsField[k - NPRIM];
    const double* src = prim ? prim_f(c, c->cur, k) : aux_f(c, c->cur, k - NPRIM);
    CUDA_TRY(cudaMemcpy2DAsync(host_interior(c, c->bound[field], 1), (size_t)(c->imax + 13) * 8, src,
                               (size_t)c->pitch * 8, (size_t)c->nx * 8, (size_t)c->ny, cudaMemcpyDeviceToHost,
                               c->xfer));
    CUDA_TRY(cudaEventRecord(c->ev_field[k], c->xfer));
    c->field_pending[k] = true;
  }
  CUDA_TRY(cudaEventRecord(c->ev_xfer_done, c->xfer));
  c->dl_pending = true;
  return CUEVA_OK;
}

int32_t cueva_step(cueva_ctx* c, int32_t nsteps) {
  if (int32_t e = check_ctx(c)) return e;
  if (nsteps < 0) return fail(CUEVA_ERR_ARG, "nsteps < 0");
  if (!c->primed) return fail(CUEVA_ERR_UNBOUND, "no state on the device: cueva_upload(CUEVA_G_PRIMS) first");
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int n = 0; n < nsteps; ++n) {
    // steps after which the writer reports (h == 1 or mod(h, hglb) == 0)
    // run a graph whose last stage also keeps varfin's D and tau
    const bool rec = diag_step(c, c->h + 1);
    cudaGraphExec_t& g = rec ? c->graph_diag[c->cur][c->qin] : c->graph[c->cur][c->qin];
    if (!g) {
      // capture one step starting from this (cur, qin) parity
      const int cur0 = c->cur, qin0 = c->qin;
      cudaGraph_t graph = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int32_t e = enqueue_step(c, rec ? c->d_diag_cons : nullptr);
      cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      if (e) { if (graph) cudaGraphDestroy(graph); return e; }
      if (ce != cudaSuccess) return fail(CUEVA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(CUEVA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
      c->cur = cur0; c->qin = qin0;
    }
    CUDA_TRY(cudaGraphLaunch(g, c->stream));
    for (int l = 0; l < c->T.s; ++l) c->qin ^= 1;
    if (!c->P.primitive_rec) c->cur ^= 1;   // with the reconstruction the step flips the buffers twice
    c->h += 1;
    c->t = c->t + c->dt;
    if (rec) {
      cueva_diag_record* slot = c->d_diag_rec + (c->diag_written % c->diag.capacity);
      CUDA_TRY(launch_diag(c->h_inst, c->cur, c->d_diag_cons, c->d_diag_cons + c->fstride, c->diag.b0,
                           c->d_diag_part, c->h, c->t, slot, c->stream));
      c->diag_written += 1;
    }
  }
  return CUEVA_OK;
}

int32_t cueva_profile_steps(cueva_ctx* c, int32_t nsteps, double ms_out[3], int32_t launches_out[3]) {
  if (int32_t e = check_ctx(c)) return e;
  if (nsteps < 0 || !ms_out || !launches_out) return fail(CUEVA_ERR_ARG, "bad profile arguments");
  if (!c->primed) return fail(CUEVA_ERR_UNBOUND, "no state on the device: cueva_upload(CUEVA_G_PRIMS) first");
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int k = 0; k < 3; ++k) { ms_out[k] = 0.0; launches_out[k] = 0; }
  cudaEvent_t ev[3] = {};
  for (auto& e : ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      for (auto& f : ev) if (f) cudaEventDestroy(f);
      return fail(CUEVA_ERR_CUDA, "cudaEventCreate failed");
    }
  int32_t rc = CUEVA_OK;
  for (int n = 0; n < nsteps && rc == CUEVA_OK; ++n) {
    if (c->P.primitive_rec) {   // timed with the other kernels in ms_out[2]
      cudaError_t ce = cudaEventRecord(ev[0], c->stream);
      if (ce == cudaSuccess)
        ce = launch_recons_begin((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur, c->qin, c->T.Abt[0][0]);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], c->stream);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
      if (ce != cudaSuccess) { rc = fail(CUEVA_ERR_CUDA, cudaGetErrorString(ce)); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      ms_out[2] += ms;
      launches_out[2] += 1;
      c->cur ^= 1;
    }
    for (int l = 1; l <= c->T.s && rc == CUEVA_OK; ++l) {
      const StageArgs sa = stage_args(c, l, 0);
      cudaError_t ce = launch_stage(c->P.rec_mp, c->P.flux_solver, c->P.precision, c->shape, c->stream, c->d_inst, 1,
                                    sa, ev);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[2]);
      if (ce != cudaSuccess) { rc = fail(CUEVA_ERR_CUDA, cudaGetErrorString(ce)); break; }
      for (int k = 0; k < 2; ++k) {
        if (k == 0 && c->shape.fused) continue;   // no separate y-face launch
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
        ms_out[k] += ms;
        launches_out[k] += 1;
      }
      c->qin ^= 1;
    }
    if (rc == CUEVA_OK && learned_tc(c->h_inst, c->d_mlp)) {
      cudaError_t ce = cudaEventRecord(ev[0], c->stream);
      if (ce == cudaSuccess)
        ce = launch_c2p_step(c->stream, c->d_inst, 1, c->h_inst.block_count[LK_C2P], c->d_mlp, c->cur, c->qin,
                             c->T.Abt[0][0]);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], c->stream);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
      if (ce != cudaSuccess) { rc = fail(CUEVA_ERR_CUDA, cudaGetErrorString(ce)); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[0], ev[1]);
      ms_out[2] += ms;
      launches_out[2] += 1;
    }
    c->cur ^= 1;
    c->h += 1;
    c->t = c->t + c->dt;
  }
  for (auto& e : ev) cudaEventDestroy(e);
  if (rc) return rc;
  return read_status(c);
}

int32_t cueva_sync(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  return read_status(c);
}

int32_t cueva_status(cueva_ctx* c, uint32_t* st) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  CUDA_TRY(cudaMemcpyAsync(st, c->d_status, 4, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CUEVA_OK;
}

int32_t cueva_clear_status(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  CUDA_TRY(cudaMemsetAsync(c->d_status, 0, 4, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return CUEVA_OK;
}

int32_t cueva_counters(cueva_ctx* c, int64_t out3[3]) {
  if (int32_t e = check_ctx(c)) return e;
  unsigned long long h[3];
  CUDA_TRY(cudaMemcpyAsync(h, c->d_counters, 24, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int k = 0; k < 3; ++k) out3[k] = (int64_t)h[k];
  return CUEVA_OK;
}

// ------------------------------------------------------------ run diagnostics
int32_t cueva_set_clock(cueva_ctx* c, int64_t h, double t) {
  if (int32_t e = check_ctx(c)) return e;
  if (h < 0) return fail(CUEVA_ERR_ARG, "step index h < 0");
  c->h = h;
  c->t = t;
  return CUEVA_OK;
}

int32_t cueva_get_clock(const cueva_ctx* c, int64_t* h, double* t) {
  if (!c) return fail(CUEVA_ERR_ARG, "null context");
  if (h) *h = c->h;
  if (t) *t = c->t;
  return CUEVA_OK;
}

int32_t cueva_diag_enable(cueva_ctx* c, const cueva_diag_config* cfg) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  destroy_graphs(c);   // the record graphs hold the buffers' addresses
  free_diag(c);
  if (!cfg) return CUEVA_OK;
  if (cfg->hglb < 1) return fail(CUEVA_ERR_ARG, "hglb must be >= 1");
  if (cfg->capacity < 1) return fail(CUEVA_ERR_ARG, "capacity must be >= 1");
  if (!(cfg->b0 != 0.0) || !(cfg->lr != 0.0) || !(cfg->delta_rec != 0.0))
    return fail(CUEVA_ERR_ARG, "b0, lr and delta_rec must be non-zero");
  const size_t part = (size_t)diag_blocks(c->imax, c->jmax) * diag_partials();
  if (cudaMalloc(&c->d_diag_cons, 2 * (size_t)c->fstride * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_diag_part, part * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_diag_rec, ((size_t)cfg->capacity + 1) * sizeof(cueva_diag_record)) != cudaSuccess) {
    cudaGetLastError();
    free_diag(c);
    return fail(CUEVA_ERR_CUDA, "cudaMalloc of the diagnostics buffers failed");
  }
  c->diag = *cfg;
  c->diag_on = true;
  c->diag_written = c->diag_read = 0;
  return CUEVA_OK;
}

// writer unit 67 (22_writer.f95:1014-1019), evaluated on the host
static void fill_delta_rec(const cueva_ctx* c, cueva_diag_record& r) {
  const int jmed = c->jmax / 2;
  const double posy = -(0.5 * c->diag.ly) + (double)(jmed + 1) * c->dely;
  const double rr = std::sqrt(1.0 - (posy * posy) / (c->diag.lr * c->diag.lr));
  r.v[CUEVA_DG_DELTA_REC] =
      (((c->diag.b0 * rr) * std::tanh(c->delx / c->diag.delta_rec)) * c->diag.delta_rec) / r.v[CUEVA_DG_BY_MED];
}

int32_t cueva_diag_read(cueva_ctx* c, cueva_diag_record* out, int32_t max_records, int32_t* n_out) {
  if (int32_t e = check_ctx(c)) return e;
  if (!n_out || max_records < 0 || (max_records > 0 && !out)) return fail(CUEVA_ERR_ARG, "bad read arguments");
  *n_out = 0;
  if (!c->diag_on) return fail(CUEVA_ERR_ARG, "diagnostics are not enabled (cueva_diag_enable)");
  CUDA_TRY(cudaSetDevice(c->dev));
  const long long cap = c->diag.capacity;
  if (c->diag_written - c->diag_read > cap) c->diag_read = c->diag_written - cap;   // overwritten ones
  const long long n = std::min<long long>(c->diag_written - c->diag_read, max_records);
  for (long long k = 0; k < n;) {
    const long long slot = (c->diag_read + k) % cap;
    const long long run = std::min<long long>(n - k, cap - slot);
    CUDA_TRY(cudaMemcpyAsync(out + k, c->d_diag_rec + slot, (size_t)run * sizeof(cueva_diag_record),
                             cudaMemcpyDeviceToHost, c->stream));
    k += run;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (long long k = 0; k < n; ++k) fill_delta_rec(c, out[k]);
  c->diag_read += n;
  *n_out = (int32_t)n;
  return read_status(c);
}

int32_t cueva_diag_now(cueva_ctx* c, cueva_diag_record* out) {
  if (int32_t e = check_ctx(c)) return e;
  if (!out) return fail(CUEVA_ERR_ARG, "null record");
  if (!c->diag_on) return fail(CUEVA_ERR_ARG, "diagnostics are not enabled (cueva_diag_enable)");
  if (!c->primed) return fail(CUEVA_ERR_UNBOUND, "no state on the device: cueva_upload(CUEVA_G_PRIMS) first");
  CUDA_TRY(cudaSetDevice(c->dev));
  cueva_diag_record* slot = c->d_diag_rec + c->diag.capacity;
  const double* a = c->h_inst.aux[c->cur];
  CUDA_TRY(launch_diag(c->h_inst, c->cur, a + (long long)A_D * c->fstride, a + (long long)A_TAU * c->fstride,
                       c->diag.b0, c->d_diag_part, c->h, c->t, slot, c->stream));
  CUDA_TRY(cudaMemcpyAsync(out, slot, sizeof(cueva_diag_record), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  fill_delta_rec(c, *out);
  return read_status(c);
}

// ------------------------------------------------------------ checkpoints
struct CkHeader {
  char magic[8];          // "CUEVACK1"
  uint32_t version;       // 1
  uint32_t header_bytes;  // sizeof(CkHeader)
  int32_t imax, jmax, nfields, pad;
  int64_t h;              // clock of the state
  double t;
  cueva_params params;    // configuration that wrote it (informational)
  uint64_t checksum;      // FNV-1a over the payload's 64-bit words
};

static uint64_t ck_hash(const double* p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t k = 0; k < n; ++k) {
    uint64_t w;
    std::memcpy(&w, p + k, 8);
    h = (h ^ w) * 1099511628211ull;
  }
  return h;
}

int32_t cueva_checkpoint_save(cueva_ctx* c, const char* path) {
  if (int32_t e = check_ctx(c)) return e;
  if (!path) return fail(CUEVA_ERR_ARG, "null path");
  if (!c->primed) return fail(CUEVA_ERR_UNBOUND, "no state on the device: cueva_upload(CUEVA_G_PRIMS) first");
  CUDA_TRY(cudaSetDevice(c->dev));
  const size_t npt = (size_t)c->nx * c->ny;
  std::vector<double> buf((size_t)NPRIM * npt);
  for (int f = 0; f < NPRIM; ++f)
    CUDA_TRY(cudaMemcpy2DAsync(buf.data() + f * npt, (size_t)c->nx * 8, prim_f(c, c->cur, f), (size_t)c->pitch * 8,
                               (size_t)c->nx * 8, (size_t)c->ny, cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (int32_t e = read_status(c)) return e;   // a non-physical state is not written
  CkHeader hd{};
  std::memcpy(hd.magic, "CUEVACK1", 8);
  hd.version = 1;
  hd.header_bytes = sizeof(CkHeader);
  hd.imax = c->imax; hd.jmax = c->jmax; hd.nfields = NPRIM;
  hd.h = c->h; hd.t = c->t;
  hd.params = c->P;
  hd.checksum = ck_hash(buf.data(), buf.size());
  const std::string tmp = std::string(path) + ".partial";
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return fail(CUEVA_ERR_ARG, "cannot create " + tmp);
  const bool ok = std::fwrite(&hd, sizeof hd, 1, f) == 1 && std::fwrite(buf.data(), 8, buf.size(), f) == buf.size();
  if (std::fclose(f) != 0 || !ok || std::rename(tmp.c_str(), path) != 0) {
    std::remove(tmp.c_str());
    return fail(CUEVA_ERR_ARG, std::string("cannot write ") + path);
  }
  return CUEVA_OK;
}

int32_t cueva_checkpoint_load(cueva_ctx* c, const char* path) {
  if (int32_t e = check_ctx(c)) return e;
  if (!path) return fail(CUEVA_ERR_ARG, "null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(CUEVA_ERR_ARG, std::string("cannot open ") + path);
  CkHeader hd{};
  if (std::fread(&hd, sizeof hd, 1, f) != 1 || std::memcmp(hd.magic, "CUEVACK1", 8) != 0 || hd.version != 1 ||
      hd.header_bytes != sizeof(CkHeader) || hd.nfields != NPRIM) {
    std::fclose(f);
    return fail(CUEVA_ERR_ARG, std::string(path) + " is not a version-1 cueva checkpoint");
  }
  if (hd.imax != c->imax || hd.jmax != c->jmax) {
    std::fclose(f);
    return fail(CUEVA_ERR_ARG, "checkpoint grid " + std::to_string(hd.imax) + " x " + std::to_string(hd.jmax) +
                                   " does not match the context's " + std::to_string(c->imax) + " x " +
                                   std::to_string(c->jmax));
  }
  const size_t npt = (size_t)c->nx * c->ny;
  std::vector<double> buf((size_t)NPRIM * npt);
  const size_t got = std::fread(buf.data(), 8, buf.size(), f);
  const bool extra = std::fgetc(f) != EOF;
  std::fclose(f);
  if (got != buf.size() || extra) return fail(CUEVA_ERR_ARG, std::string(path) + ": wrong payload size");
  if (ck_hash(buf.data(), buf.size()) != hd.checksum) return fail(CUEVA_ERR_ARG, std::string(path) + ": checksum mismatch");
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int k = 0; k < NPRIM; ++k)
    CUDA_TRY(cudaMemcpy2DAsync(prim_f(c, c->cur, k), (size_t)c->pitch * 8, buf.data() + k * npt, (size_t)c->nx * 8,
                               (size_t)c->nx * 8, (size_t)c->ny, cudaMemcpyHostToDevice, c->stream));
  if (int32_t e = run_begin_step(c)) return e;
  CUDA_TRY(cudaStreamSynchronize(c->stream));   // buf is released on return
  c->h = hd.h;
  c->t = hd.t;
  return CUEVA_OK;
}

// ------------------------------------------------------------ routine mirrors
int32_t cueva_startconvar(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int f = 0; f < NPRIM; ++f)
    if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  CUDA_TRY(launch_startconvar((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur));
  c->primed = false;
  const int map[NAUX] = {CUEVA_D, CUEVA_TAU, CUEVA_SX, CUEVA_SY, CUEVA_SZ, CUEVA_W};
  for (int f = 0; f < NAUX; ++f)
    if (c->bound[map[f]])
      if (int32_t e = d2h(c, aux_f(c, c->cur, f), map[f], 1)) return e;
  return read_status(c);
}

int32_t cueva_electricvarint(cueva_ctx* c, int32_t l) {
  if (int32_t e = check_ctx(c)) return e;
  if (l < 1 || l > c->T.s) return fail(CUEVA_ERR_ARG, "stage index out of range");
  CUDA_TRY(cudaSetDevice(c->dev));
  const int q = c->qin;
  const int in[7] = {CUEVA_EXAST, CUEVA_EYAST, CUEVA_EZAST, CUEVA_BXINT, CUEVA_BYINT, CUEVA_BZINT, CUEVA_QINT};
  const int slot[7] = {Q_EX, Q_EY, Q_EZ, Q_BX, Q_BY, Q_BZ, Q_Q};
  for (int k = 0; k < 7; ++k)
    if (int32_t e = h2d(c, stage_f(c, q, slot[k]), in[k], l)) return e;
  for (int f : {P_VX, P_VY, P_VZ})
    if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  if (int32_t e = h2d(c, aux_f(c, c->cur, A_W), CUEVA_W, 1)) return e;
  CUDA_TRY(launch_electricvarint((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur, q, c->T.Abt[l - 1][l - 1]));
  c->primed = false;
  const int out[6] = {CUEVA_EXINT, CUEVA_EYINT, CUEVA_EZINT, CUEVA_JXINT, CUEVA_JYINT, CUEVA_JZINT};
  const int oslot[6] = {Q_EX, Q_EY, Q_EZ, Q_JX, Q_JY, Q_JZ};
  for (int k = 0; k < 6; ++k)
    if (c->bound[out[k]] || k < 3)
      if (int32_t e = d2h(c, stage_f(c, q, oslot[k]), out[k], l)) return e;
  return read_status(c);
}

int32_t cueva_flux_rhs(cueva_ctx* c, int32_t l) {
  if (int32_t e = check_ctx(c)) return e;
  if (l < 1 || l > c->T.s) return fail(CUEVA_ERR_ARG, "stage index out of range");
  CUDA_TRY(cudaSetDevice(c->dev));
  const int q = c->qin;
  const int in[NSTAGE] = {CUEVA_PSIINT, CUEVA_PHIINT, CUEVA_EXINT, CUEVA_EYINT, CUEVA_EZINT, CUEVA_BXINT,
                          CUEVA_BYINT, CUEVA_BZINT, CUEVA_QINT, CUEVA_DDINT, CUEVA_TAUINT, CUEVA_SXINT,
                          CUEVA_SYINT, CUEVA_SZINT, CUEVA_JXINT, CUEVA_JYINT, CUEVA_JZINT};
  for (int k = 0; k < NSTAGE; ++k)
    if (int32_t e = h2d(c, stage_f(c, q, k), in[k], l)) return e;
  for (int f : {P_VX, P_VY, P_VZ, P_P, P_RHO})
    if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  if (int32_t e = h2d(c, aux_f(c, c->cur, A_W), CUEVA_W, 1)) return e;
  const StageArgs sa = stage_args(c, l, 1);
  CUDA_TRY(launch_stage(c->P.rec_mp, c->P.flux_solver, c->P.precision, c->shape, c->stream, c->d_inst, 1, sa));
  c->primed = false;
  const int out[NRHS] = {CUEVA_PSIFLUX, CUEVA_PHIFLUX, CUEVA_EXASTFLUX, CUEVA_EYASTFLUX, CUEVA_EZASTFLUX,
                         CUEVA_BXFLUX, CUEVA_BYFLUX, CUEVA_BZFLUX, CUEVA_QFLUX, CUEVA_DFLUX, CUEVA_TAUFLUX,
                         CUEVA_SXFLUX, CUEVA_SYFLUX, CUEVA_SZFLUX, CUEVA_EXASTSOUR, CUEVA_EYASTSOUR,
                         CUEVA_EZASTSOUR};
  for (int k = 0; k < NRHS; ++k)
    if (int32_t e = d2h(c, c->h_inst.rhs_out + (long long)k * c->fstride, out[k], l)) return e;
  return read_status(c);
}

// ---------------------------------------- routine mirrors of the flux step
namespace {
// bound array of field f, stage l, element (i, j) (Fortran indices)
double* host_at(cueva_ctx* c, int field, int l, int i, int j) {
  return c->bound[field] + (size_t)(l - 1) * host_field_elems(c) + (size_t)(i + 6) +
         (size_t)(j + 6) * (size_t)(c->imax + 13);
}
// interface flux fields by role (order of enum Role), x and y faces
const int kFaceX[NFACE] = {CUEVA_EXLAXPSI, CUEVA_BXLAXPHI, CUEVA_PHILAXBX, CUEVA_EZLAXBY, CUEVA_EYLAXBZ,
                           CUEVA_PSILAXEX, CUEVA_BZLAXEY, CUEVA_BYLAXEZ, CUEVA_JXLAX, CUEVA_FDXLAX,
                           CUEVA_FTAUXLAX, CUEVA_FSXXLAX, CUEVA_FSXYLAX, CUEVA_FSXZLAX};
const int kFaceY[NFACE] = {CUEVA_EYLAXPSI, CUEVA_BYLAXPHI, CUEVA_PHILAXBY, CUEVA_EXLAXBZ, CUEVA_EZLAXBX,
                           CUEVA_PSILAXEY, CUEVA_BXLAXEZ, CUEVA_BZLAXEX, CUEVA_JYLAX, CUEVA_FDYLAX,
                           CUEVA_FTAUYLAX, CUEVA_FSYYLAX, CUEVA_FSYZLAX, CUEVA_FSYXLAX};

int32_t check_faces_bound(cueva_ctx* c) {
  for (int r = 0; r < NFACE; ++r)
    for (int f : {kFaceX[r], kFaceY[r]})
      if (!c->bound[f]) return fail(CUEVA_ERR_UNBOUND, "field " + std::to_string(f) + " not bound");
  return CUEVA_OK;
}

// the stage inputs shared by cueva_flux_rhs, cueva_flux_flow, cueva_fluxandsource
int32_t upload_stage_inputs(cueva_ctx* c, int l) {
  const int q = c->qin;
  const int in[NSTAGE] = {CUEVA_PSIINT, CUEVA_PHIINT, CUEVA_EXINT, CUEVA_EYINT, CUEVA_EZINT, CUEVA_BXINT,
                          CUEVA_BYINT, CUEVA_BZINT, CUEVA_QINT, CUEVA_DDINT, CUEVA_TAUINT, CUEVA_SXINT,
                          CUEVA_SYINT, CUEVA_SZINT, CUEVA_JXINT, CUEVA_JYINT, CUEVA_JZINT};
  for (int k = 0; k < NSTAGE; ++k)
    if (int32_t e = h2d(c, stage_f(c, q, k), in[k], l)) return e;
  for (int f : {P_VX, P_VY, P_VZ, P_P, P_RHO})
    if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  return h2d(c, aux_f(c, c->cur, A_W), CUEVA_W, 1);
}
int32_t download_rhs(cueva_ctx* c, int l) {
  const int out[NRHS] = {CUEVA_PSIFLUX, CUEVA_PHIFLUX, CUEVA_EXASTFLUX, CUEVA_EYASTFLUX, CUEVA_EZASTFLUX,
                         CUEVA_BXFLUX, CUEVA_BYFLUX, CUEVA_BZFLUX, CUEVA_QFLUX, CUEVA_DFLUX, CUEVA_TAUFLUX,
                         CUEVA_SXFLUX, CUEVA_SYFLUX, CUEVA_SZFLUX, CUEVA_EXASTSOUR, CUEVA_EYASTSOUR,
                         CUEVA_EZASTSOUR};
  for (int k = 0; k < NRHS; ++k)
    if (int32_t e = d2h(c, c->h_inst.rhs_out + (long long)k * c->fstride, out[k], l)) return e;
  return CUEVA_OK;
}
}  // namespace

int32_t cueva_flux_flow(cueva_ctx* c, int32_t l) {
  if (int32_t e = check_ctx(c)) return e;
  if (l < 1 || l > c->T.s) return fail(CUEVA_ERR_ARG, "stage index out of range");
  if (int32_t e = check_faces_bound(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  if (int32_t e = upload_stage_inputs(c, l)) return e;
  const StageArgs sa = stage_args(c, l, 2);
  CUDA_TRY(launch_stage(c->P.rec_mp, c->P.flux_solver, c->P.precision, c->shape, c->stream, c->d_inst, 1, sa));
  c->primed = false;
  const InstDesc& I = c->h_inst;
  const size_t hp = (size_t)(c->imax + 13) * 8;
  // x faces i = -1..imax of rows 0..jmax: fx[j * fpitch + (i + 1)]
  for (int r = 0; r < NFACE; ++r)
    CUDA_TRY(cudaMemcpy2DAsync(host_at(c, kFaceX[r], l, -1, 0), hp, I.fx + r * I.ffs, (size_t)I.fpitch * 8,
                               (size_t)(c->imax + 2) * 8, (size_t)(c->jmax + 1), cudaMemcpyDeviceToHost,
                               c->stream));
  // y faces j = -1..jmax of columns 0..imax: fy[(j + 1) * fpitch + i], FP32 in the mixed kernels
  if (c->P.precision == 0) {
    for (int r = 0; r < NFACE; ++r)
      CUDA_TRY(cudaMemcpy2DAsync(host_at(c, kFaceY[r], l, 0, -1), hp, I.fy + r * I.ffs, (size_t)I.fpitch * 8,
                                 (size_t)(c->imax + 1) * 8, (size_t)(c->jmax + 2), cudaMemcpyDeviceToHost,
                                 c->stream));
  } else {
    // the mixed kernels' slabs, FP32 or FP64 by role (flux_slot)
    std::vector<double> tmp((size_t)NFACE * (size_t)I.ffs);
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), I.fy, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const float* tmpf = reinterpret_cast<const float*>(tmp.data());
    for (int r = 0; r < NFACE; ++r) {
      const FluxSlot sl = flux_slot(true, c->P.flux_solver, r, I.ffs);
      for (int j = -1; j <= c->jmax; ++j) {
        double* dst = host_at(c, kFaceY[r], l, 0, j);
        const size_t o = (size_t)sl.off + (size_t)(j + 1) * I.fpitch;
        for (int i = 0; i <= c->imax; ++i) dst[i] = sl.f64 ? tmp[o + i] : double(tmpf[o + i]);
      }
    }
  }
  return read_status(c);
}

int32_t cueva_fluxandsource(cueva_ctx* c, int32_t l) {
  if (int32_t e = check_ctx(c)) return e;
  if (l < 1 || l > c->T.s) return fail(CUEVA_ERR_ARG, "stage index out of range");
  if (int32_t e = check_faces_bound(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  if (int32_t e = upload_stage_inputs(c, l)) return e;
  const InstDesc& I = c->h_inst;
  const size_t hp = (size_t)(c->imax + 13) * 8;
  for (int r = 0; r < NFACE; ++r) {
    CUDA_TRY(cudaMemcpy2DAsync(I.fx + r * I.ffs, (size_t)I.fpitch * 8, host_at(c, kFaceX[r], l, -1, 0), hp,
                               (size_t)(c->imax + 2) * 8, (size_t)(c->jmax + 1), cudaMemcpyHostToDevice,
                               c->stream));
    CUDA_TRY(cudaMemcpy2DAsync(I.fy + r * I.ffs, (size_t)I.fpitch * 8, host_at(c, kFaceY[r], l, 0, -1), hp,
                               (size_t)(c->imax + 1) * 8, (size_t)(c->jmax + 2), cudaMemcpyHostToDevice,
                               c->stream));
  }
  const StageArgs sa = stage_args(c, l, 1);
  CUDA_TRY(launch_fluxandsource((long long)c->nx * c->ny, c->stream, c->d_inst, 1, sa));
  c->primed = false;
  if (int32_t e = download_rhs(c, l)) return e;
  return read_status(c);
}

namespace {
// varfin / electricfield: the bound final sums and fields of the Q slots in
// mask go up, U += Delt * finsum on the device, the fields come back
int32_t add_finsum(cueva_ctx* c, uint32_t mask) {
  CUDA_TRY(cudaSetDevice(c->dev));
  struct Slot { int q, fin, field; double* dev; };
  const InstDesc& I = c->h_inst;
  const long long fs = c->fstride;
  const Slot slots[NCONS] = {
      {Q_PSI, CUEVA_PSIFINSUM, CUEVA_PSI, prim_f(c, c->cur, P_PSI)},
      {Q_PHI, CUEVA_PHIFINSUM, CUEVA_PHI, prim_f(c, c->cur, P_PHI)},
      {Q_EX, CUEVA_EXFINSUM, CUEVA_EX, prim_f(c, c->cur, P_EX)},
      {Q_EY, CUEVA_EYFINSUM, CUEVA_EY, prim_f(c, c->cur, P_EY)},
      {Q_EZ, CUEVA_EZFINSUM, CUEVA_EZ, prim_f(c, c->cur, P_EZ)},
      {Q_BX, CUEVA_BXFINSUM, CUEVA_BX, prim_f(c, c->cur, P_BX)},
      {Q_BY, CUEVA_BYFINSUM, CUEVA_BY, prim_f(c, c->cur, P_BY)},
      {Q_BZ, CUEVA_BZFINSUM, CUEVA_BZ, prim_f(c, c->cur, P_BZ)},
      {Q_Q, CUEVA_QFINSUM, CUEVA_Q, prim_f(c, c->cur, P_Q)},
      {Q_D, CUEVA_DFINSUM, CUEVA_D, aux_f(c, c->cur, A_D)},
      {Q_TAU, CUEVA_TAUFINSUM, CUEVA_TAU, aux_f(c, c->cur, A_TAU)},
      {Q_SX, CUEVA_SXFINSUM, CUEVA_SX, aux_f(c, c->cur, A_SX)},
      {Q_SY, CUEVA_SYFINSUM, CUEVA_SY, aux_f(c, c->cur, A_SY)},
      {Q_SZ, CUEVA_SZFINSUM, CUEVA_SZ, aux_f(c, c->cur, A_SZ)}};
  for (const Slot& s : slots) {
    if (!(mask >> s.q & 1u)) continue;
    if (int32_t e = h2d(c, I.finsum + s.q * fs, s.fin, 1)) return e;
    if (int32_t e = h2d(c, s.dev, s.field, 1)) return e;
  }
  CUDA_TRY(launch_add_finsum((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur, mask));
  c->primed = false;
  for (const Slot& s : slots)
    if (mask >> s.q & 1u)
      if (int32_t e = d2h(c, s.dev, s.field, 1)) return e;
  return read_status(c);
}
}  // namespace

int32_t cueva_varfin(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  uint32_t mask = 0;
  for (int q : {Q_PSI, Q_PHI, Q_BX, Q_BY, Q_BZ, Q_Q, Q_D, Q_TAU, Q_SX, Q_SY, Q_SZ}) mask |= 1u << q;
  return add_finsum(c, mask);
}

int32_t cueva_electricfield(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  return add_finsum(c, (1u << Q_EX) | (1u << Q_EY) | (1u << Q_EZ));
}

int32_t cueva_con2prim(cueva_ctx* c) {
  if (int32_t e = check_ctx(c)) return e;
  CUDA_TRY(cudaSetDevice(c->dev));
  for (int f = 0; f < NPRIM; ++f)
    if (int32_t e = h2d(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  const int map[5] = {CUEVA_D, CUEVA_TAU, CUEVA_SX, CUEVA_SY, CUEVA_SZ};
  for (int f = 0; f < 5; ++f)
    if (int32_t e = h2d(c, aux_f(c, c->cur, f), map[f], 1)) return e;
  CUDA_TRY(launch_con2prim((long long)c->nx * c->ny, c->stream, c->d_inst, 1, c->cur));
  c->primed = false;
  for (int f : {P_RHO, P_P, P_VX, P_VY, P_VZ})
    if (int32_t e = d2h(c, prim_f(c, c->cur, f), CUEVA_RHO + f, 1)) return e;
  return read_status(c);
}

// ------------------------------------------------------- learned c2p seed
int32_t cueva_attach_mlp(cueva_ctx* c, const cueva_mlp* mlp) {
  if (int32_t e = check_ctx(c)) return e;
  if (!mlp) return fail(CUEVA_ERR_ARG, "null network");
  if (mlp_device_of(mlp) != c->dev) return fail(CUEVA_ERR_ARG, "network and context live on different devices");
  CUDA_TRY(cudaSetDevice(c->dev));
  MLPDevice h;
  if (int32_t e = mlp_device_image(mlp, &h)) return e;
  if (!c->d_mlp) {
    CUDA_TRY(cudaMalloc(&c->d_mlp, sizeof(MLPDevice)));
    CUDA_TRY(cudaMalloc(&c->d_mlp_stats, 3 * sizeof(unsigned long long)));
  }
  h.stats = c->d_mlp_stats;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(c->d_mlp, &h, sizeof(MLPDevice), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(c->d_mlp_stats, 0, 3 * sizeof(unsigned long long)));
  c->h_inst.mlp = c->d_mlp;
  c->h_inst.c2p_tc = 1;
  destroy_graphs(c);   // the step gains the con2prim launch
  CUDA_TRY(cudaMemcpy(c->d_inst, &c->h_inst, sizeof(InstDesc), cudaMemcpyHostToDevice));
  return CUEVA_OK;
}

int32_t cueva_set_learned_kernel(cueva_ctx* c, int32_t mode) {
  if (int32_t e = check_ctx(c)) return e;
  if (mode != 0 && mode != 1) return fail(CUEVA_ERR_ARG, "mode must be 0 (in the last stage) or 1 (tensor-core kernel)");
  CUDA_TRY(cudaSetDevice(c->dev));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->h_inst.c2p_tc = mode;
  destroy_graphs(c);
  CUDA_TRY(cudaMemcpy(c->d_inst, &c->h_inst, sizeof(InstDesc), cudaMemcpyHostToDevice));
  return CUEVA_OK;
}

int32_t cueva_learned_stats(cueva_ctx* c, int64_t out3[3]) {
  if (int32_t e = check_ctx(c)) return e;
  if (!out3) return fail(CUEVA_ERR_ARG, "null argument");
  unsigned long long h[3] = {0, 0, 0};
  if (c->d_mlp_stats) {
    CUDA_TRY(cudaMemcpyAsync(h, c->d_mlp_stats, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  for (int k = 0; k < 3; ++k) out3[k] = (int64_t)h[k];
  return CUEVA_OK;
}

// --------------------------------------------------------------- KH input
int32_t cueva_kh_init(cueva_ctx* c, double v0, double a, double amp, double width, double kpert, double phase,
                      double bshear, double rho0, double p0) {
  if (int32_t e = check_ctx(c)) return e;
  for (int f = 0; f < NPRIM; ++f)
    if (!c->bound[CUEVA_RHO + f]) return fail(CUEVA_ERR_UNBOUND, "kh_init needs all 14 prim fields bound");
  const KHParams kh{v0, a, amp, width, kpert, phase, bshear, rho0, p0};
  for (int j = 0; j <= c->jmax; ++j)
    for (int i = 0; i <= c->imax; ++i) {
      const size_t k = (size_t)(i + 6) + (size_t)(j + 6) * (c->imax + 13);
      double pv[NPRIM];
      kh_point(kh, -0.5 * c->P.lx + i * c->delx, -0.5 * c->P.ly + j * c->dely, pv);
      for (int f = 0; f < NPRIM; ++f) c->bound[CUEVA_RHO + f][k] = pv[f];
    }
  return CUEVA_OK;
}

// ------------------------------------------- stage rhs without allocation
// Scratch for cueva_flux_rhs_noalloc: a 256-byte header (status word and
// fix-up counters, zeroed per call), the kernels' instance descriptor, then
// the 14 y-flux fields.  Static device memory: nothing is allocated at run
// time.
namespace {
constexpr size_t kNoallocBytes = size_t(32) << 20;
constexpr size_t kNoallocHeader = 256;
constexpr size_t kNoallocDesc = (sizeof(InstDesc) + 255) / 256 * 256;
constexpr int kMaxDevices = 64;
void* g_noalloc_base[kMaxDevices] = {};
// the once-per-device set-up (and every read of g_noalloc_base) runs under
// this lock, so host threads making their first call together set up once
std::mutex g_noalloc_mu;
}  // namespace
static __device__ __align__(256) double g_noalloc_scratch[kNoallocBytes / sizeof(double)];

int32_t cueva_flux_rhs_noalloc(const cueva_params* p, const double* prim, const double* W, const double* stage,
                               double* rhs, int32_t pitch, int64_t fstride, void* stream, uint32_t* status_bits) {
  if (!p || !prim || !W || !stage || !rhs) return fail(CUEVA_ERR_ARG, "null argument");
  if (p->imax < 6 || p->jmax < 6) return fail(CUEVA_ERR_ARG, "imax and jmax must be >= 6 (6 ghost cells)");
  if (p->flux_solver != 5 && p->flux_solver != 6 && p->flux_solver != 7)
    return fail(CUEVA_ERR_ARG, "flux_solver must be 5 (HLL+MPX), 6 (HLLE+MPX) or 7 (HLLC+MPX)");
  if (p->rec_mp < 0 || p->rec_mp > 2) return fail(CUEVA_ERR_ARG, "rec_mp must be 0, 1 or 2");
  if ((p->bc_x != 0 && p->bc_x != 1) || (p->bc_y != 0 && p->bc_y != 1))
    return fail(CUEVA_ERR_ARG, "bc_x, bc_y must be 0 (copy) or 1 (periodic)");
  if (p->precision != 0 && p->precision != 1) return fail(CUEVA_ERR_ARG, "precision must be 0 or 1");
  const int nx = p->imax + 1, ny = p->jmax + 1;
  if (pitch < nx || fstride < (int64_t)pitch * ny) return fail(CUEVA_ERR_ARG, "pitch < imax+1 or fstride < pitch*(jmax+1)");
  const int fpitch = (nx + 1 + 31) / 32 * 32;
  const long long ffs = (long long)fpitch * (ny + 1);
  const size_t need = kNoallocHeader + kNoallocDesc + (size_t)NFACE * (size_t)ffs * sizeof(double);
  if (need > kNoallocBytes)
    return fail(CUEVA_ERR_ARG, "grid too large for the no-alloc scratch: needs " + std::to_string(need) +
                                   " bytes, the static block holds " + std::to_string(kNoallocBytes));
  if (p->device < 0 || p->device >= kMaxDevices) return fail(CUEVA_ERR_ARG, "device ordinal out of range");
  CUDA_TRY(cudaSetDevice(p->device));
  cudaStream_t st = (cudaStream_t)stream;
  // the descriptor goes up from this call's stack and the status read waits
  // for the stream: neither may be recorded into a graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(st, &cap));
  if (cap != cudaStreamCaptureStatusNone)
    return fail(CUEVA_ERR_ARG, "cueva_flux_rhs_noalloc cannot run on a stream that is being captured");
  char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[p->device]) {
      // once per device, with that device current
      void* b = nullptr;
      CUDA_TRY(cudaGetSymbolAddress(&b, g_noalloc_scratch));
      for (int rm = 0; rm < 3; ++rm)
        for (int sv : {5, 6, 7})
          for (int pr = 0; pr < 2; ++pr) CUDA_TRY(prepare_stage(rm, sv, pr));
      g_noalloc_base[p->device] = b;
    }
    base = (char*)g_noalloc_base[p->device];
  }
  InstDesc I{};
  I.status = (uint32_t*)base;
  I.counters = (unsigned long long*)(base + 8);
  // the kernels read prim[cur], aux[cur] + A_W * fstride and stage[qin] in
  // the rhs-only mode; aux is placed so that its W slot is the caller's W
  I.prim[0] = I.prim[1] = const_cast<double*>(prim);
  I.aux[0] = I.aux[1] = (double*)((uintptr_t)W - (uintptr_t)A_W * (uintptr_t)fstride * sizeof(double));
  I.stage[0] = I.stage[1] = const_cast<double*>(stage);
  I.rhs_out = rhs;
  I.fx = nullptr;
  I.fy = (double*)(base + kNoallocHeader + kNoallocDesc);
  I.fpitch = fpitch;
  I.ffs = ffs;
  I.imax = p->imax; I.jmax = p->jmax; I.pitch = pitch; I.fstride = fstride;
  I.bc_x = p->bc_x; I.bc_y = p->bc_y;
  I.delx = p->lx / (double)p->imax;
  I.dely = p->ly / (double)p->jmax;
  I.sigma = p->sigma; I.gamma = p->gamma;
  {
    const double mn = (I.dely < I.delx) ? I.dely : I.delx;   // parameters.f95:329-334
    const double cp = std::sqrt(mn / 1.0);
    I.kappa_psi = 1.0 / (cp * cp);
    I.kappa_phi = 1.0 / (cp * cp);
    auto inv_pow2 = [](double d) {
      int e = 0;
      return (std::frexp(d, &e) == 0.5 && std::isnormal(1.0 / d)) ? 1.0 / d : 0.0;
    };
    I.inv_delx_pow2 = inv_pow2(I.delx);
    I.inv_dely_pow2 = inv_pow2(I.dely);
  }
  I.c2p = 1;
  I.block_begin[LK_XUPD] = I.block_begin[LK_YFACE] = I.block_begin[LK_STAGE] = 0;
  I.block_count[LK_XUPD] = xupd_tiles(p->imax, p->jmax, FACE_ROWS);
  I.block_count[LK_YFACE] = yface_tiles(p->imax, p->jmax, FACE_ROWS);
  I.block_count[LK_STAGE] = 0;   // the right-hand-side mode runs k_yface + k_xupd
  I.seg_rows = FACE_ROWS;
  StageShape sh;
  sh.rows = FACE_ROWS;
  for (int k = 0; k < 2; ++k) sh.grid[k] = sh.ntiles[k] = I.block_count[k];
  InstDesc* d_inst = (InstDesc*)(base + kNoallocHeader);
  CUDA_TRY(cudaMemsetAsync(base, 0, kNoallocHeader, st));
  CUDA_TRY(cudaMemcpyAsync(d_inst, &I, sizeof(InstDesc), cudaMemcpyHostToDevice, st));
  StageArgs sa{};
  sa.l = 1; sa.s = 1; sa.cur = 0; sa.qin = 0; sa.mode = 1;
  for (int m = 0; m < 8; ++m) sa.kslot[m] = -1;
  sa.store_k_slot = -1;
  sa.store_k_src = 0; sa.fin_load = 0; sa.fin_store = 0;
  CUDA_TRY(launch_stage(p->rec_mp, p->flux_solver, p->precision, sh, st, d_inst, 1, sa));
  if (status_bits) {
    uint32_t h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, base, 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *status_bits = h;
    if (h) {
      char buf[64];
      snprintf(buf, sizeof buf, "kernel status 0x%x", h);
      return fail(CUEVA_ERR_PHYSICS, buf);
    }
  }
  return CUEVA_OK;
}

}  // extern "C"

// =====================================================================
// Ensembles: many independent grids advanced by the same launches.  Every
// instance has its own slab and descriptor; the stage kernels map a tile
// index to (instance, tile) through the descriptors' tile ranges, so one
// y-face launch and one x-face + update launch per RK stage serve all
// instances, and one CUDA graph holds a whole ensemble step.
// =====================================================================
struct cueva_ens {
  int dev = 0;
  int n = 0;
  cueva_params P0{};                    // shared scheme: order, solver, rec_mp, precision, intsum_reset
  Tableau T;
  int nkslot = 0;
  int kslot_of[8];
  std::vector<cueva_params> P;
  std::vector<InstGeom> G;
  std::vector<InstDesc> I;
  std::vector<double*> slab;
  uint32_t* d_status = nullptr;          // one status word per instance
  unsigned long long* d_counters = nullptr;
  InstDesc* d_inst = nullptr;
  cudaStream_t stream = nullptr, own_stream = nullptr;
  StageShape shape;
  int ctas_per_sm = 0;                   // 0: one tile per CTA
  int cur = 0, qin = 0;
  bool primed = false;
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  MLPDevice* d_mlp = nullptr;
  unsigned long long* d_mlp_stats = nullptr;
  long long max_points = 0;
  int num_sms = 148;
  int c2p_ntiles = 0;     // tiles of the learned con2prim launch over all instances
};

namespace {

void ens_destroy_graphs(cueva_ens* e) {
  for (auto& row : e->graph)
    for (auto& g : row)
      if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

// tile ranges for a tile height and the launch grid for a CTA count per SM
int32_t ens_apply_shape(cueva_ens* e, int rows, int ctas_per_sm) {
  int begin[4] = {0, 0, 0, 0};
  for (int k = 0; k < e->n; ++k) {
    InstDesc& I = e->I[k];
    I.block_count[LK_XUPD] = xupd_tiles(I.imax, I.jmax, rows);
    I.block_count[LK_YFACE] = yface_tiles(I.imax, I.jmax, rows);
    I.block_count[LK_C2P] = c2p_tiles(I.imax, I.jmax);
    I.seg_rows = stage_seg_rows(I.imax, I.jmax, FACE_ROWS, 2 * e->num_sms);
    I.block_count[LK_STAGE] = stage_tiles(I.imax, I.jmax, I.seg_rows);
    for (int t = 0; t < 4; ++t) { I.block_begin[t] = begin[t]; begin[t] += I.block_count[t]; }
  }
  e->c2p_ntiles = begin[LK_C2P];
  e->shape.rows = rows;
  // the fused stage kernel has the tile height FACE_ROWS; other heights run k_yface + k_xupd
  e->shape.fused = rows == FACE_ROWS && stage_fused_available(e->P0.rec_mp, e->P0.flux_solver);
  for (int t : {LK_XUPD, LK_YFACE, LK_STAGE}) {
    e->shape.ntiles[t] = begin[t];
    const long long persistent = (long long)ctas_per_sm * e->num_sms;
    e->shape.grid[t] = (ctas_per_sm > 0 && persistent < begin[t]) ? (int)persistent : begin[t];
  }
  e->ctas_per_sm = ctas_per_sm;
  ens_destroy_graphs(e);
  CUDA_TRY(cudaMemcpyAsync(e->d_inst, e->I.data(), sizeof(InstDesc) * e->n, cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return CUEVA_OK;
}

int32_t ens_begin(cueva_ens* e) {
  CUDA_TRY(launch_begin_step(e->max_points, e->stream, e->d_inst, e->n, e->cur, e->qin, e->T.Abt[0][0]));
  e->primed = true;
  return CUEVA_OK;
}

int32_t ens_enqueue_step(cueva_ens* e) {
  if (e->P0.primitive_rec) {
    CUDA_TRY(launch_recons_begin(e->max_points, e->stream, e->d_inst, e->n, e->cur, e->qin, e->T.Abt[0][0]));
    e->cur ^= 1;
  }
  for (int l = 1; l <= e->T.s; ++l) {
    const StageArgs sa = stage_args_of(e->T, e->kslot_of, e->P0.intsum_reset, e->cur, e->qin, l, 0);
    CUDA_TRY(launch_stage(e->P0.rec_mp, e->P0.flux_solver, e->P0.precision, e->shape, e->stream, e->d_inst, e->n, sa));
    e->qin ^= 1;
  }
  bool any = false;
  for (const auto& I : e->I) any = any || learned_tc(I, e->d_mlp);
  if (any)   // one con2prim launch over the tiles of every instance with the learned method
    CUDA_TRY(launch_c2p_step(e->stream, e->d_inst, e->n, e->c2p_ntiles, e->d_mlp, e->cur, e->qin, e->T.Abt[0][0]));
  e->cur ^= 1;
  return CUEVA_OK;
}

int32_t ens_check(cueva_ens* e, int k) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  if (k < 0 || k >= e->n) return fail(CUEVA_ERR_ARG, "instance index out of range");
  return CUEVA_OK;
}

}  // namespace

extern "C" {

int32_t cueva_ens_destroy(cueva_ens* e) {
  if (!e) return CUEVA_OK;
  cudaSetDevice(e->dev);
  if (e->stream) cudaStreamSynchronize(e->stream);
  ens_destroy_graphs(e);
  for (double* s : e->slab)
    if (s) cudaFree(s);
  for (void* p : {(void*)e->d_status, (void*)e->d_counters, (void*)e->d_inst, (void*)e->d_mlp, (void*)e->d_mlp_stats})
    if (p) cudaFree(p);
  if (e->own_stream) cudaStreamDestroy(e->own_stream);
  delete e;
  return CUEVA_OK;
}

int32_t cueva_ens_create(const cueva_params* params, int32_t n, cueva_ens** out) {
  if (!params || !out || n <= 0) return fail(CUEVA_ERR_ARG, "null argument or empty ensemble");
  *out = nullptr;
  for (int k = 0; k < n; ++k) {
    if (int32_t e = validate_params(&params[k]))
      return fail(e, "instance " + std::to_string(k) + ": " + g_err);
    const cueva_params& a = params[0];
    const cueva_params& b = params[k];
    if (b.order != a.order || b.flux_solver != a.flux_solver || b.rec_mp != a.rec_mp ||
        b.precision != a.precision || b.intsum_reset != a.intsum_reset || b.device != a.device ||
        b.primitive_rec != a.primitive_rec)
      return fail(CUEVA_ERR_ARG, "instance " + std::to_string(k) +
                                     ": order, flux_solver, rec_mp, precision, intsum_reset, primitive_rec and device "
                                     "must agree");
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, "no CUDA device available");
  }
  if (params[0].device < 0 || params[0].device >= ndev) return fail(CUEVA_ERR_ARG, "device ordinal out of range");
  CUDA_TRY(cudaSetDevice(params[0].device));
  cueva_ens* e = new cueva_ens();
  e->dev = params[0].device;
  e->n = n;
  e->P0 = params[0];
  if (!make_tableau(e->P0.order, e->T)) { delete e; return fail(CUEVA_ERR_ARG, "unsupported IMEX order"); }
  e->nkslot = kslots(e->T, e->kslot_of);
  cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->dev);
  e->P.assign(params, params + n);
  e->I.resize(n);
  e->slab.assign(n, nullptr);
  cudaError_t ce = cudaMalloc(&e->d_status, sizeof(uint32_t) * n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_counters, sizeof(unsigned long long) * 3 * n);
  if (ce == cudaSuccess) ce = cudaMalloc(&e->d_inst, sizeof(InstDesc) * n);
  if (ce == cudaSuccess) ce = cudaMemset(e->d_status, 0, sizeof(uint32_t) * n);
  if (ce == cudaSuccess) ce = cudaMemset(e->d_counters, 0, sizeof(unsigned long long) * 3 * n);
  for (int k = 0; k < n && ce == cudaSuccess; ++k) {
    e->G.push_back(inst_geom(&params[k], e->nkslot));
    ce = cudaMalloc(&e->slab[k], (size_t)e->G[k].nslab * sizeof(double));
    if (ce == cudaSuccess) ce = cudaMemset(e->slab[k], 0, (size_t)e->G[k].nslab * sizeof(double));
    if (ce == cudaSuccess) {
      fill_desc(&params[k], e->G[k], e->nkslot, e->slab[k], e->d_status + k, e->d_counters + 3 * k, e->I[k]);
      const long long pts = (long long)e->G[k].nx * e->G[k].ny;
      if (pts > e->max_points) e->max_points = pts;
    }
  }
  if (ce == cudaSuccess && prepare_stage(e->P0.rec_mp, e->P0.flux_solver, e->P0.precision) != cudaSuccess)
    ce = cudaErrorInvalidValue;
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&e->own_stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) {
    cueva_ens_destroy(e);
    cudaGetLastError();
    return fail(CUEVA_ERR_CUDA, std::string("ensemble set-up: ") + cudaGetErrorString(ce));
  }
  e->stream = e->own_stream;
  if (int32_t r = ens_apply_shape(e, FACE_ROWS, 0)) { cueva_ens_destroy(e); return r; }
  *out = e;
  return CUEVA_OK;
}

int32_t cueva_ens_set_stream(cueva_ens* e, void* s) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  ens_destroy_graphs(e);
  e->stream = s ? (cudaStream_t)s : e->own_stream;
  return CUEVA_OK;
}

int32_t cueva_ens_set_shape(cueva_ens* e, int32_t rows, int32_t ctas_per_sm) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  if ((rows != 4 && rows != 8) || ctas_per_sm < 0) return fail(CUEVA_ERR_ARG, "rows must be 4 or 8, ctas_per_sm >= 0");
  CUDA_TRY(cudaSetDevice(e->dev));
  return ens_apply_shape(e, rows, ctas_per_sm);
}

int32_t cueva_ens_set_prims(cueva_ens* e, int32_t k, const double* host) {
  if (int32_t r = ens_check(e, k)) return r;
  if (!host) return fail(CUEVA_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(e->dev));
  const InstGeom& G = e->G[k];
  for (int f = 0; f < NPRIM; ++f)
    CUDA_TRY(cudaMemcpy2DAsync(e->I[k].prim[e->cur] + (long long)f * G.fstride, (size_t)G.pitch * 8,
                               host + (size_t)f * G.nx * G.ny, (size_t)G.nx * 8, (size_t)G.nx * 8, (size_t)G.ny,
                               cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  e->primed = false;
  return CUEVA_OK;
}

int32_t cueva_ens_get_prims(cueva_ens* e, int32_t k, double* host) {
  if (int32_t r = ens_check(e, k)) return r;
  if (!host) return fail(CUEVA_ERR_ARG, "null argument");
  CUDA_TRY(cudaSetDevice(e->dev));
  const InstGeom& G = e->G[k];
  for (int f = 0; f < NPRIM; ++f)
    CUDA_TRY(cudaMemcpy2DAsync(host + (size_t)f * G.nx * G.ny, (size_t)G.nx * 8,
                               e->I[k].prim[e->cur] + (long long)f * G.fstride, (size_t)G.pitch * 8,
                               (size_t)G.nx * 8, (size_t)G.ny, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return CUEVA_OK;
}

int32_t cueva_ens_kh_init(cueva_ens* e, int32_t k, double v0, double a, double amp, double width, double kpert,
                          double phase, double bshear, double rho0, double p0) {
  if (int32_t r = ens_check(e, k)) return r;
  const InstGeom& G = e->G[k];
  const KHParams kh{v0, a, amp, width, kpert, phase, bshear, rho0, p0};
  std::vector<double> h((size_t)NPRIM * G.nx * G.ny);
  for (int j = 0; j <= G.jmax; ++j)
    for (int i = 0; i <= G.imax; ++i) {
      double pv[NPRIM];
      kh_point(kh, -0.5 * e->P[k].lx + i * G.delx, -0.5 * e->P[k].ly + j * G.dely, pv);
      for (int f = 0; f < NPRIM; ++f) h[(size_t)f * G.nx * G.ny + (size_t)j * G.nx + i] = pv[f];
    }
  return cueva_ens_set_prims(e, k, h.data());
}

int32_t cueva_ens_step(cueva_ens* e, int32_t nsteps) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  if (nsteps < 0) return fail(CUEVA_ERR_ARG, "nsteps < 0");
  CUDA_TRY(cudaSetDevice(e->dev));
  if (!e->primed)
    if (int32_t r = ens_begin(e)) return r;
  for (int s = 0; s < nsteps; ++s) {
    cudaGraphExec_t& g = e->graph[e->cur][e->qin];
    if (!g) {
      const int cur0 = e->cur, qin0 = e->qin;
      cudaGraph_t graph = nullptr;
      CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
      int32_t r = ens_enqueue_step(e);
      cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
      e->cur = cur0; e->qin = qin0;
      if (r) { if (graph) cudaGraphDestroy(graph); return r; }
      if (ce != cudaSuccess) return fail(CUEVA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
      ce = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (ce != cudaSuccess) return fail(CUEVA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
    }
    CUDA_TRY(cudaGraphLaunch(g, e->stream));
    for (int l = 0; l < e->T.s; ++l) e->qin ^= 1;
    if (!e->P0.primitive_rec) e->cur ^= 1;   // with the reconstruction the step flips the buffers twice
  }
  return CUEVA_OK;
}

int32_t cueva_ens_sync(cueva_ens* e, uint32_t* status_out) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  CUDA_TRY(cudaSetDevice(e->dev));
  std::vector<uint32_t> st(e->n);
  CUDA_TRY(cudaMemcpyAsync(st.data(), e->d_status, sizeof(uint32_t) * e->n, cudaMemcpyDeviceToHost, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (status_out) std::memcpy(status_out, st.data(), sizeof(uint32_t) * e->n);
  for (int k = 0; k < e->n; ++k)
    if (st[k]) {
      char buf[128];
      snprintf(buf, sizeof buf, "instance %d: kernel status 0x%x", k, st[k]);
      return fail(CUEVA_ERR_PHYSICS, buf);
    }
  return CUEVA_OK;
}

int32_t cueva_ens_attach_mlp(cueva_ens* e, const cueva_mlp* mlp) {
  if (!e || !mlp) return fail(CUEVA_ERR_ARG, "null argument");
  if (mlp_device_of(mlp) != e->dev) return fail(CUEVA_ERR_ARG, "network and ensemble live on different devices");
  CUDA_TRY(cudaSetDevice(e->dev));
  MLPDevice h;
  if (int32_t r = mlp_device_image(mlp, &h)) return r;
  if (!e->d_mlp) {
    CUDA_TRY(cudaMalloc(&e->d_mlp, sizeof(MLPDevice)));
    CUDA_TRY(cudaMalloc(&e->d_mlp_stats, 3 * sizeof(unsigned long long)));
  }
  h.stats = e->d_mlp_stats;
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(cudaMemcpy(e->d_mlp, &h, sizeof(MLPDevice), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemset(e->d_mlp_stats, 0, 3 * sizeof(unsigned long long)));
  for (auto& I : e->I) { I.mlp = e->d_mlp; I.c2p_tc = 1; }
  ens_destroy_graphs(e);   // the step gains the con2prim launch
  CUDA_TRY(cudaMemcpy(e->d_inst, e->I.data(), sizeof(InstDesc) * e->n, cudaMemcpyHostToDevice));
  return CUEVA_OK;
}

int32_t cueva_ens_set_learned_kernel(cueva_ens* e, int32_t mode) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  if (mode != 0 && mode != 1) return fail(CUEVA_ERR_ARG, "mode must be 0 (in the last stage) or 1 (tensor-core kernel)");
  CUDA_TRY(cudaSetDevice(e->dev));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  for (auto& I : e->I) I.c2p_tc = mode;
  ens_destroy_graphs(e);
  CUDA_TRY(cudaMemcpy(e->d_inst, e->I.data(), sizeof(InstDesc) * e->n, cudaMemcpyHostToDevice));
  return CUEVA_OK;
}

// Autotuner: times one ensemble step for each launch shape -- tile height
// 8 or 4 rows, and one tile per CTA or a persistent grid of 1 or 2 (rows 8)
// / 2 or 4 (rows 4) CTAs per SM -- on the ensemble's own state, keeps the
// fastest and puts the state back.  Allocates a copy of the primitives.
int32_t cueva_ens_autotune(cueva_ens* e, int32_t* rows_out, int32_t* ctas_out, double* ms_out) {
  if (!e) return fail(CUEVA_ERR_ARG, "null ensemble");
  CUDA_TRY(cudaSetDevice(e->dev));
  std::vector<double*> save(e->n, nullptr);
  auto release = [&]() {
    for (double* p : save)
      if (p) cudaFree(p);
  };
  auto copy_prims = [&](bool to_save) -> cudaError_t {
    for (int k = 0; k < e->n; ++k) {
      const size_t bytes = (size_t)NPRIM * e->G[k].fstride * sizeof(double);
      cudaError_t ce = to_save ? cudaMemcpyAsync(save[k], e->I[k].prim[e->cur], bytes, cudaMemcpyDeviceToDevice, e->stream)
                               : cudaMemcpyAsync(e->I[k].prim[e->cur], save[k], bytes, cudaMemcpyDeviceToDevice, e->stream);
      if (ce != cudaSuccess) return ce;
    }
    return cudaSuccess;
  };
  for (int k = 0; k < e->n; ++k)
    if (cudaMalloc(&save[k], (size_t)NPRIM * e->G[k].fstride * sizeof(double)) != cudaSuccess) {
      release(); cudaGetLastError();
      return fail(CUEVA_ERR_CUDA, "autotune: no memory for the state copy");
    }
  if (copy_prims(true) != cudaSuccess) { release(); return fail(CUEVA_ERR_CUDA, "autotune: state copy failed"); }
  const int cand[6][2] = {{8, 0}, {8, 2}, {8, 1}, {4, 0}, {4, 4}, {4, 2}};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  double best = 1e300;
  int brow = FACE_ROWS, bctas = 0;
  int32_t rc = CUEVA_OK;
  const int cur0 = e->cur, qin0 = e->qin;
  for (const auto& c : cand) {
    e->cur = cur0; e->qin = qin0;
    if ((rc = ens_apply_shape(e, c[0], c[1]))) break;
    if (copy_prims(false) != cudaSuccess) { rc = fail(CUEVA_ERR_CUDA, "autotune: state restore failed"); break; }
    e->primed = false;
    if ((rc = cueva_ens_step(e, 1))) break;   // captures the graphs, warms the caches
    cudaEventRecord(ev0, e->stream);
    if ((rc = cueva_ens_step(e, 2))) break;
    cudaEventRecord(ev1, e->stream);
    if (cudaEventSynchronize(ev1) != cudaSuccess) { rc = fail(CUEVA_ERR_CUDA, "autotune: timing failed"); break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (ms / 2.0 < best) { best = ms / 2.0; brow = c[0]; bctas = c[1]; }
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  e->cur = cur0; e->qin = qin0;
  if (!rc) rc = ens_apply_shape(e, brow, bctas);
  if (!rc && copy_prims(false) != cudaSuccess) rc = fail(CUEVA_ERR_CUDA, "autotune: state restore failed");
  if (!rc && cudaMemsetAsync(e->d_status, 0, sizeof(uint32_t) * e->n, e->stream) != cudaSuccess)
    rc = fail(CUEVA_ERR_CUDA, "autotune: status reset failed");
  cudaStreamSynchronize(e->stream);
  release();
  e->primed = false;
  if (rc) return rc;
  if (rows_out) *rows_out = brow;
  if (ctas_out) *ctas_out = bctas;
  if (ms_out) *ms_out = best;
  return CUEVA_OK;
}

int32_t cueva_ens_learned_stats(cueva_ens* e, int64_t out3[3]) {
  if (!e || !out3) return fail(CUEVA_ERR_ARG, "null argument");
  unsigned long long h[3] = {0, 0, 0};
  if (e->d_mlp_stats) {
    CUDA_TRY(cudaMemcpyAsync(h, e->d_mlp_stats, sizeof h, cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
  }
  for (int k = 0; k < 3; ++k) out3[k] = (int64_t)h[k];
  return CUEVA_OK;
}

}  // extern "C"
