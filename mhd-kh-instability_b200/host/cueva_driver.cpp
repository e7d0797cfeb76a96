// cueva_driver.cpp -- C++ stand-in for the reference's driver program
// (cueva_2D_base/main_cueva_code.f95) on top of the C-ABI of include/cueva.h.
//
// It does what the Fortran driver does with the library linked in (the
// Fortran form binds the same calls through fortran/cueva_gpu.f90): the run configuration of
// parameters.f95 as a key = value file, the module arrays as host arrays with
// the Fortran layout (-6:imax+6, -6:jmax+6), initial data (the KH shear
// layer) or a restart from a backup file (RESTART = 1, 03_restart_primitive.f95),
// the time loop h = hini .. hmax-1 with t_advance starting at (hini-1)*Delt
// and growing by Delt each step,
// the writer's time series after every step with h == 1 or mod(h, hglb) == 0
// (01_openfiles.f95 file names, 22_writer.f95:950-988 line content, reduced
// on the device), and the backup files data_restart/all_variables_NNNN.dat
// every hloc steps (22_writer.f95:1105-1150, ghost points filled by the
// BOUND rule first, as the writer runs after `boundary`).
//
// Usage: cueva_driver <config file>      (cueva_driver --help lists the keys)
// Exit status: 0 done, 1 bad configuration or I/O, 2 a kernel hit a
// reference STOP condition, 3 CUDA failure (e.g. no device).
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "cueva.h"

namespace {

// ------------------------------------------------------------ configuration
struct Key { const char* name; const char* dflt; const char* help; };
const Key kKeys[] = {
    {"imax", "256", "grid points 0..imax along x (parameters.f95:110)"},
    {"jmax", "128", "grid points 0..jmax along y (parameters.f95:111)"},
    {"order", "2", "IMEX tableau: 1, 2 SSP2(2,2,2), 3 SSP2(3,3,2), 4 SSP3(4,3,3), 5, 6, 8"},
    {"flux_solver", "5", "1 Lax-Friedrichs with MC slopes, 2 HLL / 3 HLLE / 4 HLLC with MC reconstruction, 5 HLL, 6 HLLE, 7 HLLC (MPX reconstruction)"},
    {"rec_mp", "0", "0 MP5, 1 MP7, 2 MP9"},
    {"conserved_to_primitive", "1", "1 Cardano, 0 Newton-Raphson"},
    {"BOUND", "6", "1 copy/copy, 2 periodic/periodic, 6 x copy / y periodic (04_boundary.f95)"},
    {"Longx", "2.0", "domain length along x"},
    {"Longy", "1.0", "domain length along y"},
    {"Longz", "1.0", "Delz"},
    {"CFL", "0.25", "Delt = CFL * min(Delx, Dely, Delz) unless Delt is given"},
    {"Delt", "0", "time step (0: from CFL)"},
    {"sigma", "1.0e3", "conductivity"},
    {"gamma", "1.3333333333333333", "adiabatic index"},
    {"hini", "1", "first step index"},
    {"hmax", "201", "the loop runs h = hini .. hmax-1"},
    {"hglb", "10", "time-series records after h == 1 or mod(h, hglb) == 0"},
    {"hloc", "100", "backup file after mod(h, hloc) == 0"},
    {"RESTART", "0", "0: KH initial data, 1: read restart_file"},
    {"restart_file", "all_variables.dat", "backup file read when RESTART = 1"},
    {"precision", "0", "0 FP64, 1 FP32 reconstruction and Riemann solves"},
    {"intsum_reset", "0", "1 zeroes the stage sums before every stage"},
    {"primitive_rec", "0", "1 reconstructs the primitives at the start of every step (05_reconstruct.f95)"},
    {"device", "0", "CUDA device ordinal"},
    {"kh_v0", "0.5", "shear velocity"},
    {"kh_a", "0.01", "shear width"},
    {"kh_amp", "0.01", "perturbation amplitude"},
    {"kh_width", "0.01", "perturbation Gaussian width (x^2 / width)"},
    {"kh_kpert", "6.283185307179586", "perturbation wave number"},
    {"kh_phase", "0.0", "perturbation phase"},
    {"kh_bshear", "0.1", "uniform field along the flow"},
    {"kh_rho0", "1.0", "density"},
    {"kh_p0", "1.0", "pressure"},
    {"B0", "0.1", "writer: max_val_bx = max(Bx) / B0"},
    {"Lr", "3.0", "writer: unit 67"},
    {"Ly", "1.0", "writer: unit 67"},
    {"delta_rec", "0", "writer: unit 67 (0: S_l**(-1/3) * Lr with S_l = 1e3)"},
    {"output_dir", ".", "directory that receives data_global/ and data_restart/"},
    {"checkpoint_in", "", "binary checkpoint to start from (replaces initial data; sets the clock)"},
    {"checkpoint_out", "", "binary checkpoint written after the last step"},
    {"max_chunk", "1000", "largest number of steps launched between host checks"},
};

struct Config {
  std::map<std::string, std::string> v;
  std::string str(const char* k) const { return v.at(k); }
  double num(const char* k) const { return std::strtod(v.at(k).c_str(), nullptr); }
  int integer(const char* k) const { return (int)std::strtol(v.at(k).c_str(), nullptr, 10); }
};

bool parse_config(const char* path, Config& c, std::string& err) {
  for (const Key& k : kKeys) c.v[k.name] = k.dflt;
  std::ifstream in(path);
  if (!in) { err = std::string("cannot open ") + path; return false; }
  std::string line;
  int ln = 0;
  while (std::getline(in, line)) {
    ++ln;
    const size_t bang = line.find('!');
    if (bang != std::string::npos) line.erase(bang);
    const size_t eq = line.find('=');
    auto trim = [](std::string s) {
      const size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
      return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
    };
    if (trim(line).empty()) continue;
    if (eq == std::string::npos) { err = "line " + std::to_string(ln) + ": expected key = value"; return false; }
    const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    if (!c.v.count(key)) { err = "line " + std::to_string(ln) + ": unknown key '" + key + "'"; return false; }
    c.v[key] = val;
  }
  return true;
}

void usage() {
  std::printf("usage: cueva_driver <config file>\n\nkeys (key = value, '!' starts a comment):\n");
  for (const Key& k : kKeys) std::printf("  %-24s default %-20s %s\n", k.name, k.dflt[0] ? k.dflt : "(none)", k.help);
}

// ------------------------------------------------------------ host fields
struct Fields {
  int imax, jmax;
  std::vector<double> a[CUEVA_W + 1];   // the 14 primitives, then D, tau, Sx, Sy, Sz, W
  size_t id(int i, int j) const { return (size_t)(i + 6) + (size_t)(j + 6) * (size_t)(imax + 13); }
};

// ghost points of the BOUND rule: copy = the edge point, periodic = the
// node duplicate (-k -> N-k, N+k -> k), corners from both rules
void fill_ghosts(Fields& F, int bc_x, int bc_y) {
  auto mi = [&](int i) { return i < 0 ? (bc_x ? i + F.imax : 0) : (i > F.imax ? (bc_x ? i - F.imax : F.imax) : i); };
  auto mj = [&](int j) { return j < 0 ? (bc_y ? j + F.jmax : 0) : (j > F.jmax ? (bc_y ? j - F.jmax : F.jmax) : j); };
  for (int f = 0; f <= CUEVA_Q; ++f) {
    double* x = F.a[f].data();
    for (int j = -6; j <= F.jmax + 6; ++j)
      for (int i = -6; i <= F.imax + 6; ++i)
        if (i < 0 || i > F.imax || j < 0 || j > F.jmax) x[F.id(i, j)] = x[F.id(mi(i), mj(j))];
  }
}

// ------------------------------------------------------------ writer files
// 01_openfiles.f95:62-111 (DIM == 2): unit -> file, and the record slot it prints
struct Series { int unit; const char* file; int slot; };
const Series kSeries[] = {
    {67, "delta_rec_t_2D.dat", CUEVA_DG_DELTA_REC}, {68, "rate_rec_ez_2D.dat", CUEVA_DG_EZ_MED},
    {80, "2d_data_psi_integral_vol.dat", CUEVA_DG_SUM_PSI}, {81, "2d_data_phi_integral_vol.dat", CUEVA_DG_SUM_PHI},
    {82, "2d_data_ex_integral_vol.dat", CUEVA_DG_SUM_EX}, {83, "2d_data_ey_integral_vol.dat", CUEVA_DG_SUM_EY},
    {84, "2d_data_ez_integral_vol.dat", CUEVA_DG_SUM_EZ}, {85, "2d_data_exey_integral_vol.dat", CUEVA_DG_SUM_EXEY},
    {86, "2d_data_exez_integral_vol.dat", CUEVA_DG_SUM_EXEZ}, {87, "2d_data_eyez_integral_vol.dat", CUEVA_DG_SUM_EYEZ},
    {88, "2d_data_bx_integral_vol.dat", CUEVA_DG_SUM_BX}, {90, "2d_data_by_integral_vol.dat", CUEVA_DG_SUM_BY},
    {91, "2d_data_bz_integral_vol.dat", CUEVA_DG_SUM_BZ}, {92, "2d_data_bxby_integral_vol.dat", CUEVA_DG_SUM_BXBY},
    {93, "2d_data_bxbz_integral_vol.dat", CUEVA_DG_SUM_BXBZ}, {94, "2d_data_bybz_integral_vol.dat", CUEVA_DG_SUM_BYBZ},
    {95, "2d_data_v2_integral_vol.dat", CUEVA_DG_SUM_VXVYVZ}, {96, "2d_data_b2_integral_vol.dat", CUEVA_DG_SUM_BXBYBZ},
    {97, "2d_data_vx_integral_vol.dat", CUEVA_DG_SUM_VX}, {98, "2d_data_vy_integral_vol.dat", CUEVA_DG_SUM_VY},
    {99, "2d_data_vz_integral_vol.dat", CUEVA_DG_SUM_VZ}, {200, "2d_data_vxvy_integral_vol.dat", CUEVA_DG_SUM_VXVY},
    {201, "2d_data_vxvz_integral_vol.dat", CUEVA_DG_SUM_VXVZ}, {202, "2d_data_vyvz_integral_vol.dat", CUEVA_DG_SUM_VYVZ},
    {203, "2d_data_q_integral_vol.dat", CUEVA_DG_SUM_Q}, {204, "2d_data_p_integral_vol.dat", CUEVA_DG_SUM_P},
    {205, "2d_data_rho_integral_vol.dat", CUEVA_DG_SUM_RHO}, {206, "2d_data_ekin_c_integral_vol.dat", CUEVA_DG_EKIN_C},
    {207, "2d_data_ekin_r_integral_vol.dat", CUEVA_DG_EKIN_R}, {208, "2d_data_etot_integral_vol.dat", CUEVA_DG_ETOT},
    {209, "2d_data_efluid_r_integral_vol.dat", CUEVA_DG_EFLUID_R}, {210, "2d_data_emag_integral_vol.dat", CUEVA_DG_EMAG},
    {211, "2d_data_eint_c_integral_vol.dat", CUEVA_DG_EINT_C}, {212, "2d_data_eint_r_integral_vol.dat", CUEVA_DG_EINT_R},
    {213, "2d_data_lorentz_integral_vol.dat", CUEVA_DG_LORENTZ}, {214, "2d_data_D_integral_vol.dat", CUEVA_DG_SUM_D},
    {215, "2d_data_D_zona_media_integral_vol.dat", CUEVA_DG_SUM_D_MED},
    {216, "2d_data_bx_max_val.dat", CUEVA_DG_MAX_BX}, {217, "2d_data_phi_max_val.dat", CUEVA_DG_MAX_PHI},
};
constexpr int kNSeries = sizeof(kSeries) / sizeof(kSeries[0]);

bool make_dir(const std::string& d) { return ::mkdir(d.c_str(), 0755) == 0 || errno == EEXIST; }

int fail_with(const char* what, int32_t rc) {
  std::fprintf(stderr, "cueva_driver: %s: %s\n", what, cueva_last_error());
  if (rc == CUEVA_ERR_PHYSICS) return 2;
  if (rc == CUEVA_ERR_CUDA) return 3;
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 2 || !std::strcmp(argv[1], "--help") || !std::strcmp(argv[1], "-h")) {
    usage();
    return argc == 2 ? 0 : 1;
  }
  Config C;
  std::string err;
  if (!parse_config(argv[1], C, err)) {
    std::fprintf(stderr, "cueva_driver: %s: %s\n", argv[1], err.c_str());
    return 1;
  }
  const int bound = C.integer("BOUND");
  int bc_x, bc_y;
  if (bound == 1) { bc_x = 0; bc_y = 0; }
  else if (bound == 2) { bc_x = 1; bc_y = 1; }
  else if (bound == 6) { bc_x = 0; bc_y = 1; }
  else { std::fprintf(stderr, "cueva_driver: BOUND must be 1, 2 or 6\n"); return 1; }
  const int hini = C.integer("hini"), hmax = C.integer("hmax"), hglb = C.integer("hglb"), hloc = C.integer("hloc");
  if (hini < 1 || hmax < hini || hglb < 1 || hloc < 1) {
    std::fprintf(stderr, "cueva_driver: need 1 <= hini <= hmax, hglb >= 1, hloc >= 1\n");
    return 1;
  }

  cueva_params p{};
  p.imax = C.integer("imax"); p.jmax = C.integer("jmax"); p.order = C.integer("order");
  p.flux_solver = C.integer("flux_solver"); p.rec_mp = C.integer("rec_mp"); p.c2p = C.integer("conserved_to_primitive");
  p.bc_x = bc_x; p.bc_y = bc_y; p.precision = C.integer("precision"); p.device = C.integer("device");
  p.intsum_reset = C.integer("intsum_reset");
  p.primitive_rec = C.integer("primitive_rec");
  p.lx = C.num("Longx"); p.ly = C.num("Longy"); p.lz = C.num("Longz"); p.cfl = C.num("CFL");
  p.sigma = C.num("sigma"); p.gamma = C.num("gamma"); p.dt = C.num("Delt");

  cueva_ctx* ctx = nullptr;
  if (int32_t rc = cueva_ctx_create(&p, &ctx)) return fail_with("cueva_ctx_create", rc);
  const double Delt = cueva_dt(ctx);

  // module arrays with the Fortran layout, bound once (cueva_attach of cueva_gpu.f90)
  Fields F{p.imax, p.jmax, {}};
  const size_t nfield = (size_t)(p.imax + 13) * (size_t)(p.jmax + 13);
  for (int f = 0; f <= CUEVA_W; ++f) {
    F.a[f].assign(nfield, 0.0);
    if (int32_t rc = cueva_bind_field(ctx, f, F.a[f].data())) return fail_with("cueva_bind_field", rc);
  }
  double* prim_tab[CUEVA_Q + 1];
  for (int f = 0; f <= CUEVA_Q; ++f) prim_tab[f] = F.a[f].data();

  // initial data (main_cueva_code.f95:18-34)
  int32_t rc = 0;
  const std::string ck_in = C.str("checkpoint_in");
  if (!ck_in.empty()) {
    if ((rc = cueva_checkpoint_load(ctx, ck_in.c_str()))) return fail_with("cueva_checkpoint_load", rc);
  } else {
    if (C.integer("RESTART") == 1) {
      rc = cueva_read_all_variables(C.str("restart_file").c_str(), p.imax, p.jmax, prim_tab, 0);
      if (rc) return fail_with("reading the restart file", rc);
    } else {
      rc = cueva_kh_init(ctx, C.num("kh_v0"), C.num("kh_a"), C.num("kh_amp"), C.num("kh_width"), C.num("kh_kpert"),
                         C.num("kh_phase"), C.num("kh_bshear"), C.num("kh_rho0"), C.num("kh_p0"));
      if (rc) return fail_with("cueva_kh_init", rc);
    }
    if ((rc = cueva_upload(ctx, CUEVA_G_PRIMS))) return fail_with("cueva_upload", rc);
    // t_advance = (hini-1) * Delt (main_cueva_code.f95:45)
    if ((rc = cueva_set_clock(ctx, hini - 1, (hini - 1) * Delt))) return fail_with("cueva_set_clock", rc);
  }

  // writer files (01_openfiles.f95) and device-side records
  const std::string out = C.str("output_dir");
  if (!make_dir(out) || !make_dir(out + "/data_global") || !make_dir(out + "/data_restart")) {
    std::fprintf(stderr, "cueva_driver: cannot create the output directories under %s\n", out.c_str());
    return 1;
  }
  std::vector<FILE*> series(kNSeries, nullptr);
  for (int k = 0; k < kNSeries; ++k) {
    series[k] = std::fopen((out + "/data_global/" + kSeries[k].file).c_str(), "w");
    if (!series[k]) { std::fprintf(stderr, "cueva_driver: cannot open %s\n", kSeries[k].file); return 1; }
  }
  FILE* courant = std::fopen((out + "/data_global/2d_data_courant.dat").c_str(), "w");
  if (!courant) { std::fprintf(stderr, "cueva_driver: cannot open 2d_data_courant.dat\n"); return 1; }
  const int max_chunk = std::max(1, C.integer("max_chunk"));
  cueva_diag_config dc{};
  dc.hglb = hglb;
  dc.capacity = max_chunk / hglb + 2;
  dc.b0 = C.num("B0"); dc.lr = C.num("Lr"); dc.ly = C.num("Ly");
  dc.delta_rec = C.num("delta_rec") != 0.0 ? C.num("delta_rec") : std::pow(1.0e3, -1.0 / 3.0) * dc.lr;
  if ((rc = cueva_diag_enable(ctx, &dc))) return fail_with("cueva_diag_enable", rc);
  std::vector<cueva_diag_record> recs(dc.capacity);

  int64_t h0 = 0;
  double t0 = 0.0;
  cueva_get_clock(ctx, &h0, &t0);
  const long long first = h0 + 1, last = hmax - 1;
  const auto wall0 = std::chrono::steady_clock::now();
  int status = 0;
  for (long long h = first; h <= last;) {
    // launch up to the next backup step (or max_chunk steps) without host checks
    long long stop = std::min<long long>(last, h + max_chunk - 1);
    const long long next_bck = ((h + hloc - 1) / hloc) * hloc;
    if (next_bck <= stop) stop = next_bck;
    if ((rc = cueva_step(ctx, (int32_t)(stop - h + 1)))) { status = fail_with("cueva_step", rc); break; }
    int32_t n = 0;
    rc = cueva_diag_read(ctx, recs.data(), (int32_t)recs.size(), &n);
    for (int32_t r = 0; r < n; ++r) {   // write(80,*) h, t_advance, sum_psi, ... (22_writer.f95:950-988)
      for (int k = 0; k < kNSeries; ++k)
        std::fprintf(series[k], "%12lld %25.16E %25.16E\n", (long long)recs[r].h, recs[r].t, recs[r].v[kSeries[k].slot]);
      std::fprintf(courant, "%12lld %25.16E %25.16E %25.16E %25.16E\n", (long long)recs[r].h, recs[r].t,
                   recs[r].v[CUEVA_DG_MAX_V], recs[r].v[CUEVA_DG_MAX_W], recs[r].v[CUEVA_DG_COURANT]);
      std::printf(" ::::::::::: loop ::::::::::::\n iteration = %lld   time = %.16E\n", (long long)recs[r].h, recs[r].t);
    }
    if (rc) { status = fail_with("cueva_diag_read", rc); break; }
    if (stop % hloc == 0) {   // backup (22_writer.f95:1105-1150) after boundary
      if ((rc = cueva_download(ctx, CUEVA_G_PRIMS))) { status = fail_with("cueva_download", rc); break; }
      fill_ghosts(F, bc_x, bc_y);
      char name[64];
      std::snprintf(name, sizeof name, "all_variables_%04lld.dat", stop / hloc);
      rc = cueva_write_all_variables((out + "/data_restart/" + name).c_str(), p.imax, p.jmax, prim_tab, 0, 0);
      if (rc) { status = fail_with("writing the backup file", rc); break; }
    }
    h = stop + 1;
  }
  if (status == 0) {
    if ((rc = cueva_sync(ctx))) status = fail_with("cueva_sync", rc);
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
  for (FILE* f : series) std::fclose(f);
  std::fclose(courant);
  int64_t hend = 0;
  double tend = 0.0;
  cueva_get_clock(ctx, &hend, &tend);
  if (status == 0) {
    const std::string ck_out = C.str("checkpoint_out");
    if (!ck_out.empty() && (rc = cueva_checkpoint_save(ctx, ck_out.c_str()))) status = fail_with("cueva_checkpoint_save", rc);
  }
  int64_t cnt[3] = {0, 0, 0};
  cueva_counters(ctx, cnt);
  const double steps = (double)(hend - h0);
  std::printf("cueva_driver: %lld steps to h = %lld, t = %.16E, %.3f s, %.4e zone-updates/s; "
              "fix-ups rho %lld p %lld v %lld\n",
              (long long)(hend - h0), (long long)hend, tend, wall,
              wall > 0 ? steps * (double)p.imax * (double)p.jmax / wall : 0.0, (long long)cnt[0], (long long)cnt[1],
              (long long)cnt[2]);
  cueva_ctx_destroy(ctx);
  return status;
}
