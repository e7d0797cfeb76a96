// cueva_oracle.cpp -- CPU restatement (test infrastructure only) of the CUEVA
// per-step hot path.  See cueva_oracle.h for scope and parity status.
//
// Every routine mirrors one Fortran routine of cueva_2D_base/ (paths relative
// to the reference project) and keeps its array layout: fields live on
// (-6:imax+6, -6:jmax+6), i fastest, exactly like the Fortran module arrays
// (threevectors.f95:12-81, fourvectors.f95:12-170).  Ghost cells are filled
// by the boundary maps of 04_boundary.f95 / 24_boundary_conserved.f95 /
// 24_boundary_flux_conserved.f95 / 25_boundary_electric.f95 (per-axis copy or
// periodic, node-duplicate convention).
//
// Build: g++ -O2 -ffp-contract=off -fno-fast-math -fopenmp -shared -fPIC
#include "cueva_oracle.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// gfortran expands constant integer powers with powi: x**2 = x*x,
// x**3 = (x*x)*x, x**4 = (x*x)*(x*x).
inline double pw2(double x) { return x * x; }
inline double pw3(double x) { return (x * x) * x; }
inline double pw4(double x) { double t = x * x; return t * t; }
// Fortran SIGN(a,b) with signed zeros (gfortran -fsign-zero default)
inline double fsign(double a, double b) { return std::copysign(std::fabs(a), b); }
inline double fmin2(double a, double b) { return (b < a) ? b : a; }
inline double fmax2(double a, double b) { return (b > a) ? b : a; }
inline double fmin3(double a, double b, double c) { return fmin2(fmin2(a, b), c); }
inline double fmax3(double a, double b, double c) { return fmax2(fmax2(a, b), c); }

constexpr double PI = 3.14159265358979323846264338327950288419716939937510582097494459230781640628620899862803;
constexpr double THIRD = 0.33333333333333333333333333333333333333333333333333333333333333333333333333333333333;

enum Status : int32_t {
  ST_OK = 0,
  ST_C2P_FAIL = 1,        // Cardano "stop" branches (12_varprimitive.f95:382-428,485)
  ST_SUPERLUMINAL = 2,    // 12_varprimitive.f95:678,691 ; 12_varprimitive_nr.f95:217
  ST_HLLC_NOCONV = 4,     // funciones.f95:240-245
  ST_HLLC_VSTAR = 8,      // 16_hllc_flow_mpx.f95:4294,4605
  ST_NONFINITE = 16,
  ST_HLLE_SPEED = 32,     // 16_hlle_flow_mpx.f95:2796-2803, 2974-2981
};

// ---------------------------------------------------------------- tableaux
// imex_scheme.f95:13-507 (MIRK = 0 branches)
struct Tableau { int s; double wb[8], wbt[8], Ab[8][8], Abt[8][8]; };

bool make_tableau(int order, Tableau& T) {
  std::memset(&T, 0, sizeof(T));
  const double cst = 1.0 - 1.0 / std::sqrt(2.0);            // parameters.f95:240
  const double alpha1 = 0.24169426078821, beta1 = 0.06042356519705, etha1 = 0.12915286960590;
  switch (order) {
  case 1:  // imex_scheme.f95:15-20
    T.s = 1; T.wb[0] = 1.0; T.wbt[0] = 0.0; T.Ab[0][0] = 1.0; T.Abt[0][0] = 0.0; return true;
  case 2:  // SSP2(2,2,2) imex_scheme.f95:42-49
    T.s = 2; T.wb[0] = 0.5; T.wb[1] = 0.5; T.wbt[0] = 0.5; T.wbt[1] = 0.5;
    T.Ab[1][0] = 1.0;
    T.Abt[0][0] = cst; T.Abt[1][0] = 1.0 - 2.0 * cst; T.Abt[1][1] = cst; return true;
  case 3:  // SSP2(3,3,2)-LUM imex_scheme.f95:77-86
    T.s = 3; for (int k = 0; k < 3; ++k) { T.wb[k] = 1.0 / 3.0; T.wbt[k] = 1.0 / 3.0; }
    T.Ab[1][0] = 0.5; T.Ab[2][0] = 0.5; T.Ab[2][1] = 0.5;
    T.Abt[0][0] = 1.0 / 5.0; T.Abt[1][0] = 1.0 / 10.0; T.Abt[1][1] = 1.0 / 5.0;
    T.Abt[2][0] = 1.0 / 3.0; T.Abt[2][1] = 1.0 / 3.0; T.Abt[2][2] = 1.0 / 3.0; return true;
  case 4:  // SSP3(4,3,3) imex_scheme.f95:280-291
    T.s = 4;
    T.wb[0] = 0.0; T.wb[1] = 1.0 / 6.0; T.wb[2] = 1.0 / 6.0; T.wb[3] = 2.0 / 3.0;
    for (int k = 0; k < 4; ++k) T.wbt[k] = T.wb[k];
    T.Ab[2][1] = 1.0; T.Ab[3][1] = 0.25; T.Ab[3][2] = 0.25;
    T.Abt[0][0] = alpha1;
    T.Abt[1][0] = -1.0 * alpha1; T.Abt[1][1] = alpha1;
    T.Abt[2][1] = 1.0 - alpha1; T.Abt[2][2] = alpha1;
    T.Abt[3][0] = beta1; T.Abt[3][1] = etha1; T.Abt[3][2] = 0.5 - beta1 - etha1 - alpha1; T.Abt[3][3] = alpha1;
    return true;
  case 5: {  // ARS(4,4,3) imex_scheme.f95:328-341
    T.s = 5;
    const double wb[5] = {1.0 / 4.0, 7.0 / 4.0, 3.0 / 4.0, -7.0 / 4.0, 0.0};
    const double wbt[5] = {0.0, 3.0 / 2.0, -3.0 / 2.0, 0.5, 0.5};
    const double Ab[5][5] = {{0, 0, 0, 0, 0}, {0.5, 0, 0, 0, 0}, {11.0 / 18.0, 1.0 / 18.0, 0, 0, 0},
                             {5.0 / 6.0, -5.0 / 6.0, 0.5, 0, 0}, {1.0 / 4.0, 7.0 / 4.0, 3.0 / 4.0, -7.0 / 4.0, 0}};
    const double Abt[5][5] = {{0, 0, 0, 0, 0}, {0, 0.5, 0, 0, 0}, {0, 1.0 / 6.0, 0.5, 0, 0},
                              {0, -0.5, 0.5, 0.5, 0}, {0, 3.0 / 2.0, -3.0 / 2.0, 0.5, 0.5}};
    for (int a = 0; a < 5; ++a) { T.wb[a] = wb[a]; T.wbt[a] = wbt[a];
      for (int b = 0; b < 5; ++b) { T.Ab[a][b] = Ab[a][b]; T.Abt[a][b] = Abt[a][b]; } }
    return true; }
  case 6: {  // IMEX-RK36S_E imex_scheme.f95:366-395
    T.s = 6;
    const double w[6] = {-0.035877095577305, 0.673080876788404, 0.149064711243777,
                         0.137173305022086, 0.150219587614740, -0.073661385091702};
    const double A[6][6] = {
      {0, 0, 0, 0, 0, 0},
      {0.342975342284516, 0, 0, 0, 0, 0},
      {0.016193013787920, 0.309787886268879, 0, 0, 0, 0},
      {-0.135950059698287, 0.640189764616023, 0.342154021907072, 0, 0, 0},
      {-0.042056958294301, 0.660781723165128, -0.381308869908091, 1.001236515566727, 0, 0},
      {0.099109299514465, -0.466919631638661, 1.030492210860962, 0.564549736036252, -0.119257987827582, 0}};
    const double At[6][6] = {
      {0.449855695709406, 0, 0, 0, 0, 0},
      {-0.295189486209790, 0.449855695709406, 0, 0, 0, 0},
      {0.879036496969614, -0.042071370873823, 0.449855695709406, 0, 0, 0},
      {0.751731896214317, -0.222508174774298, 0.220689305480633, 0.449855695709406, 0, 0},
      {-0.039570781554756, 0.788509712948086, 0.685131268735182, -0.144071924307435, 0.449855695709406, 0},
      {0.382760589609172, -0.196622622060158, 0.904049611197476, 0.680864149962184, 0.571862669923976, 0.449855695709406}};
    for (int a = 0; a < 6; ++a) { T.wb[a] = w[a]; T.wbt[a] = w[a];
      for (int b = 0; b < 6; ++b) { T.Ab[a][b] = A[a][b]; T.Abt[a][b] = At[a][b]; } }
    return true; }
  case 8: {  // IMEX-RK48SSP imex_scheme.f95:469-507
    T.s = 8;
    const double w[8] = {0.0, 277.0 / 1720.0, 385.0 / 1314.0, 587.0 / 1885.0, 31.0 / 18247.0, 665.0 / 2906.0, 0.0, 23.0 / 5731.0};
    const double A[8][8] = {
      {0, 0, 0, 0, 0, 0, 0, 0},
      {0, 0, 0, 0, 0, 0, 0, 0},
      {0, 966.0 / 2039.0, 0, 0, 0, 0, 0, 0},
      {0, 199.0 / 5291.0, 735.0 / 1709.0, 0, 0, 0, 0, 0},
      {0, 306.0 / 4373.0, 533.0 / 1060.0, 773.0 / 628.0, 0, 0, 0, 0},
      {0, 61.0 / 10399.0, 552.0 / 8267.0, 881.0 / 1054.0, 52.0 / 9395.0, 0, 0, 0},
      {184.0 / 2869.0, 141.0 / 3059.0, 826.0 / 1929.0, 1567.0 / 757.0, 1754.0 / 977.0, 161.0 / 599.0, 0, 0},
      {0, 27.0 / 359.0, 227.0 / 2338.0, 53.0 / 557.0, 569.0 / 4644.0, 859.0 / 1966.0, 0, 0}};
    const double g = 1026.0 / 3919.0;
    const double At[8][8] = {
      {g, 0, 0, 0, 0, 0, 0, 0},
      {-1148.0 / 4385.0, g, 0, 0, 0, 0, 0, 0},
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

// ------------------------------------------------------------ MP5/7/9 line
// mp5.f95:2-278, mp7.f95:2-315, mp9.f95:2-320 for ONE slot of one grid line.
// The Fortran routine processes 68 slots at once, but every slot is computed
// independently (the only cross-slot code is the positivity fix, which reads
// and writes its own slot), so one slot at a time is the same arithmetic.
// u, up, um are indexed -6..n+6 (pointer offset +6).  posfix selects the
// p/rho positivity fix of mp5.f95:177-262 (applied to slots 24,25 / 61,62).

// slope limiter of the primitive reconstruction, limit = 2 (monotonized
// central), funciones.f95:104-147
inline double limiter_mc(double ga, double gb) {
  return 0.5 * (fsign(1.0, ga) + fsign(1.0, gb)) * fmin3(2.0 * std::fabs(ga), 2.0 * std::fabs(gb), 0.5 * std::fabs(ga + gb));
}
inline double DMM(double x, double y) {  // funciones.f95:148-162
  return 0.5 * (fsign(1.0, x) + fsign(1.0, y)) * fmin2(std::fabs(x), std::fabs(y));
}
inline double DM4(double w, double xx, double y, double z) {  // funciones.f95:165-185
  return 0.125 * (fsign(1.0, w) + fsign(1.0, xx))
         * std::fabs((fsign(1.0, w) + fsign(1.0, y)) * (fsign(1.0, w) + fsign(1.0, z)))
         * fmin2(fmin2(fmin2(std::fabs(w), std::fabs(xx)), std::fabs(y)), std::fabs(z));
}

void mp_line(int rec_mp, int n, const double* U, int posfix, double* UP, double* UM) {
  const double* u = U + 6;
  double* up = UP + 6;
  double* um = UM + 6;
  const double b2 = 4.0 / 3.0, epsm = 1.0e-10, alpha_mp = 2.0;
  const int mm = 0, nn = n;
  // du, d2 over mm-3..nn+3 (mm-4/mm-5 for MP7/MP9; the extra points are never read)
  std::vector<double> duv(n + 13, 0.0), d2v(n + 13, 0.0), vorpv(n + 13, 0.0), vormv(n + 13, 0.0),
      vmppv(n + 13, 0.0), vmpmv(n + 13, 0.0);
  double* du = duv.data() + 6;
  double* d2 = d2v.data() + 6;
  double* vorp = vorpv.data() + 6;
  double* vorm = vormv.data() + 6;
  double* vmpp = vmppv.data() + 6;
  double* vmpm = vmpmv.data() + 6;
  for (int i = mm - 3; i <= nn + 3; ++i) {
    du[i] = u[i] - u[i - 1];
    d2[i] = u[i - 1] - 2.0 * u[i] + u[i + 1];
  }
  for (int i = mm - 2; i <= nn + 2; ++i) {
    if (rec_mp == 0) {
      const double b1 = 1.0 / 60.0;   // mp5.f95:23, 79-83
      vorp[i] = b1 * (2.0 * u[i - 2] - 13.0 * u[i - 1] + 47.0 * u[i] + 27.0 * u[i + 1] - 3.0 * u[i + 2]);
      vorm[i] = b1 * (-3.0 * u[i - 2] + 27.0 * u[i - 1] + 47.0 * u[i] - 13.0 * u[i + 1] + 2.0 * u[i + 2]);
    } else if (rec_mp == 1) {
      const double b1 = 1.0 / 420.0;  // mp7.f95:23, 110-117
      vorp[i] = b1 * (-3.0 * u[i - 3] + 25.0 * u[i - 2] - 101.0 * u[i - 1] + 319.0 * u[i] + 214.0 * u[i + 1]
                      - 38.0 * u[i + 2] + 4.0 * u[i + 3]);
      vorm[i] = b1 * (-3.0 * u[i + 3] + 25.0 * u[i + 2] - 101.0 * u[i + 1] + 319.0 * u[i] + 214.0 * u[i - 1]
                      - 38.0 * u[i - 2] + 4.0 * u[i - 3]);
    } else {
      const double b1 = 1.0 / 2520.0; // mp9.f95:25, 114-124
      vorp[i] = b1 * (4.0 * u[i - 4] - 41.0 * u[i - 3] + 199.0 * u[i - 2] - 641.0 * u[i - 1] + 1879.0 * u[i]
                      + 1375.0 * u[i + 1] - 305.0 * u[i + 2] + 55.0 * u[i + 3] - 5.0 * u[i + 4]);
      vorm[i] = b1 * (4.0 * u[i + 4] - 41.0 * u[i + 3] + 199.0 * u[i + 2] - 641.0 * u[i + 1] + 1879.0 * u[i]
                      + 1375.0 * u[i - 1] - 305.0 * u[i - 2] + 55.0 * u[i - 3] - 5.0 * u[i - 4]);
    }
    vmpp[i] = u[i] + DMM(du[i + 1], alpha_mp * du[i]);
    vmpm[i] = u[i] + DMM(-du[i], -alpha_mp * du[i + 1]);
  }
  for (int i = mm - 2; i <= nn + 2; ++i) { up[i] = vorp[i]; um[i] = vorm[i]; }
  for (int i = mm - 2; i <= nn + 2; ++i) {  // mp5.f95:104-136
    if ((vorp[i] - u[i]) * (vorp[i] - vmpp[i]) <= epsm) {
      up[i] = vorp[i];
    } else {
      const double dm4jph = DM4(4.0 * d2[i] - d2[i + 1], 4.0 * d2[i + 1] - d2[i], d2[i], d2[i + 1]);
      const double dm4jmh = DM4(4.0 * d2[i] - d2[i - 1], 4.0 * d2[i - 1] - d2[i], d2[i], d2[i - 1]);
      const double vul = u[i] + alpha_mp * du[i];
      const double vav = 0.5 * (u[i] + u[i + 1]);
      const double vmd = vav - 0.5 * dm4jph;
      const double vlc = u[i] + 0.5 * du[i] + b2 * dm4jmh;
      const double vmin = fmax2(fmin3(u[i], u[i + 1], vmd), fmin3(u[i], vul, vlc));
      const double vmax = fmin2(fmax3(u[i], u[i + 1], vmd), fmax3(u[i], vul, vlc));
      up[i] = vorp[i] + DMM(vmin - vorp[i], vmax - vorp[i]);
    }
  }
  for (int i = mm - 2; i <= nn + 2; ++i) {  // mp5.f95:142-167
    if ((vorm[i] - u[i]) * (vorm[i] - vmpm[i]) <= epsm) {
      um[i] = vorm[i];
    } else {
      const double dm4jph = DM4(4.0 * d2[i] - d2[i + 1], 4.0 * d2[i + 1] - d2[i], d2[i], d2[i + 1]);
      const double dm4jmh = DM4(4.0 * d2[i] - d2[i - 1], 4.0 * d2[i - 1] - d2[i], d2[i], d2[i - 1]);
      const double vul = u[i] - alpha_mp * du[i + 1];
      const double vav = 0.5 * (u[i] + u[i - 1]);
      const double vmd = vav - 0.5 * dm4jmh;
      const double vlc = u[i] - 0.5 * du[i + 1] + b2 * dm4jph;
      const double vmin = fmax2(fmin3(u[i], u[i - 1], vmd), fmin3(u[i], vul, vlc));
      const double vmax = fmin2(fmax3(u[i], u[i - 1], vmd), fmax3(u[i], vul, vlc));
      um[i] = vorm[i] + DMM(vmin - vorm[i], vmax - vorm[i]);
    }
  }
  if (posfix) {  // mp5.f95:177-216 (and 226-262 for the y slots)
    for (int i = mm - 2; i <= nn + 2; ++i) {
      if (up[i] < 0.0) { up[i] = u[i] + 0.50 * DMM(du[i], du[i + 1]); um[i] = u[i]; }
    }
    for (int i = mm - 2; i <= nn + 2; ++i) {
      if (um[i] < 0.0) { um[i] = u[i] - 0.50 * DMM(du[i], du[i + 1]); up[i] = u[i]; }
    }
  }
}

// ---------------------------------------------------------- get_hllc_vel
// funciones.f95:188-259.  The Fortran evaluates f at the local v before it
// is ever assigned (line 229); this restatement starts from v = oldv, the
// seed the routine documents ("Initial seed ... limited to [-1,1]").
double get_hllc_vel(double a, double b, double c, double rt, int32_t* st) {
  const int maxiter = 100;
  const double minerr = 1.0e-12, diferr = 1.0e-3;
  double oldv = fmax2(-1.0, fmin2(1.0, rt));
  double v = oldv;
  int iter = 0;
  for (;;) {
    const double fv = a * v * v - b * v + c;
    const double dfdv = 2.0 * a * v - b;
    v = fmax2(-1.0, fmin2(1.0, oldv - fv / dfdv));
    const double err = std::fabs(oldv - v);
    oldv = v;
    iter = iter + 1;
    if (iter >= maxiter) { if (st) *st |= ST_HLLC_NOCONV; break; }
    if (!(err > minerr)) break;
  }
  return fmax2(-1.0 + diferr, fmin2(1.0 - diferr, v));
}

// ------------------------------------------------ Cardano seed arithmetic
// The Cardano branch of 12_varprimitive.f95:351-452 needs acos, cos and
// x**THIRD.  Their last bit depends on the math library (glibc here, CUDA's
// on the device), and that last bit of the W seed is amplified by the
// reference's limiter switches: a 1-ulp change of the seed moves config-1
// prims by ~1e-5 (relative L1) after 200 steps.  The default "deterministic"
// mode therefore evaluates the seed with +,-,*,/ only, identically on host
// and device:
//  * the three angles of the trigonometric solution, cos((acos(y)+2 pi k)/3),
//    are the three roots of 4c^3 - 3c = y (triple-angle identity
//    cos 3a = 4 cos^3 a - 3 cos a), found by monotone Newton iterations from
//    c = 1 and c = -1 and, for the middle root, from -(c0 + c1) (the roots
//    sum to zero);
//  * x**(1/3) is a Newton cube root on the mantissa (frexp/ldexp are exact).
// oracle_set_libm_seed(1) switches back to acos/cos/pow of the C library.
int g_libm_seed = 0;

void chebyshev_roots(double y, double& c0, double& c1, double& c2) {
  double c = 1.0;
  for (int it = 0; it < 80; ++it) {
    const double cn = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
    if (!(cn < c)) break;
    c = cn;
  }
  c0 = c;
  c = -1.0;
  for (int it = 0; it < 80; ++it) {
    const double cn = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
    if (!(cn > c)) break;
    c = cn;
  }
  c1 = c;
  c = -(c0 + c1);
  for (int it = 0; it < 3; ++it) c = c - ((4.0 * c * c - 3.0) * c - y) / (12.0 * c * c - 3.0);
  c2 = c;
}

// Deviation from 12_varprimitive.f95 (one-real-root branch): d_2 + 2 z_1
// vanishes where the depressed quartic is biquadratic (d_1 = 0), which the
// V0 = 0.8 KH layer crosses at |v| ~ 0.74; rounding can leave it at -1e-15,
// and the reference's sqrt then returns NaN with no status raised (W, rho, p
// and v of the point become NaN).  A negative value within rounding of zero
// (<= 1e-12 |d_2|) is taken as zero, the biquadratic limit; other values are
// unchanged, so every state the reference inverts to a finite result is
// unaffected.
double biquad_guard(double s2, double d_2) { return (s2 < 0.0 && -s2 <= 1.0e-12 * std::fabs(d_2)) ? 0.0 : s2; }

double cbrt_newton(double x) {
  if (!(x > 0.0) || !(x < INFINITY)) return x;
  int e;
  double m = std::frexp(x, &e);
  const int r = ((e % 3) + 3) % 3;
  const int q = (e - r) / 3;
  m = std::ldexp(m, r);                 // x = m 2^(3q), m in [0.5, 4)
  double y = 1.0;
  for (int it = 0; it < 8; ++it) y = y - (y * y * y - m) / (3.0 * y * y);
  return std::ldexp(y, q);
}

// -------------------------------------------------------- con2prim, point
struct C2PIn { double D, tau, Sx, Sy, Sz, Ex, Ey, Ez, Bx, By, Bz, vx0, vy0, vz0, rho0, p0; };
struct C2POut { double vx, vy, vz, rho, p, W; };

// 12_varprimitive.f95:48-813 with l_swap = 1, VDRIFT = 0, low_vel = 0, REC_ELEC = 0
int32_t c2p_cardano(const C2PIn& in, double gamma, double eps1, C2POut& o, int64_t* cnt) {
  int32_t st = 0;
  const double TOL = 1.0e-10;
  const int nrmax = 40;
  double Vx_elec_0 = in.vx0, Vy_elec_0 = in.vy0, Vz_elec_0 = in.vz0;
  const double Ex_elec_0 = in.Ex, Ey_elec_0 = in.Ey, Ez_elec_0 = in.Ez;
  const double Bx_elec = in.Bx, By_elec = in.By, Bz_elec = in.Bz;
  const double D_elec = in.D, Sx_elec = in.Sx, Sy_elec = in.Sy, Sz_elec = in.Sz;
  double tau_elec = in.tau;
  double rho_elec = in.rho0, p_elec = in.p0, enthpy_elec = 0.0;
  double W_elec, V2c, Vx_elec = 0, Vy_elec = 0, Vz_elec = 0;
  double E2B2 = 0.5 * (Ex_elec_0 * Ex_elec_0 + Ey_elec_0 * Ey_elec_0 + Ez_elec_0 * Ez_elec_0 +
                       Bx_elec * Bx_elec + By_elec * By_elec + Bz_elec * Bz_elec);
  double gamma_1 = (gamma - 1.0) / gamma;
  // do while loop with REC_ELEC = 0 runs exactly once (12_varprimitive.f95:222,756-767)
  {
    V2c = pw2(Vx_elec_0) + pw2(Vy_elec_0) + pw2(Vz_elec_0);
    W_elec = 1.0 / std::sqrt(1.0 - V2c);
    if (V2c > 1.0) {
      V2c = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V2c));
      W_elec = 1.0 / std::sqrt(1.0 - V2c);
    }
    E2B2 = 0.5 * (pw2(Ex_elec_0) + pw2(Ey_elec_0) + pw2(Ez_elec_0) + pw2(Bx_elec) + pw2(By_elec) + pw2(Bz_elec));
    gamma_1 = (gamma - 1.0) / gamma;
    const double C_1 = pw2(Sx_elec - Ey_elec_0 * Bz_elec + Ez_elec_0 * By_elec)
                     + pw2(Sy_elec - Ez_elec_0 * Bx_elec + Ex_elec_0 * Bz_elec)
                     + pw2(Sz_elec - Ex_elec_0 * By_elec + Ey_elec_0 * Bx_elec);
    const double C_2 = tau_elec - E2B2;
    const double a_4 = C_1 - pw2(C_2);
    const double a_3 = 2.0 * gamma_1 * C_2 * D_elec;
    const double a_2 = pw2(C_2) - 2.0 * gamma_1 * C_1 - pw2(gamma_1) * pw2(D_elec);
    const double a_1 = -2.0 * gamma_1 * C_2 * D_elec;
    const double a_0 = pw2(gamma_1) * (C_1 + pw2(D_elec));
    const double b_3 = a_3 / a_4, b_2 = a_2 / a_4, b_1 = a_1 / a_4, b_0 = a_0 / a_4;
    const double d_2 = b_2 - (3.0 * pw2(b_3)) / 8.0;
    const double d_1 = b_1 - (b_3 * b_2) / 2.0 + (pw3(b_3)) / 8.0;
    const double d_0 = b_0 - (b_3 * b_1) / 4.0 + (pw2(b_3) * b_2) / 16.0 - (3.0 * pw4(b_3)) / 256.0;
    double Wnro = NAN;
    const double e = (20.0 * d_2) / 8.0;
    const double f = -(d_0 - 2.0 * pw2(d_2));
    const double g = -(pw2(d_1) + 4.0 * d_2 * d_0 - 4.0 * pw3(d_2)) / 8.0;
    const double Q_1 = (pw2(e) - 3.0 * f) / 9.0;
    const double R_1 = (2.0 * pw3(e) - 9.0 * e * f + 27.0 * g) / 54.0;
    double s = 0, t = 0, det = 0, z_1 = 0;
    if (pw2(R_1) < pw3(Q_1)) {
      double ca, cb, cc;   // cos(T/3), cos((T+2pi)/3), cos((T-2pi)/3)
      if (g_libm_seed) {
        const double T_1 = std::acos(R_1 / std::fabs(std::sqrt(pw3(Q_1))));
        ca = std::cos((T_1) / 3.0); cb = std::cos((T_1 + 2.0 * PI) / 3.0); cc = std::cos((T_1 - 2.0 * PI) / 3.0);
      } else {
        chebyshev_roots(R_1 / std::fabs(std::sqrt(pw3(Q_1))), ca, cb, cc);
      }
      const double z_1a = -2.0 * std::fabs(std::sqrt(Q_1)) * ca - e / 3.0;
      const double s_1a = d_2 + 2.0 * z_1a;
      const double t_1a = pw2(z_1a) + 2.0 * d_2 * z_1a + pw2(d_2) - d_0;
      const double z_1b = -2.0 * std::fabs(std::sqrt(Q_1)) * cb - e / 3.0;
      const double s_1b = d_2 + 2.0 * z_1b;
      const double t_1b = pw2(z_1b) + 2.0 * d_2 * z_1b + pw2(d_2) - d_0;
      const double z_1c = -2.0 * std::fabs(std::sqrt(Q_1)) * cc - e / 3.0;
      const double s_1c = d_2 + 2.0 * z_1c;
      const double t_1c = pw2(z_1c) + 2.0 * d_2 * z_1c + pw2(d_2) - d_0;
      if (s_1a >= 0.0 && t_1a >= 0.0) {
        s = std::fabs(std::sqrt(s_1a)); t = std::fabs(std::sqrt(t_1a));
        det = pw2(s) - 4.0 * (d_2 + z_1a - t); z_1 = z_1a;
        if (det < 0.0) st |= ST_C2P_FAIL;
      } else if (s_1b >= 0.0 && t_1b >= 0.0) {
        s = std::fabs(std::sqrt(s_1b)); t = std::fabs(std::sqrt(t_1b));
        det = pw2(s) - 4.0 * (d_2 + z_1b - t); z_1 = z_1b;
        if (det < 0.0) st |= ST_C2P_FAIL;
      } else if (s_1c >= 0.0 && t_1c >= 0.0) {
        s = std::fabs(std::sqrt(s_1c)); t = std::fabs(std::sqrt(t_1c));
        det = pw2(s) - 4.0 * (d_2 + z_1c - t); z_1 = z_1c;
        if (det < 0.0) st |= ST_C2P_FAIL;
      } else {
        st |= ST_C2P_FAIL;
      }
    } else {
      const double xx1 = std::fabs(R_1) + std::fabs(std::sqrt(pw2(R_1) - pw3(Q_1)));
      const double cr = g_libm_seed ? std::pow(xx1, THIRD) : cbrt_newton(xx1);
      const double AA_1 = -fsign(1.0, R_1) * fsign(std::fabs(cr), xx1);
      const double BB_1 = (AA_1 != 0.0) ? Q_1 / AA_1 : 0.0;
      z_1 = (AA_1 + BB_1) - e / 3.0;
      s = std::fabs(std::sqrt(biquad_guard(d_2 + 2.0 * z_1, d_2)));
      t = std::fabs(std::sqrt(pw2(z_1) + 2.0 * d_2 * z_1 + pw2(d_2) - d_0));
      det = pw2(s) - 4.0 * (d_2 + z_1 - t);
    }
    const double Q_2 = -0.5 * (-s + fsign(1.0, -s) * std::fabs(std::sqrt(det)));
    const double y_1 = Q_2 - b_3 / 4.0;
    const double y_2 = (d_2 + z_1 - t) / Q_2 - b_3 / 4.0;
    if (y_1 >= 1.0 && y_2 >= 1.0) Wnro = fmin2(y_1, y_2);
    if (y_1 <= 1.0 && y_2 <= 1.0) st |= ST_C2P_FAIL;
    if (y_1 >= 1.0 && y_2 <= 1.0) Wnro = y_1;
    if (y_1 <= 1.0 && y_2 >= 1.0) Wnro = y_2;
    // Newton-Raphson polish of W (12_varprimitive.f95:510-526)
    int nrw = 1;
    double CHA1 = 1.0;
    while (CHA1 > TOL && nrw < nrmax) {
      const double Wnr = Wnro - (pw4(Wnro) + b_3 * pw3(Wnro) + b_2 * pw2(Wnro) + b_1 * Wnro + b_0) /
                                (4.0 * pw3(Wnro) + 3.0 * b_3 * pw2(Wnro) + 2.0 * b_2 * Wnro + b_1);
      CHA1 = std::fabs(Wnr - Wnro) / (0.5 * (Wnr + Wnro));
      Wnro = Wnr;
      nrw = nrw + 1;
    }
    W_elec = Wnro;
    rho_elec = D_elec / W_elec;
    if (rho_elec < 0.0) {  // 12_varprimitive.f95:536-548
      if (cnt) cnt[0] += 1;
      rho_elec = fmax2(in.rho0 * 1.0e-1, rho_elec);
    }
    enthpy_elec = (tau_elec - E2B2 - gamma_1 * rho_elec) / (pw2(W_elec) - gamma_1);
    p_elec = gamma_1 * (enthpy_elec - rho_elec);
    // "pressure NR" with frozen epsilon (12_varprimitive.f95:558-587)
    double pnro = p_elec;
    int nr = 1;
    const double epsilonnr = (tau_elec - E2B2 - D_elec * W_elec + pnro * (1.0 - pw2(W_elec))) / (D_elec * W_elec);
    const double Cs2 = (gamma * (gamma - 1.0) * epsilonnr) / (1.0 + gamma * epsilonnr);
    double CHA = 1.0;
    while (CHA >= TOL && nr <= nrmax) {
      const double pnr = pnro - ((gamma - 1.0) * rho_elec * epsilonnr - pnro) / (V2c * Cs2 - 1.0);
      CHA = std::fabs(pnr - pnro) / (0.5 * (pnr + pnro));
      pnro = pnr;
      nr = nr + 1;
    }
    if (pnro < 0.0) {  // 12_varprimitive.f95:592-607
      if (cnt) cnt[1] += 1;
      pnro = fmax2(in.p0 * 1.0e-4, pnro);
    }
    p_elec = pnro;
    tau_elec = E2B2 + enthpy_elec * pw2(W_elec) - p_elec;
    Vx_elec = (Sx_elec - Ey_elec_0 * Bz_elec + Ez_elec_0 * By_elec) / (tau_elec - E2B2 + p_elec);
    Vy_elec = (Sy_elec - Ez_elec_0 * Bx_elec + Ex_elec_0 * Bz_elec) / (tau_elec - E2B2 + p_elec);
    Vz_elec = (Sz_elec - Ex_elec_0 * By_elec + Ey_elec_0 * Bx_elec) / (tau_elec - E2B2 + p_elec);
    V2c = pw2(Vx_elec) + pw2(Vy_elec) + pw2(Vz_elec);
    W_elec = 1.0 / std::sqrt(1.0 - V2c);
    if (V2c >= 1.0) {  // 12_varprimitive.f95:627-696
      const double ErotB = Ey_elec_0 * Bz_elec - Ez_elec_0 * By_elec + Ez_elec_0 * Bx_elec - Ex_elec_0 * Bz_elec +
                           Ex_elec_0 * By_elec - Ey_elec_0 * Bx_elec;
      const double B2_drift = pw2(Bx_elec) + pw2(By_elec) + pw2(Bz_elec);
      if (B2_drift / rho_elec >= 10.0) {
        const double v_drift = ErotB / B2_drift;
        const double W_drift = 1.0 / std::sqrt(1.0 - pw2(v_drift));
        rho_elec = D_elec / W_drift;
        enthpy_elec = (tau_elec - E2B2 - gamma_1 * rho_elec) / (pw2(W_drift) - gamma_1);
        p_elec = gamma_1 * (enthpy_elec - rho_elec);
        tau_elec = E2B2 + enthpy_elec * pw2(W_elec) - p_elec;
        Vx_elec = (Sx_elec - Ey_elec_0 * Bz_elec + Ez_elec_0 * By_elec) / (tau_elec - E2B2 + p_elec);
        Vy_elec = (Sy_elec - Ez_elec_0 * Bx_elec + Ex_elec_0 * Bz_elec) / (tau_elec - E2B2 + p_elec);
        Vz_elec = (Sz_elec - Ex_elec_0 * By_elec + Ey_elec_0 * Bx_elec) / (tau_elec - E2B2 + p_elec);
        V2c = pw2(Vx_elec) + pw2(Vy_elec) + pw2(Vz_elec);
        W_elec = 1.0 / std::sqrt(1.0 - V2c);
        if (cnt) cnt[2] += 1;
        if (V2c >= 1.0) st |= ST_SUPERLUMINAL;
      } else {
        st |= ST_SUPERLUMINAL;
      }
    }
    Vx_elec_0 = Vx_elec; Vy_elec_0 = Vy_elec; Vz_elec_0 = Vz_elec;  // label 111
  }
  o.vx = Vx_elec_0; o.vy = Vy_elec_0; o.vz = Vz_elec_0;
  o.rho = rho_elec; o.p = p_elec; o.W = W_elec;
  return st;
}

// 12_varprimitive_nr.f95:28-338 with l_swap = 1, REC_ELEC = 0
int32_t c2p_nr(const C2PIn& in, double gamma, C2POut& o) {
  int32_t st = 0;
  const double TOL = 1.0e-10;
  const int nrmax = 40;
  const double Ex = in.Ex, Ey = in.Ey, Ez = in.Ez, Bx = in.Bx, By = in.By, Bz = in.Bz;
  const double D = in.D, tau = in.tau, Sx = in.Sx, Sy = in.Sy, Sz = in.Sz;
  double p_elec = in.p0;
  const double E2B2 = 0.5 * (pw2(Ex) + pw2(Ey) + pw2(Ez) + pw2(Bx) + pw2(By) + pw2(Bz));
  double Vx = (Sx - Ey * Bz + Ez * By) / (tau - E2B2 + p_elec);
  double Vy = (Sy - Ez * Bx + Ex * Bz) / (tau - E2B2 + p_elec);
  double Vz = (Sz - Ex * By + Ey * Bx) / (tau - E2B2 + p_elec);
  double V2c = pw2(Vx) + pw2(Vy) + pw2(Vz);
  double W = 1.0 / std::sqrt(1.0 - V2c);
  double W_2 = 1.0 / (1.0 - V2c);
  double rho = D / W;
  const double epsilonnr = (tau - E2B2 - D * W + p_elec * (1.0 - W_2)) / (D * W);
  const double Cs2 = (gamma * (gamma - 1.0) * epsilonnr) / (1.0 + gamma * epsilonnr);
  double CHA = 1.0;
  int nr = 1;
  double pnro = p_elec;
  while (CHA >= TOL && nr <= nrmax) {
    const double pnr = pnro - ((gamma - 1.0) * rho * epsilonnr - pnro) / (V2c * Cs2 - 1.0);
    CHA = std::fabs(pnr - pnro) / (0.5 * (pnr + pnro));
    pnro = pnr;
    nr = nr + 1;
  }
  p_elec = pnro;
  Vx = (Sx - Ey * Bz + Ez * By) / (tau - E2B2 + p_elec);
  Vy = (Sy - Ez * Bx + Ex * Bz) / (tau - E2B2 + p_elec);
  Vz = (Sz - Ex * By + Ey * Bx) / (tau - E2B2 + p_elec);
  V2c = pw2(Vx) + pw2(Vy) + pw2(Vz);
  W = 1.0 / std::sqrt(1.0 - V2c);
  W_2 = 1.0 / (1.0 - V2c);
  (void)W_2;
  rho = D / W;
  if (V2c >= 1.0) st |= ST_SUPERLUMINAL;
  o.vx = Vx; o.vy = Vy; o.vz = Vz; o.rho = rho; o.p = p_elec; o.W = W;
  return st;
}

// ------------------------------------------------------------------ state
struct Arr {
  std::vector<double> v;
};

struct Oracle {
  oracle_params P;
  int imax, jmax, nxg, nyg;
  size_t ng;
  double Delx, Dely, Delz, Delt, kappa_psi, kappa_phi, gamma, sigma;
  double eps1_c2p;
  Tableau T;
  int lmax;
  int32_t status = 0;
  int64_t counters[3] = {0, 0, 0};

  std::map<std::string, std::vector<double>> A;    // named ghosted arrays
  std::vector<std::map<std::string, std::vector<double>>> K;  // per-stage fluxes/sources

  size_t id(int i, int j) const { return (size_t)(i + 6) + (size_t)(j + 6) * nxg; }
  double* a(const char* n) { return A[n].data(); }

  void alloc(const char* n) { A[n].assign(ng, 0.0); }

  // ghost map: copy (clamp to [0,N]) or periodic (node duplicate: -k -> N-k, N+k -> k)
  int mapi(int i) const {
    if (i >= 0 && i <= imax) return i;
    if (P.bc_x == 1) return i < 0 ? i + imax : i - imax;
    return i < 0 ? 0 : imax;
  }
  int mapj(int j) const {
    if (j >= 0 && j <= jmax) return j;
    if (P.bc_y == 1) return j < 0 ? j + jmax : j - jmax;
    return j < 0 ? 0 : jmax;
  }
  // composite of the per-axis ghost fills (same final values for the y-then-x
  // order of 04_boundary.f95:2867-3033 and the x-then-y order of
  // 24_boundary_flux_conserved.f95:2088-2788 when imax, jmax >= 6)
  void fill_ghosts(double* f) {
    for (int j = -6; j <= jmax + 6; ++j)
      for (int i = -6; i <= imax + 6; ++i) {
        if (i >= 0 && i <= imax && j >= 0 && j <= jmax) continue;
        f[id(i, j)] = f[id(mapi(i), mapj(j))];
      }
  }

  explicit Oracle(const oracle_params& p) : P(p) {
    imax = p.imax; jmax = p.jmax;
    nxg = imax + 13; nyg = jmax + 13; ng = (size_t)nxg * nyg;
    Delx = p.lx / (double)imax;             // parameters.f95:306-308
    Dely = p.ly / (double)jmax;
    Delz = p.lz / 1.0;
    const double mn = fmin2(fmin2(Delx, Dely), Delz);
    Delt = (p.dt > 0.0) ? p.dt : p.cfl * mn; // parameters.f95:312
    const double cp_psi = std::sqrt(fmin2(Delx, Dely) / 1.0);  // parameters.f95:329-334
    const double cp_phi = std::sqrt(fmin2(Delx, Dely) / 1.0);
    kappa_psi = 1.0 / pw2(cp_psi);
    kappa_phi = 1.0 / pw2(cp_phi);
    gamma = p.gamma; sigma = p.sigma;
    // value the module variable eps1 holds when con2prim runs (set last by the flux routine)
    // (the Lax routine of flux_solver 1 and the MCL routine of flux_solver 2
    // never set it: the zero-initialised module variable; only the
    // superluminal seed clamp reads it)
    eps1_c2p = (p.flux_solver == 7) ? (double)1.0e-6f : (p.flux_solver <= 2 ? 0.0 : 1.0e-6);
    make_tableau(p.order, T);
    lmax = T.s;
    const char* names[] = {
      "psi", "phi", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "Vx", "Vy", "Vz", "q", "p", "rho",
      "V2", "W", "E2", "B2", "epsiln", "enthpy", "D", "tau", "Sx", "Sy", "Sz",
      "psiintsum", "phiintsum", "Bxintsum", "Byintsum", "Bzintsum", "Exastsum", "Eyastsum", "Ezastsum",
      "qintsum", "Dintsum", "tauintsum", "Sxintsum", "Syintsum", "Szintsum",
      "psifinsum", "phifinsum", "Bxfinsum", "Byfinsum", "Bzfinsum", "Exfinsum", "Eyfinsum", "Ezfinsum",
      "qfinsum", "Dfinsum", "taufinsum", "Sxfinsum", "Syfinsum", "Szfinsum",
      "psiint", "phiint", "Exast", "Eyast", "Ezast", "Exint", "Eyint", "Ezint", "Bxint", "Byint", "Bzint",
      "qint", "DDint", "tauint", "Sxint", "Syint", "Szint", "Jxint", "Jyint", "Jzint",
      // interface fluxes (16_*_flow_mpx.f95 outputs read by 17_fluxandsource.f95)
      "Exlaxpsi", "Eylaxpsi", "Bxlaxphi", "Bylaxphi", "philaxBx", "EzlaxBx", "EzlaxBy", "philaxBy",
      "EylaxBz", "ExlaxBz", "psilaxEx", "BzlaxEx", "BzlaxEy", "psilaxEy", "BylaxEz", "BxlaxEz",
      "Jxlax", "Jylax", "FDxlax", "FDylax", "Ftauxlax", "Ftauylax",
      "FSxxlax", "FSxylax", "FSxzlax", "FSyxlax", "FSyylax", "FSyzlax"};
    for (const char* n : names) alloc(n);
    K.resize(lmax);
    const char* kn[] = {"psiflux", "phiflux", "Bxflux", "Byflux", "Bzflux", "Exastflux", "Eyastflux",
                        "Ezastflux", "qflux", "Dflux", "tauflux", "Sxflux", "Syflux", "Szflux",
                        "Exastsour", "Eyastsour", "Ezastsour"};
    for (int l = 0; l < lmax; ++l)
      for (const char* n : kn) K[l][n].assign(ng, 0.0);
  }

  // ------------------------------------------------- 06_conserved_var.f95:79-140
  void startconvar() {
    double *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz"), *Ex = a("Ex"), *Ey = a("Ey"), *Ez = a("Ez");
    double *Bx = a("Bx"), *By = a("By"), *Bz = a("Bz"), *p = a("p"), *rho = a("rho");
    double *V2 = a("V2"), *W = a("W"), *E2 = a("E2"), *B2 = a("B2"), *eps = a("epsiln"), *h = a("enthpy");
    double *D = a("D"), *tau = a("tau"), *Sx = a("Sx"), *Sy = a("Sy"), *Sz = a("Sz");
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j);
        V2[k] = pw2(Vx[k]) + pw2(Vy[k]) + pw2(Vz[k]);
        W[k] = 1.0 / std::sqrt(1.0 - V2[k]);
        E2[k] = pw2(Ex[k]) + pw2(Ey[k]) + pw2(Ez[k]);
        B2[k] = pw2(Bx[k]) + pw2(By[k]) + pw2(Bz[k]);
        eps[k] = p[k] / ((gamma - 1.0) * rho[k]);
        h[k] = rho[k] * (1.0 + eps[k]) + p[k];
        D[k] = rho[k] * W[k];
        tau[k] = 0.5 * (E2[k] + B2[k]) + h[k] * pw2(W[k]) - p[k];
        Sx[k] = (Bz[k] * Ey[k] - By[k] * Ez[k]) + h[k] * pw2(W[k]) * Vx[k];
        Sy[k] = (Bx[k] * Ez[k] - Bz[k] * Ex[k]) + h[k] * pw2(W[k]) * Vy[k];
        Sz[k] = (By[k] * Ex[k] - Bx[k] * Ey[k]) + h[k] * pw2(W[k]) * Vz[k];
      }
  }

  // ---------------------------------------------------- 07_clean_var.f95:18-58
  void cleanvarint() {
    const char* s[] = {"psiintsum", "phiintsum", "Bxintsum", "Byintsum", "Bzintsum", "Exastsum", "Eyastsum",
                       "Ezastsum", "qintsum", "Dintsum", "tauintsum", "Sxintsum", "Syintsum", "Szintsum",
                       "psifinsum", "phifinsum", "Bxfinsum", "Byfinsum", "Bzfinsum", "Exfinsum", "Eyfinsum",
                       "Ezfinsum", "qfinsum", "Dfinsum", "taufinsum", "Sxfinsum", "Syfinsum", "Szfinsum"};
    for (const char* n : s) std::fill(A[n].begin(), A[n].end(), 0.0);
  }

  // ------------------------------------------------------- 09_sumint.f95:18-67
  // EGLM terms carry FAC_EGLM = 0 (parameters.f95:44) and are dropped.
  void sumint(int l, int m) {  // l, m are 1-based like the Fortran
    const double ab = T.Ab[l - 1][m - 1], abt = T.Abt[l - 1][m - 1];
    auto& Km = K[m - 1];
    const char* s[] = {"psiintsum", "phiintsum", "Bxintsum", "Byintsum", "Bzintsum", "qintsum", "Dintsum",
                       "tauintsum", "Sxintsum", "Syintsum", "Szintsum"};
    const char* f[] = {"psiflux", "phiflux", "Bxflux", "Byflux", "Bzflux", "qflux", "Dflux",
                       "tauflux", "Sxflux", "Syflux", "Szflux"};
    for (int c = 0; c < 11; ++c) {
      double* S = a(s[c]);
      const double* F = Km[f[c]].data();
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); S[k] = S[k] + ab * F[k]; }
    }
    const char* es[] = {"Exastsum", "Eyastsum", "Ezastsum"};
    const char* ef[] = {"Exastflux", "Eyastflux", "Ezastflux"};
    const char* eo[] = {"Exastsour", "Eyastsour", "Ezastsour"};
    for (int c = 0; c < 3; ++c) {
      double* S = a(es[c]);
      const double* F = Km[ef[c]].data();
      const double* O = Km[eo[c]].data();
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); S[k] = S[k] + (ab * F[k] - abt * O[k]); }
    }
  }

  // -------------------------------------------------------- 10_varint.f95:18-72
  void varint() {
    const char* dst[] = {"psiint", "phiint", "Bxint", "Byint", "Bzint", "Exast", "Eyast", "Ezast",
                         "qint", "DDint", "tauint", "Sxint", "Syint", "Szint"};
    const char* src[] = {"psi", "phi", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "q", "D", "tau", "Sx", "Sy", "Sz"};
    const char* sum[] = {"psiintsum", "phiintsum", "Bxintsum", "Byintsum", "Bzintsum", "Exastsum", "Eyastsum",
                         "Ezastsum", "qintsum", "Dintsum", "tauintsum", "Sxintsum", "Syintsum", "Szintsum"};
    for (int c = 0; c < 14; ++c) {
      double* d = a(dst[c]);
      const double* s = a(src[c]);
      const double* S = a(sum[c]);
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); d[k] = s[k] + Delt * S[k]; }
    }
    const char* bc[] = {"psiint", "phiint", "Bxint", "Byint", "Bzint", "qint", "DDint", "tauint",
                        "Sxint", "Syint", "Szint"};
    for (const char* n : bc) fill_ghosts(a(n));   // boundary_conserved
  }

  // ------------------------------------------- 11_elecvarint.f95:279-328 (IMEX)
  // a(l) and matx(l) are per-cell temporaries here (the Fortran shares them
  // between OpenMP threads, 11_elecvarint.f95:13).
  void electricvarint(int l) {
    const double abtll = T.Abt[l - 1][l - 1];
    double *W = a("W"), *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz");
    double *Bx = a("Bxint"), *By = a("Byint"), *Bz = a("Bzint");
    double *Exa = a("Exast"), *Eya = a("Eyast"), *Eza = a("Ezast");
    double *Exi = a("Exint"), *Eyi = a("Eyint"), *Ezi = a("Ezint");
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j);
        const double al = abtll * sigma * Delt;
        const double Wk = W[k], vx = Vx[k], vy = Vy[k], vz = Vz[k];
        const double matx = pw2(Wk) * al + Wk * pw2(al) + Wk + al;
        const double vrotB_x = (Bz[k] * vy - By[k] * vz);
        const double vrotB_y = (Bx[k] * vz - Bz[k] * vx);
        const double vrotB_z = (By[k] * vx - Bx[k] * vy);
        Exi[k] = (1.0 / matx) * (
            (al + Wk + al * pw2(Wk) * pw2(vx)) * Exa[k] +
            al * pw2(Wk) * vx * vy * Eya[k] +
            al * pw2(Wk) * vx * vz * Eza[k] -
            abtll * sigma * Wk * Delt * (
              (al + Wk + al * pw2(Wk) * pw2(vx)) * vrotB_x +
              al * pw2(Wk) * vx * vy * vrotB_y +
              al * pw2(Wk) * vx * vz * vrotB_z));
        Eyi[k] = (1.0 / matx) * (
            al * pw2(Wk) * vx * vy * Exa[k] +
            (al + Wk + al * pw2(Wk) * pw2(vy)) * Eya[k] +
            al * pw2(Wk) * vy * vz * Eza[k] -
            abtll * sigma * Wk * Delt * (
              al * pw2(Wk) * vx * vy * vrotB_x +
              (al + Wk + al * pw2(Wk) * pw2(vy)) * vrotB_y +
              al * pw2(Wk) * vy * vz * vrotB_z));
        Ezi[k] = (1.0 / matx) * (
            al * pw2(Wk) * vx * vz * Exa[k] +
            al * pw2(Wk) * vy * vz * Eya[k] +
            (al + Wk + al * pw2(Wk) * pw2(vz)) * Eza[k] -
            abtll * sigma * Wk * Delt * (
              al * pw2(Wk) * vx * vz * vrotB_x +
              al * pw2(Wk) * vy * vz * vrotB_y +
              (al + Wk + al * pw2(Wk) * pw2(vz)) * vrotB_z));
      }
    fill_ghosts(Exi); fill_ghosts(Eyi); fill_ghosts(Ezi);   // boundary_electric
  }

  // ------------------------------------------- 14_flowinit.f95:264-302 (J only;
  // the centre fluxes are only read when flux_rec_mp5 = 1)
  void flowinit() {
    double *W = a("W"), *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz");
    double *Ex = a("Exint"), *Ey = a("Eyint"), *Ez = a("Ezint");
    double *Bx = a("Bxint"), *By = a("Byint"), *Bz = a("Bzint"), *q = a("qint");
    double *Jx = a("Jxint"), *Jy = a("Jyint"), *Jz = a("Jzint");
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j);
        const double Edotv = Ex[k] * Vx[k] + Ey[k] * Vy[k] + Ez[k] * Vz[k];
        const double vrotB_x = (Bz[k] * Vy[k] - By[k] * Vz[k]);
        const double vrotB_y = (Bx[k] * Vz[k] - Bz[k] * Vx[k]);
        const double vrotB_z = (By[k] * Vx[k] - Bx[k] * Vy[k]);
        Jx[k] = sigma * W[k] * (Ex[k] + vrotB_x - Edotv * Vx[k]) + q[k] * Vx[k];
        Jy[k] = sigma * W[k] * (Ey[k] + vrotB_y - Edotv * Vy[k]) + q[k] * Vy[k];
        Jz[k] = sigma * W[k] * (Ez[k] + vrotB_z - Edotv * Vz[k]) + q[k] * Vz[k];
      }
    fill_ghosts(Jx); fill_ghosts(Jy); fill_ghosts(Jz);   // boundary_flux_conserved
  }

  // ----------------------------------------- reconstruction passes (MPX 2D)
  // x slots of 16_hll_flow_mpx.f95:784-894 and y slots of :1086-1197
  enum XS { X_PSI = 0, X_PHI, X_EX, X_EY, X_EZ, X_EXM, X_EYM, X_EZM, X_BX, X_BY, X_BZ, X_BXM, X_BYM, X_BZM,
            X_Q, X_D, X_TAU, X_SX, X_SY, X_SZ, X_VX, X_VY, X_VZ, X_P, X_RHO, X_JX, X_JZ, X_N };
  enum YS { Y_PSI = 0, Y_PHI, Y_EX, Y_EY, Y_EZ, Y_EXM, Y_EYM, Y_EZM, Y_BX, Y_BY, Y_BZ, Y_BXM, Y_BYM, Y_BZM,
            Y_Q, Y_D, Y_TAU, Y_SX, Y_SY, Y_SZ, Y_VX, Y_VY, Y_VZ, Y_P, Y_RHO, Y_JY, Y_N };
  std::vector<std::vector<double>> XL, XR, YL, YR;   // [slot][ghosted 2D]

  void slot_src(int slot, bool xdir, const double*& src, double& sgn) {
    sgn = 1.0;
    // identical ordering for x and y up to the current slot
    switch (slot) {
      case X_PSI: src = a("psiint"); break;
      case X_PHI: src = a("phiint"); break;
      case X_EX: src = a("Exint"); break;
      case X_EY: src = a("Eyint"); break;
      case X_EZ: src = a("Ezint"); break;
      case X_EXM: src = a("Exint"); sgn = -1.0; break;
      case X_EYM: src = a("Eyint"); sgn = -1.0; break;
      case X_EZM: src = a("Ezint"); sgn = -1.0; break;
      case X_BX: src = a("Bxint"); break;
      case X_BY: src = a("Byint"); break;
      case X_BZ: src = a("Bzint"); break;
      case X_BXM: src = a("Bxint"); sgn = -1.0; break;
      case X_BYM: src = a("Byint"); sgn = -1.0; break;
      case X_BZM: src = a("Bzint"); sgn = -1.0; break;
      case X_Q: src = a("qint"); break;
      case X_D: src = a("DDint"); break;
      case X_TAU: src = a("tauint"); break;
      case X_SX: src = a("Sxint"); break;
      case X_SY: src = a("Syint"); break;
      case X_SZ: src = a("Szint"); break;
      case X_VX: src = a("Vx"); break;
      case X_VY: src = a("Vy"); break;
      case X_VZ: src = a("Vz"); break;
      case X_P: src = a("p"); break;
      case X_RHO: src = a("rho"); break;
      case X_JX: src = xdir ? a("Jxint") : a("Jyint"); break;   // slot 26 (x) / 63 (y)
      case X_JZ: src = a("Jzint"); break;                      // slot 27 (x only)
      default: src = nullptr;
    }
  }

  // --------------------- second-order MC reconstruction (16_hll_flow_mcl.f95:565-1112)
  // face i+1/2 of a line: L = u(i) + FAC mcl(u(i+1)-u(i), u(i)-u(i-1)),
  // R = u(i+1) - FAC mcl(u(i+2)-u(i+1), u(i+1)-u(i)) with FAC = FAC_SR = 0.5
  // (parameters.f95:42-43) and mcl the monotonized-central slope (slop = 2,
  // funciones.f95:56-95).  The "_m" values of E and B keep the slope's sign
  // and negate only the cell value: L_m = -u(i) + FAC mcl(...),
  // R_m = -u(i+1) - FAC mcl(...) (:655-667, :708-735), which is not -L / -R.
  void mcl_line(int n, const double* u, bool negate, double* L, double* R) {
    for (int i = -1; i <= n + 1; ++i) {
      const double um1 = u[i - 1 + 6], u0 = u[i + 6], u1 = u[i + 1 + 6], u2 = u[i + 2 + 6];
      const double sl = 0.5 * limiter_mc(u1 - u0, u0 - um1);
      const double sr = 0.5 * limiter_mc(u2 - u1, u1 - u0);
      L[i + 6] = negate ? -u0 + sl : u0 + sl;
      R[i + 6] = negate ? -u1 - sr : u1 - sr;
    }
  }
  void reconstruct_mcl() {
    XL.assign(X_N, std::vector<double>(ng, 0.0)); XR.assign(X_N, std::vector<double>(ng, 0.0));
    YL.assign(Y_N, std::vector<double>(ng, 0.0)); YR.assign(Y_N, std::vector<double>(ng, 0.0));
#pragma omp parallel
    {
      std::vector<double> u(imax + 13), L(imax + 13), R(imax + 13);
#pragma omp for schedule(static)
      for (int jj = -1; jj <= jmax + 1; ++jj)
        for (int s = 0; s < X_JX; ++s) {
          const double* src; double sg;
          slot_src(s, true, src, sg);
          for (int i = -6; i <= imax + 6; ++i) u[i + 6] = src[id(i, jj)];
          mcl_line(imax, u.data(), sg < 0, L.data(), R.data());
          for (int i = -1; i <= imax + 1; ++i) { XL[s][id(i, jj)] = L[i + 6]; XR[s][id(i, jj)] = R[i + 6]; }
        }
    }
#pragma omp parallel
    {
      std::vector<double> u(jmax + 13), L(jmax + 13), R(jmax + 13);
#pragma omp for schedule(static)
      for (int ii = -1; ii <= imax + 1; ++ii)
        for (int s = 0; s < Y_JY; ++s) {
          const double* src; double sg;
          slot_src(s, false, src, sg);
          for (int j = -6; j <= jmax + 6; ++j) u[j + 6] = src[id(ii, j)];
          mcl_line(jmax, u.data(), sg < 0, L.data(), R.data());
          for (int j = -1; j <= jmax + 1; ++j) { YL[s][id(ii, j)] = L[j + 6]; YR[s][id(ii, j)] = R[j + 6]; }
        }
    }
  }

  // ------------- Lax-Friedrichs flux with MC slopes (flux_solver 1), 15_lax_flow.f95:733-1457
  // Every cell (ghosts included) carries the pair p = F + Sp U, m = F - Sp U
  // of each flux F and the conserved variable U it transports, with Sp = 1
  // (const_sp = 0, parameters.f95:274).  Face i+1/2 of a line:
  //   L = p(i)   + FAC mcl(p(i+1) - p(i),   p(i)   - p(i-1))
  //   R = m(i+1) - FAC mcl(p(i+2) - p(i+1), p(i+1) - p(i))      (slopes of p on both sides)
  //   F(i+1/2) = 0.5 (L + R), negated for EzlaxBy, ExlaxBz, BzlaxEx, BylaxEz,
  // whose cell flux is written with the opposite sign (-Ez + By, ...).
  // F of the fluid comes from flowinit (14_flowinit.f95:258-360): stage
  // E, B, D, S with the time-n v, W, enthpy and p, computed on the interior
  // and copied to the ghosts by boundary_flux_conserved; the current F is
  // the stage J of flowinit.
  void lax_flow() {
    double *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz"), *W = a("W"), *h = a("enthpy"), *p = a("p");
    double *Ex = a("Exint"), *Ey = a("Eyint"), *Ez = a("Ezint"), *Bx = a("Bxint"), *By = a("Byint"),
           *Bz = a("Bzint"), *DD = a("DDint");
    enum { FDX, FDY, FTX, FTY, FSXX, FSXY, FSXZ, FSYX, FSYY, FSYZ, NCF };
    std::vector<std::vector<double>> cf(NCF, std::vector<double>(ng, 0.0));
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j);
        const double E2 = pw2(Ex[k]) + pw2(Ey[k]) + pw2(Ez[k]);
        const double B2 = pw2(Bx[k]) + pw2(By[k]) + pw2(Bz[k]);
        const double hW2 = h[k] * pw2(W[k]);
        cf[FDX][k] = DD[k] * Vx[k];
        cf[FDY][k] = DD[k] * Vy[k];
        cf[FTX][k] = (Bz[k] * Ey[k] - By[k] * Ez[k]) + hW2 * Vx[k];
        cf[FTY][k] = (Bx[k] * Ez[k] - Bz[k] * Ex[k]) + hW2 * Vy[k];
        cf[FSXX][k] = -pw2(Ex[k]) - pw2(Bx[k]) + hW2 * pw2(Vx[k]) + 0.5 * (E2 + B2) + p[k];
        cf[FSXY][k] = -Ex[k] * Ey[k] - Bx[k] * By[k] + hW2 * Vx[k] * Vy[k];
        cf[FSXZ][k] = -Ex[k] * Ez[k] - Bx[k] * Bz[k] + hW2 * Vx[k] * Vz[k];
        cf[FSYX][k] = -Ex[k] * Ey[k] - Bx[k] * By[k] + hW2 * Vx[k] * Vy[k];
        cf[FSYY][k] = -pw2(Ey[k]) - pw2(By[k]) + hW2 * pw2(Vy[k]) + 0.5 * (E2 + B2) + p[k];
        cf[FSYZ][k] = -Ey[k] * Ez[k] - By[k] * Bz[k] + hW2 * Vy[k] * Vz[k];
      }
    for (auto& f : cf) fill_ghosts(f.data());
    struct Pairing { const double* F; bool negF; const double* U; bool ydir; bool negface; };
    const double *psi = a("psiint"), *phi = a("phiint"), *q = a("qint"), *tau = a("tauint");
    const double *Sx = a("Sxint"), *Sy = a("Syint"), *Sz = a("Szint");
    const Pairing pr[28] = {
        {Ex, false, psi, false, false},              // Exlaxpsi
        {Ey, false, psi, true, false},               // Eylaxpsi
        {Bx, false, phi, false, false},              // Bxlaxphi
        {By, false, phi, true, false},               // Bylaxphi
        {phi, false, Bx, false, false},              // philaxBx
        {Ez, false, Bx, true, false},                // EzlaxBx
        {Ez, true, By, false, true},                 // EzlaxBy
        {phi, false, By, true, false},               // philaxBy
        {Ey, false, Bz, false, false},               // EylaxBz
        {Ex, true, Bz, true, true},                  // ExlaxBz
        {psi, false, Ex, false, false},              // psilaxEx
        {Bz, true, Ex, true, true},                  // BzlaxEx
        {Bz, false, Ey, false, false},               // BzlaxEy
        {psi, false, Ey, true, false},               // psilaxEy
        {By, true, Ez, false, true},                 // BylaxEz
        {Bx, false, Ez, true, false},                // BxlaxEz
        {a("Jxint"), false, q, false, false},        // Jxlax
        {a("Jyint"), false, q, true, false},         // Jylax
        {cf[FDX].data(), false, DD, false, false},   // FDxlax
        {cf[FDY].data(), false, DD, true, false},    // FDylax
        {cf[FTX].data(), false, tau, false, false},  // Ftauxlax
        {cf[FTY].data(), false, tau, true, false},   // Ftauylax
        {cf[FSXX].data(), false, Sx, false, false},  // FSxxlax
        {cf[FSXY].data(), false, Sy, false, false},  // FSxylax
        {cf[FSXZ].data(), false, Sz, false, false},  // FSxzlax
        {cf[FSYX].data(), false, Sx, true, false},   // FSyxlax
        {cf[FSYY].data(), false, Sy, true, false},   // FSyylax
        {cf[FSYZ].data(), false, Sz, true, false}};  // FSyzlax
    const char* on[] = {"Exlaxpsi", "Eylaxpsi", "Bxlaxphi", "Bylaxphi", "philaxBx", "EzlaxBx", "EzlaxBy",
                        "philaxBy", "EylaxBz", "ExlaxBz", "psilaxEx", "BzlaxEx", "BzlaxEy", "psilaxEy",
                        "BylaxEz", "BxlaxEz", "Jxlax", "Jylax", "FDxlax", "FDylax", "Ftauxlax", "Ftauylax",
                        "FSxxlax", "FSxylax", "FSxzlax", "FSyxlax", "FSyylax", "FSyzlax"};
    const double Sp = 1.0;
    for (int c = 0; c < 28; ++c) {
      const Pairing& P2 = pr[c];
      double* o = a(on[c]);
      auto pv = [&](size_t k) { return (P2.negF ? -P2.F[k] : P2.F[k]) + Sp * P2.U[k]; };
      auto mv = [&](size_t k) { return (P2.negF ? -P2.F[k] : P2.F[k]) - Sp * P2.U[k]; };
#pragma omp parallel for schedule(static)
      for (int j = -1; j <= jmax; ++j)
        for (int i = -1; i <= imax; ++i) {
          auto at = [&](int s) { return P2.ydir ? id(i, j + s) : id(i + s, j); };
          const double pm1 = pv(at(-1)), p0 = pv(at(0)), p1 = pv(at(1)), p2 = pv(at(2));
          const double L = p0 + 0.5 * limiter_mc(p1 - p0, p0 - pm1);
          const double R = mv(at(1)) - 0.5 * limiter_mc(p2 - p1, p1 - p0);
          o[id(i, j)] = P2.negface ? -(0.5 * (L + R)) : 0.5 * (L + R);
        }
    }
  }

  void reconstruct() {
    if (P.flux_solver == 1) return;   // lax_flow works on the cell pairs directly
    if (P.flux_solver >= 2 && P.flux_solver <= 4) { reconstruct_mcl(); return; }
    const int rec = P.rec_mp;
    XL.assign(X_N, std::vector<double>(ng, 0.0)); XR.assign(X_N, std::vector<double>(ng, 0.0));
    YL.assign(Y_N, std::vector<double>(ng, 0.0)); YR.assign(Y_N, std::vector<double>(ng, 0.0));
    // x pass: lines imp = -1..jmax+1 (16_hll_flow_mpx.f95:781)
#pragma omp parallel
    {
      std::vector<double> u(imax + 13), up(imax + 13), um(imax + 13);
#pragma omp for schedule(static)
      for (int jj = -1; jj <= jmax + 1; ++jj) {
        for (int s = 0; s < X_N; ++s) {
          const double* src; double sg;
          slot_src(s, true, src, sg);
          for (int i = -6; i <= imax + 6; ++i) u[i + 6] = (sg < 0) ? -src[id(i, jj)] : src[id(i, jj)];
          mp_line(rec, imax, u.data(), (s == X_P || s == X_RHO), up.data(), um.data());
          for (int i = -1; i <= imax + 1; ++i) {    // :942-1036
            XL[s][id(i, jj)] = up[i + 6];
            XR[s][id(i, jj)] = um[i + 1 + 6];
          }
        }
      }
    }
    // y pass: lines imp = -1..imax+1 (16_hll_flow_mpx.f95:1083)
#pragma omp parallel
    {
      std::vector<double> u(jmax + 13), up(jmax + 13), um(jmax + 13);
#pragma omp for schedule(static)
      for (int ii = -1; ii <= imax + 1; ++ii) {
        for (int s = 0; s < Y_N; ++s) {
          const double* src; double sg;
          slot_src(s, false, src, sg);
          for (int j = -6; j <= jmax + 6; ++j) u[j + 6] = (sg < 0) ? -src[id(ii, j)] : src[id(ii, j)];
          mp_line(rec, jmax, u.data(), (s == Y_P || s == Y_RHO), up.data(), um.data());
          for (int j = -1; j <= jmax + 1; ++j) {    // :1240-1329
            YL[s][id(ii, j)] = up[j + 6];
            YR[s][id(ii, j)] = um[j + 1 + 6];
          }
        }
      }
    }
  }

  // per-interface reconstructed state of one side
  struct Side {
    double psi, phi, Ex, Ey, Ez, Exm, Eym, Ezm, Bx, By, Bz, Bxm, Bym, Bzm, q, D, tau, Sx, Sy, Sz;
    double vx, vy, vz, p, rho, J;   // J = Jx (x side) or Jy (y side)
  };
  Side side(const std::vector<std::vector<double>>& R, size_t k) {
    Side s;
    s.psi = R[X_PSI][k]; s.phi = R[X_PHI][k];
    s.Ex = R[X_EX][k]; s.Ey = R[X_EY][k]; s.Ez = R[X_EZ][k];
    s.Exm = R[X_EXM][k]; s.Eym = R[X_EYM][k]; s.Ezm = R[X_EZM][k];
    s.Bx = R[X_BX][k]; s.By = R[X_BY][k]; s.Bz = R[X_BZ][k];
    s.Bxm = R[X_BXM][k]; s.Bym = R[X_BYM][k]; s.Bzm = R[X_BZM][k];
    s.q = R[X_Q][k]; s.D = R[X_D][k]; s.tau = R[X_TAU][k];
    s.Sx = R[X_SX][k]; s.Sy = R[X_SY][k]; s.Sz = R[X_SZ][k];
    s.vx = R[X_VX][k]; s.vy = R[X_VY][k]; s.vz = R[X_VZ][k];
    s.p = R[X_P][k]; s.rho = R[X_RHO][k]; s.J = R[X_JX][k];
    return s;
  }

  // physical fluxes of one side (16_hll_flow_mpx.f95:1464-1733, flux_rec_mp5 = 0)
  struct PhysX { double W, h, FD, Ftau, FSx, FSy, FSz; };
  PhysX physx(const Side& s) {  // x direction
    PhysX f;
    const double V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
    f.W = 1.0 / std::sqrt(1.0 - V2);
    const double E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
    const double eps = s.p / ((gamma - 1.0) * s.rho);
    f.h = s.rho * (1.0 + eps) + s.p;
    f.FD = s.D * s.vx;
    f.Ftau = (s.Bz * s.Ey - s.By * s.Ez) + f.h * pw2(f.W) * s.vx;
    f.FSx = -pw2(s.Ex) - pw2(s.Bx) + f.h * pw2(f.W) * pw2(s.vx) + 0.5 * E2B2 + s.p;
    f.FSy = -s.Ex * s.Ey - s.Bx * s.By + f.h * pw2(f.W) * s.vx * s.vy;
    f.FSz = -s.Ex * s.Ez - s.Bx * s.Bz + f.h * pw2(f.W) * s.vx * s.vz;
    return f;
  }
  PhysX physy(const Side& s) {  // y direction: FSx is FSyx, FSy is FSyy, FSz is FSyz
    PhysX f;
    const double V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
    f.W = 1.0 / std::sqrt(1.0 - V2);
    const double E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
    const double eps = s.p / ((gamma - 1.0) * s.rho);
    f.h = s.rho * (1.0 + eps) + s.p;
    f.FD = s.D * s.vy;
    f.Ftau = (s.Bx * s.Ez - s.Bz * s.Ex) + f.h * pw2(f.W) * s.vy;
    f.FSx = -s.Ex * s.Ey - s.Bx * s.By + f.h * pw2(f.W) * s.vx * s.vy;
    f.FSy = -pw2(s.Ey) - pw2(s.By) + f.h * pw2(f.W) * pw2(s.vy) + 0.5 * E2B2 + s.p;
    f.FSz = -s.Ey * s.Ez - s.By * s.Bz + f.h * pw2(f.W) * s.vy * s.vz;
    return f;
  }
  // HLLE variant of the physical fluxes: W from 1 - vx^2 - vy^2 - vz^2
  // (16_hlle_flow_mpx.f95:2289-2292)
  void hlle_w(PhysX& f, const Side& s) {
    f.W = 1.0 / std::sqrt(1.0 - pw2(s.vx) - pw2(s.vy) - pw2(s.vz));
  }

  static double hllf(double FL, double FR, double UL, double UR) {
    const double s1 = -1.0, s2 = 1.0;   // parameters.f95:283-284
    return (s2 * FL - s1 * FR + s1 * s2 * (UR - UL)) / (s2 - s1);
  }

  // HLL fluxes of the MC-reconstructed states (16_hll_flow_mcl.f95:1014-1396):
  // the same arrays as the MPX routines, with W = 1/sqrt(1 - vx^2 - vy^2 - vz^2)
  // (:900-905), the current J computed from the reconstructed states of
  // each side instead of reconstructed (:1026-1042), and the "_m" values in
  // the fluxes EzlaxBy, ExlaxBz, BylaxEz, BzlaxEx
  void mcl_fluxes(const Side& xl, const Side& xr, const Side& yl, const Side& yr, double* out) {
    PhysX fxl = physx(xl), fxr = physx(xr), fyl = physy(yl), fyr = physy(yr);
    hlle_w(fxl, xl); hlle_w(fxr, xr); hlle_w(fyl, yl); hlle_w(fyr, yr);
    fxl = physx_w(xl, fxl.W); fxr = physx_w(xr, fxr.W); fyl = physy_w(yl, fyl.W); fyr = physy_w(yr, fyr.W);
    auto jx = [&](const Side& s, double W) {
      const double vrotB = s.Bz * s.vy - s.By * s.vz;
      const double Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
      return sigma * W * (s.Ex + vrotB - Edotv * s.vx) + s.q * s.vx;
    };
    auto jy = [&](const Side& s, double W) {
      const double vrotB = s.Bx * s.vz - s.Bz * s.vx;
      const double Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
      return sigma * W * (s.Ey + vrotB - Edotv * s.vy) + s.q * s.vy;
    };
    out[0] = hllf(xl.Ex, xr.Ex, xl.psi, xr.psi);                 // Exlaxpsi
    out[1] = hllf(yl.Ey, yr.Ey, yl.psi, yr.psi);                 // Eylaxpsi
    out[2] = hllf(xl.Bx, xr.Bx, xl.phi, xr.phi);                 // Bxlaxphi
    out[3] = hllf(yl.By, yr.By, yl.phi, yr.phi);                 // Bylaxphi
    out[4] = hllf(xl.phi, xr.phi, xl.Bx, xr.Bx);                 // philaxBx
    out[5] = hllf(yl.Ez, yr.Ez, yl.Bx, yr.Bx);                   // EzlaxBx
    out[6] = -hllf(xl.Ezm, xr.Ezm, xl.By, xr.By);                // EzlaxBy
    out[7] = hllf(yl.phi, yr.phi, yl.By, yr.By);                 // philaxBy
    out[8] = hllf(xl.Ey, xr.Ey, xl.Bz, xr.Bz);                   // EylaxBz
    out[9] = -hllf(yl.Exm, yr.Exm, yl.Bz, yr.Bz);                // ExlaxBz
    out[10] = hllf(xl.psi, xr.psi, xl.Ex, xr.Ex);                // psilaxEx
    out[11] = -hllf(yl.Bzm, yr.Bzm, yl.Ex, yr.Ex);               // BzlaxEx
    out[12] = hllf(xl.Bz, xr.Bz, xl.Ey, xr.Ey);                  // BzlaxEy
    out[13] = hllf(yl.psi, yr.psi, yl.Ey, yr.Ey);                // psilaxEy
    out[14] = -hllf(xl.Bym, xr.Bym, xl.Ez, xr.Ez);               // BylaxEz
    out[15] = hllf(yl.Bx, yr.Bx, yl.Ez, yr.Ez);                  // BxlaxEz
    out[16] = hllf(jx(xl, fxl.W), jx(xr, fxr.W), xl.q, xr.q);    // Jxlax
    out[17] = hllf(jy(yl, fyl.W), jy(yr, fyr.W), yl.q, yr.q);    // Jylax
    out[18] = hllf(fxl.FD, fxr.FD, xl.D, xr.D);
    out[19] = hllf(fyl.FD, fyr.FD, yl.D, yr.D);
    out[20] = hllf(fxl.Ftau, fxr.Ftau, xl.tau, xr.tau);
    out[21] = hllf(fyl.Ftau, fyr.Ftau, yl.tau, yr.tau);
    out[22] = hllf(fxl.FSx, fxr.FSx, xl.Sx, xr.Sx);
    out[23] = hllf(fxl.FSy, fxr.FSy, xl.Sy, xr.Sy);
    out[24] = hllf(fxl.FSz, fxr.FSz, xl.Sz, xr.Sz);
    out[25] = hllf(fyl.FSx, fyr.FSx, yl.Sx, yr.Sx);
    out[26] = hllf(fyl.FSy, fyr.FSy, yl.Sy, yr.Sy);
    out[27] = hllf(fyl.FSz, fyr.FSz, yl.Sz, yr.Sz);
  }

  // ------------------------------------------- Riemann loop (2D, i=-1..imax, j=-1..jmax)
  void riemann() {
    const int solver = P.flux_solver;
    if (solver == 1) { lax_flow(); return; }
    double *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz"), *rho = a("rho");
    double* o[28];
    const char* on[] = {"Exlaxpsi", "Eylaxpsi", "Bxlaxphi", "Bylaxphi", "philaxBx", "EzlaxBx", "EzlaxBy",
                        "philaxBy", "EylaxBz", "ExlaxBz", "psilaxEx", "BzlaxEx", "BzlaxEy", "psilaxEy",
                        "BylaxEz", "BxlaxEz", "Jxlax", "Jylax", "FDxlax", "FDylax", "Ftauxlax", "Ftauylax",
                        "FSxxlax", "FSxylax", "FSxzlax", "FSyxlax", "FSyylax", "FSyzlax"};
    for (int c = 0; c < 28; ++c) o[c] = a(on[c]);
    int32_t st_acc = 0;
#pragma omp parallel for schedule(static) reduction(| : st_acc)
    for (int j = -1; j <= jmax; ++j)
      for (int i = -1; i <= imax; ++i) {
        const size_t k = id(i, j);
        Side xl = side(XL, k), xr = side(XR, k);
        Side yl = side(YL, k), yr = side(YR, k);
        yl.J = YL[Y_JY][k]; yr.J = YR[Y_JY][k];
        if (solver == 5 || solver == 7) {
          // superluminal fall-back, 16_hll_flow_mpx.f95:1393-1462
          double V2xl = pw2(xl.vx) + pw2(xl.vy) + pw2(xl.vz);
          double V2xr = pw2(xr.vx) + pw2(xr.vy) + pw2(xr.vz);
          double V2yl = pw2(yl.vx) + pw2(yl.vy) + pw2(yl.vz);
          double V2yr = pw2(yr.vx) + pw2(yr.vy) + pw2(yr.vz);
          auto fallback = [&]() {
            xl.vx = Vx[id(i, j)]; xr.vx = Vx[id(i - 1, j)];
            xl.vy = Vy[id(i, j)]; xr.vy = Vy[id(i - 1, j)];
            xl.vz = Vz[id(i, j)]; xr.vz = Vz[id(i - 1, j)];
            yl.vx = Vx[id(i, j)]; yr.vx = Vx[id(i, j - 1)];
            yl.vy = Vy[id(i, j)]; yr.vy = Vy[id(i, j - 1)];
            yl.vz = Vz[id(i, j)]; yr.vz = Vz[id(i, j - 1)];
            V2yl = pw2(yl.vx) + pw2(yl.vy) + pw2(yl.vz);
            V2yr = pw2(yr.vx) + pw2(yr.vy) + pw2(yr.vz);
            V2xl = pw2(xl.vx) + pw2(xl.vy) + pw2(xl.vz);
            V2xr = pw2(xr.vx) + pw2(xr.vy) + pw2(xr.vz);
          };
          if (V2xl >= 1.0 || V2xr >= 1.0) fallback();
          if (V2yl >= 1.0 || V2yr >= 1.0) fallback();
        }
        if (solver == 2) {   // 16_hll_flow_mcl.f95:1014-1396 (const_sp = 0: Sp = 1, SLC = 0)
          double out[28];
          mcl_fluxes(xl, xr, yl, yr, out);
          for (int c = 0; c < 28; ++c) o[c][k] = out[c];
          continue;
        }
        if (solver == 3) {   // 16_hlle_flow_mcl.f95:1647-4345
          PhysX fxl = physx(xl), fxr = physx(xr), fyl = physy(yl), fyr = physy(yr);
          hlle_w(fxl, xl); hlle_w(fxr, xr); hlle_w(fyl, yl); hlle_w(fyr, yr);
          fxl = physx_w(xl, fxl.W); fxr = physx_w(xr, fxr.W); fyl = physy_w(yl, fyl.W); fyr = physy_w(yr, fyr.W);
          double out[28];
          st_acc |= hllemc_x(xl, xr, fxl, fxr, side_jx(xl, fxl.W), side_jx(xr, fxr.W), out);
          st_acc |= hllemc_y(yl, yr, fyl, fyr, side_jy(yl, fyl.W), side_jy(yr, fyr.W), out);
          for (int c = 0; c < 28; ++c) o[c][k] = out[c];
          continue;
        }
        if (solver == 7) {
          // density fix-up chain, 16_hllc_flow_mpx.f95:2663-2690
          if (yl.rho < 0.0) yl.rho = rho[k] * 1.0e-1;
          else if (yr.rho < 0.0) yr.rho = rho[k] * 1.0e-1;
          else if (xl.rho < 0.0) xl.rho = rho[k] * 1.0e-1;
          else if (xr.rho < 0.0) xr.rho = rho[k] * 1.0e-1;
        }
        PhysX fxl = physx(xl), fxr = physx(xr), fyl = physy(yl), fyr = physy(yr);
        if (solver == 6 || solver == 4) { hlle_w(fxl, xl); hlle_w(fxr, xr); hlle_w(fyl, yl); hlle_w(fyr, yr);
          fxl = physx_w(xl, fxl.W); fxr = physx_w(xr, fxr.W); fyl = physy_w(yl, fyl.W); fyr = physy_w(yr, fyr.W); }
        if (solver == 4) {   // 16_hllc_flow_mcl.f95: the current of each side's MC state
          xl.J = side_jx(xl, fxl.W); xr.J = side_jx(xr, fxr.W);
          yl.J = side_jy(yl, fyl.W); yr.J = side_jy(yr, fyr.W);
        }
        double out[28];
        // EM + charge fluxes are HLL for every solver (HLLC star EM fluxes equal the HLL ones)
        out[0] = hllf(xl.Ex, xr.Ex, xl.psi, xr.psi);                 // Exlaxpsi
        out[1] = hllf(yl.Ey, yr.Ey, yl.psi, yr.psi);                 // Eylaxpsi
        out[2] = hllf(xl.Bx, xr.Bx, xl.phi, xr.phi);                 // Bxlaxphi
        out[3] = hllf(yl.By, yr.By, yl.phi, yr.phi);                 // Bylaxphi
        out[4] = hllf(xl.phi, xr.phi, xl.Bx, xr.Bx);                 // philaxBx
        out[5] = hllf(yl.Ez, yr.Ez, yl.Bx, yr.Bx);                   // EzlaxBx
        out[6] = -hllf(xl.Ezm, xr.Ezm, xl.By, xr.By);                // EzlaxBy
        out[7] = hllf(yl.phi, yr.phi, yl.By, yr.By);                 // philaxBy
        out[8] = hllf(xl.Ey, xr.Ey, xl.Bz, xr.Bz);                   // EylaxBz
        out[9] = -hllf(yl.Exm, yr.Exm, yl.Bz, yr.Bz);                // ExlaxBz
        out[10] = hllf(xl.psi, xr.psi, xl.Ex, xr.Ex);                // psilaxEx
        out[11] = -hllf(yl.Bzm, yr.Bzm, yl.Ex, yr.Ex);               // BzlaxEx
        out[12] = hllf(xl.Bz, xr.Bz, xl.Ey, xr.Ey);                  // BzlaxEy
        out[13] = hllf(yl.psi, yr.psi, yl.Ey, yr.Ey);                // psilaxEy
        out[14] = -hllf(xl.Bym, xr.Bym, xl.Ez, xr.Ez);               // BylaxEz
        out[15] = hllf(yl.Bx, yr.Bx, yl.Ez, yr.Ez);                  // BxlaxEz
        out[16] = hllf(xl.J, xr.J, xl.q, xr.q);                      // Jxlax
        out[17] = hllf(yl.J, yr.J, yl.q, yr.q);                      // Jylax
        if (solver == 5) {  // 16_hll_flow_mpx.f95:1871-1924
          out[18] = hllf(fxl.FD, fxr.FD, xl.D, xr.D);
          out[19] = hllf(fyl.FD, fyr.FD, yl.D, yr.D);
          out[20] = hllf(fxl.Ftau, fxr.Ftau, xl.tau, xr.tau);
          out[21] = hllf(fyl.Ftau, fyr.Ftau, yl.tau, yr.tau);
          out[22] = hllf(fxl.FSx, fxr.FSx, xl.Sx, xr.Sx);
          out[23] = hllf(fxl.FSy, fxr.FSy, xl.Sy, xr.Sy);
          out[24] = hllf(fxl.FSz, fxr.FSz, xl.Sz, xr.Sz);
          out[25] = hllf(fyl.FSx, fyr.FSx, yl.Sx, yr.Sx);
          out[26] = hllf(fyl.FSy, fyr.FSy, yl.Sy, yr.Sy);
          out[27] = hllf(fyl.FSz, fyr.FSz, yl.Sz, yr.Sz);
        } else if (solver == 7) {
          st_acc |= hllc_x(xl, xr, fxl, fxr, out);
          st_acc |= hllc_y(yl, yr, fyl, fyr, out);
        } else if (solver == 4) {   // 16_hllc_flow_mcl.f95:2580-2600: |v*| <= 1e-6 counts as 0
          st_acc |= hllc_x(xl, xr, fxl, fxr, out, 1.0e-6);
          st_acc |= hllc_y(yl, yr, fyl, fyr, out, 1.0e-6);
        } else {
          st_acc |= hlle_x(xl, xr, fxl, fxr, out);
          st_acc |= hlle_y(yl, yr, fyl, fyr, out);
        }
        for (int c = 0; c < 28; ++c) o[c][k] = out[c];
      }
    status |= st_acc;
  }

  PhysX physx_w(const Side& s, double W) {
    PhysX f = physx(s); f.W = W;
    const double eps = s.p / ((gamma - 1.0) * s.rho);
    f.h = s.rho * (1.0 + eps) + s.p;
    const double E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
    f.Ftau = (s.Bz * s.Ey - s.By * s.Ez) + f.h * pw2(f.W) * s.vx;
    f.FSx = -pw2(s.Ex) - pw2(s.Bx) + f.h * pw2(f.W) * pw2(s.vx) + 0.5 * E2B2 + s.p;
    f.FSy = -s.Ex * s.Ey - s.Bx * s.By + f.h * pw2(f.W) * s.vx * s.vy;
    f.FSz = -s.Ex * s.Ez - s.Bx * s.Bz + f.h * pw2(f.W) * s.vx * s.vz;
    return f;
  }
  PhysX physy_w(const Side& s, double W) {
    PhysX f = physy(s); f.W = W;
    const double eps = s.p / ((gamma - 1.0) * s.rho);
    f.h = s.rho * (1.0 + eps) + s.p;
    const double E2B2 = pw2(s.Ex) + pw2(s.Ey) + pw2(s.Ez) + pw2(s.Bx) + pw2(s.By) + pw2(s.Bz);
    f.Ftau = (s.Bx * s.Ez - s.Bz * s.Ex) + f.h * pw2(f.W) * s.vy;
    f.FSx = -s.Ex * s.Ey - s.Bx * s.By + f.h * pw2(f.W) * s.vx * s.vy;
    f.FSy = -pw2(s.Ey) - pw2(s.By) + f.h * pw2(f.W) * pw2(s.vy) + 0.5 * E2B2 + s.p;
    f.FSz = -s.Ey * s.Ez - s.By * s.Bz + f.h * pw2(f.W) * s.vy * s.vz;
    return f;
  }

  // ----------------------------------------- HLLC, x direction
  // The HLLC of the MC family (16_hllc_flow_mcl.f95, flux_solver 4, 2D
  // :1751-4056) has the same HLL states, star states and flux choice on the
  // MC sides (the "_m" values in Ez / By, the current of each side, W from
  // 1 - vx^2 - vy^2 - vz^2) and zeroes |v*| <= 1e-6 (vzero) instead of 1e-9.
  // 16_hllc_flow_mpx.f95:2816-3100 (HLL states/fluxes), 3184-3335 (v*),
  // 3485-3520 (star states), 3592-3740 (star fluxes), 3908-4300 (selection)
  int32_t hllc_x(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double* out,
                  double vzero = 1.0e-9) {
    int32_t st = 0;
    const double s1 = -1.0, s2 = 1.0;
    const double psi_hll = (s2 * R.psi - s1 * L.psi + L.Ex - R.Ex) / (s2 - s1);
    const double phi_hll = (s2 * R.phi - s1 * L.phi + L.Bx - R.Bx) / (s2 - s1);
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.psi - R.psi) / (s2 - s1);
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.Bz - R.Bz) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bym - R.Bym) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.phi - R.phi) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.Ezm - R.Ezm) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Ey - R.Ey) / (s2 - s1);
    const double DD_hll = (s2 * R.D - s1 * L.D + fl.FD - fr.FD) / (s2 - s1);
    const double tau_hll = (s2 * R.tau - s1 * L.tau + fl.Ftau - fr.Ftau) / (s2 - s1);
    const double Sx_hll = (s2 * R.Sx - s1 * L.Sx + fl.FSx - fr.FSx) / (s2 - s1);
    const double Sy_hll = (s2 * R.Sy - s1 * L.Sy + fl.FSy - fr.FSy) / (s2 - s1);
    const double Sz_hll = (s2 * R.Sz - s1 * L.Sz + fl.FSz - fr.FSz) / (s2 - s1);
    const double psi_f = 0.5 * (L.Ex + R.Ex - (R.psi - L.psi));
    const double phi_f = 0.5 * (L.Bx + R.Bx - (R.phi - L.phi));
    const double Bx_f = 0.5 * (L.phi + R.phi - (R.Bx - L.Bx));
    const double By_f = 0.5 * (L.Ezm + R.Ezm - (R.By - L.By));
    const double Bz_f = 0.5 * (L.Ey + R.Ey - (R.Bz - L.Bz));
    const double Ex_f = 0.5 * (L.psi + R.psi - (R.Ex - L.Ex));
    const double Ey_f = 0.5 * (L.Bz + R.Bz - (R.Ey - L.Ey));
    const double Ez_f = 0.5 * (L.Bym + R.Bym - (R.Ez - L.Ez));
    const double q_f = 0.5 * (L.J + R.J - (R.q - L.q));
    const double DD_f = 0.5 * (fl.FD + fr.FD - (R.D - L.D));
    const double tau_f = 0.5 * (fl.Ftau + fr.Ftau - (R.tau - L.tau));
    const double Sx_f = 0.5 * (fl.FSx + fr.FSx - (R.Sx - L.Sx));
    const double Sy_f = 0.5 * (fl.FSy + fr.FSy - (R.Sy - L.Sy));
    const double Sz_f = 0.5 * (fl.FSz + fr.FSz - (R.Sz - L.Sz));
    // star E, B are the HLL averages (L and R identical)
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Eys) + pw2(Ezs));
    const double B2_perp = (pw2(Bys) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_x;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sx_f;
    const double c_hll = Sx_hll - ErotB_x;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = 1.0e-6;  // 16_hllc_flow_mpx.f95:3217
    if (std::fabs(V) <= vzero) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sx_f + (pw2(Exs) + pw2(Bxs)) - (tau_f - ErotB_x) * V;
    const double psiR = (s2 * psi_hll - V * Ex_f) / (s2 - V);
    const double psiL = (-s1 * psi_hll + V * Ex_f) / (V - s1);
    const double phiR = (s2 * phi_hll - V * Bx_f) / (s2 - V);
    const double phiL = (-s1 * phi_hll + V * Bx_f) / (V - s1);
    const double SxR = (s2 * Sx_hll - tau_f * V) / (s2 - V);
    const double SxL = (-s1 * Sx_hll + tau_f * V) / (V - s1);
    const double SyR = (s2 * Sy_hll - Sy_f - ErotB_y * V - Exs * Eys - Bxs * Bys) / (s2 - V);
    const double SyL = (-s1 * Sy_hll + Sy_f + ErotB_y * V + Exs * Eys + Bxs * Bys) / (V - s1);
    const double SzR = (s2 * Sz_hll - Sz_f - ErotB_z * V - Exs * Ezs - Bxs * Bzs) / (s2 - V);
    const double SzL = (-s1 * Sz_hll + Sz_f + ErotB_z * V + Exs * Ezs + Bxs * Bzs) / (V - s1);
    const double tauR = (SxR - ErotB_x) / V - pstr + E2B2_str;
    const double tauL = (SxL - ErotB_x) / V - pstr + E2B2_str;
    const double DR = (s2 * DD_hll - DD_f) / (s2 - V);
    const double DL = (-s1 * DD_hll + DD_f) / (V - s1);
    double fpsiR, fpsiL, fphiR, fphiL, fDR, fDL, ftR, ftL, fSxR, fSxL, fSyR, fSyL, fSzR, fSzL;
    if (V == 0.0) {
      fpsiR = fpsiL = psi_f; fphiR = fphiL = phi_f; fDR = fDL = DD_f; ftR = ftL = tau_f;
      fSxR = fSxL = Sx_f; fSyR = fSyL = Sy_f; fSzR = fSzL = Sz_f;
    } else {
      fpsiR = psi_f + (s2 * (V - s1) * (psiR - psiL)) / (s2 - s1);
      fpsiL = psi_f - (s1 * (s2 - V) * (psiR - psiL)) / (s2 - s1);
      fphiR = phi_f + (s2 * (V - s1) * (phiR - phiL)) / (s2 - s1);
      fphiL = phi_f - (s1 * (s2 - V) * (phiR - phiL)) / (s2 - s1);
      fDR = DD_f + s2 * (V - s1) * (DR - DL) / (s2 - s1);
      fDL = DD_f - s1 * (s2 - V) * (DR - DL) / (s2 - s1);
      ftR = tau_f + s2 * (V - s1) * (tauR - tauL) / (s2 - s1);
      ftL = tau_f - s1 * (s2 - V) * (tauR - tauL) / (s2 - s1);
      fSxR = Sx_f + s2 * (V - s1) * (SxR - SxL) / (s2 - s1);
      fSxL = Sx_f - s1 * (s2 - V) * (SxR - SxL) / (s2 - s1);
      fSyR = Sy_f + s2 * (V - s1) * (SyR - SyL) / (s2 - s1);
      fSyL = Sy_f - s1 * (s2 - V) * (SyR - SyL) / (s2 - s1);
      fSzR = Sz_f + s2 * (V - s1) * (SzR - SzL) / (s2 - s1);
      fSzL = Sz_f - s1 * (s2 - V) * (SzR - SzL) / (s2 - s1);
    }
    if (s1 < 0.0 && 0.0 < V) {
      out[0] = fpsiL; out[2] = fphiL; out[18] = fDL; out[20] = ftL; out[22] = fSxL; out[23] = fSyL; out[24] = fSzL;
      out[4] = Bx_f; out[6] = -By_f; out[8] = Bz_f; out[10] = Ex_f; out[12] = Ey_f; out[14] = -Ez_f; out[16] = q_f;
    } else if (V < 0.0 && 0.0 < s2) {
      out[0] = fpsiR; out[2] = fphiR; out[18] = fDR; out[20] = ftR; out[22] = fSxR; out[23] = fSyR; out[24] = fSzR;
      out[4] = Bx_f; out[6] = -By_f; out[8] = Bz_f; out[10] = Ex_f; out[12] = Ey_f; out[14] = -Ez_f; out[16] = q_f;
    } else if (V == 0.0) {
      out[0] = 0.5 * (fpsiR + fpsiL); out[2] = 0.5 * (fphiR + fphiL);
      out[4] = 0.5 * (Bx_f + Bx_f); out[6] = -0.5 * (By_f + By_f); out[8] = 0.5 * (Bz_f + Bz_f);
      out[10] = 0.5 * (Ex_f + Ex_f); out[12] = 0.5 * (Ey_f + Ey_f); out[14] = -0.5 * (Ez_f + Ez_f);
      out[16] = 0.5 * (q_f + q_f); out[18] = 0.5 * (fDR + fDL); out[20] = 0.5 * (ftR + ftL);
      out[22] = 0.5 * (fSxR + fSxL); out[23] = 0.5 * (fSyR + fSyL); out[24] = 0.5 * (fSzR + fSzL);
    } else {
      st |= ST_HLLC_VSTAR;
      for (int c : {0, 2, 4, 6, 8, 10, 12, 14, 16, 18, 20, 22, 23, 24}) out[c] = NAN;
    }
    return st;
  }

  // ----------------------------------------- HLLC, y direction
  // 16_hllc_flow_mpx.f95:2960-3100, 3340-3475, 3522-3570, 3742-3905, 4305-4610
  int32_t hllc_y(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double* out,
                  double vzero = 1.0e-9) {
    int32_t st = 0;
    const double s1 = -1.0, s2 = 1.0;
    const double psi_hll = (s2 * R.psi - s1 * L.psi + L.Ey - R.Ey) / (s2 - s1);
    const double phi_hll = (s2 * R.phi - s1 * L.phi + L.By - R.By) / (s2 - s1);
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.psi - R.psi) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bx - R.Bx) / (s2 - s1);
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.Bzm - R.Bzm) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.phi - R.phi) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Exm - R.Exm) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.Ez - R.Ez) / (s2 - s1);
    const double DD_hll = (s2 * R.D - s1 * L.D + fl.FD - fr.FD) / (s2 - s1);
    const double tau_hll = (s2 * R.tau - s1 * L.tau + fl.Ftau - fr.Ftau) / (s2 - s1);
    const double Sy_hll = (s2 * R.Sy - s1 * L.Sy + fl.FSy - fr.FSy) / (s2 - s1);
    const double Sz_hll = (s2 * R.Sz - s1 * L.Sz + fl.FSz - fr.FSz) / (s2 - s1);
    const double Sx_hll = (s2 * R.Sx - s1 * L.Sx + fl.FSx - fr.FSx) / (s2 - s1);
    const double psi_f = 0.5 * (L.Ey + R.Ey - (R.psi - L.psi));
    const double phi_f = 0.5 * (L.By + R.By - (R.phi - L.phi));
    const double By_f = 0.5 * (L.phi + R.phi - (R.By - L.By));
    const double Bz_f = 0.5 * (L.Exm + R.Exm - (R.Bz - L.Bz));
    const double Bx_f = 0.5 * (L.Ez + R.Ez - (R.Bx - L.Bx));
    const double Ey_f = 0.5 * (L.psi + R.psi - (R.Ey - L.Ey));
    const double Ez_f = 0.5 * (L.Bx + R.Bx - (R.Ez - L.Ez));
    const double Ex_f = 0.5 * (L.Bzm + R.Bzm - (R.Ex - L.Ex));
    const double q_f = 0.5 * (L.J + R.J - (R.q - L.q));
    const double DD_f = 0.5 * (fl.FD + fr.FD - (R.D - L.D));
    const double tau_f = 0.5 * (fl.Ftau + fr.Ftau - (R.tau - L.tau));
    const double Sy_f = 0.5 * (fl.FSy + fr.FSy - (R.Sy - L.Sy));
    const double Sz_f = 0.5 * (fl.FSz + fr.FSz - (R.Sz - L.Sz));
    const double Sx_f = 0.5 * (fl.FSx + fr.FSx - (R.Sx - L.Sx));
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Exs) + pw2(Ezs));
    const double B2_perp = (pw2(Bxs) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_y;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sy_f;
    const double c_hll = Sy_hll - ErotB_y;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = (double)1.0e-6f;  // single-precision literal, 16_hllc_flow_mpx.f95:3354
    if (std::fabs(V) <= vzero) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sy_f + (pw2(Eys) + pw2(Bys)) - (tau_f - ErotB_y) * V;
    const double psiR = (s2 * psi_hll - V * Ey_f) / (s2 - V);
    const double psiL = (-s1 * psi_hll + V * Ey_f) / (V - s1);
    const double phiR = (s2 * phi_hll - V * By_f) / (s2 - V);
    const double phiL = (-s1 * phi_hll + V * By_f) / (V - s1);
    const double SyR = (s2 * Sy_hll - tau_f * V) / (s2 - V);
    const double SyL = (-s1 * Sy_hll + tau_f * V) / (V - s1);
    const double SzR = (s2 * Sz_hll - Sz_f - ErotB_z * V - Eys * Ezs - Bys * Bzs) / (s2 - V);
    const double SzL = (-s1 * Sz_hll + Sz_f + ErotB_z * V + Eys * Ezs + Bys * Bzs) / (V - s1);
    const double SxR = (s2 * Sx_hll - Sx_f - ErotB_x * V - Eys * Exs - Bys * Bxs) / (s2 - V);
    const double SxL = (-s1 * Sx_hll + Sx_f + ErotB_x * V + Eys * Exs + Bys * Bxs) / (V - s1);
    const double tauR = (SyR - ErotB_y) / V - pstr + E2B2_str;
    const double tauL = (SyL - ErotB_y) / V - pstr + E2B2_str;
    const double DR = (s2 * DD_hll - DD_f) / (s2 - V);
    const double DL = (-s1 * DD_hll + DD_f) / (V - s1);
    double fpsiR, fpsiL, fphiR, fphiL, fDR, fDL, ftR, ftL, fSxR, fSxL, fSyR, fSyL, fSzR, fSzL;
    if (V == 0.0) {
      fpsiR = fpsiL = psi_f; fphiR = fphiL = phi_f; fDR = fDL = DD_f; ftR = ftL = tau_f;
      fSxR = fSxL = Sx_f; fSyR = fSyL = Sy_f; fSzR = fSzL = Sz_f;
    } else {
      fpsiR = psi_f + (s2 * (V - s1) * (psiR - psiL)) / (s2 - s1);
      fpsiL = psi_f - (s1 * (s2 - V) * (psiR - psiL)) / (s2 - s1);
      fphiR = phi_f + (s2 * (V - s1) * (phiR - phiL)) / (s2 - s1);
      fphiL = phi_f - (s1 * (s2 - V) * (phiR - phiL)) / (s2 - s1);
      fDR = DD_f + s2 * (V - s1) * (DR - DL) / (s2 - s1);
      fDL = DD_f - s1 * (s2 - V) * (DR - DL) / (s2 - s1);
      ftR = tau_f + s2 * (V - s1) * (tauR - tauL) / (s2 - s1);
      ftL = tau_f - s1 * (s2 - V) * (tauR - tauL) / (s2 - s1);
      fSxR = Sx_f + s2 * (V - s1) * (SxR - SxL) / (s2 - s1);
      fSxL = Sx_f - s1 * (s2 - V) * (SxR - SxL) / (s2 - s1);
      fSyR = Sy_f + s2 * (V - s1) * (SyR - SyL) / (s2 - s1);
      fSyL = Sy_f - s1 * (s2 - V) * (SyR - SyL) / (s2 - s1);
      fSzR = Sz_f + s2 * (V - s1) * (SzR - SzL) / (s2 - s1);
      fSzL = Sz_f - s1 * (s2 - V) * (SzR - SzL) / (s2 - s1);
    }
    if (s1 < 0.0 && 0.0 < V) {
      out[1] = fpsiL; out[3] = fphiL; out[19] = fDL; out[21] = ftL; out[25] = fSxL; out[26] = fSyL; out[27] = fSzL;
      out[5] = Bx_f; out[7] = By_f; out[9] = -Bz_f; out[11] = -Ex_f; out[13] = Ey_f; out[15] = Ez_f; out[17] = q_f;
    } else if (V < 0.0 && 0.0 < s2) {
      out[1] = fpsiR; out[3] = fphiR; out[19] = fDR; out[21] = ftR; out[25] = fSxR; out[26] = fSyR; out[27] = fSzR;
      out[5] = Bx_f; out[7] = By_f; out[9] = -Bz_f; out[11] = -Ex_f; out[13] = Ey_f; out[15] = Ez_f; out[17] = q_f;
    } else if (V == 0.0) {
      out[1] = 0.5 * (fpsiR + fpsiL); out[3] = 0.5 * (fphiR + fphiL);
      out[5] = 0.5 * (Bx_f + Bx_f); out[7] = 0.5 * (By_f + By_f); out[9] = -0.5 * (Bz_f + Bz_f);
      out[11] = -0.5 * (Ex_f + Ex_f); out[13] = 0.5 * (Ey_f + Ey_f); out[15] = 0.5 * (Ez_f + Ez_f);
      out[17] = 0.5 * (q_f + q_f); out[19] = 0.5 * (fDR + fDL); out[21] = 0.5 * (ftR + ftL);
      out[25] = 0.5 * (fSxR + fSxL); out[26] = 0.5 * (fSyR + fSyL); out[27] = 0.5 * (fSzR + fSzL);
    } else {
      st |= ST_HLLC_VSTAR;
      for (int c : {1, 3, 5, 7, 9, 11, 13, 15, 17, 19, 21, 25, 26, 27}) out[c] = NAN;
    }
    return st;
  }

  // ----------------------------------------- HLLE (16_hlle_flow_mpx.f95, 2D)
  // EM fields, psi and phi take the fixed-speed HLL fluxes (s = -1, +1,
  // :2526-2588, the star psi/phi fluxes are the HLL ones, :3489-3604); q, D,
  // tau and S use the bounds sx1 = min(lambda-), sx2 = max(lambda+) from the
  // relativistic sound speed (:2709-2826), and D, tau, S get the HLLC-type
  // contact of the same quadratic for v* (:3165-3420).  Flux choice
  // (:4021-4286): sx1 >= 0 left physical flux, sx1 <= 0 <= v* left star,
  // v* <= 0 <= sx2 right star, sx2 < 0 right physical flux.
  // Wave bounds of one side; vn is the normal velocity.  The reference
  // writes vn (not vn^2) in the second factor under the root (:2722-2735).
  void hlle_bounds(const Side& s, const PhysX& f, double vn, double& lm, double& lp) const {
    const double Cs = std::sqrt(gamma * s.p / (f.h));
    const double V2 = pw2(s.vx) + pw2(s.vy) + pw2(s.vz);
    const double root = std::sqrt((1.0 - V2) * (1.0 - V2 * pw2(Cs) - vn * (1.0 - pw2(Cs))));
    lp = (vn * (1.0 - pw2(Cs)) + Cs * root) / (1.0 - pw2(Cs) * V2);
    lm = (vn * (1.0 - pw2(Cs)) - Cs * root) / (1.0 - pw2(Cs) * V2);
  }
  // sx1, sx2 with the NaN stop (:2796-2803) and the clamp to 1 - 1e-9 (:2805-2819)
  static int32_t hlle_speeds(double lmL, double lmR, double lpL, double lpR, double& s1, double& s2) {
    s1 = fmin2(lmL, lmR);
    s2 = fmax2(lpL, lpR);
    int32_t st = 0;
    if (std::isnan(s1) || std::isnan(s2)) st |= ST_HLLE_SPEED;
    const double eps2 = 1.0e-9;
    if (std::fabs(s1) > 1.0) s1 = fmax2(-1.0 + eps2, fmin2(1.0 - eps2, s1));
    if (std::fabs(s2) > 1.0) s2 = fmax2(-1.0 + eps2, fmin2(1.0 - eps2, s2));
    return st;
  }

  // ------------------- HLLE with the MC reconstruction (16_hlle_flow_mcl.f95, 2D, :1638-4345)
  // Sides come from the MC reconstruction (the "_m" values of Ez / By in x,
  // Ex / Bz in y), W from 1 - vx^2 - vy^2 - vz^2 and the current J from each
  // side's state, as in the HLL routine of the family.  The averaged states
  // the routine also forms (p_L, rho_L, enthpy_L, ...) feed only its
  // diagnostics prints.  Wave bounds and the v* quadratic are those of the
  // MPX HLLE; the star states and fluxes differ (:2911-3029 for x):
  //   S_n* = (s S_n,hll - F(S_n)_hll +- (p* - B_n*^2 - E_n*^2 - (E*xB*)_n v*)) / (s - v*),
  //   tau* = (s tau_hll - F(tau)_hll +- ((p* - |E*B*|^2/2) v* + (E*xB*)_n)) / (s - v*),
  //   F*   = F(side) + s (U* - U(side))            (s = sx1 left, sx2 right),
  // and for v* != 0 the EM fluxes are the fluxes of the star state
  // (psi: E_n*, E_n: psi*, E_t1: B_t2*, E_t2: -B_t1*, ...), for v* == 0 the
  // fixed-speed HLL fluxes (:3042-3150).  Flux choice (:3236-4343): sx1 > 0
  // left physical flux, sx1 <= 0 <= v* left star, v* < 0 <= sx2 right star,
  // sx2 < 0 right physical flux.  A NaN v* leaves the reference's EM arrays
  // unset; it is reported here with NaN fluxes.
  double side_jx(const Side& s, double W) const {
    const double vrotB = s.Bz * s.vy - s.By * s.vz;
    const double Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
    return sigma * W * (s.Ex + vrotB - Edotv * s.vx) + s.q * s.vx;
  }
  double side_jy(const Side& s, double W) const {
    const double vrotB = s.Bx * s.vz - s.Bz * s.vx;
    const double Edotv = s.Ex * s.vx + s.Ey * s.vy + s.Ez * s.vz;
    return sigma * W * (s.Ey + vrotB - Edotv * s.vy) + s.q * s.vy;
  }
  int32_t hllemc_x(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double JL, double JR,
                   double* out) {
    const double s1 = -1.0, s2 = 1.0;
    const double psi_hll = (s2 * R.psi - s1 * L.psi + L.Ex - R.Ex) / (s2 - s1);
    const double phi_hll = (s2 * R.phi - s1 * L.phi + L.Bx - R.Bx) / (s2 - s1);
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.psi - R.psi) / (s2 - s1);
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.Bz - R.Bz) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bym - R.Bym) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.phi - R.phi) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.Ezm - R.Ezm) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Ey - R.Ey) / (s2 - s1);
    double lmL, lpL, lmR, lpR, sx1, sx2;
    hlle_bounds(R, fr, R.vx, lmR, lpR);
    hlle_bounds(L, fl, L.vx, lmL, lpL);
    int32_t st = hlle_speeds(lmL, lmR, lpL, lpR, sx1, sx2);
    const double DD_hll = (sx2 * R.D - sx1 * L.D + fl.FD - fr.FD) / (sx2 - sx1);
    const double tau_hll = (sx2 * R.tau - sx1 * L.tau + fl.Ftau - fr.Ftau) / (sx2 - sx1);
    const double Sx_hll = (sx2 * R.Sx - sx1 * L.Sx + fl.FSx - fr.FSx) / (sx2 - sx1);
    const double Sy_hll = (sx2 * R.Sy - sx1 * L.Sy + fl.FSy - fr.FSy) / (sx2 - sx1);
    const double Sz_hll = (sx2 * R.Sz - sx1 * L.Sz + fl.FSz - fr.FSz) / (sx2 - sx1);
    auto hlle = [&](double FL, double FR, double UL, double UR) {
      return (sx2 * FL - sx1 * FR + sx1 * sx2 * (UR - UL)) / (sx2 - sx1);
    };
    const double q_f = hlle(JL, JR, L.q, R.q);
    const double DD_f = hlle(fl.FD, fr.FD, L.D, R.D);
    const double tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
    const double Sx_f = hlle(fl.FSx, fr.FSx, L.Sx, R.Sx);
    const double Sy_f = hlle(fl.FSy, fr.FSy, L.Sy, R.Sy);
    const double Sz_f = hlle(fl.FSz, fr.FSz, L.Sz, R.Sz);
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Eys) + pw2(Ezs));
    const double B2_perp = (pw2(Bys) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_x;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sx_f;
    const double c_hll = Sx_hll - ErotB_x;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = 1.0e-6;
    if (std::fabs(V) <= 1.0e-9) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sx_f + (pw2(Exs) + pw2(Bxs)) - (tau_f - ErotB_x) * V;
    const double SxR = (sx2 * Sx_hll - Sx_f + pstr - pw2(Bxs) - pw2(Exs) - ErotB_x * V) / (sx2 - V);
    const double SxL = (-sx1 * Sx_hll + Sx_f - pstr + pw2(Bxs) + pw2(Exs) + ErotB_x * V) / (V - sx1);
    const double SyR = (sx2 * Sy_hll - Sy_f - ErotB_y * V - Exs * Eys - Bxs * Bys) / (sx2 - V);
    const double SyL = (-sx1 * Sy_hll + Sy_f + ErotB_y * V + Exs * Eys + Bxs * Bys) / (V - sx1);
    const double SzR = (sx2 * Sz_hll - Sz_f - ErotB_z * V - Exs * Ezs - Bxs * Bzs) / (sx2 - V);
    const double SzL = (-sx1 * Sz_hll + Sz_f + ErotB_z * V + Exs * Ezs + Bxs * Bzs) / (V - sx1);
    const double tauR = (sx2 * tau_hll - tau_f + (pstr - E2B2_str) * V + ErotB_x) / (sx2 - V);
    const double tauL = (-sx1 * tau_hll + tau_f - (pstr - E2B2_str) * V - ErotB_x) / (V - sx1);
    const double DR = (sx2 * DD_hll - DD_f) / (sx2 - V);
    const double DL = (-sx1 * DD_hll + DD_f) / (V - sx1);
    double fpsi, fphi, fEx, fEy, fEz, fBx, fBy, fBz;
    double fDR = DD_f, fDL = DD_f, ftR = tau_f, ftL = tau_f, fSxR = Sx_f, fSxL = Sx_f, fSyR = Sy_f, fSyL = Sy_f,
           fSzR = Sz_f, fSzL = Sz_f;
    if (V == 0.0) {
      fpsi = hllf(L.Ex, R.Ex, L.psi, R.psi); fphi = hllf(L.Bx, R.Bx, L.phi, R.phi);
      fBx = hllf(L.phi, R.phi, L.Bx, R.Bx); fBy = hllf(L.Ezm, R.Ezm, L.By, R.By);
      fBz = hllf(L.Ey, R.Ey, L.Bz, R.Bz); fEx = hllf(L.psi, R.psi, L.Ex, R.Ex);
      fEy = hllf(L.Bz, R.Bz, L.Ey, R.Ey); fEz = hllf(L.Bym, R.Bym, L.Ez, R.Ez);
    } else {
      fpsi = Exs; fphi = Bxs; fEx = psi_hll; fEy = Bzs; fEz = -Bys; fBx = phi_hll; fBy = -Ezs; fBz = Eys;
      fDR = fr.FD + sx2 * (DR - R.D);        fDL = fl.FD + sx1 * (DL - L.D);
      ftR = fr.Ftau + sx2 * (tauR - R.tau);  ftL = fl.Ftau + sx1 * (tauL - L.tau);
      fSxR = fr.FSx + sx2 * (SxR - R.Sx);    fSxL = fl.FSx + sx1 * (SxL - L.Sx);
      fSyR = fr.FSy + sx2 * (SyR - R.Sy);    fSyL = fl.FSy + sx1 * (SyL - L.Sy);
      fSzR = fr.FSz + sx2 * (SzR - R.Sz);    fSzL = fl.FSz + sx1 * (SzL - L.Sz);
    }
    if (0.0 <= V || V < 0.0) {   // both star sides carry the same EM fluxes
      out[0] = fpsi; out[2] = fphi; out[4] = fBx; out[6] = -fBy; out[8] = fBz; out[10] = fEx; out[12] = fEy;
      out[14] = -fEz;
    } else {
      st |= ST_HLLC_VSTAR;
      for (int c : {0, 2, 4, 6, 8, 10, 12, 14}) out[c] = NAN;
    }
    if (sx1 > 0.0) {
      out[16] = JL; out[18] = fl.FD; out[20] = fl.Ftau; out[22] = fl.FSx; out[23] = fl.FSy; out[24] = fl.FSz;
    } else if (sx1 <= 0.0 && 0.0 <= V) {
      out[16] = q_f; out[18] = fDL; out[20] = ftL; out[22] = fSxL; out[23] = fSyL; out[24] = fSzL;
    } else if (V < 0.0 && 0.0 <= sx2) {
      out[16] = q_f; out[18] = fDR; out[20] = ftR; out[22] = fSxR; out[23] = fSyR; out[24] = fSzR;
    } else if (sx2 < 0.0) {
      out[16] = JR; out[18] = fr.FD; out[20] = fr.Ftau; out[22] = fr.FSx; out[23] = fr.FSy; out[24] = fr.FSz;
    } else {   // the reference stops
      st |= ST_HLLC_VSTAR;
      for (int c : {16, 18, 20, 22, 23, 24}) out[c] = NAN;
    }
    return st;
  }
  // y faces (16_hlle_flow_mcl.f95 y branches): physy's FSx, FSy, FSz are FSyx, FSyy, FSyz
  int32_t hllemc_y(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double JL, double JR,
                   double* out) {
    const double s1 = -1.0, s2 = 1.0;
    const double psi_hll = (s2 * R.psi - s1 * L.psi + L.Ey - R.Ey) / (s2 - s1);
    const double phi_hll = (s2 * R.phi - s1 * L.phi + L.By - R.By) / (s2 - s1);
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.psi - R.psi) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bx - R.Bx) / (s2 - s1);
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.Bzm - R.Bzm) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.phi - R.phi) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Exm - R.Exm) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.Ez - R.Ez) / (s2 - s1);
    double lmL, lpL, lmR, lpR, sy1, sy2;
    hlle_bounds(R, fr, R.vy, lmR, lpR);
    hlle_bounds(L, fl, L.vy, lmL, lpL);
    int32_t st = hlle_speeds(lmL, lmR, lpL, lpR, sy1, sy2);
    const double DD_hll = (sy2 * R.D - sy1 * L.D + fl.FD - fr.FD) / (sy2 - sy1);
    const double tau_hll = (sy2 * R.tau - sy1 * L.tau + fl.Ftau - fr.Ftau) / (sy2 - sy1);
    const double Sy_hll = (sy2 * R.Sy - sy1 * L.Sy + fl.FSy - fr.FSy) / (sy2 - sy1);
    const double Sz_hll = (sy2 * R.Sz - sy1 * L.Sz + fl.FSz - fr.FSz) / (sy2 - sy1);
    const double Sx_hll = (sy2 * R.Sx - sy1 * L.Sx + fl.FSx - fr.FSx) / (sy2 - sy1);
    auto hlle = [&](double FL, double FR, double UL, double UR) {
      return (sy2 * FL - sy1 * FR + sy1 * sy2 * (UR - UL)) / (sy2 - sy1);
    };
    const double q_f = hlle(JL, JR, L.q, R.q);
    const double DD_f = hlle(fl.FD, fr.FD, L.D, R.D);
    const double tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
    const double Sy_f = hlle(fl.FSy, fr.FSy, L.Sy, R.Sy);
    const double Sz_f = hlle(fl.FSz, fr.FSz, L.Sz, R.Sz);
    const double Sx_f = hlle(fl.FSx, fr.FSx, L.Sx, R.Sx);
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Exs) + pw2(Ezs));
    const double B2_perp = (pw2(Bxs) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_y;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sy_f;
    const double c_hll = Sy_hll - ErotB_y;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = 1.0e-6;
    if (std::fabs(V) <= 1.0e-9) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sy_f + (pw2(Eys) + pw2(Bys)) - (tau_f - ErotB_y) * V;
    const double SyR = (sy2 * Sy_hll - Sy_f + pstr - pw2(Bys) - pw2(Eys) - ErotB_y * V) / (sy2 - V);
    const double SyL = (-sy1 * Sy_hll + Sy_f - pstr + pw2(Bys) + pw2(Eys) + ErotB_y * V) / (V - sy1);
    const double SzR = (sy2 * Sz_hll - Sz_f - ErotB_z * V - Eys * Ezs - Bys * Bzs) / (sy2 - V);
    const double SzL = (-sy1 * Sz_hll + Sz_f + ErotB_z * V + Eys * Ezs + Bys * Bzs) / (V - sy1);
    const double SxR = (sy2 * Sx_hll - Sx_f - ErotB_x * V - Eys * Exs - Bys * Bxs) / (sy2 - V);
    const double SxL = (-sy1 * Sx_hll + Sx_f + ErotB_x * V + Eys * Exs + Bys * Bxs) / (V - sy1);
    const double tauR = (sy2 * tau_hll - tau_f + (pstr - E2B2_str) * V + ErotB_y) / (sy2 - V);
    const double tauL = (-sy1 * tau_hll + tau_f - (pstr - E2B2_str) * V - ErotB_y) / (V - sy1);
    const double DR = (sy2 * DD_hll - DD_f) / (sy2 - V);
    const double DL = (-sy1 * DD_hll + DD_f) / (V - sy1);
    double fpsi, fphi, fEx, fEy, fEz, fBx, fBy, fBz;
    double fDR = DD_f, fDL = DD_f, ftR = tau_f, ftL = tau_f, fSxR = Sx_f, fSxL = Sx_f, fSyR = Sy_f, fSyL = Sy_f,
           fSzR = Sz_f, fSzL = Sz_f;
    if (V == 0.0) {
      fpsi = hllf(L.Ey, R.Ey, L.psi, R.psi); fphi = hllf(L.By, R.By, L.phi, R.phi);
      fBy = hllf(L.phi, R.phi, L.By, R.By); fBz = hllf(L.Exm, R.Exm, L.Bz, R.Bz);
      fBx = hllf(L.Ez, R.Ez, L.Bx, R.Bx); fEy = hllf(L.psi, R.psi, L.Ey, R.Ey);
      fEz = hllf(L.Bx, R.Bx, L.Ez, R.Ez); fEx = hllf(L.Bzm, R.Bzm, L.Ex, R.Ex);
    } else {
      fpsi = Eys; fphi = Bys; fEx = -Bzs; fEy = psi_hll; fEz = Bxs; fBx = Ezs; fBy = phi_hll; fBz = -Exs;
      fDR = fr.FD + sy2 * (DR - R.D);        fDL = fl.FD + sy1 * (DL - L.D);
      ftR = fr.Ftau + sy2 * (tauR - R.tau);  ftL = fl.Ftau + sy1 * (tauL - L.tau);
      fSxR = fr.FSx + sy2 * (SxR - R.Sx);    fSxL = fl.FSx + sy1 * (SxL - L.Sx);
      fSyR = fr.FSy + sy2 * (SyR - R.Sy);    fSyL = fl.FSy + sy1 * (SyL - L.Sy);
      fSzR = fr.FSz + sy2 * (SzR - R.Sz);    fSzL = fl.FSz + sy1 * (SzL - L.Sz);
    }
    if (0.0 <= V || V < 0.0) {
      out[1] = fpsi; out[3] = fphi; out[5] = fBx; out[7] = fBy; out[9] = -fBz; out[11] = -fEx; out[13] = fEy;
      out[15] = fEz;
    } else {
      st |= ST_HLLC_VSTAR;
      for (int c : {1, 3, 5, 7, 9, 11, 13, 15}) out[c] = NAN;
    }
    if (sy1 > 0.0) {
      out[17] = JL; out[19] = fl.FD; out[21] = fl.Ftau; out[25] = fl.FSx; out[26] = fl.FSy; out[27] = fl.FSz;
    } else if (sy1 <= 0.0 && 0.0 <= V) {
      out[17] = q_f; out[19] = fDL; out[21] = ftL; out[25] = fSxL; out[26] = fSyL; out[27] = fSzL;
    } else if (V < 0.0 && 0.0 <= sy2) {
      out[17] = q_f; out[19] = fDR; out[21] = ftR; out[25] = fSxR; out[26] = fSyR; out[27] = fSzR;
    } else if (sy2 < 0.0) {
      out[17] = JR; out[19] = fr.FD; out[21] = fr.Ftau; out[25] = fr.FSx; out[26] = fr.FSy; out[27] = fr.FSz;
    } else {
      st |= ST_HLLC_VSTAR;
      for (int c : {17, 19, 21, 25, 26, 27}) out[c] = NAN;
    }
    return st;
  }

  int32_t hlle_x(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double* out) {
    const double s1 = -1.0, s2 = 1.0;
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.psi - R.psi) / (s2 - s1);
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.Bz - R.Bz) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bym - R.Bym) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.phi - R.phi) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.Ezm - R.Ezm) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Ey - R.Ey) / (s2 - s1);
    double lmL, lpL, lmR, lpR, sx1, sx2;
    hlle_bounds(R, fr, R.vx, lmR, lpR);
    hlle_bounds(L, fl, L.vx, lmL, lpL);
    int32_t st = hlle_speeds(lmL, lmR, lpL, lpR, sx1, sx2);
    const double DD_hll = (sx2 * R.D - sx1 * L.D + fl.FD - fr.FD) / (sx2 - sx1);
    const double tau_hll = (sx2 * R.tau - sx1 * L.tau + fl.Ftau - fr.Ftau) / (sx2 - sx1);
    const double Sx_hll = (sx2 * R.Sx - sx1 * L.Sx + fl.FSx - fr.FSx) / (sx2 - sx1);
    const double Sy_hll = (sx2 * R.Sy - sx1 * L.Sy + fl.FSy - fr.FSy) / (sx2 - sx1);
    const double Sz_hll = (sx2 * R.Sz - sx1 * L.Sz + fl.FSz - fr.FSz) / (sx2 - sx1);
    auto hlle = [&](double FL, double FR, double UL, double UR) {
      return (sx2 * FL - sx1 * FR + sx1 * sx2 * (UR - UL)) / (sx2 - sx1);
    };
    const double q_f = hlle(L.J, R.J, L.q, R.q);
    const double DD_f = hlle(fl.FD, fr.FD, L.D, R.D);
    const double tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
    const double Sx_f = hlle(fl.FSx, fr.FSx, L.Sx, R.Sx);
    const double Sy_f = hlle(fl.FSy, fr.FSy, L.Sy, R.Sy);
    const double Sz_f = hlle(fl.FSz, fr.FSz, L.Sz, R.Sz);
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Eys) + pw2(Ezs));
    const double B2_perp = (pw2(Bys) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_x;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sx_f;
    const double c_hll = Sx_hll - ErotB_x;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = 1.0e-6;   // double literal here, 16_hlle_flow_mpx.f95:3172
    if (std::fabs(V) <= 1.0e-9) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sx_f + (pw2(Exs) + pw2(Bxs)) - (tau_f - ErotB_x) * V;
    const double SxR = (sx2 * Sx_hll - tau_f * V) / (sx2 - V);
    const double SxL = (-sx1 * Sx_hll + tau_f * V) / (V - sx1);
    const double SyR = (sx2 * Sy_hll - Sy_f - ErotB_y * V - Exs * Eys - Bxs * Bys) / (sx2 - V);
    const double SyL = (-sx1 * Sy_hll + Sy_f + ErotB_y * V + Exs * Eys + Bxs * Bys) / (V - sx1);
    const double SzR = (sx2 * Sz_hll - Sz_f - ErotB_z * V - Exs * Ezs - Bxs * Bzs) / (sx2 - V);
    const double SzL = (-sx1 * Sz_hll + Sz_f + ErotB_z * V + Exs * Ezs + Bxs * Bzs) / (V - sx1);
    const double tauR = (SxR - ErotB_x) / V - pstr + E2B2_str;
    const double tauL = (SxL - ErotB_x) / V - pstr + E2B2_str;
    const double DR = (sx2 * DD_hll - DD_f) / (sx2 - V);
    const double DL = (-sx1 * DD_hll + DD_f) / (V - sx1);
    double fDR = DD_f, fDL = DD_f, ftR = tau_f, ftL = tau_f, fSxR = Sx_f, fSxL = Sx_f, fSyR = Sy_f, fSyL = Sy_f,
           fSzR = Sz_f, fSzL = Sz_f;
    if (V != 0.0) {
      fDR = DD_f + sx2 * (V - sx1) * (DR - DL) / (sx2 - sx1);
      fDL = DD_f - sx1 * (sx2 - V) * (DR - DL) / (sx2 - sx1);
      ftR = tau_f + sx2 * (V - sx1) * (tauR - tauL) / (sx2 - sx1);
      ftL = tau_f - sx1 * (sx2 - V) * (tauR - tauL) / (sx2 - sx1);
      fSxR = Sx_f + sx2 * (V - sx1) * (SxR - SxL) / (sx2 - sx1);
      fSxL = Sx_f - sx1 * (sx2 - V) * (SxR - SxL) / (sx2 - sx1);
      fSyR = Sy_f + sx2 * (V - sx1) * (SyR - SyL) / (sx2 - sx1);
      fSyL = Sy_f - sx1 * (sx2 - V) * (SyR - SyL) / (sx2 - sx1);
      fSzR = Sz_f + sx2 * (V - sx1) * (SzR - SzL) / (sx2 - sx1);
      fSzL = Sz_f - sx1 * (sx2 - V) * (SzR - SzL) / (sx2 - sx1);
    }
    // EM, psi, phi: HLL fluxes (out[0..15], set by the caller) in both v* branches
    if (sx1 >= 0.0) {
      out[16] = L.J; out[18] = fl.FD; out[20] = fl.Ftau; out[22] = fl.FSx; out[23] = fl.FSy; out[24] = fl.FSz;
    } else if (sx1 <= 0.0 && 0.0 <= V) {
      out[16] = q_f; out[18] = fDL; out[20] = ftL; out[22] = fSxL; out[23] = fSyL; out[24] = fSzL;
    } else if (V <= 0.0 && 0.0 <= sx2) {
      out[16] = q_f; out[18] = fDR; out[20] = ftR; out[22] = fSxR; out[23] = fSyR; out[24] = fSzR;
    } else if (sx2 < 0.0) {
      out[16] = R.J; out[18] = fr.FD; out[20] = fr.Ftau; out[22] = fr.FSx; out[23] = fr.FSy; out[24] = fr.FSz;
    } else {   // the reference stops, :4284-4285
      st |= ST_HLLC_VSTAR;
      for (int c : {16, 18, 20, 22, 23, 24}) out[c] = NAN;
    }
    return st;
  }

  int32_t hlle_y(const Side& L, const Side& R, const PhysX& fl, const PhysX& fr, double* out) {
    const double s1 = -1.0, s2 = 1.0;
    const double Ey_hll = (s2 * R.Ey - s1 * L.Ey + L.psi - R.psi) / (s2 - s1);
    const double Ez_hll = (s2 * R.Ez - s1 * L.Ez + L.Bx - R.Bx) / (s2 - s1);
    const double Ex_hll = (s2 * R.Ex - s1 * L.Ex + L.Bzm - R.Bzm) / (s2 - s1);
    const double By_hll = (s2 * R.By - s1 * L.By + L.phi - R.phi) / (s2 - s1);
    const double Bz_hll = (s2 * R.Bz - s1 * L.Bz + L.Exm - R.Exm) / (s2 - s1);
    const double Bx_hll = (s2 * R.Bx - s1 * L.Bx + L.Ez - R.Ez) / (s2 - s1);
    double lmL, lpL, lmR, lpR, sy1, sy2;
    hlle_bounds(R, fr, R.vy, lmR, lpR);
    hlle_bounds(L, fl, L.vy, lmL, lpL);
    int32_t st = hlle_speeds(lmL, lmR, lpL, lpR, sy1, sy2);
    const double DD_hll = (sy2 * R.D - sy1 * L.D + fl.FD - fr.FD) / (sy2 - sy1);
    const double tau_hll = (sy2 * R.tau - sy1 * L.tau + fl.Ftau - fr.Ftau) / (sy2 - sy1);
    const double Sy_hll = (sy2 * R.Sy - sy1 * L.Sy + fl.FSy - fr.FSy) / (sy2 - sy1);
    const double Sz_hll = (sy2 * R.Sz - sy1 * L.Sz + fl.FSz - fr.FSz) / (sy2 - sy1);
    const double Sx_hll = (sy2 * R.Sx - sy1 * L.Sx + fl.FSx - fr.FSx) / (sy2 - sy1);
    auto hlle = [&](double FL, double FR, double UL, double UR) {
      return (sy2 * FL - sy1 * FR + sy1 * sy2 * (UR - UL)) / (sy2 - sy1);
    };
    const double q_f = hlle(L.J, R.J, L.q, R.q);
    const double DD_f = hlle(fl.FD, fr.FD, L.D, R.D);
    const double tau_f = hlle(fl.Ftau, fr.Ftau, L.tau, R.tau);
    const double Sy_f = hlle(fl.FSy, fr.FSy, L.Sy, R.Sy);
    const double Sz_f = hlle(fl.FSz, fr.FSz, L.Sz, R.Sz);
    const double Sx_f = hlle(fl.FSx, fr.FSx, L.Sx, R.Sx);
    const double Exs = Ex_hll, Eys = Ey_hll, Ezs = Ez_hll, Bxs = Bx_hll, Bys = By_hll, Bzs = Bz_hll;
    const double ErotB_x = (Bzs * Eys - Bys * Ezs);
    const double ErotB_y = (Bxs * Ezs - Bzs * Exs);
    const double ErotB_z = (Bys * Exs - Bxs * Eys);
    const double E2_perp = (pw2(Exs) + pw2(Ezs));
    const double B2_perp = (pw2(Bxs) + pw2(Bzs));
    const double E2B2_str = 0.5 * ((pw2(Exs) + pw2(Eys) + pw2(Ezs)) + (pw2(Bxs) + pw2(Bys) + pw2(Bzs)));
    const double a_hll = tau_f - ErotB_y;
    const double b_hll = E2_perp + B2_perp - tau_hll - Sy_f;
    const double c_hll = Sy_hll - ErotB_y;
    const double det_hll = pw2(b_hll) - 4.0 * a_hll * c_hll;
    const double q_root1 = -0.5 * (b_hll + fsign(1.0, b_hll) * std::fabs(std::sqrt(det_hll)));
    double rt2 = c_hll / q_root1;
    if (det_hll < 0.0) rt2 = c_hll / b_hll;
    double V = get_hllc_vel(a_hll, -b_hll, c_hll, rt2, &st);
    const double eps1 = 1.0e-6;
    if (std::fabs(V) <= 1.0e-9) V = 0.0;
    else if (std::fabs(V) > 1.0) V = fmax2(-1.0 + eps1, fmin2(1.0 - eps1, V));
    const double pstr = Sy_f + (pw2(Eys) + pw2(Bys)) - (tau_f - ErotB_y) * V;
    const double SyR = (sy2 * Sy_hll - tau_f * V) / (sy2 - V);
    const double SyL = (-sy1 * Sy_hll + tau_f * V) / (V - sy1);
    const double SzR = (sy2 * Sz_hll - Sz_f - ErotB_z * V - Eys * Ezs - Bys * Bzs) / (sy2 - V);
    const double SzL = (-sy1 * Sz_hll + Sz_f + ErotB_z * V + Eys * Ezs + Bys * Bzs) / (V - sy1);
    const double SxR = (sy2 * Sx_hll - Sx_f - ErotB_x * V - Eys * Exs - Bys * Bxs) / (sy2 - V);
    const double SxL = (-sy1 * Sx_hll + Sx_f + ErotB_x * V + Eys * Exs + Bys * Bxs) / (V - sy1);
    const double tauR = (SyR - ErotB_y) / V - pstr + E2B2_str;
    const double tauL = (SyL - ErotB_y) / V - pstr + E2B2_str;
    const double DR = (sy2 * DD_hll - DD_f) / (sy2 - V);
    const double DL = (-sy1 * DD_hll + DD_f) / (V - sy1);
    double fDR = DD_f, fDL = DD_f, ftR = tau_f, ftL = tau_f, fSxR = Sx_f, fSxL = Sx_f, fSyR = Sy_f, fSyL = Sy_f,
           fSzR = Sz_f, fSzL = Sz_f;
    if (V != 0.0) {
      fDR = DD_f + sy2 * (V - sy1) * (DR - DL) / (sy2 - sy1);
      fDL = DD_f - sy1 * (sy2 - V) * (DR - DL) / (sy2 - sy1);
      ftR = tau_f + sy2 * (V - sy1) * (tauR - tauL) / (sy2 - sy1);
      ftL = tau_f - sy1 * (sy2 - V) * (tauR - tauL) / (sy2 - sy1);
      fSxR = Sx_f + sy2 * (V - sy1) * (SxR - SxL) / (sy2 - sy1);
      fSxL = Sx_f - sy1 * (sy2 - V) * (SxR - SxL) / (sy2 - sy1);
      fSyR = Sy_f + sy2 * (V - sy1) * (SyR - SyL) / (sy2 - sy1);
      fSyL = Sy_f - sy1 * (sy2 - V) * (SyR - SyL) / (sy2 - sy1);
      fSzR = Sz_f + sy2 * (V - sy1) * (SzR - SzL) / (sy2 - sy1);
      fSzL = Sz_f - sy1 * (sy2 - V) * (SzR - SzL) / (sy2 - sy1);
    }
    if (sy1 >= 0.0) {
      out[17] = L.J; out[19] = fl.FD; out[21] = fl.Ftau; out[25] = fl.FSx; out[26] = fl.FSy; out[27] = fl.FSz;
    } else if (sy1 <= 0.0 && 0.0 <= V) {
      out[17] = q_f; out[19] = fDL; out[21] = ftL; out[25] = fSxL; out[26] = fSyL; out[27] = fSzL;
    } else if (V <= 0.0 && 0.0 <= sy2) {
      out[17] = q_f; out[19] = fDR; out[21] = ftR; out[25] = fSxR; out[26] = fSyR; out[27] = fSzR;
    } else if (sy2 < 0.0) {
      out[17] = R.J; out[19] = fr.FD; out[21] = fr.Ftau; out[25] = fr.FSx; out[26] = fr.FSy; out[27] = fr.FSz;
    } else {   // the reference stops, :4612-4613
      st |= ST_HLLC_VSTAR;
      for (int c : {17, 19, 21, 25, 26, 27}) out[c] = NAN;
    }
    return st;
  }

  // ---------------------------------------------- 17_fluxandsource.f95:441-635
  // z differences (X(i,j)-X(i,j))/Delz are kept as literal zeros.
  void fluxandsource(int l) {
    auto& Kl = K[l - 1];
    double *Ex = a("Exint"), *Ey = a("Eyint"), *Ez = a("Ezint"), *Bx = a("Bxint"), *By = a("Byint"),
           *Bz = a("Bzint"), *q = a("qint"), *psi = a("psiint"), *phi = a("phiint");
    double *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz"), *W = a("W");
    double *Exlaxpsi = a("Exlaxpsi"), *Eylaxpsi = a("Eylaxpsi"), *Bxlaxphi = a("Bxlaxphi"), *Bylaxphi = a("Bylaxphi");
    double *philaxBx = a("philaxBx"), *EzlaxBx = a("EzlaxBx"), *EzlaxBy = a("EzlaxBy"), *philaxBy = a("philaxBy");
    double *EylaxBz = a("EylaxBz"), *ExlaxBz = a("ExlaxBz"), *psilaxEx = a("psilaxEx"), *BzlaxEx = a("BzlaxEx");
    double *BzlaxEy = a("BzlaxEy"), *psilaxEy = a("psilaxEy"), *BylaxEz = a("BylaxEz"), *BxlaxEz = a("BxlaxEz");
    double *Jxlax = a("Jxlax"), *Jylax = a("Jylax"), *FDxlax = a("FDxlax"), *FDylax = a("FDylax");
    double *Ftauxlax = a("Ftauxlax"), *Ftauylax = a("Ftauylax");
    double *FSxxlax = a("FSxxlax"), *FSxylax = a("FSxylax"), *FSxzlax = a("FSxzlax");
    double *FSyxlax = a("FSyxlax"), *FSyylax = a("FSyylax"), *FSyzlax = a("FSyzlax");
    double *psiflux = Kl["psiflux"].data(), *phiflux = Kl["phiflux"].data(), *Bxflux = Kl["Bxflux"].data(),
           *Byflux = Kl["Byflux"].data(), *Bzflux = Kl["Bzflux"].data(), *Exf = Kl["Exastflux"].data(),
           *Eyf = Kl["Eyastflux"].data(), *Ezf = Kl["Ezastflux"].data(), *qflux = Kl["qflux"].data(),
           *Dflux = Kl["Dflux"].data(), *tauflux = Kl["tauflux"].data(), *Sxflux = Kl["Sxflux"].data(),
           *Syflux = Kl["Syflux"].data(), *Szflux = Kl["Szflux"].data(), *Exs = Kl["Exastsour"].data(),
           *Eys = Kl["Eyastsour"].data(), *Ezs = Kl["Ezastsour"].data();
    const double z = 0.0;  // (X(i,j,1,l) - X(i,j,1,l))/Delz for finite X
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j), km = id(i - 1, j), kn = id(i, j - 1);
        const double Edotv = Ex[k] * Vx[k] + Ey[k] * Vy[k] + Ez[k] * Vz[k];
        const double vrotB_x = (Bz[k] * Vy[k] - By[k] * Vz[k]);
        const double vrotB_y = (Bx[k] * Vz[k] - Bz[k] * Vx[k]);
        const double vrotB_z = (By[k] * Vx[k] - Bx[k] * Vy[k]);
        const double Vx_elec = Vx[k], Vy_elec = Vy[k], Vz_elec = Vz[k], W_elec = W[k];
        psiflux[k] = -(Exlaxpsi[k] - Exlaxpsi[km]) / Delx - (Eylaxpsi[k] - Eylaxpsi[kn]) / Dely - z / Delz
                     + q[k] - kappa_psi * psi[k];
        phiflux[k] = -(Bxlaxphi[k] - Bxlaxphi[km]) / Delx - (Bylaxphi[k] - Bylaxphi[kn]) / Dely - z / Delz
                     - kappa_phi * phi[k];
        Bxflux[k] = -(EzlaxBx[k] - EzlaxBx[kn]) / Dely + z / Delz - (philaxBx[k] - philaxBx[km]) / Delx;
        Byflux[k] = -(z) / Delz + (EzlaxBy[k] - EzlaxBy[km]) / Delx - (philaxBy[k] - philaxBy[kn]) / Dely;
        Bzflux[k] = -(EylaxBz[k] - EylaxBz[km]) / Delx + (ExlaxBz[k] - ExlaxBz[kn]) / Dely - z / Delz;
        Exf[k] = (BzlaxEx[k] - BzlaxEx[kn]) / Dely - z / Delz - (psilaxEx[k] - psilaxEx[km]) / Delx - q[k] * Vx_elec;
        Eyf[k] = z / Delz - (BzlaxEy[k] - BzlaxEy[km]) / Delx - (psilaxEy[k] - psilaxEy[kn]) / Dely - q[k] * Vy_elec;
        Ezf[k] = (BylaxEz[k] - BylaxEz[km]) / Delx - (BxlaxEz[k] - BxlaxEz[kn]) / Dely - z / Delz - q[k] * Vz_elec;
        Exs[k] = sigma * W_elec * (Ex[k] + vrotB_x - Edotv * Vx_elec);
        Eys[k] = sigma * W_elec * (Ey[k] + vrotB_y - Edotv * Vy_elec);
        Ezs[k] = sigma * W_elec * (Ez[k] + vrotB_z - Edotv * Vz_elec);
        qflux[k] = -(Jxlax[k] - Jxlax[km]) / Delx - (Jylax[k] - Jylax[kn]) / Dely - z / Delz;
        Dflux[k] = -(FDxlax[k] - FDxlax[km]) / Delx - (FDylax[k] - FDylax[kn]) / Dely - z / Delz;
        tauflux[k] = -(Ftauxlax[k] - Ftauxlax[km]) / Delx - (Ftauylax[k] - Ftauylax[kn]) / Dely - z / Delz;
        Sxflux[k] = -(FSxxlax[k] - FSxxlax[km]) / Delx - (FSyxlax[k] - FSyxlax[kn]) / Dely - z / Delz;
        Syflux[k] = -(FSxylax[k] - FSxylax[km]) / Delx - (FSyylax[k] - FSyylax[kn]) / Dely - z / Delz;
        Szflux[k] = -(FSxzlax[k] - FSxzlax[km]) / Delx - (FSyzlax[k] - FSyzlax[kn]) / Dely - z / Delz;
      }
  }

  // ------------------------------------------------------- 18_sumfin.f95:20-66
  void sumfin(int l) {
    auto& Kl = K[l - 1];
    const double w = T.wb[l - 1], wt = T.wbt[l - 1];
    const char* s[] = {"psifinsum", "phifinsum", "Bxfinsum", "Byfinsum", "Bzfinsum", "qfinsum", "Dfinsum",
                       "taufinsum", "Sxfinsum", "Syfinsum", "Szfinsum"};
    const char* f[] = {"psiflux", "phiflux", "Bxflux", "Byflux", "Bzflux", "qflux", "Dflux",
                       "tauflux", "Sxflux", "Syflux", "Szflux"};
    for (int c = 0; c < 11; ++c) {
      double* S = a(s[c]);
      const double* F = Kl[f[c]].data();
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); S[k] = S[k] + w * F[k]; }
    }
    const char* es[] = {"Exfinsum", "Eyfinsum", "Ezfinsum"};
    const char* ef[] = {"Exastflux", "Eyastflux", "Ezastflux"};
    const char* eo[] = {"Exastsour", "Eyastsour", "Ezastsour"};
    for (int c = 0; c < 3; ++c) {
      double* S = a(es[c]);
      const double* F = Kl[ef[c]].data();
      const double* O = Kl[eo[c]].data();
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); S[k] = S[k] + (w * F[k] - wt * O[k]); }
    }
  }

  // ----------------------------- 19_varfin.f95:16-54, 20_electricfield.f95:153-167
  void varfin_electricfield() {
    const char* dst[] = {"psi", "phi", "Bx", "By", "Bz", "q", "D", "tau", "Sx", "Sy", "Sz", "Ex", "Ey", "Ez"};
    const char* sum[] = {"psifinsum", "phifinsum", "Bxfinsum", "Byfinsum", "Bzfinsum", "qfinsum", "Dfinsum",
                         "taufinsum", "Sxfinsum", "Syfinsum", "Szfinsum", "Exfinsum", "Eyfinsum", "Ezfinsum"};
    for (int c = 0; c < 14; ++c) {
      double* d = a(dst[c]);
      const double* S = a(sum[c]);
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) { const size_t k = id(i, j); d[k] = d[k] + Delt * S[k]; }
    }
  }

  // ------------------------------------------------------ con2prim (l_swap = 1)
  void con2prim() {
    double *D = a("D"), *tau = a("tau"), *Sx = a("Sx"), *Sy = a("Sy"), *Sz = a("Sz");
    double *Ex = a("Ex"), *Ey = a("Ey"), *Ez = a("Ez"), *Bx = a("Bx"), *By = a("By"), *Bz = a("Bz");
    double *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz"), *rho = a("rho"), *p = a("p"), *W = a("W");
    int32_t st_acc = 0;
    int64_t c0 = 0, c1 = 0, c2 = 0;
#pragma omp parallel for schedule(static) reduction(| : st_acc) reduction(+ : c0, c1, c2)
    for (int j = 0; j <= jmax; ++j)
      for (int i = 0; i <= imax; ++i) {
        const size_t k = id(i, j);
        C2PIn in{D[k], tau[k], Sx[k], Sy[k], Sz[k], Ex[k], Ey[k], Ez[k], Bx[k], By[k], Bz[k],
                 Vx[k], Vy[k], Vz[k], rho[k], p[k]};
        C2POut o;
        int64_t cnt[3] = {0, 0, 0};
        int32_t st = (P.c2p == 1) ? c2p_cardano(in, gamma, eps1_c2p, o, cnt) : c2p_nr(in, gamma, o);
        // NaN states pass the reference's checks silently; report them
        if (!(std::isfinite(o.rho) && std::isfinite(o.p) && std::isfinite(o.vx) && std::isfinite(o.vy) &&
              std::isfinite(o.vz)))
          st |= ST_NONFINITE;
        st_acc |= st;
        c0 += cnt[0]; c1 += cnt[1]; c2 += cnt[2];
        Vx[k] = o.vx; Vy[k] = o.vy; Vz[k] = o.vz; rho[k] = o.rho; p[k] = o.p; W[k] = o.W;
      }
    status |= st_acc;
    counters[0] += c0; counters[1] += c1; counters[2] += c2;
  }

  void boundary_prims() {
    const char* n[] = {"psi", "phi", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "Vx", "Vy", "Vz", "q", "p", "rho"};
    for (const char* s : n) fill_ghosts(a(s));
  }

  // ------------------------- 05_reconstruct.f95:525-746 (primitive_rec = 1, DIM == 2)
  // MC-limited slopes along the grid diagonal (i-1,j-1), (i,j), (i+1,j+1),
  // (i+2,j+2): L(i,j) = u + slope/2, R(i+1,j+1) = u(i+1,j+1) - slope'/2, and
  // the new value is the mean of R and L of the point.  Both faces of a
  // point take the same limiter arguments, so the mean equals u up to the
  // rounding of (u - x) + (u + x); the reference does exactly this.
  void recons_var_primitive() {
    const char* n[] = {"psi", "phi", "Bx", "By", "Bz", "Ex", "Ey", "Ez", "Vx", "Vy", "Vz", "q", "p", "rho"};
    std::vector<double> L(ng, 0.0), R(ng, 0.0);
    for (const char* f : n) {
      double* u = a(f);
#pragma omp parallel for schedule(static)
      for (int j = -2; j <= jmax; ++j)
        for (int i = -2; i <= imax; ++i) {
          const double um1 = u[id(i - 1, j - 1)], m = u[id(i, j)], p1 = u[id(i + 1, j + 1)], p2 = u[id(i + 2, j + 2)];
          L[id(i, j)] = m + 0.5 * limiter_mc(p1 - m, m - um1);
          R[id(i + 1, j + 1)] = p1 - 0.5 * limiter_mc(p2 - p1, p1 - m);
        }
#pragma omp parallel for schedule(static)
      for (int j = 0; j <= jmax; ++j)
        for (int i = 0; i <= imax; ++i) u[id(i, j)] = 0.5 * (R[id(i, j)] + L[id(i, j)]);
    }
  }

  // main_cueva_code.f95:53-328 stages part
  void begin_step() {
    boundary_prims();   // :53
    if (P.primitive_rec) {   // :170-175
      recons_var_primitive();
      boundary_prims();
    }
    startconvar();      // :181
    cleanvarint();      // :184
  }
  void stage(int l) {
    if (P.intsum_reset) {   // optional textbook variant; the reference zeroes intsum once per step
      const char* sn[] = {"psiintsum", "phiintsum", "Bxintsum", "Byintsum", "Bzintsum", "Exastsum", "Eyastsum",
                          "Ezastsum", "qintsum", "Dintsum", "tauintsum", "Sxintsum", "Syintsum", "Szintsum"};
      for (const char* n : sn) std::fill(A[n].begin(), A[n].end(), 0.0);
    }
    for (int m = 1; m <= l - 1; ++m) sumint(l, m);   // :205-211
    varint();                                       // :214
    {
      // Exast ghosts are never read; only E_l carries boundary data
    }
    electricvarint(l);                              // :216
    flowinit();                                     // :238 (+ boundary_flux_conserved :242)
    reconstruct();                                  // 16_*_flow_mpx.f95 passes
    riemann();
    fluxandsource(l);                               // :284
    sumfin(l);                                      // :286
  }
  void finish_step() {
    varfin_electricfield();                         // :295-297
    con2prim();                                     // :312-326
    boundary_prims();                               // :328
  }
  int32_t step(int n) {
    for (int h = 0; h < n; ++h) {
      begin_step();
      for (int l = 1; l <= lmax; ++l) stage(l);
      finish_step();
    }
    return status;
  }
  // ------------------------------------- 22_writer.f95:821-1019 (lector, DIM == 2)
  // The writer's sums in its own loop order (i outer, j inner), each term
  // evaluated as written; abs[k] collects sum |term| of every sum (both
  // terms of eint_r and efluid_r).  The writer also stores W, epsiln,
  // enthpy, E2 and B2 into the module arrays; startconvar recomputes all of
  // them before they are read again, so they stay local here.
  void lector(double B0, double Lr, double Ly, double delta_rec, double* v, double* ab) {
    const double *psi = a("psi"), *phi = a("phi"), *Ex = a("Ex"), *Ey = a("Ey"), *Ez = a("Ez");
    const double *Bx = a("Bx"), *By = a("By"), *Bz = a("Bz"), *Vx = a("Vx"), *Vy = a("Vy"), *Vz = a("Vz");
    const double *q = a("q"), *p = a("p"), *rho = a("rho"), *D = a("D"), *tau = a("tau");
    double s[35] = {0.0}, sa[35] = {0.0};
    double mbx = -INFINITY, mphi = -INFINITY, mv = -INFINITY, mW = -INFINITY, mlx = -INFINITY, mly = -INFINITY;
    auto add = [&](int k, double t) { s[k] = s[k] + t; sa[k] = sa[k] + std::fabs(t); };
    const double dx = Delx, dy = Dely;
    for (int i = 0; i <= imax; ++i)
      for (int j = 0; j <= jmax; ++j) {
        const size_t k = id(i, j);
        add(0, psi[k] * dx * dy);
        add(1, phi[k] * dx * dy);
        add(2, pw2(Ex[k]) * dx * dy);
        add(3, pw2(Ey[k]) * dx * dy);
        add(4, pw2(Ez[k]) * dx * dy);
        add(5, Ex[k] * Ey[k] * dx * dy);
        add(6, Ex[k] * Ez[k] * dx * dy);
        add(7, Ey[k] * Ez[k] * dx * dy);
        add(8, pw2(Bx[k]) * dx * dy);
        add(9, pw2(By[k]) * dx * dy);
        add(10, pw2(Bz[k]) * dx * dy);
        mbx = std::fmax(mbx, Bx[k] / B0);      // max_bx(i,j) = Bx / B0
        mphi = std::fmax(mphi, phi[k]);
        add(11, Bx[k] * By[k] * dx * dy);
        add(12, Bx[k] * Bz[k] * dx * dy);
        add(13, By[k] * Bz[k] * dx * dy);
        add(15, (pw2(Bx[k]) + pw2(By[k]) + pw2(Bz[k])) * dx * dy);   // sum_bxbybz
        add(14, (pw2(Vx[k]) + pw2(Vy[k]) + pw2(Vz[k])) * dx * dy);   // sum_vxvyvz
        add(16, pw2(Vx[k]) * dx * dy);
        add(17, pw2(Vy[k]) * dx * dy);
        add(18, pw2(Vz[k]) * dx * dy);
        add(19, Vx[k] * Vy[k] * dx * dy);
        add(20, Vx[k] * Vz[k] * dx * dy);
        add(21, Vy[k] * Vz[k] * dx * dy);
        add(22, q[k] * dx * dy);
        add(23, p[k] * dx * dy);
        add(24, rho[k] * dx * dy);
        add(33, D[k] * dx * dy);
        const double eps = p[k] / ((gamma - 1.0) * rho[k]);
        const double enth = rho[k] * (1.0 + eps) + p[k];
        const double W = 1.0 / std::sqrt(1.0 - (pw2(Vx[k]) + pw2(Vy[k]) + pw2(Vz[k])));
        const double E2 = pw2(Ex[k]) + pw2(Ey[k]) + pw2(Ez[k]);
        const double B2 = pw2(By[k]) + pw2(Bz[k]);
        add(25, 0.5 * rho[k] * (pw2(Vx[k]) + pw2(Vy[k]) + pw2(Vz[k])) * dx * dy);   // ekin_c
        add(26, D[k] * (W - 1.0) * dx * dy);                                        // ekin_r
        add(30, rho[k] * eps * dx * dy);                                            // eint_c
        {  // eint_r = eint_r + W**2 * (rho*eps + p) - p * Delx * Dely
          const double t1 = pw2(W) * (rho[k] * eps + p[k]), t2 = p[k] * dx * dy;
          s[31] = s[31] + t1 - t2;
          sa[31] = sa[31] + std::fabs(t1) + std::fabs(t2);
        }
        add(27, tau[k] * dx * dy);                                                  // etot
        {  // efluid_r = efluid_r + enthpy * W**2 - p * Delx * Dely
          const double t1 = enth * pw2(W), t2 = p[k] * dx * dy;
          s[28] = s[28] + t1 - t2;
          sa[28] = sa[28] + std::fabs(t1) + std::fabs(t2);
        }
        add(29, 0.5 * (E2 + B2) * dx * dy);                                         // emag (0.5 is exact in REAL*4)
        add(32, W * dx * dy);                                                       // lorentz
        // Courant check (no counterpart in the writer)
        const double V2 = pw2(Vx[k]) + pw2(Vy[k]) + pw2(Vz[k]);
        const double cs2 = gamma * p[k] / enth;
        mv = std::fmax(mv, std::sqrt(V2));
        mW = std::fmax(mW, W);
        mlx = std::fmax(mlx, sound_lambda(Vx[k], V2, cs2));
        mly = std::fmax(mly, sound_lambda(Vy[k], V2, cs2));
      }
    const int imed1 = (int)std::floor(0.25 * imax), imed2 = (int)std::floor(0.75 * imax);
    for (int i = imed1; i <= imed2; ++i)
      for (int j = 0; j <= jmax; ++j) add(34, D[id(i, j)] * dx * dy);
    for (int k = 0; k < 35; ++k) { v[k] = s[k]; if (ab) ab[k] = sa[k]; }
    v[35] = mbx;
    v[36] = mphi;
    const int imed = imax / 2, jmed = jmax / 2;    // floor(0.5d0*imax), floor(0.5d0*jmax)
    const double posy = -0.5 * Ly + (jmed + 1) * Dely;
    const double r = std::sqrt(1.0 - pw2(posy) / pw2(Lr));
    const double by = a("By")[id(std::min(imed + 1, imax), std::min(jmed + 1, jmax))];
    v[37] = B0 * r * std::tanh(Delx / delta_rec) * delta_rec / by;
    v[38] = a("Ez")[id(imed, jmed)];
    v[39] = by;
    v[40] = mv;
    v[41] = mW;
    v[42] = mlx;
    v[43] = mly;
    v[44] = std::fmax(Delt * (mlx / Delx), Delt * (mly / Dely));
  }
  // largest |lambda| of the two relativistic sound waves along a direction
  // with normal velocity vn (cs2 = gamma p / (rho h))
  static double sound_lambda(double vn, double V2, double cs2) {
    const double cs = std::sqrt(cs2);
    const double root = std::sqrt((1.0 - V2) * (1.0 - V2 * cs2 - vn * vn * (1.0 - cs2)));
    const double den = 1.0 - cs2 * V2;
    const double lp = (vn * (1.0 - cs2) + cs * root) / den;
    const double lm = (vn * (1.0 - cs2) - cs * root) / den;
    return std::fmax(std::fabs(lp), std::fabs(lm));
  }
};

const char* prim_names[OR_NPRIM] = {"rho", "p", "Vx", "Vy", "Vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"};

}  // namespace

// ============================================================== C API
extern "C" {

void* oracle_create(const oracle_params* p) {
  if (!p || p->imax < 6 || p->jmax < 6) return nullptr;
  if (p->flux_solver < 1 || p->flux_solver > 7) return nullptr;   // main_cueva_code.f95:247-279
  if (p->rec_mp < 0 || p->rec_mp > 2) return nullptr;
  if (p->primitive_rec < 0 || p->primitive_rec > 1) return nullptr;
  Tableau T;
  if (!make_tableau(p->order, T)) return nullptr;
  return new Oracle(*p);
}
void oracle_destroy(void* h) { delete static_cast<Oracle*>(h); }
void oracle_set_libm_seed(int32_t on) { g_libm_seed = on ? 1 : 0; }
void oracle_chebyshev_roots(double y, double* out3) { chebyshev_roots(y, out3[0], out3[1], out3[2]); }
double oracle_cbrt(double x) { return cbrt_newton(x); }
void oracle_set_threads(int32_t n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}
double oracle_dt(void* h) { return static_cast<Oracle*>(h)->Delt; }

void oracle_set_prims(void* h, const double* const* f) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int c = 0; c < OR_NPRIM; ++c) {
    double* d = o->a(prim_names[c]);
    for (int j = 0; j <= o->jmax; ++j)
      for (int i = 0; i <= o->imax; ++i) d[o->id(i, j)] = f[c][(size_t)i + (size_t)j * (o->imax + 1)];
  }
  o->boundary_prims();
}
void oracle_get_prims(void* h, double* const* f) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int c = 0; c < OR_NPRIM; ++c) {
    const double* d = o->a(prim_names[c]);
    for (int j = 0; j <= o->jmax; ++j)
      for (int i = 0; i <= o->imax; ++i) f[c][(size_t)i + (size_t)j * (o->imax + 1)] = d[o->id(i, j)];
  }
}
int32_t oracle_step(void* h, int32_t n) { return static_cast<Oracle*>(h)->step(n); }
int32_t oracle_run_stages(void* h, int32_t upto) {
  Oracle* o = static_cast<Oracle*>(h);
  o->begin_step();
  for (int l = 1; l <= upto && l <= o->lmax; ++l) o->stage(l);
  return o->status;
}
int32_t oracle_get_named(void* h, const char* name, int32_t l, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const double* src = nullptr;
  auto it = o->A.find(name);
  if (it != o->A.end()) src = it->second.data();
  else if (l >= 1 && l <= o->lmax) {
    auto jt = o->K[l - 1].find(name);
    if (jt != o->K[l - 1].end()) src = jt->second.data();
  }
  if (!src) return -1;
  for (int j = 0; j <= o->jmax; ++j)
    for (int i = 0; i <= o->imax; ++i) out[(size_t)i + (size_t)j * (o->imax + 1)] = src[o->id(i, j)];
  return 0;
}
// the whole ghosted array (-6..imax+6) x (-6..jmax+6), i fastest
int32_t oracle_get_named_full(void* h, const char* name, int32_t l, double* out) {
  Oracle* o = static_cast<Oracle*>(h);
  const double* src = nullptr;
  auto it = o->A.find(name);
  if (it != o->A.end()) src = it->second.data();
  else if (l >= 1 && l <= o->lmax) {
    auto jt = o->K[l - 1].find(name);
    if (jt != o->K[l - 1].end()) src = jt->second.data();
  }
  if (!src) return -1;
  std::copy(src, src + o->ng, out);
  return 0;
}
void oracle_counters(void* h, int64_t* out3) {
  Oracle* o = static_cast<Oracle*>(h);
  for (int c = 0; c < 3; ++c) out3[c] = o->counters[c];
}

void oracle_kh_init(int32_t imax, int32_t jmax, double lx, double ly, double v0, double a, double amp,
                    double width, double kpert, double phase, double bshear, double rho0, double p0,
                    double* const* f) {
  const double Delx = lx / (double)imax, Dely = ly / (double)jmax;
  for (int j = 0; j <= jmax; ++j)
    for (int i = 0; i <= imax; ++i) {
      const size_t k = (size_t)i + (size_t)j * (imax + 1);
      const double posx = -0.5 * lx + i * Delx;   // reference x = problem y (shear normal)
      const double posy = -0.5 * ly + j * Dely;   // reference y = problem x (periodic, along the flow)
      const double vx = amp * std::sin(kpert * posy + phase) * std::exp(-(posx * posx) / width);
      const double vy = v0 * std::tanh(posx / a);
      const double vz = 0.0;
      const double Bx = 0.0, By = bshear, Bz = 0.0;
      f[OR_RHO][k] = rho0; f[OR_P][k] = p0;
      f[OR_VX][k] = vx; f[OR_VY][k] = vy; f[OR_VZ][k] = vz;
      f[OR_PSI][k] = 0.0; f[OR_PHI][k] = 0.0; f[OR_Q][k] = 0.0;
      f[OR_BX][k] = Bx; f[OR_BY][k] = By; f[OR_BZ][k] = Bz;
      f[OR_EX][k] = -(vy * Bz - vz * By);
      f[OR_EY][k] = -(vz * Bx - vx * Bz);
      f[OR_EZ][k] = -(vx * By - vy * Bx);
    }
}

void oracle_mp_line(int32_t rec_mp, int32_t n, const double* u, int32_t posfix, double* up, double* um) {
  mp_line(rec_mp, n, u, posfix, up, um);
}
double oracle_hllc_vel(double a, double b, double c, double rt) { return get_hllc_vel(a, b, c, rt, nullptr); }
int32_t oracle_c2p_cardano(const double* in, double gamma, double eps1, double* out) {
  C2PIn i{in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], in[9], in[10],
          in[11], in[12], in[13], in[14], in[15]};
  C2POut o;
  int32_t st = c2p_cardano(i, gamma, eps1, o, nullptr);
  out[0] = o.vx; out[1] = o.vy; out[2] = o.vz; out[3] = o.rho; out[4] = o.p; out[5] = o.W;
  return st;
}
int32_t oracle_c2p_nr(const double* in, double gamma, double* out) {
  C2PIn i{in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8], in[9], in[10],
          in[11], in[12], in[13], in[14], in[15]};
  C2POut o;
  int32_t st = c2p_nr(i, gamma, o);
  out[0] = o.vx; out[1] = o.vy; out[2] = o.vz; out[3] = o.rho; out[4] = o.p; out[5] = o.W;
  return st;
}
void oracle_lector(void* h, double b0, double lr, double ly, double delta_rec, int32_t d_from_startconvar,
                   double* out45, double* abs45) {
  Oracle* o = static_cast<Oracle*>(h);
  if (d_from_startconvar) o->startconvar();
  o->lector(b0, lr, ly, delta_rec, out45, abs45);
}
int32_t oracle_tableau(int32_t order, double* wb8, double* wbt8, double* ab64, double* abt64) {
  Tableau T;
  if (!make_tableau(order, T)) return -1;
  for (int a = 0; a < 8; ++a) {
    wb8[a] = T.wb[a]; wbt8[a] = T.wbt[a];
    for (int b = 0; b < 8; ++b) { ab64[a * 8 + b] = T.Ab[a][b]; abt64[a * 8 + b] = T.Abt[a][b]; }
  }
  return T.s;
}

}  // extern "C"
