// acs_oracle.cpp -- CPU ORACLE for the artificial-compressibility pseudo-time loop.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (the CUDA library, its C ABI or the
// Python host layer) links, loads or calls this file.  It is used by tests/, by the smoke
// check in __graft_entry__.py and by the CPU-baseline leg of bench.py, always as the checker
// or the timed CPU baseline, never as the thing measured or shipped.
//
// It restates, expression by expression, the OpenMP Fortran reference (paths are relative to
// the reference project):
//   OpenMp_Multicore/equations.f90   RESU :2-116, upwind_Ui :120-178, upwind_Uj :182-240,
//                                    solve_U :244-301, RESV :305-420, upwind_Vi :423-481,
//                                    upwind_Vj :485-542, solve_V :546-603, solve_P :607-665,
//                                    solve_Z :669-719, RESZ :723-765, solve_C :769-819,
//                                    RESC :823-867
//   OpenMp_Multicore/boundary.f90    bcUV :1-49, bcP :52-73, bcZ :76-116, bcC :119-159
//   OpenMp_Multicore/main.f90        pseudo/physical loop :104-186
//   OpenMp_Multicore/nonsymetric_mesh.f90  mesh, metrics, flag -> epsilon1/liga_poros :1-218
//   OpenMp_Multicore/initial.f90     IC :20-49
//   OpenMp_Multicore/comum.f90       constants :29-46, 79-85, 112-115
//
// Floating point: every expression keeps the Fortran evaluation order (left to right for
// + - * /, `x**2.d0` -> x*x, `x**0.5d0` -> sqrt(x)) and the file is compiled with
// -ffp-contract=off so no multiply-add is fused.  Max reductions are order independent, so
// the OpenMP build gives bit-identical results for any thread count.
//
// Generalisations (all off by default, i.e. reference behaviour):
//   * runtime imax/jmax, physical constants, dt, dtau, beta, eps, itc_max;
//   * scheme 1 = first-order upwind everywhere (the upwind_U*/upwind_V* coefficients);
//   * bc 1 = channel: inlet on the left, outflow on the right, no-slip walls top and bottom
//     (the rules are written out in bc_uv_channel/bc_p_channel/bc_s_channel below);
//   * a channel mesh generator (uniform x, two-sided tanh clustering in y) and a
//     rectangular porous block, both reusing the reference flag-dilation rule.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {

// Parameter block.  Field order is mirrored by oracle/oracle.py (ctypes).
struct orc_params {
  int imax, jmax;      // p-node counts in x and y (the reference's imax, jmax)
  int scheme;          // 0 = QUICK + first-order upwind next to the edges, 1 = upwind everywhere
  int bc;              // 0 = reference boundary passes, 1 = channel
  int solve_scalars;   // 1 = solve_Z and solve_C run in the pseudo loop
  int itc_max;         // pseudo-iteration cap per physical step (main.f90:120)
  double Re, Pe, Sc;   // comum.f90:112-115
  double Da, Cf;       // Darcy number, Forchheimer coefficient (comum.f90:30-31)
  double g;            // body force on u (comum.f90:79), applied as -g*epsilon1 (equations.f90:104)
  double InvFr2;       // buoyancy coefficient (comum.f90:85; Richardson number in the channel set-up)
  double v_in;         // inflow velocity: v_i (bottom) for bc 0, u on the left for bc 1
  double T_in;         // Tinf: T on the inflow boundary (boundary.f90:86)
  double C_in;         // C on the inflow boundary (0 in boundary.f90:129)
  double b_art;        // artificial bulk viscosity (iterations.dat)
  double beta;         // artificial compressibility
  double dt, dtau;     // physical and pseudo time steps (main.f90:105-106)
  double eps;          // convergence tolerance on max(res_u, res_v, res_p)
  int arith;           // solver option of the product (ignored here: the oracle has one arithmetic)
  int continuity;      // 0 = RP is the face-flux balance (equations.f90:623-625); 1 = the same
                       // divided by the p-cell volume vol_p (nonsymetric_mesh.f90:234-238)
};

}  // extern "C"

namespace {

struct Case {
  orc_params p;
  int nx, ny;
  // 1-based metric arrays, index 0 unused.
  std::vector<double> x, y, xm, ym;
  std::vector<double> eps, liga;  // nx*ny, column-major
  // Scratch that the reference keeps in module/local arrays.
  std::vector<double> RU, ui, RV, vi, RZ, Zi, RC, Ci, Pi, RPa, resp;
  Case(const orc_params& prm) : p(prm), nx(prm.imax), ny(prm.jmax) {}

  // Column-major 1-based accessors.  um: (nx+1) x ny, vm: nx x (ny+1), scalars: nx x ny.
  inline size_t iu(int i, int j) const { return (size_t)(i - 1) + (size_t)(j - 1) * (nx + 1); }
  inline size_t iv(int i, int j) const { return (size_t)(i - 1) + (size_t)(j - 1) * nx; }
  inline size_t ip(int i, int j) const { return (size_t)(i - 1) + (size_t)(j - 1) * nx; }

  double areau_ns(int i) const { return x[i] - x[i - 1]; }     // nonsymetric_mesh.f90:82-85
  double areau_ew(int j) const { return ym[j + 1] - ym[j]; }   // :87-90
  double areav_ns(int i) const { return xm[i + 1] - xm[i]; }   // :93-96
  double areav_ew(int j) const { return y[j] - y[j - 1]; }     // :98-101
};

inline double fmax0(double a) { return a > 0.0 ? a : 0.0; }

// ---------------------------------------------------------------------------------------
// RESU  (equations.f90:2-116) and its edge rows (upwind_Ui :120-178, upwind_Uj :182-240)
// ---------------------------------------------------------------------------------------
inline double resu_quick(const Case& c, const double* um, const double* vm, const double* p,
                         int i, int j) {
  const orc_params& P = c.p;
  const double e = c.eps[c.ip(i, j)], lg = c.liga[c.ip(i, j)];
  const double An = c.areau_ns(i), As = c.areau_ns(i), Ae = c.areau_ew(j), Aw = c.areau_ew(j);
  double fn = 0.5 * (vm[c.iv(i, j + 1)] + vm[c.iv(i - 1, j + 1)]) * An / e;
  double fs = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i - 1, j)]) * As / e;
  double fe = 0.5 * (um[c.iu(i + 1, j)] + um[c.iu(i, j)]) * Ae / e;
  double fw = 0.5 * (um[c.iu(i, j)] + um[c.iu(i - 1, j)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / P.Re) * An / (c.y[j + 1] - c.y[j]);
  double Ds = (e / P.Re) * As / (c.y[j] - c.y[j - 1]);
  double De = (e / P.Re) * Ae / (c.xm[i + 1] - c.xm[i]);
  double Dw = (e / P.Re) * Aw / (c.xm[i] - c.xm[i - 1]);
  // alpha flags (:27-49).  A flux of exactly 0 leaves the flag unchanged in the reference;
  // every flag only multiplies its own flux, so 0 or 1 give the same coefficients.
  double afw = fw > 0.0 ? 1.0 : 0.0, afe = fe > 0.0 ? 1.0 : 0.0;
  double afn = fn > 0.0 ? 1.0 : 0.0, afs = fs > 0.0 ? 1.0 : 0.0;
  double aw = Dw + 0.75 * afw * fw + 0.125 * afe * fe + 0.375 * (1.0 - afw) * fw;
  double ae = De - 0.375 * afe * fe - 0.75 * (1.0 - afe) * fe - 0.125 * (1.0 - afw) * fw;
  double as = Ds + 0.75 * afs * fs + 0.125 * afn * fn + 0.375 * (1.0 - afs) * fs;
  double an = Dn - 0.375 * afn * fn - 0.75 * (1.0 - afn) * fn - 0.125 * (1.0 - afs) * fs;
  double aww = -0.125 * afw * fw;
  double aee = 0.125 * (1.0 - afe) * fe;
  double ass = -0.125 * afs * fs;
  double ann = 0.125 * (1.0 - afn) * fn;
  double ap = aw + ae + as + an + aww + aee + ass + ann + df;
  double uW = um[c.iu(i - 1, j)], uWW = um[c.iu(i - 2, j)], uE = um[c.iu(i + 1, j)],
         uEE = um[c.iu(i + 2, j)], uS = um[c.iu(i, j - 1)], uSS = um[c.iu(i, j - 2)],
         uN = um[c.iu(i, j + 1)], uNN = um[c.iu(i, j + 2)], uP = um[c.iu(i, j)],
         vP = vm[c.iv(i, j)];
  double dudxdx = Ae * (uE - uP) / (c.xm[i + 1] - c.xm[i]) - Aw * (uP - uW) / (c.xm[i] - c.xm[i - 1]);
  double dxdvdy = Ae * (vm[c.iv(i, j + 1)] - vm[c.iv(i, j)]) / (c.ym[j + 1] - c.ym[j]) -
                  Aw * (vm[c.iv(i - 1, j + 1)] - vm[c.iv(i - 1, j)]) / (c.ym[j + 1] - c.ym[j]);
  double artDivU = -(P.b_art * (dudxdx + dxdvdy));
  double q_art = e * (p[c.ip(i, j)] - p[c.ip(i - 1, j)]) / (c.x[i] - c.x[i - 1]) + artDivU;
  return 1.0 / (c.x[i] - c.x[i - 1]) / (c.y[j] - c.y[j - 1]) *
             (-(ap * uP) + aww * uWW + aw * uW + aee * uEE + ae * uE + ass * uSS + as * uS +
              ann * uNN + an * uN) -
         q_art -
         e * (uP / (P.Re * P.Da) + P.Cf / std::sqrt(e * P.Da) * uP * std::sqrt(uP * uP + vP * vP)) * lg -
         P.g * e;
}

inline double resu_upwind(const Case& c, const double* um, const double* vm, const double* p,
                          int i, int j) {
  const orc_params& P = c.p;
  const double e = c.eps[c.ip(i, j)], lg = c.liga[c.ip(i, j)];
  const double An = c.areau_ns(i), As = c.areau_ns(i), Ae = c.areau_ew(j), Aw = c.areau_ew(j);
  double fn = 0.5 * (vm[c.iv(i, j + 1)] + vm[c.iv(i - 1, j + 1)]) * An / e;
  double fs = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i - 1, j)]) * As / e;
  double fe = 0.5 * (um[c.iu(i + 1, j)] + um[c.iu(i, j)]) * Ae / e;
  double fw = 0.5 * (um[c.iu(i, j)] + um[c.iu(i - 1, j)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / P.Re) * An / (c.y[j + 1] - c.y[j]);
  double Ds = (e / P.Re) * As / (c.y[j] - c.y[j - 1]);
  double De = (e / P.Re) * Ae / (c.xm[i + 1] - c.xm[i]);
  double Dw = (e / P.Re) * Aw / (c.xm[i] - c.xm[i - 1]);
  double aw = Dw + fmax0(fw);
  double as = Ds + fmax0(fs);
  double ae = De + fmax0(-fe);
  double an = Dn + fmax0(-fn);
  double ap = aw + ae + as + an + df;
  double uW = um[c.iu(i - 1, j)], uE = um[c.iu(i + 1, j)], uS = um[c.iu(i, j - 1)],
         uN = um[c.iu(i, j + 1)], uP = um[c.iu(i, j)], vP = vm[c.iv(i, j)];
  double dudxdx = Ae * (uE - uP) / (c.xm[i + 1] - c.xm[i]) - Aw * (uP - uW) / (c.xm[i] - c.xm[i - 1]);
  double dxdvdy = Ae * (vm[c.iv(i, j + 1)] - vm[c.iv(i, j)]) / (c.ym[j + 1] - c.ym[j]) -
                  Aw * (vm[c.iv(i - 1, j + 1)] - vm[c.iv(i - 1, j)]) / (c.ym[j + 1] - c.ym[j]);
  double q_art = e * (p[c.ip(i, j)] - p[c.ip(i - 1, j)]) / (c.x[i] - c.x[i - 1]) - P.b_art * (dudxdx + dxdvdy);
  return 1.0 / (c.x[i] - c.x[i - 1]) / (c.y[j] - c.y[j - 1]) *
             (-(ap * uP) + aw * uW + ae * uE + as * uS + an * uN) -
         q_art -
         e * (uP / (P.Re * P.Da) + P.Cf / std::sqrt(e * P.Da) * uP * std::sqrt(uP * uP + vP * vP)) * lg -
         P.g * e;
}

// RU over the u update region i = 3..imax-1, j = 2..jmax-1 (solve_U :262-263).  The reference
// also fills the columns i = 2 and i = imax with upwind values (:112-113); the update never
// reads them, so they are computed here too only to keep RU identical.
void RESU(Case& c, const double* um, const double* vm, const double* p, double* RU) {
  const int nx = c.nx, ny = c.ny;
  const bool upw_all = c.p.scheme == 1;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j) {
    for (int i = 2; i <= nx; ++i) {
      bool quick = !upw_all && j >= 3 && j <= ny - 2 && i >= 3 && i <= nx - 1;
      RU[c.iu(i, j)] = quick ? resu_quick(c, um, vm, p, i, j) : resu_upwind(c, um, vm, p, i, j);
    }
  }
}

// ---------------------------------------------------------------------------------------
// RESV  (equations.f90:305-420), upwind_Vi :423-481, upwind_Vj :485-542
// ---------------------------------------------------------------------------------------
inline double buoy(const Case& c, const double* T, int i, int j) {
  return c.p.InvFr2 * (1.0 - 1.0 / ((T[c.ip(i, j)] + T[c.ip(i, j - 1)]) * 0.5));
}

inline double resv_quick(const Case& c, const double* um, const double* vm, const double* p,
                         const double* T, int i, int j) {
  const orc_params& P = c.p;
  const double e = c.eps[c.ip(i, j)], lg = c.liga[c.ip(i, j)];
  const double An = c.areav_ns(i), As = c.areav_ns(i), Ae = c.areav_ew(j), Aw = c.areav_ew(j);
  double fn = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i, j + 1)]) * An / e;
  double fs = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i, j - 1)]) * As / e;
  double fe = 0.5 * (um[c.iu(i + 1, j)] + um[c.iu(i + 1, j - 1)]) * Ae / e;
  double fw = 0.5 * (um[c.iu(i, j)] + um[c.iu(i, j - 1)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / P.Re) * An / (c.ym[j + 1] - c.ym[j]);
  double Ds = (e / P.Re) * As / (c.ym[j] - c.ym[j - 1]);
  double De = (e / P.Re) * Ae / (c.x[i + 1] - c.x[i]);
  double Dw = (e / P.Re) * Aw / (c.x[i] - c.x[i - 1]);
  double afw = fw > 0.0 ? 1.0 : 0.0, afe = fe > 0.0 ? 1.0 : 0.0;
  double afn = fn > 0.0 ? 1.0 : 0.0, afs = fs > 0.0 ? 1.0 : 0.0;
  double aw = Dw + 0.75 * afw * fw + 0.125 * afe * fe + 0.375 * (1.0 - afw) * fw;
  double ae = De - 0.375 * afe * fe - 0.75 * (1.0 - afe) * fe - 0.125 * (1.0 - afw) * fw;
  double as = Ds + 0.75 * afs * fs + 0.125 * afn * fn + 0.375 * (1.0 - afs) * fs;
  double an = Dn - 0.375 * afn * fn - 0.75 * (1.0 - afn) * fn - 0.125 * (1.0 - afs) * fs;
  double aww = -0.125 * afw * fw;
  double aee = 0.125 * (1.0 - afe) * fe;
  double ass = -0.125 * afs * fs;
  double ann = 0.125 * (1.0 - afn) * fn;
  double ap = aw + ae + as + an + aww + aee + ass + ann + df;
  double vW = vm[c.iv(i - 1, j)], vWW = vm[c.iv(i - 2, j)], vE = vm[c.iv(i + 1, j)],
         vEE = vm[c.iv(i + 2, j)], vS = vm[c.iv(i, j - 1)], vSS = vm[c.iv(i, j - 2)],
         vN = vm[c.iv(i, j + 1)], vNN = vm[c.iv(i, j + 2)], vP = vm[c.iv(i, j)],
         uP = um[c.iu(i, j)];
  double dvdydy = An * (vN - vP) / (c.ym[j + 1] - c.ym[j]) - As * (vP - vS) / (c.ym[j] - c.ym[j - 1]);
  double dydudx = An * (um[c.iu(i + 1, j)] - um[c.iu(i, j)]) / (c.xm[i + 1] - c.xm[i]) -
                  As * (um[c.iu(i + 1, j - 1)] - um[c.iu(i, j - 1)]) / (c.xm[i + 1] - c.xm[i]);
  double artDivV = -(P.b_art * (dydudx + dvdydy));
  double q_art = e * (p[c.ip(i, j)] - p[c.ip(i, j - 1)]) / (c.y[j] - c.y[j - 1]) + artDivV;
  return 1.0 / (c.x[i] - c.x[i - 1]) / (c.y[j] - c.y[j - 1]) *
             (-(ap * vP) + aww * vWW + aw * vW + aee * vEE + ae * vE + ass * vSS + as * vS +
              ann * vNN + an * vN) -
         q_art + buoy(c, T, i, j) -
         e * (vP / (P.Re * P.Da) + P.Cf / std::sqrt(e * P.Da) * vP * std::sqrt(uP * uP + vP * vP)) * lg;
}

inline double resv_upwind(const Case& c, const double* um, const double* vm, const double* p,
                          const double* T, int i, int j) {
  const orc_params& P = c.p;
  const double e = c.eps[c.ip(i, j)], lg = c.liga[c.ip(i, j)];
  const double An = c.areav_ns(i), As = c.areav_ns(i), Ae = c.areav_ew(j), Aw = c.areav_ew(j);
  double fn = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i, j + 1)]) * An / e;
  double fs = 0.5 * (vm[c.iv(i, j)] + vm[c.iv(i, j - 1)]) * As / e;
  double fe = 0.5 * (um[c.iu(i + 1, j)] + um[c.iu(i + 1, j - 1)]) * Ae / e;
  double fw = 0.5 * (um[c.iu(i, j)] + um[c.iu(i, j - 1)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / P.Re) * An / (c.ym[j + 1] - c.ym[j]);
  double Ds = (e / P.Re) * As / (c.ym[j] - c.ym[j - 1]);
  double De = (e / P.Re) * Ae / (c.x[i + 1] - c.x[i]);
  double Dw = (e / P.Re) * Aw / (c.x[i] - c.x[i - 1]);
  double aw = Dw + fmax0(fw);
  double as = Ds + fmax0(fs);
  double ae = De + fmax0(-fe);
  double an = Dn + fmax0(-fn);
  double ap = aw + ae + as + an + df;
  double vW = vm[c.iv(i - 1, j)], vE = vm[c.iv(i + 1, j)], vS = vm[c.iv(i, j - 1)],
         vN = vm[c.iv(i, j + 1)], vP = vm[c.iv(i, j)], uP = um[c.iu(i, j)];
  double dvdydy = An * (vN - vP) / (c.ym[j + 1] - c.ym[j]) - As * (vP - vS) / (c.ym[j] - c.ym[j - 1]);
  double dydudx = An * (um[c.iu(i + 1, j)] - um[c.iu(i, j)]) / (c.xm[i + 1] - c.xm[i]) -
                  As * (um[c.iu(i + 1, j - 1)] - um[c.iu(i, j - 1)]) / (c.xm[i + 1] - c.xm[i]);
  double q_art = e * (p[c.ip(i, j)] - p[c.ip(i, j - 1)]) / (c.y[j] - c.y[j - 1]) - P.b_art * (dydudx + dvdydy);
  return 1.0 / (c.x[i] - c.x[i - 1]) / (c.y[j] - c.y[j - 1]) *
             (-(ap * vP) + aw * vW + ae * vE + as * vS + an * vN) -
         q_art + buoy(c, T, i, j) -
         e * (vP / (P.Re * P.Da) + P.Cf / std::sqrt(e * P.Da) * vP * std::sqrt(uP * uP + vP * vP)) * lg;
}

// RV over i = 2..imax-1, j = 3..jmax-1 (the update region of solve_V :564-565) plus the rows
// j = 2 and j = jmax that upwind_Vi fills (:413-414) and the update never reads.
void RESV(Case& c, const double* um, const double* vm, const double* p, const double* T, double* RV) {
  const int nx = c.nx, ny = c.ny;
  const bool upw_all = c.p.scheme == 1;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny; ++j) {
    for (int i = 2; i <= nx - 1; ++i) {
      bool quick = !upw_all && i >= 3 && i <= nx - 2 && j >= 3 && j <= ny - 1;
      RV[c.iv(i, j)] = quick ? resv_quick(c, um, vm, p, T, i, j) : resv_upwind(c, um, vm, p, T, i, j);
    }
  }
}

// ---------------------------------------------------------------------------------------
// Boundary passes.  bc 0 = boundary.f90 verbatim; bc 1 = channel.
// ---------------------------------------------------------------------------------------
void bc_uv_reference(Case& c, double* um, double* vm) {  // boundary.f90:1-49
  const int nx = c.nx, ny = c.ny;
  const double vi = c.p.v_in;
  for (int i = 1; i <= nx; ++i) { vm[c.iv(i, 1)] = vi; vm[c.iv(i, 2)] = vm[c.iv(i, 1)]; }
  for (int i = 2; i <= nx; ++i) um[c.iu(i, 1)] = 0.0;
  for (int i = 2; i <= nx; ++i) {
    vm[c.iv(i, ny)] = 2.0 * vm[c.iv(i, ny - 2)] - vm[c.iv(i, ny - 1)];
    vm[c.iv(i, ny + 1)] = 2.0 * vm[c.iv(i, ny - 1)] - vm[c.iv(i, ny)];
  }
  for (int i = 2; i <= nx; ++i) um[c.iu(i, ny)] = um[c.iu(i, ny - 1)];
  for (int j = 1; j <= ny; ++j) { um[c.iu(2, j)] = 0.0; um[c.iu(1, j)] = 0.0; }
  for (int j = 1; j <= ny + 1; ++j) vm[c.iv(1, j)] = vm[c.iv(2, j)];
  for (int j = 1; j <= ny; ++j) { um[c.iu(nx, j)] = 0.0; um[c.iu(nx + 1, j)] = 0.0; }
  for (int j = 2; j <= ny; ++j) vm[c.iv(nx, j)] = vm[c.iv(nx - 1, j)];
}

// Channel: inflow u = v_in through the face xm(2); zero-gradient outflow through xm(imax);
// no-slip walls on the faces ym(2) and ym(jmax) (odd ghost reflection).  The columns are set
// first, then the wall rows, so every value depends only on the current interior.
void bc_uv_channel(Case& c, double* um, double* vm) {
  const int nx = c.nx, ny = c.ny;
  const double uin = c.p.v_in;
  for (int j = 1; j <= ny; ++j) {
    um[c.iu(1, j)] = uin;
    um[c.iu(2, j)] = uin;
    um[c.iu(nx, j)] = um[c.iu(nx - 1, j)];
    um[c.iu(nx + 1, j)] = um[c.iu(nx, j)];
  }
  for (int i = 1; i <= nx + 1; ++i) {
    um[c.iu(i, 1)] = -um[c.iu(i, 2)];
    um[c.iu(i, ny)] = -um[c.iu(i, ny - 1)];
  }
  for (int j = 1; j <= ny + 1; ++j) {
    vm[c.iv(1, j)] = -vm[c.iv(2, j)];
    vm[c.iv(nx, j)] = vm[c.iv(nx - 1, j)];
  }
  for (int i = 1; i <= nx; ++i) {
    vm[c.iv(i, 2)] = 0.0;
    vm[c.iv(i, ny)] = 0.0;
    vm[c.iv(i, 1)] = -vm[c.iv(i, 3)];
    vm[c.iv(i, ny + 1)] = -vm[c.iv(i, ny - 1)];
  }
}

void bcUV(Case& c, double* um, double* vm) {
  if (c.p.bc == 1) bc_uv_channel(c, um, vm); else bc_uv_reference(c, um, vm);
}

void bcP(Case& c, double* pn) {
  const int nx = c.nx, ny = c.ny;
  if (c.p.bc == 0) {  // boundary.f90:52-73
    for (int i = 1; i <= nx; ++i) {
      pn[c.ip(i, 1)] = pn[c.ip(i, 2)];
      pn[c.ip(i, ny)] = pn[c.ip(i, ny - 1)] + 1.0 * (pn[c.ip(i, ny - 1)] - pn[c.ip(i, ny - 2)]);
    }
    for (int j = 1; j <= ny; ++j) { pn[c.ip(1, j)] = pn[c.ip(2, j)]; pn[c.ip(nx, j)] = pn[c.ip(nx - 1, j)]; }
  } else {  // channel: Neumann at the inlet, linear extrapolation at the outflow, Neumann walls
    for (int j = 1; j <= ny; ++j) {
      pn[c.ip(1, j)] = pn[c.ip(2, j)];
      pn[c.ip(nx, j)] = pn[c.ip(nx - 1, j)] + 1.0 * (pn[c.ip(nx - 1, j)] - pn[c.ip(nx - 2, j)]);
    }
    for (int i = 1; i <= nx; ++i) { pn[c.ip(i, 1)] = pn[c.ip(i, 2)]; pn[c.ip(i, ny)] = pn[c.ip(i, ny - 1)]; }
  }
}

// bcZ (boundary.f90:76-116, inflow value Tinf) and bcC (:119-159, inflow value 0) differ only
// in the inflow value; the channel variant mirrors them with the inflow on the left.
void bcS(Case& c, double* z, double zin) {
  const int nx = c.nx, ny = c.ny;
  if (c.p.bc == 0) {
    for (int i = 1; i <= nx; ++i) {
      z[c.ip(i, 1)] = zin;
      z[c.ip(i, ny)] = z[c.ip(i, ny - 1)] + 1.0 * (z[c.ip(i, ny - 1)] - z[c.ip(i, ny - 2)]);
    }
    for (int j = 1; j <= ny; ++j) { z[c.ip(1, j)] = z[c.ip(2, j)]; z[c.ip(nx, j)] = z[c.ip(nx - 1, j)]; }
  } else {
    for (int j = 1; j <= ny; ++j) {
      z[c.ip(1, j)] = zin;
      z[c.ip(nx, j)] = z[c.ip(nx - 1, j)] + 1.0 * (z[c.ip(nx - 1, j)] - z[c.ip(nx - 2, j)]);
    }
    for (int i = 1; i <= nx; ++i) { z[c.ip(i, 1)] = z[c.ip(i, 2)]; z[c.ip(i, ny)] = z[c.ip(i, ny - 1)]; }
  }
}
inline double c_inflow(const Case& c) { return c.p.C_in; }

// ---------------------------------------------------------------------------------------
// solve_U (equations.f90:244-301)
// ---------------------------------------------------------------------------------------
double solve_U(Case& c, const double* um, const double* um_tau, double* vm_tau, const double* p,
               double* um_n_tau) {
  const int nx = c.nx, ny = c.ny;
  const double dt = c.p.dt, dtau = c.p.dtau;
  double* RU = c.RU.data();
  double* ui = c.ui.data();
  RESU(c, um_tau, vm_tau, p, RU);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i) {
      size_t k = c.iu(i, j);
      double r = ((um[k] - um_tau[k]) + RU[k] * dt) * dtau;
      ui[k] = um_tau[k] + r;
    }
  bcUV(c, ui, vm_tau);
  RESU(c, ui, vm_tau, p, RU);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i) {
      size_t k = c.iu(i, j);
      double r = ((um[k] - um_tau[k]) + RU[k] * dt) * dtau;
      ui[k] = 0.75 * um_tau[k] + 0.25 * (ui[k] + r);
    }
  bcUV(c, ui, vm_tau);
  RESU(c, ui, vm_tau, p, RU);
  double mx = 0.0;
#pragma omp parallel for schedule(static) reduction(max : mx)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 3; i <= nx - 1; ++i) {
      size_t k = c.iu(i, j);
      double r = ((um[k] - um_tau[k]) + RU[k] * dt) * dtau;
      um_n_tau[k] = 1.0 / 3.0 * um_tau[k] + 2.0 / 3.0 * (ui[k] + r);
      double a = std::fabs(r);
      if (a > mx || a != a) mx = a;
    }
  bcUV(c, um_n_tau, vm_tau);
  return mx;
}

// solve_V (equations.f90:546-603)
double solve_V(Case& c, const double* vm, double* um_tau, const double* vm_tau, const double* p,
               const double* T, double* vm_n_tau) {
  const int nx = c.nx, ny = c.ny;
  const double dt = c.p.dt, dtau = c.p.dtau;
  double* RV = c.RV.data();
  double* vi = c.vi.data();
  RESV(c, um_tau, vm_tau, p, T, RV);
#pragma omp parallel for schedule(static)
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.iv(i, j);
      double r = ((vm[k] - vm_tau[k]) + RV[k] * dt) * dtau;
      vi[k] = (vm_tau[k] + r);
    }
  bcUV(c, um_tau, vi);
  RESV(c, um_tau, vi, p, T, RV);
#pragma omp parallel for schedule(static)
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.iv(i, j);
      double r = ((vm[k] - vm_tau[k]) + RV[k] * dt) * dtau;
      vi[k] = (0.75 * vm_tau[k] + 0.25 * (vi[k] + r));
    }
  bcUV(c, um_tau, vi);
  RESV(c, um_tau, vi, p, T, RV);
  double mx = 0.0;
#pragma omp parallel for schedule(static) reduction(max : mx)
  for (int j = 3; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.iv(i, j);
      double r = ((vm[k] - vm_tau[k]) + RV[k] * dt) * dtau;
      vm_n_tau[k] = 1.0 / 3.0 * vm_tau[k] + 2.0 / 3.0 * (vi[k] + r);
      double a = std::fabs(r);
      if (a > mx || a != a) mx = a;
    }
  bcUV(c, um_tau, vm_n_tau);
  return mx;
}

// solve_P (equations.f90:607-665).  RP is frozen over the three stages.
double solve_P(Case& c, const double* p, const double* um_n, const double* vm_n, double* pn) {
  const int nx = c.nx, ny = c.ny;
  const double dtau = c.p.dtau, beta = c.p.beta;
  double* pi = c.Pi.data();
  double* RP = c.RPa.data();
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      double dudx = um_n[c.iu(i + 1, j)] * c.areau_ew(j) - um_n[c.iu(i, j)] * c.areau_ew(j);
      double dvdy = vm_n[c.iv(i, j + 1)] * c.areav_ns(i) - vm_n[c.iv(i, j)] * c.areav_ns(i);
      size_t k = c.ip(i, j);
      RP[k] = -(dudx + dvdy);
      if (c.p.continuity == 1) RP[k] = RP[k] / ((c.ym[j + 1] - c.ym[j]) * (c.xm[i + 1] - c.xm[i]));
      pi[k] = p[k] + dtau * RP[k] * beta;
    }
  bcP(c, pi);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.ip(i, j);
      pi[k] = 0.75 * p[k] + 0.25 * (pi[k] + dtau * RP[k] * beta);
    }
  bcP(c, pi);
  double mx = 0.0;
#pragma omp parallel for schedule(static) reduction(max : mx)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.ip(i, j);
      double r = dtau * RP[k] * beta;
      pn[k] = 1.0 / 3.0 * p[k] + 2.0 / 3.0 * (pi[k] + r);
      double a = std::fabs(r);
      if (a > mx || a != a) mx = a;
    }
  bcP(c, pn);
  return mx;
}

// RESZ (equations.f90:723-765)
void RESZ(Case& c, const double* um_n, const double* vm_n, const double* Z, double* RZ) {
  const int nx = c.nx, ny = c.ny;
  const double iPe = 1.0 / c.p.Pe;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      double Zp = Z[c.ip(i, j)], Ze = Z[c.ip(i + 1, j)], Zw = Z[c.ip(i - 1, j)],
             Zn = Z[c.ip(i, j + 1)], Zs = Z[c.ip(i, j - 1)];
      double dZudx = 0.5 * (Ze + Zp) * um_n[c.iu(i + 1, j)] * c.areau_ew(j) -
                     0.5 * (Zw + Zp) * um_n[c.iu(i, j)] * c.areau_ew(j);
      double dZvdy = 0.5 * (Zn + Zp) * vm_n[c.iv(i, j + 1)] * c.areav_ns(i) -
                     0.5 * (Zs + Zp) * vm_n[c.iv(i, j)] * c.areav_ns(i);
      double De = (c.ym[j + 1] - c.ym[j]) * iPe / (c.x[i + 1] - c.x[i]);
      double Dw = (c.ym[j + 1] - c.ym[j]) * iPe / (c.x[i] - c.x[i - 1]);
      double Dn = (c.xm[i + 1] - c.xm[i]) * iPe / (c.y[j + 1] - c.y[j]);
      double Ds = (c.xm[i + 1] - c.xm[i]) * iPe / (c.y[j] - c.y[j - 1]);
      double Dp = De + Dw + Dn + Ds;
      double lg = c.liga[c.ip(i, j)], e = c.eps[c.ip(i, j)];
      RZ[c.ip(i, j)] = 1.0 / (c.xm[i + 1] - c.xm[i]) / (c.ym[j + 1] - c.ym[j]) *
                       (-(Dp * Zp) + De * Ze + Dw * Zw + Dn * Zn + Ds * Zs - (1.0 - lg) * (dZudx + dZvdy)) /
                       (lg * (e - 1.0) + 1.0);
    }
}

// RESC (equations.f90:823-867)
void RESC(Case& c, const double* um_n, const double* vm_n, const double* C, double* RC) {
  const int nx = c.nx, ny = c.ny;
  const double iReSc = 1.0 / c.p.Re / c.p.Sc;
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      double Cp = C[c.ip(i, j)], Ce = C[c.ip(i + 1, j)], Cw = C[c.ip(i - 1, j)],
             Cn = C[c.ip(i, j + 1)], Cs = C[c.ip(i, j - 1)];
      double dCudx = 0.5 * (Ce + Cp) * um_n[c.iu(i + 1, j)] * c.areau_ew(j) -
                     0.5 * (Cw + Cp) * um_n[c.iu(i, j)] * c.areau_ew(j);
      double dCvdy = 0.5 * (Cn + Cp) * vm_n[c.iv(i, j + 1)] * c.areav_ns(i) -
                     0.5 * (Cs + Cp) * vm_n[c.iv(i, j)] * c.areav_ns(i);
      double De = (c.ym[j + 1] - c.ym[j]) * iReSc / (c.x[i + 1] - c.x[i]);
      double Dw = (c.ym[j + 1] - c.ym[j]) * iReSc / (c.x[i] - c.x[i - 1]);
      double Dn = (c.xm[i + 1] - c.xm[i]) * iReSc / (c.y[j + 1] - c.y[j]);
      double Ds = (c.xm[i + 1] - c.xm[i]) * iReSc / (c.y[j] - c.y[j - 1]);
      double Dp = De + Dw + Dn + Ds;
      double lg = c.liga[c.ip(i, j)], e = c.eps[c.ip(i, j)];
      RC[c.ip(i, j)] = 1.0 / (c.xm[i + 1] - c.xm[i]) / (c.ym[j + 1] - c.ym[j]) *
                       (-(Dp * Cp) + De * Ce + Dw * Cw + Dn * Cn + Ds * Cs -
                        (dCudx + dCvdy) / (lg * (e - 1.0) + 1.0));
    }
}

// solve_Z (equations.f90:669-719) and solve_C (:769-819): same three stages, different residual.
template <bool IS_C>
void solve_S(Case& c, const double* um_n, const double* vm_n, const double* Z, double* Z_n_tau,
             const double* Z_tau) {
  const int nx = c.nx, ny = c.ny;
  const double dt = c.p.dt, dtau = c.p.dtau;
  double* R = IS_C ? c.RC.data() : c.RZ.data();
  double* Zi = IS_C ? c.Ci.data() : c.Zi.data();
  const double zin = IS_C ? c_inflow(c) : c.p.T_in;
  auto res = [&](const double* s) { if (IS_C) RESC(c, um_n, vm_n, s, R); else RESZ(c, um_n, vm_n, s, R); };
  res(Z_tau);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.ip(i, j);
      double r = ((Z[k] - Z_tau[k]) + R[k] * dt) * dtau;
      Zi[k] = Z_tau[k] + r;
    }
  bcS(c, Zi, zin);
  res(Zi);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.ip(i, j);
      double r = ((Z[k] - Z_tau[k]) + R[k] * dt) * dtau;
      Zi[k] = 0.75 * Z_tau[k] + 0.25 * (Zi[k] + r);
    }
  bcS(c, Zi, zin);
  res(Zi);
#pragma omp parallel for schedule(static)
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i) {
      size_t k = c.ip(i, j);
      double r = ((Z[k] - Z_tau[k]) + R[k] * dt) * dtau;
      Z_n_tau[k] = 1.0 / 3.0 * Z_tau[k] + 2.0 / 3.0 * (Zi[k] + r);
    }
  bcS(c, Z_n_tau, zin);
}

// ---------------------------------------------------------------------------------------
// Mesh (nonsymetric_mesh.f90:1-218) and the porous flag (:166-218)
// ---------------------------------------------------------------------------------------
enum { C_F = 0, C_B = 1, C_I = 2, C_BS = 3 };

// flag dilation (:177-218): interior cells next to fluid become C_B, fluid cells next to C_B
// become C_BS.  The last loop of the reference reads flag(0,j) and flag(i,0).  Fortran stores
// flag column-major without bounds checks, so flag(0,j) is the word flag(imax,j-1) for j >= 2;
// that aliasing is kept.  flag(i,0) and flag(0,1) lie before the array and are taken as
// "not C_B".
void flag_dilate(int nx, int ny, int* flag) {
  auto F = [&](int i, int j) -> int& { return flag[(i - 1) + (j - 1) * nx]; };
  auto Fr = [&](int i, int j) -> int {
    long lin = (long)(i - 1) + (long)(j - 1) * nx;
    return (lin < 0 || lin >= (long)nx * ny) ? -1 : flag[lin];
  };
  for (int j = 2; j <= ny - 1; ++j)
    for (int i = 2; i <= nx - 1; ++i)
      if ((F(i, j) == C_I && F(i - 1, j) == C_F) || (F(i, j) == C_I && F(i, j - 1) == C_F) ||
          (F(i, j) == C_I && F(i + 1, j) == C_F) || (F(i, j) == C_I && F(i, j + 1) == C_F))
        F(i, j) = C_B;
  {
    int i = 1;
    for (int j = 2; j <= ny - 1; ++j)
      if ((F(i, j) == C_I && F(i, j - 1) == C_F) || (F(i, j) == C_I && F(i, j + 1) == C_F)) F(i, j) = C_B;
  }
  for (int j = 1; j <= ny - 1; ++j)
    for (int i = 1; i <= nx - 1; ++i)
      if ((F(i, j) == C_F && Fr(i - 1, j) == C_B) || (F(i, j) == C_F && Fr(i, j - 1) == C_B) ||
          (F(i, j) == C_F && Fr(i + 1, j) == C_B) || (F(i, j) == C_F && Fr(i, j + 1) == C_B))
        F(i, j) = C_BS;
}

// staggered mid-points (:48-60)
void midpoints(int nx, int ny, const double* x, const double* y, double* xm, double* ym) {
  xm[1] = -(x[2] + x[1]) * 0.5;
  xm[nx + 1] = (x[nx] + x[nx - 1]) * 0.5 + (x[nx] - x[nx - 1]);
  for (int i = 2; i <= nx; ++i) xm[i] = (x[i] + x[i - 1]) * 0.5;
  ym[1] = y[1] - (y[2] - y[1]) * 0.5;
  ym[ny + 1] = (y[ny] + y[ny - 1]) * 0.5 + (y[ny] - y[ny - 1]);
  for (int j = 2; j <= ny; ++j) ym[j] = (y[j] + y[j - 1]) * 0.5;
}

}  // namespace

extern "C" {

// jmax of the reference for a given imax: (Hvert/dx_c)+1 truncated (comum.f90:40-46).
int orc_reference_jmax(int imax) {
  const double Lhori = 12.0, y_up = 15.0, y_down = 5.0, Hvert = y_up + y_down;
  const double dx_c = Lhori / (imax - 1);
  return (int)(Hvert / dx_c + 1.0);
}

// Reference mesh (nonsymetric_mesh.f90:1-60, 166-218).  Arrays are 1-based views: the caller
// passes x[nx], y[ny], xm[nx+1], ym[ny+1], flag/eps/liga[nx*ny].
int orc_mesh_reference(int imax, double porosity, double* x0, double* y0, double* xm0, double* ym0,
                       int* flag, double* eps, double* liga) {
  const double Lhori = 12.0, y_up = 15.0, y_down = 5.0, Hvert = y_up + y_down;
  const double Px = 1.0, Py = 1.6, Q = 1.0;
  const int nx = imax;
  const double dx_c = Lhori / (imax - 1);
  const int ny = (int)(Hvert / dx_c + 1.0);
  double* X = x0 - 1;
  double* Y = y0 - 1;
  for (int i = 1; i <= nx; ++i) X[i] = ((double)i - 1.0) * dx_c - Lhori / 2.0;
  for (int j = 1; j <= ny; ++j) Y[j] = ((double)j - 1.0) * dx_c - y_down;
  const int mid = nx / 2 + 1;
  for (int i = mid; i <= nx; ++i) {
    double etax = (X[i] - X[nx]) / (X[mid] - X[nx]);
    double sx = Px * etax + (1.0 - Px) * (1.0 - (std::tanh(Q * (1.0 - etax))) / std::tanh(Q));
    X[i] = X[nx] - sx * (X[nx] - X[mid]);
  }
  for (int i = mid; i >= 1; --i) {
    double etax = (X[i] + X[nx]) / (X[mid] + X[nx]);
    double sx = Px * etax + (1.0 - Px) * (1.0 - (std::tanh(Q * (1.0 - etax))) / std::tanh(Q));
    X[i] = -X[nx] - sx * (-X[nx] - X[mid]);
  }
  const int jm = (int)(y_down / dx_c) + 1;
  for (int j = jm; j <= ny; ++j) {
    double etay = (Y[j] - Y[ny]) / (Y[jm] - Y[ny]);
    double sy = Py * etay + (1.0 - Py) * (1.0 - (std::tanh(Q * (1.0 - etay))) / std::tanh(Q));
    Y[j] = Y[ny] - sy * (Y[ny] - Y[jm]);
  }
  for (int j = jm; j >= 1; --j) {
    double etay = (Y[j] + Y[ny]) / (Y[jm] + Y[ny]);
    double sy = Py * etay + (1.0 - Py) * (1.0 - (std::tanh(Q * (1.0 - etay))) / std::tanh(Q));
    Y[j] = -Y[ny] - sy * (-Y[ny] - Y[jm]);
  }
  midpoints(nx, ny, X, Y, xm0 - 1, ym0 - 1);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      flag[(i - 1) + (j - 1) * nx] = (X[i] <= -4.0 && Y[j] >= 0.5) ? C_I : C_F;
  flag_dilate(nx, ny, flag);
  for (int k = 0; k < nx * ny; ++k) {
    eps[k] = flag[k] != C_F ? porosity : 1.0;
    liga[k] = flag[k] != C_F ? 1.0 : 0.0;
  }
  return ny;
}

// Channel mesh: x uniform on [0, Lx]; y on [0, Ly] clustered toward both walls by
// y = Ly/2 (1 + tanh(s (2 xi - 1)) / tanh(s)), xi = (j-1)/(jmax-1) (s = 0: uniform).
// Porous block: nodes with bx0 <= x <= bx1 and by0 <= y <= by1 are C_I, then the reference
// dilation rule.  A second block (cx0..cx1, cy0..cy1) is optional (cx0 > cx1 disables it).
int orc_mesh_channel(int nx, int ny, double Lx, double Ly, double s, double bx0, double bx1,
                     double by0, double by1, double cx0, double cx1, double cy0, double cy1,
                     double porosity, double* x0, double* y0, double* xm0, double* ym0, int* flag,
                     double* eps, double* liga) {
  double* X = x0 - 1;
  double* Y = y0 - 1;
  for (int i = 1; i <= nx; ++i) X[i] = Lx * ((double)(i - 1) / (double)(nx - 1));
  for (int j = 1; j <= ny; ++j) {
    double xi = (double)(j - 1) / (double)(ny - 1);
    Y[j] = s > 0.0 ? 0.5 * Ly * (1.0 + std::tanh(s * (2.0 * xi - 1.0)) / std::tanh(s)) : Ly * xi;
  }
  midpoints(nx, ny, X, Y, xm0 - 1, ym0 - 1);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) {
      bool in1 = X[i] >= bx0 && X[i] <= bx1 && Y[j] >= by0 && Y[j] <= by1;
      bool in2 = X[i] >= cx0 && X[i] <= cx1 && Y[j] >= cy0 && Y[j] <= cy1;
      flag[(i - 1) + (j - 1) * nx] = (in1 || in2) ? C_I : C_F;
    }
  flag_dilate(nx, ny, flag);
  for (int k = 0; k < nx * ny; ++k) {
    eps[k] = flag[k] != C_F ? porosity : 1.0;
    liga[k] = flag[k] != C_F ? 1.0 : 0.0;
  }
  return 0;
}

// Seeded uniform noise shared (by specification) with the product's host generator:
// splitmix64 of a key built from (seed, case, field, index); u in [0,1) from the top 53 bits.
double orc_noise(uint64_t seed, uint64_t case_id, uint64_t field, uint64_t index, double amp) {
  uint64_t z = (seed + 1) * 0x9E3779B97F4A7C15ULL + case_id * 0xD1B54A32D192ED03ULL +
               field * 0x8CB92BA72F3D8DD7ULL + index * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  double u = (double)(z >> 11) * 0x1.0p-53;
  return amp * (2.0 * u - 1.0);
}

// orc_noise at n indices (the case builders' initial perturbation, without a Python loop)
void orc_noise_array(uint64_t seed, uint64_t case_id, uint64_t field, const uint64_t* index, long long n,
                     double amp, double* out) {
  for (long long k = 0; k < n; ++k) out[k] = orc_noise(seed, case_id, field, index[k], amp);
}

struct orc_case;
orc_case* orc_create(const orc_params* prm, const double* x, const double* y, const double* xm,
                     const double* ym, const double* eps, const double* liga) {
  Case* c = new Case(*prm);
  const int nx = c->nx, ny = c->ny;
  c->x.assign(nx + 1, 0.0); c->y.assign(ny + 1, 0.0);
  c->xm.assign(nx + 2, 0.0); c->ym.assign(ny + 2, 0.0);
  for (int i = 1; i <= nx; ++i) c->x[i] = x[i - 1];
  for (int j = 1; j <= ny; ++j) c->y[j] = y[j - 1];
  for (int i = 1; i <= nx + 1; ++i) c->xm[i] = xm[i - 1];
  for (int j = 1; j <= ny + 1; ++j) c->ym[j] = ym[j - 1];
  c->eps.assign(eps, eps + (size_t)nx * ny);
  c->liga.assign(liga, liga + (size_t)nx * ny);
  size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1), np = (size_t)nx * ny;
  c->RU.assign(nu, 0.0); c->ui.assign(nu, 0.0);
  c->RV.assign(nv, 0.0); c->vi.assign(nv, 0.0);
  c->RZ.assign(np, 0.0); c->Zi.assign(np, 0.0);
  c->RC.assign(np, 0.0); c->Ci.assign(np, 0.0);
  c->Pi.assign(np, 0.0); c->RPa.assign(np, 0.0); c->resp.assign(np, 0.0);
  return reinterpret_cast<orc_case*>(c);
}

void orc_destroy(orc_case* h) { delete reinterpret_cast<Case*>(h); }

// Per-routine entry points (argument order of the Fortran subroutines, unused ones dropped).
void orc_resu(orc_case* h, const double* um, const double* vm, const double* p, double* RU) {
  RESU(*reinterpret_cast<Case*>(h), um, vm, p, RU);
}
void orc_resv(orc_case* h, const double* um, const double* vm, const double* p, const double* T, double* RV) {
  RESV(*reinterpret_cast<Case*>(h), um, vm, p, T, RV);
}
void orc_resz(orc_case* h, const double* um, const double* vm, const double* Z, double* RZ) {
  RESZ(*reinterpret_cast<Case*>(h), um, vm, Z, RZ);
}
void orc_resc(orc_case* h, const double* um, const double* vm, const double* C, double* RC) {
  RESC(*reinterpret_cast<Case*>(h), um, vm, C, RC);
}
double orc_solve_u(orc_case* h, const double* um, const double* um_tau, double* vm_tau, const double* p,
                   double* um_n_tau) {
  return solve_U(*reinterpret_cast<Case*>(h), um, um_tau, vm_tau, p, um_n_tau);
}
double orc_solve_v(orc_case* h, const double* vm, double* um_tau, const double* vm_tau, const double* p,
                   const double* T, double* vm_n_tau) {
  return solve_V(*reinterpret_cast<Case*>(h), vm, um_tau, vm_tau, p, T, vm_n_tau);
}
double orc_solve_p(orc_case* h, const double* p, const double* um_n, const double* vm_n, double* pn) {
  return solve_P(*reinterpret_cast<Case*>(h), p, um_n, vm_n, pn);
}
void orc_solve_z(orc_case* h, const double* um_n, const double* vm_n, const double* Z, double* Z_n_tau,
                 const double* Z_tau) {
  solve_S<false>(*reinterpret_cast<Case*>(h), um_n, vm_n, Z, Z_n_tau, Z_tau);
}
void orc_solve_c(orc_case* h, const double* um_n, const double* vm_n, const double* C, double* C_n_tau,
                 const double* C_tau) {
  solve_S<true>(*reinterpret_cast<Case*>(h), um_n, vm_n, C, C_n_tau, C_tau);
}
void orc_bc_uv(orc_case* h, double* um, double* vm) { bcUV(*reinterpret_cast<Case*>(h), um, vm); }
void orc_bc_p(orc_case* h, double* p) { bcP(*reinterpret_cast<Case*>(h), p); }
void orc_bc_z(orc_case* h, double* z) { Case& c = *reinterpret_cast<Case*>(h); bcS(c, z, c.p.T_in); }
void orc_bc_c(orc_case* h, double* z) { Case& c = *reinterpret_cast<Case*>(h); bcS(c, z, c.p.C_in); }

// Loop state, all arrays caller-owned (main.f90:15-20).
struct orc_state {
  double *um, *vm, *um_tau, *vm_tau, *um_n_tau, *vm_n_tau;
  double *p, *pn;
  double *T, *T_tau, *T_n_tau, *C, *C_tau, *C_n_tau;
};

// n_steps physical steps of main.f90:116-186.  *itc carries the pseudo counter across calls
// (1 before the first step, main.f90:77).  iters[s] = pseudo-iterations taken in step s,
// err[s] = the last error of step s.  Returns the total pseudo-iterations.
long orc_run(orc_case* h, orc_state* s, int n_steps, int* itc_io, int* iters, double* err) {
  Case& c = *reinterpret_cast<Case*>(h);
  const size_t nu = (size_t)(c.nx + 1) * c.ny, nv = (size_t)c.nx * (c.ny + 1), np = (size_t)c.nx * c.ny;
  int itc = *itc_io;
  long total = 0;
  for (int st = 0; st < n_steps; ++st) {
    double error = 100.0;
    int k = 0;
    while (itc < c.p.itc_max) {
      double ru = solve_U(c, s->um, s->um_tau, s->vm_tau, s->pn, s->um_n_tau);
      double rv = solve_V(c, s->vm, s->um_tau, s->vm_tau, s->pn, s->T, s->vm_n_tau);
      double rp = solve_P(c, s->p, s->um_n_tau, s->vm_n_tau, s->pn);
      if (c.p.solve_scalars) {
        solve_S<false>(c, s->um_n_tau, s->vm_n_tau, s->T, s->T_n_tau, s->T_tau);
        solve_S<true>(c, s->um_n_tau, s->vm_n_tau, s->C, s->C_n_tau, s->C_tau);
      }
      ++k;
      // error = MAX(residual_u, residual_v, residual_p) (main.f90:139)
      error = ru;
      if (rv > error || rv != rv) error = rv;
      if (rp > error || rp != rp) error = rp;
      if (itc != 1 && error < c.p.eps) break;
      std::memcpy(s->um_tau, s->um_n_tau, nu * sizeof(double));
      std::memcpy(s->vm_tau, s->vm_n_tau, nv * sizeof(double));
      std::memcpy(s->p, s->pn, np * sizeof(double));
      if (c.p.solve_scalars) {
        std::memcpy(s->T_tau, s->T_n_tau, np * sizeof(double));
        std::memcpy(s->C_tau, s->C_n_tau, np * sizeof(double));
      }
      ++itc;
    }
    std::memcpy(s->um, s->um_n_tau, nu * sizeof(double));
    std::memcpy(s->vm, s->vm_n_tau, nv * sizeof(double));
    if (c.p.solve_scalars) {
      std::memcpy(s->T, s->T_n_tau, np * sizeof(double));
      std::memcpy(s->C, s->C_n_tau, np * sizeof(double));
    }
    itc = 0;
    if (iters) iters[st] = k;
    if (err) err[st] = error;
    total += k;
  }
  *itc_io = itc;
  return total;
}

}  // extern "C"
