// points_exact.cuh -- per-node residuals with the reference's exact operation order.
//
// Shared by the stage kernels (kernels_exact.cu) and the persistent cluster engine
// (engine_exact.cu); every including unit is compiled with -fmad=false so each product and sum
// is rounded separately.  Field loads go through LD(), which reads from L2 (ld.global.cg): in
// the persistent engine other CTAs of the cluster write these arrays between barriers.
//
// Reference (OpenMp_Multicore/): RESU equations.f90:2-116 (+ upwind_Ui/Uj :120-240),
// RESV :305-420 (+ upwind_Vi/Vj :423-542), RESZ :723-765, RESC :823-867.
#pragma once
#include <cuda_runtime.h>
#include "acs_dev.cuh"

#ifndef LD
#define LD(ptr, idx) __ldcg((ptr) + (idx))
#endif

namespace acs {
namespace exact {

struct G {
  const double *x, *y, *xm, *ym;
  int p;
  __device__ G(const CaseDev& d) : x(d.x), y(d.y), xm(d.xm), ym(d.ym), p(d.pitch) {}
  __device__ long long o(int i, int j) const { return lin(i, j, p); }
};

__device__ inline double pos(double a) { return a > 0.0 ? a : 0.0; }

// ---- RESU: QUICK interior (equations.f90:14-104) --------------------------------------------
__device__ inline double resu_quick(const CaseDev& d, const G& g, const double* um, const double* vm,
                             const double* p, int i, int j) {
  const double e = LD(d.epsf, g.o(i, j)), lg = LD(d.liga, g.o(i, j));
  const double An = g.x[i] - g.x[i - 1], As = An, Ae = g.ym[j + 1] - g.ym[j], Aw = Ae;
  double fn = 0.5 * (LD(vm, g.o(i, j + 1)) + LD(vm, g.o(i - 1, j + 1))) * An / e;
  double fs = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i - 1, j))) * As / e;
  double fe = 0.5 * (LD(um, g.o(i + 1, j)) + LD(um, g.o(i, j))) * Ae / e;
  double fw = 0.5 * (LD(um, g.o(i, j)) + LD(um, g.o(i - 1, j))) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.y[j + 1] - g.y[j]);
  double Ds = (e / d.Re) * As / (g.y[j] - g.y[j - 1]);
  double De = (e / d.Re) * Ae / (g.xm[i + 1] - g.xm[i]);
  double Dw = (e / d.Re) * Aw / (g.xm[i] - g.xm[i - 1]);
  double afw = fw > 0.0 ? 1.0 : 0.0, afe = fe > 0.0 ? 1.0 : 0.0;
  double afn = fn > 0.0 ? 1.0 : 0.0, afs = fs > 0.0 ? 1.0 : 0.0;
  double aw = Dw + 0.75 * afw * fw + 0.125 * afe * fe + 0.375 * (1.0 - afw) * fw;
  double ae = De - 0.375 * afe * fe - 0.75 * (1.0 - afe) * fe - 0.125 * (1.0 - afw) * fw;
  double as = Ds + 0.75 * afs * fs + 0.125 * afn * fn + 0.375 * (1.0 - afs) * fs;
  double an = Dn - 0.375 * afn * fn - 0.75 * (1.0 - afn) * fn - 0.125 * (1.0 - afs) * fs;
  double aww = -0.125 * afw * fw, aee = 0.125 * (1.0 - afe) * fe;
  double ass = -0.125 * afs * fs, ann = 0.125 * (1.0 - afn) * fn;
  double ap = aw + ae + as + an + aww + aee + ass + ann + df;
  double uW = LD(um, g.o(i - 1, j)), uWW = LD(um, g.o(i - 2, j)), uE = LD(um, g.o(i + 1, j)),
         uEE = LD(um, g.o(i + 2, j)), uS = LD(um, g.o(i, j - 1)), uSS = LD(um, g.o(i, j - 2)),
         uN = LD(um, g.o(i, j + 1)), uNN = LD(um, g.o(i, j + 2)), uP = LD(um, g.o(i, j)), vP = LD(vm, g.o(i, j));
  double q_art = e * (LD(p, g.o(i, j)) - LD(p, g.o(i - 1, j))) / (g.x[i] - g.x[i - 1]);
  if (d.flags & F_BART) {
    double dudxdx = Ae * (uE - uP) / (g.xm[i + 1] - g.xm[i]) - Aw * (uP - uW) / (g.xm[i] - g.xm[i - 1]);
    double dxdvdy = Ae * (LD(vm, g.o(i, j + 1)) - LD(vm, g.o(i, j))) / (g.ym[j + 1] - g.ym[j]) -
                    Aw * (LD(vm, g.o(i - 1, j + 1)) - LD(vm, g.o(i - 1, j))) / (g.ym[j + 1] - g.ym[j]);
    q_art = q_art + -(d.b_art * (dudxdx + dxdvdy));
  }
  double r = 1.0 / (g.x[i] - g.x[i - 1]) / (g.y[j] - g.y[j - 1]) *
                 (-(ap * uP) + aww * uWW + aw * uW + aee * uEE + ae * uE + ass * uSS + as * uS +
                  ann * uNN + an * uN) -
             q_art;
  if (d.flags & F_POROUS)
    r = r - e * (uP / (d.Re * d.Da) + d.Cf / sqrt(e * d.Da) * uP * sqrt(uP * uP + vP * vP)) * lg;
  return r - d.g * e;
}

// ---- RESU: first-order upwind rows (upwind_Ui/upwind_Uj, equations.f90:133-174) ----------------
__device__ inline double resu_upwind(const CaseDev& d, const G& g, const double* um, const double* vm,
                              const double* p, int i, int j) {
  const double e = LD(d.epsf, g.o(i, j)), lg = LD(d.liga, g.o(i, j));
  const double An = g.x[i] - g.x[i - 1], As = An, Ae = g.ym[j + 1] - g.ym[j], Aw = Ae;
  double fn = 0.5 * (LD(vm, g.o(i, j + 1)) + LD(vm, g.o(i - 1, j + 1))) * An / e;
  double fs = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i - 1, j))) * As / e;
  double fe = 0.5 * (LD(um, g.o(i + 1, j)) + LD(um, g.o(i, j))) * Ae / e;
  double fw = 0.5 * (LD(um, g.o(i, j)) + LD(um, g.o(i - 1, j))) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.y[j + 1] - g.y[j]);
  double Ds = (e / d.Re) * As / (g.y[j] - g.y[j - 1]);
  double De = (e / d.Re) * Ae / (g.xm[i + 1] - g.xm[i]);
  double Dw = (e / d.Re) * Aw / (g.xm[i] - g.xm[i - 1]);
  double aw = Dw + pos(fw), as = Ds + pos(fs), ae = De + pos(-fe), an = Dn + pos(-fn);
  double ap = aw + ae + as + an + df;
  double uW = LD(um, g.o(i - 1, j)), uE = LD(um, g.o(i + 1, j)), uS = LD(um, g.o(i, j - 1)),
         uN = LD(um, g.o(i, j + 1)), uP = LD(um, g.o(i, j)), vP = LD(vm, g.o(i, j));
  double q_art = e * (LD(p, g.o(i, j)) - LD(p, g.o(i - 1, j))) / (g.x[i] - g.x[i - 1]);
  if (d.flags & F_BART) {
    double dudxdx = Ae * (uE - uP) / (g.xm[i + 1] - g.xm[i]) - Aw * (uP - uW) / (g.xm[i] - g.xm[i - 1]);
    double dxdvdy = Ae * (LD(vm, g.o(i, j + 1)) - LD(vm, g.o(i, j))) / (g.ym[j + 1] - g.ym[j]) -
                    Aw * (LD(vm, g.o(i - 1, j + 1)) - LD(vm, g.o(i - 1, j))) / (g.ym[j + 1] - g.ym[j]);
    q_art = q_art - d.b_art * (dudxdx + dxdvdy);
  }
  double r = 1.0 / (g.x[i] - g.x[i - 1]) / (g.y[j] - g.y[j - 1]) *
                 (-(ap * uP) + aw * uW + ae * uE + as * uS + an * uN) -
             q_art;
  if (d.flags & F_POROUS)
    r = r - e * (uP / (d.Re * d.Da) + d.Cf / sqrt(e * d.Da) * uP * sqrt(uP * uP + vP * vP)) * lg;
  return r - d.g * e;
}

// ---- RESV (equations.f90:317-408, upwind :436-477) -------------------------------------------
__device__ inline double buoyancy(const CaseDev& d, const G& g, const double* T, int i, int j) {
  return d.InvFr2 * (1.0 - 1.0 / ((LD(T, g.o(i, j)) + LD(T, g.o(i, j - 1))) * 0.5));
}

__device__ inline double resv_quick(const CaseDev& d, const G& g, const double* um, const double* vm,
                             const double* p, const double* T, int i, int j) {
  const double e = LD(d.epsf, g.o(i, j)), lg = LD(d.liga, g.o(i, j));
  const double An = g.xm[i + 1] - g.xm[i], As = An, Ae = g.y[j] - g.y[j - 1], Aw = Ae;
  double fn = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i, j + 1))) * An / e;
  double fs = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i, j - 1))) * As / e;
  double fe = 0.5 * (LD(um, g.o(i + 1, j)) + LD(um, g.o(i + 1, j - 1))) * Ae / e;
  double fw = 0.5 * (LD(um, g.o(i, j)) + LD(um, g.o(i, j - 1))) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.ym[j + 1] - g.ym[j]);
  double Ds = (e / d.Re) * As / (g.ym[j] - g.ym[j - 1]);
  double De = (e / d.Re) * Ae / (g.x[i + 1] - g.x[i]);
  double Dw = (e / d.Re) * Aw / (g.x[i] - g.x[i - 1]);
  double afw = fw > 0.0 ? 1.0 : 0.0, afe = fe > 0.0 ? 1.0 : 0.0;
  double afn = fn > 0.0 ? 1.0 : 0.0, afs = fs > 0.0 ? 1.0 : 0.0;
  double aw = Dw + 0.75 * afw * fw + 0.125 * afe * fe + 0.375 * (1.0 - afw) * fw;
  double ae = De - 0.375 * afe * fe - 0.75 * (1.0 - afe) * fe - 0.125 * (1.0 - afw) * fw;
  double as = Ds + 0.75 * afs * fs + 0.125 * afn * fn + 0.375 * (1.0 - afs) * fs;
  double an = Dn - 0.375 * afn * fn - 0.75 * (1.0 - afn) * fn - 0.125 * (1.0 - afs) * fs;
  double aww = -0.125 * afw * fw, aee = 0.125 * (1.0 - afe) * fe;
  double ass = -0.125 * afs * fs, ann = 0.125 * (1.0 - afn) * fn;
  double ap = aw + ae + as + an + aww + aee + ass + ann + df;
  double vW = LD(vm, g.o(i - 1, j)), vWW = LD(vm, g.o(i - 2, j)), vE = LD(vm, g.o(i + 1, j)),
         vEE = LD(vm, g.o(i + 2, j)), vS = LD(vm, g.o(i, j - 1)), vSS = LD(vm, g.o(i, j - 2)),
         vN = LD(vm, g.o(i, j + 1)), vNN = LD(vm, g.o(i, j + 2)), vP = LD(vm, g.o(i, j)), uP = LD(um, g.o(i, j));
  double q_art = e * (LD(p, g.o(i, j)) - LD(p, g.o(i, j - 1))) / (g.y[j] - g.y[j - 1]);
  if (d.flags & F_BART) {
    double dvdydy = An * (vN - vP) / (g.ym[j + 1] - g.ym[j]) - As * (vP - vS) / (g.ym[j] - g.ym[j - 1]);
    double dydudx = An * (LD(um, g.o(i + 1, j)) - LD(um, g.o(i, j))) / (g.xm[i + 1] - g.xm[i]) -
                    As * (LD(um, g.o(i + 1, j - 1)) - LD(um, g.o(i, j - 1))) / (g.xm[i + 1] - g.xm[i]);
    q_art = q_art + -(d.b_art * (dydudx + dvdydy));
  }
  double r = 1.0 / (g.x[i] - g.x[i - 1]) / (g.y[j] - g.y[j - 1]) *
                 (-(ap * vP) + aww * vWW + aw * vW + aee * vEE + ae * vE + ass * vSS + as * vS +
                  ann * vNN + an * vN) -
             q_art;
  if (d.flags & F_BUOY) r = r + buoyancy(d, g, T, i, j);
  if (d.flags & F_POROUS)
    r = r - e * (vP / (d.Re * d.Da) + d.Cf / sqrt(e * d.Da) * vP * sqrt(uP * uP + vP * vP)) * lg;
  return r;
}

__device__ inline double resv_upwind(const CaseDev& d, const G& g, const double* um, const double* vm,
                              const double* p, const double* T, int i, int j) {
  const double e = LD(d.epsf, g.o(i, j)), lg = LD(d.liga, g.o(i, j));
  const double An = g.xm[i + 1] - g.xm[i], As = An, Ae = g.y[j] - g.y[j - 1], Aw = Ae;
  double fn = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i, j + 1))) * An / e;
  double fs = 0.5 * (LD(vm, g.o(i, j)) + LD(vm, g.o(i, j - 1))) * As / e;
  double fe = 0.5 * (LD(um, g.o(i + 1, j)) + LD(um, g.o(i + 1, j - 1))) * Ae / e;
  double fw = 0.5 * (LD(um, g.o(i, j)) + LD(um, g.o(i, j - 1))) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.ym[j + 1] - g.ym[j]);
  double Ds = (e / d.Re) * As / (g.ym[j] - g.ym[j - 1]);
  double De = (e / d.Re) * Ae / (g.x[i + 1] - g.x[i]);
  double Dw = (e / d.Re) * Aw / (g.x[i] - g.x[i - 1]);
  double aw = Dw + pos(fw), as = Ds + pos(fs), ae = De + pos(-fe), an = Dn + pos(-fn);
  double ap = aw + ae + as + an + df;
  double vW = LD(vm, g.o(i - 1, j)), vE = LD(vm, g.o(i + 1, j)), vS = LD(vm, g.o(i, j - 1)),
         vN = LD(vm, g.o(i, j + 1)), vP = LD(vm, g.o(i, j)), uP = LD(um, g.o(i, j));
  double q_art = e * (LD(p, g.o(i, j)) - LD(p, g.o(i, j - 1))) / (g.y[j] - g.y[j - 1]);
  if (d.flags & F_BART) {
    double dvdydy = An * (vN - vP) / (g.ym[j + 1] - g.ym[j]) - As * (vP - vS) / (g.ym[j] - g.ym[j - 1]);
    double dydudx = An * (LD(um, g.o(i + 1, j)) - LD(um, g.o(i, j))) / (g.xm[i + 1] - g.xm[i]) -
                    As * (LD(um, g.o(i + 1, j - 1)) - LD(um, g.o(i, j - 1))) / (g.xm[i + 1] - g.xm[i]);
    q_art = q_art - d.b_art * (dydudx + dvdydy);
  }
  double r = 1.0 / (g.x[i] - g.x[i - 1]) / (g.y[j] - g.y[j - 1]) *
                 (-(ap * vP) + aw * vW + ae * vE + as * vS + an * vN) -
             q_art;
  if (d.flags & F_BUOY) r = r + buoyancy(d, g, T, i, j);
  if (d.flags & F_POROUS)
    r = r - e * (vP / (d.Re * d.Da) + d.Cf / sqrt(e * d.Da) * vP * sqrt(uP * uP + vP * vP)) * lg;
  return r;
}

// ---- RESZ / RESC (equations.f90:738-759, 839-861) -------------------------------------------
template <bool IS_C>
__device__ inline double res_scalar(const CaseDev& d, const G& g, const double* un, const double* vn,
                             const double* Z, int i, int j) {
  const double k = IS_C ? 1.0 / d.Re / d.Sc : 1.0 / d.Pe;
  double Zp = LD(Z, g.o(i, j)), Ze = LD(Z, g.o(i + 1, j)), Zw = LD(Z, g.o(i - 1, j)), Zn = LD(Z, g.o(i, j + 1)),
         Zs = LD(Z, g.o(i, j - 1));
  double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
  double dzu = 0.5 * (Ze + Zp) * LD(un, g.o(i + 1, j)) * Aew - 0.5 * (Zw + Zp) * LD(un, g.o(i, j)) * Aew;
  double dzv = 0.5 * (Zn + Zp) * LD(vn, g.o(i, j + 1)) * Ans - 0.5 * (Zs + Zp) * LD(vn, g.o(i, j)) * Ans;
  double De = (g.ym[j + 1] - g.ym[j]) * k / (g.x[i + 1] - g.x[i]);
  double Dw = (g.ym[j + 1] - g.ym[j]) * k / (g.x[i] - g.x[i - 1]);
  double Dn = (g.xm[i + 1] - g.xm[i]) * k / (g.y[j + 1] - g.y[j]);
  double Ds = (g.xm[i + 1] - g.xm[i]) * k / (g.y[j] - g.y[j - 1]);
  double Dp = De + Dw + Dn + Ds;
  double lg = LD(d.liga, g.o(i, j)), e = LD(d.epsf, g.o(i, j));
  if (IS_C)
    return 1.0 / (g.xm[i + 1] - g.xm[i]) / (g.ym[j + 1] - g.ym[j]) *
           (-(Dp * Zp) + De * Ze + Dw * Zw + Dn * Zn + Ds * Zs - (dzu + dzv) / (lg * (e - 1.0) + 1.0));
  return 1.0 / (g.xm[i + 1] - g.xm[i]) / (g.ym[j + 1] - g.ym[j]) *
         (-(Dp * Zp) + De * Ze + Dw * Zw + Dn * Zn + Ds * Zs - (1.0 - lg) * (dzu + dzv)) /
         (lg * (e - 1.0) + 1.0);
}

}  // namespace exact
}  // namespace acs
