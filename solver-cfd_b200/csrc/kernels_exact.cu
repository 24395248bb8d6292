// kernels_exact.cu -- FP64 kernels that reproduce the reference's rounding bit for bit.
//
// Built with -fmad=false: every product and sum is rounded separately and each expression keeps
// the Fortran evaluation order (left to right, `x**2.d0` = x*x, `x**0.5d0` = sqrt(x)), so the
// results are bit-identical to the reference arithmetic compiled without fused multiply-add.
// One thread per node, one launch per Runge-Kutta stage; boundary passes are separate
// one-block-per-case launches.  Every launch covers all active cases of a batch through a tile
// table; inactive cases (converged or failed) return at once.
//
// Reference (OpenMp_Multicore/): RESU equations.f90:2-116 (+ upwind_Ui/Uj :120-240),
// solve_U :244-301, RESV :305-420 (+ upwind_Vi/Vj :423-542), solve_V :546-603, solve_P :607-665,
// solve_Z :669-719, RESZ :723-765, solve_C :769-819, RESC :823-867, boundary.f90:1-159,
// main.f90:116-186 (control).
#include <cuda_runtime.h>
#include "acs_dev.cuh"
#include "kernels.h"

namespace acs {
namespace {

struct G {
  const double *x, *y, *xm, *ym;
  int p;
  __device__ G(const CaseDev& d) : x(d.x), y(d.y), xm(d.xm), ym(d.ym), p(d.pitch) {}
  __device__ long long o(int i, int j) const { return lin(i, j, p); }
};

__device__ inline double pos(double a) { return a > 0.0 ? a : 0.0; }

// ---- RESU: QUICK interior (equations.f90:14-104) --------------------------------------------
__device__ double resu_quick(const CaseDev& d, const G& g, const double* um, const double* vm,
                             const double* p, int i, int j) {
  const double e = d.epsf[g.o(i, j)], lg = d.liga[g.o(i, j)];
  const double An = g.x[i] - g.x[i - 1], As = An, Ae = g.ym[j + 1] - g.ym[j], Aw = Ae;
  double fn = 0.5 * (vm[g.o(i, j + 1)] + vm[g.o(i - 1, j + 1)]) * An / e;
  double fs = 0.5 * (vm[g.o(i, j)] + vm[g.o(i - 1, j)]) * As / e;
  double fe = 0.5 * (um[g.o(i + 1, j)] + um[g.o(i, j)]) * Ae / e;
  double fw = 0.5 * (um[g.o(i, j)] + um[g.o(i - 1, j)]) * Aw / e;
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
  double uW = um[g.o(i - 1, j)], uWW = um[g.o(i - 2, j)], uE = um[g.o(i + 1, j)],
         uEE = um[g.o(i + 2, j)], uS = um[g.o(i, j - 1)], uSS = um[g.o(i, j - 2)],
         uN = um[g.o(i, j + 1)], uNN = um[g.o(i, j + 2)], uP = um[g.o(i, j)], vP = vm[g.o(i, j)];
  double q_art = e * (p[g.o(i, j)] - p[g.o(i - 1, j)]) / (g.x[i] - g.x[i - 1]);
  if (d.flags & F_BART) {
    double dudxdx = Ae * (uE - uP) / (g.xm[i + 1] - g.xm[i]) - Aw * (uP - uW) / (g.xm[i] - g.xm[i - 1]);
    double dxdvdy = Ae * (vm[g.o(i, j + 1)] - vm[g.o(i, j)]) / (g.ym[j + 1] - g.ym[j]) -
                    Aw * (vm[g.o(i - 1, j + 1)] - vm[g.o(i - 1, j)]) / (g.ym[j + 1] - g.ym[j]);
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
__device__ double resu_upwind(const CaseDev& d, const G& g, const double* um, const double* vm,
                              const double* p, int i, int j) {
  const double e = d.epsf[g.o(i, j)], lg = d.liga[g.o(i, j)];
  const double An = g.x[i] - g.x[i - 1], As = An, Ae = g.ym[j + 1] - g.ym[j], Aw = Ae;
  double fn = 0.5 * (vm[g.o(i, j + 1)] + vm[g.o(i - 1, j + 1)]) * An / e;
  double fs = 0.5 * (vm[g.o(i, j)] + vm[g.o(i - 1, j)]) * As / e;
  double fe = 0.5 * (um[g.o(i + 1, j)] + um[g.o(i, j)]) * Ae / e;
  double fw = 0.5 * (um[g.o(i, j)] + um[g.o(i - 1, j)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.y[j + 1] - g.y[j]);
  double Ds = (e / d.Re) * As / (g.y[j] - g.y[j - 1]);
  double De = (e / d.Re) * Ae / (g.xm[i + 1] - g.xm[i]);
  double Dw = (e / d.Re) * Aw / (g.xm[i] - g.xm[i - 1]);
  double aw = Dw + pos(fw), as = Ds + pos(fs), ae = De + pos(-fe), an = Dn + pos(-fn);
  double ap = aw + ae + as + an + df;
  double uW = um[g.o(i - 1, j)], uE = um[g.o(i + 1, j)], uS = um[g.o(i, j - 1)],
         uN = um[g.o(i, j + 1)], uP = um[g.o(i, j)], vP = vm[g.o(i, j)];
  double q_art = e * (p[g.o(i, j)] - p[g.o(i - 1, j)]) / (g.x[i] - g.x[i - 1]);
  if (d.flags & F_BART) {
    double dudxdx = Ae * (uE - uP) / (g.xm[i + 1] - g.xm[i]) - Aw * (uP - uW) / (g.xm[i] - g.xm[i - 1]);
    double dxdvdy = Ae * (vm[g.o(i, j + 1)] - vm[g.o(i, j)]) / (g.ym[j + 1] - g.ym[j]) -
                    Aw * (vm[g.o(i - 1, j + 1)] - vm[g.o(i - 1, j)]) / (g.ym[j + 1] - g.ym[j]);
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
  return d.InvFr2 * (1.0 - 1.0 / ((T[g.o(i, j)] + T[g.o(i, j - 1)]) * 0.5));
}

__device__ double resv_quick(const CaseDev& d, const G& g, const double* um, const double* vm,
                             const double* p, const double* T, int i, int j) {
  const double e = d.epsf[g.o(i, j)], lg = d.liga[g.o(i, j)];
  const double An = g.xm[i + 1] - g.xm[i], As = An, Ae = g.y[j] - g.y[j - 1], Aw = Ae;
  double fn = 0.5 * (vm[g.o(i, j)] + vm[g.o(i, j + 1)]) * An / e;
  double fs = 0.5 * (vm[g.o(i, j)] + vm[g.o(i, j - 1)]) * As / e;
  double fe = 0.5 * (um[g.o(i + 1, j)] + um[g.o(i + 1, j - 1)]) * Ae / e;
  double fw = 0.5 * (um[g.o(i, j)] + um[g.o(i, j - 1)]) * Aw / e;
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
  double vW = vm[g.o(i - 1, j)], vWW = vm[g.o(i - 2, j)], vE = vm[g.o(i + 1, j)],
         vEE = vm[g.o(i + 2, j)], vS = vm[g.o(i, j - 1)], vSS = vm[g.o(i, j - 2)],
         vN = vm[g.o(i, j + 1)], vNN = vm[g.o(i, j + 2)], vP = vm[g.o(i, j)], uP = um[g.o(i, j)];
  double q_art = e * (p[g.o(i, j)] - p[g.o(i, j - 1)]) / (g.y[j] - g.y[j - 1]);
  if (d.flags & F_BART) {
    double dvdydy = An * (vN - vP) / (g.ym[j + 1] - g.ym[j]) - As * (vP - vS) / (g.ym[j] - g.ym[j - 1]);
    double dydudx = An * (um[g.o(i + 1, j)] - um[g.o(i, j)]) / (g.xm[i + 1] - g.xm[i]) -
                    As * (um[g.o(i + 1, j - 1)] - um[g.o(i, j - 1)]) / (g.xm[i + 1] - g.xm[i]);
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

__device__ double resv_upwind(const CaseDev& d, const G& g, const double* um, const double* vm,
                              const double* p, const double* T, int i, int j) {
  const double e = d.epsf[g.o(i, j)], lg = d.liga[g.o(i, j)];
  const double An = g.xm[i + 1] - g.xm[i], As = An, Ae = g.y[j] - g.y[j - 1], Aw = Ae;
  double fn = 0.5 * (vm[g.o(i, j)] + vm[g.o(i, j + 1)]) * An / e;
  double fs = 0.5 * (vm[g.o(i, j)] + vm[g.o(i, j - 1)]) * As / e;
  double fe = 0.5 * (um[g.o(i + 1, j)] + um[g.o(i + 1, j - 1)]) * Ae / e;
  double fw = 0.5 * (um[g.o(i, j)] + um[g.o(i, j - 1)]) * Aw / e;
  double df = fe - fw + fn - fs;
  double Dn = (e / d.Re) * An / (g.ym[j + 1] - g.ym[j]);
  double Ds = (e / d.Re) * As / (g.ym[j] - g.ym[j - 1]);
  double De = (e / d.Re) * Ae / (g.x[i + 1] - g.x[i]);
  double Dw = (e / d.Re) * Aw / (g.x[i] - g.x[i - 1]);
  double aw = Dw + pos(fw), as = Ds + pos(fs), ae = De + pos(-fe), an = Dn + pos(-fn);
  double ap = aw + ae + as + an + df;
  double vW = vm[g.o(i - 1, j)], vE = vm[g.o(i + 1, j)], vS = vm[g.o(i, j - 1)],
         vN = vm[g.o(i, j + 1)], vP = vm[g.o(i, j)], uP = um[g.o(i, j)];
  double q_art = e * (p[g.o(i, j)] - p[g.o(i, j - 1)]) / (g.y[j] - g.y[j - 1]);
  if (d.flags & F_BART) {
    double dvdydy = An * (vN - vP) / (g.ym[j + 1] - g.ym[j]) - As * (vP - vS) / (g.ym[j] - g.ym[j - 1]);
    double dydudx = An * (um[g.o(i + 1, j)] - um[g.o(i, j)]) / (g.xm[i + 1] - g.xm[i]) -
                    As * (um[g.o(i + 1, j - 1)] - um[g.o(i, j - 1)]) / (g.xm[i + 1] - g.xm[i]);
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
__device__ double res_scalar(const CaseDev& d, const G& g, const double* un, const double* vn,
                             const double* Z, int i, int j) {
  const double k = IS_C ? 1.0 / d.Re / d.Sc : 1.0 / d.Pe;
  double Zp = Z[g.o(i, j)], Ze = Z[g.o(i + 1, j)], Zw = Z[g.o(i - 1, j)], Zn = Z[g.o(i, j + 1)],
         Zs = Z[g.o(i, j - 1)];
  double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
  double dzu = 0.5 * (Ze + Zp) * un[g.o(i + 1, j)] * Aew - 0.5 * (Zw + Zp) * un[g.o(i, j)] * Aew;
  double dzv = 0.5 * (Zn + Zp) * vn[g.o(i, j + 1)] * Ans - 0.5 * (Zs + Zp) * vn[g.o(i, j)] * Ans;
  double De = (g.ym[j + 1] - g.ym[j]) * k / (g.x[i + 1] - g.x[i]);
  double Dw = (g.ym[j + 1] - g.ym[j]) * k / (g.x[i] - g.x[i - 1]);
  double Dn = (g.xm[i + 1] - g.xm[i]) * k / (g.y[j + 1] - g.y[j]);
  double Ds = (g.xm[i + 1] - g.xm[i]) * k / (g.y[j] - g.y[j - 1]);
  double Dp = De + Dw + Dn + Ds;
  double lg = d.liga[g.o(i, j)], e = d.epsf[g.o(i, j)];
  if (IS_C)
    return 1.0 / (g.xm[i + 1] - g.xm[i]) / (g.ym[j + 1] - g.ym[j]) *
           (-(Dp * Zp) + De * Ze + Dw * Zw + Dn * Zn + Ds * Zs - (dzu + dzv) / (lg * (e - 1.0) + 1.0));
  return 1.0 / (g.xm[i + 1] - g.xm[i]) / (g.ym[j + 1] - g.ym[j]) *
         (-(Dp * Zp) + De * Ze + Dw * Zw + Dn * Zn + Ds * Zs - (1.0 - lg) * (dzu + dzv)) /
         (lg * (e - 1.0) + 1.0);
}

// Block-wide max of non-negative values, then one atomic per block.
__device__ inline void block_max_to(unsigned long long* slot, double v) {
  __shared__ double red[32];
  unsigned m = 0xffffffffu;
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(m, v, o);
    v = (w > v || w != w) ? w : v;
  }
  int tid = threadIdx.x + threadIdx.y * blockDim.x;
  int nw = (blockDim.x * blockDim.y + 31) / 32;
  if ((tid & 31) == 0) red[tid >> 5] = v;
  __syncthreads();
  if (tid < 32) {
    v = tid < nw ? red[tid] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      double w = __shfl_xor_sync(m, v, o);
      v = (w > v || w != w) ? w : v;
    }
    if (tid == 0 && v != 0.0) atomic_max_nonneg(slot, v);
  }
}

}  // namespace

// ---- solve_U stage s (s = 1,2,3; equations.f90:259-298) ---------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(256) k_u_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* uin = STAGE == 1 ? d.U[k.ru[R_TAU]] : d.S[STAGE - 2];
  double* uout = STAGE == 3 ? d.U[k.ru[R_NTAU]] : d.S[STAGE - 1];
  const double* utau = d.U[k.ru[R_TAU]];
  const double* um = d.U[k.ru[R_PHYS]];
  const double* vt = d.V[k.rv[R_TAU]];
  const double* pn = d.P[k.rp_read];
  double a = 0.0;
  if (i >= 3 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const bool quick = d.scheme == 0 && j >= 3 && j <= d.ny - 2;
    const double RU = quick ? resu_quick(d, g, uin, vt, pn, i, j) : resu_upwind(d, g, uin, vt, pn, i, j);
    const long long q = g.o(i, j);
    const double r = ((um[q] - utau[q]) + RU * d.dt) * d.dtau;
    if (STAGE == 1) uout[q] = utau[q] + r;
    if (STAGE == 2) uout[q] = 0.75 * utau[q] + 0.25 * (uin[q] + r);
    if (STAGE == 3) uout[q] = 1.0 / 3.0 * utau[q] + 2.0 / 3.0 * (uin[q] + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_u, a);
}

// ---- solve_V stage s (equations.f90:561-600) --------------------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(256) k_v_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* vin = STAGE == 1 ? d.V[k.rv[R_TAU]] : d.S[STAGE - 2];
  double* vout = STAGE == 3 ? d.V[k.rv[R_NTAU]] : d.S[STAGE - 1];
  const double* vtau = d.V[k.rv[R_TAU]];
  const double* vm = d.V[k.rv[R_PHYS]];
  const double* ut = d.U[k.ru[R_TAU]];
  const double* pn = d.P[k.rp_read];
  const double* T = d.T[k.rt[R_PHYS]];
  double a = 0.0;
  if (i >= 2 && i <= d.nx - 1 && j >= 3 && j <= d.ny - 1) {
    const bool quick = d.scheme == 0 && i >= 3 && i <= d.nx - 2;
    const double RV = quick ? resv_quick(d, g, ut, vin, pn, T, i, j) : resv_upwind(d, g, ut, vin, pn, T, i, j);
    const long long q = g.o(i, j);
    const double r = ((vm[q] - vtau[q]) + RV * d.dt) * d.dtau;
    if (STAGE == 1) vout[q] = (vtau[q] + r);
    if (STAGE == 2) vout[q] = (0.75 * vtau[q] + 0.25 * (vin[q] + r));
    if (STAGE == 3) vout[q] = 1.0 / 3.0 * vtau[q] + 2.0 / 3.0 * (vin[q] + r);
    a = fabs(r);
  }
  if (STAGE == 3) block_max_to(&ctl[t.c].res_v, a);
}

// ---- solve_P: the three stages share RP, so they fuse pointwise (equations.f90:620-662) -----
__global__ void __launch_bounds__(256) k_p_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                 const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  const double* p = d.P[k.rp[0]];
  double* pn = d.P[k.rp[1]];
  const double* un = d.U[k.ru[R_NTAU]];
  const double* vn = d.V[k.rv[R_NTAU]];
  double a = 0.0;
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double Aew = g.ym[j + 1] - g.ym[j], Ans = g.xm[i + 1] - g.xm[i];
    const double dudx = un[g.o(i + 1, j)] * Aew - un[g.o(i, j)] * Aew;
    const double dvdy = vn[g.o(i, j + 1)] * Ans - vn[g.o(i, j)] * Ans;
    double RP = -(dudx + dvdy);
    if (d.continuity == 1) RP = RP / ((g.ym[j + 1] - g.ym[j]) * (g.xm[i + 1] - g.xm[i]));
    const long long q = g.o(i, j);
    const double p0 = p[q];
    const double pi1 = p0 + d.dtau * RP * d.beta;
    const double pi2 = 0.75 * p0 + 0.25 * (pi1 + d.dtau * RP * d.beta);
    const double r = d.dtau * RP * d.beta;
    pn[q] = 1.0 / 3.0 * p0 + 2.0 / 3.0 * (pi2 + r);
    a = fabs(r);
  }
  block_max_to(&ctl[t.c].res_p, a);
}

// ---- solve_Z / solve_C stage s (equations.f90:679-716, 779-816) -------------------------------
template <bool IS_C, int STAGE>
__global__ void __launch_bounds__(256) k_s_stage_exact(const CaseDev* __restrict__ cs, CaseCtl* __restrict__ ctl,
                                                       const Tile* __restrict__ tiles) {
  const Tile t = tiles[blockIdx.x];
  if (!ctl[t.c].active || !ctl[t.c].scalars) return;
  const CaseDev& d = cs[t.c];
  const CaseCtl& k = ctl[t.c];
  const G g(d);
  const int i = t.i0 + threadIdx.x, j = t.j0 + threadIdx.y;
  double* const* F = IS_C ? d.C : d.T;
  const int* rr = IS_C ? k.rc : k.rt;
  const double* zin = STAGE == 1 ? F[rr[R_TAU]] : d.S[STAGE - 2];
  double* zout = STAGE == 3 ? F[rr[R_NTAU]] : d.S[STAGE - 1];
  const double* ztau = F[rr[R_TAU]];
  const double* z = F[rr[R_PHYS]];
  const double* un = d.U[k.ru[R_NTAU]];
  const double* vn = d.V[k.rv[R_NTAU]];
  if (i >= 2 && i <= d.nx - 1 && j >= 2 && j <= d.ny - 1) {
    const double R = res_scalar<IS_C>(d, g, un, vn, zin, i, j);
    const long long q = g.o(i, j);
    const double r = ((z[q] - ztau[q]) + R * d.dt) * d.dtau;
    if (STAGE == 1) zout[q] = ztau[q] + r;
    if (STAGE == 2) zout[q] = 0.75 * ztau[q] + 0.25 * (zin[q] + r);
    if (STAGE == 3) zout[q] = 1.0 / 3.0 * ztau[q] + 2.0 / 3.0 * (zin[q] + r);
  }
}

// ---- boundary passes (boundary.f90), one block per case --------------------------------------
// which: 0..2 = u written by U stage s (S0, S1, U[ntau]) with vm = V[tau];
//        3..5 = um = U[tau] with v written by V stage s (S0, S1, V[ntau]).
__device__ void bc_uv_block(const CaseDev& d, double* um, double* vm) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (d.bc == 0) {
    // bottom, top rows (boundary.f90:9-26), per column i
    for (int i = 1 + tid; i <= nx; i += nt) {
      vm[lin(i, 1, P)] = d.v_in;
      vm[lin(i, 2, P)] = vm[lin(i, 1, P)];
      if (i >= 2) {
        um[lin(i, 1, P)] = 0.0;
        vm[lin(i, ny, P)] = 2.0 * vm[lin(i, ny - 2, P)] - vm[lin(i, ny - 1, P)];
        vm[lin(i, ny + 1, P)] = 2.0 * vm[lin(i, ny - 1, P)] - vm[lin(i, ny, P)];
        um[lin(i, ny, P)] = um[lin(i, ny - 1, P)];
      }
    }
    __syncthreads();
    // left (:29-36) and right (:39-46) columns
    for (int j = 1 + tid; j <= ny + 1; j += nt) {
      if (j <= ny) {
        um[lin(2, j, P)] = 0.0; um[lin(1, j, P)] = 0.0;
        um[lin(nx, j, P)] = 0.0; um[lin(nx + 1, j, P)] = 0.0;
      }
      vm[lin(1, j, P)] = vm[lin(2, j, P)];
      if (j >= 2 && j <= ny) vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    }
  } else {
    // channel: inflow/outflow columns first, then the wall rows
    for (int j = 1 + tid; j <= ny + 1; j += nt) {
      if (j <= ny) {
        um[lin(1, j, P)] = d.v_in;
        um[lin(2, j, P)] = d.v_in;
        um[lin(nx, j, P)] = um[lin(nx - 1, j, P)];
        um[lin(nx + 1, j, P)] = um[lin(nx, j, P)];
      }
      vm[lin(1, j, P)] = -vm[lin(2, j, P)];
      vm[lin(nx, j, P)] = vm[lin(nx - 1, j, P)];
    }
    __syncthreads();
    for (int i = 1 + tid; i <= nx + 1; i += nt) {
      um[lin(i, 1, P)] = -um[lin(i, 2, P)];
      um[lin(i, ny, P)] = -um[lin(i, ny - 1, P)];
      if (i <= nx) {
        vm[lin(i, 2, P)] = 0.0;
        vm[lin(i, ny, P)] = 0.0;
        vm[lin(i, 1, P)] = -vm[lin(i, 3, P)];
        vm[lin(i, ny + 1, P)] = -vm[lin(i, ny - 1, P)];
      }
    }
  }
}

// bcP / bcZ / bcC (boundary.f90:52-159); `neumann_in` = true for p (inflow boundary copies the
// neighbour), false for scalars (inflow boundary takes zin).
__device__ void bc_cell_block(const CaseDev& d, double* z, bool neumann_in, double zin) {
  const int nx = d.nx, ny = d.ny, P = d.pitch;
  const int tid = threadIdx.x, nt = blockDim.x;
  if (d.bc == 0) {
    for (int i = 1 + tid; i <= nx; i += nt) {
      z[lin(i, 1, P)] = neumann_in ? z[lin(i, 2, P)] : zin;
      z[lin(i, ny, P)] = z[lin(i, ny - 1, P)] + 1.0 * (z[lin(i, ny - 1, P)] - z[lin(i, ny - 2, P)]);
    }
    __syncthreads();
    for (int j = 1 + tid; j <= ny; j += nt) {
      z[lin(1, j, P)] = z[lin(2, j, P)];
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)];
    }
  } else {
    for (int j = 1 + tid; j <= ny; j += nt) {
      z[lin(1, j, P)] = neumann_in ? z[lin(2, j, P)] : zin;
      z[lin(nx, j, P)] = z[lin(nx - 1, j, P)] + 1.0 * (z[lin(nx - 1, j, P)] - z[lin(nx - 2, j, P)]);
    }
    __syncthreads();
    for (int i = 1 + tid; i <= nx; i += nt) {
      z[lin(i, 1, P)] = z[lin(i, 2, P)];
      z[lin(i, ny, P)] = z[lin(i, ny - 1, P)];
    }
  }
}

__global__ void k_bc_uv(const CaseDev* __restrict__ cs, const CaseCtl* __restrict__ ctl, int which) {
  const int c = blockIdx.x;
  if (!ctl[c].active) return;
  const CaseDev& d = cs[c];
  const CaseCtl& k = ctl[c];
  double *um, *vm;
  if (which < 3) {
    um = which == 2 ? d.U[k.ru[R_NTAU]] : d.S[which];
    vm = d.V[k.rv[R_TAU]];
  } else {
    um = d.U[k.ru[R_TAU]];
    vm = which == 5 ? d.V[k.rv[R_NTAU]] : d.S[which - 3];
  }
  bc_uv_block(d, um, vm);
}

// which: 0 = p (P[pn]); 1..3 = T written by stage (S0, S1, T[ntau]); 4..6 = C likewise.
__global__ void k_bc_cell(const CaseDev* __restrict__ cs, const CaseCtl* __restrict__ ctl, int which) {
  const int c = blockIdx.x;
  if (!ctl[c].active) return;
  const CaseDev& d = cs[c];
  const CaseCtl& k = ctl[c];
  if (which == 0) { bc_cell_block(d, d.P[k.rp[1]], true, 0.0); return; }
  if (!k.scalars) return;
  const bool isC = which >= 4;
  const int s = isC ? which - 4 : which - 1;
  double* z = s == 2 ? (isC ? d.C[k.rc[R_NTAU]] : d.T[k.rt[R_NTAU]]) : d.S[s];
  bc_cell_block(d, z, false, isC ? d.C_in : d.T_in);
}

namespace {
template <int S>
void go_u(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_u_stage_exact<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <int S>
void go_v(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_v_stage_exact<S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
template <bool IC, int S>
void go_s(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_s_stage_exact<IC, S><<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
}  // namespace

void launch_u_stage_exact(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_u<1>(c, k, t, n, s);
  else if (stage == 2) go_u<2>(c, k, t, n, s);
  else go_u<3>(c, k, t, n, s);
}
void launch_v_stage_exact(int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (stage == 1) go_v<1>(c, k, t, n, s);
  else if (stage == 2) go_v<2>(c, k, t, n, s);
  else go_v<3>(c, k, t, n, s);
}
void launch_s_stage_exact(bool is_c, int stage, const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  if (is_c) {
    if (stage == 1) go_s<true, 1>(c, k, t, n, s);
    else if (stage == 2) go_s<true, 2>(c, k, t, n, s);
    else go_s<true, 3>(c, k, t, n, s);
  } else {
    if (stage == 1) go_s<false, 1>(c, k, t, n, s);
    else if (stage == 2) go_s<false, 2>(c, k, t, n, s);
    else go_s<false, 3>(c, k, t, n, s);
  }
}
void launch_p_exact(const CaseDev* c, CaseCtl* k, const Tile* t, int n, cudaStream_t s) {
  k_p_exact<<<n, dim3(TILE_X, TILE_Y), 0, s>>>(c, k, t);
}
void launch_bc_uv(const CaseDev* c, const CaseCtl* k, int ncases, int which, cudaStream_t s) {
  k_bc_uv<<<ncases, 128, 0, s>>>(c, k, which);
}
void launch_bc_cell(const CaseDev* c, const CaseCtl* k, int ncases, int which, cudaStream_t s) {
  k_bc_cell<<<ncases, 128, 0, s>>>(c, k, which);
}

}  // namespace acs
