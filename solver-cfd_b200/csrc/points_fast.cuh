// points_fast.cuh -- per-node residuals with the FAST arithmetic, shared by the persistent
// cluster engine (engine_fast.cu) and the per-stage kernels of the graph engine
// (kernels_fast.cu).
//
// Same discretisation as the reference, rearranged for fewer FP64 operations:
//   * every division by a metric difference becomes a product with a reciprocal precomputed
//     once per case in 1-D tables (MX per column i, MY per row j);
//   * the QUICK / upwind coefficient sums  -ap*uP + sum(a_nb*u_nb)  are evaluated in the
//     equivalent face-value form  fw*phi_w - fe*phi_e + fs*phi_s - fn*phi_n  plus the diffusive
//     face differences (the identity is exact in real arithmetic);
//   * porosity enters through a 1-byte mask and per-case constants (1/phi, phi/(Re Da),
//     Cf/sqrt(phi Da)) instead of two FP64 fields;
//   * solve_P's three stages with frozen RP collapse to pn = p + dtau*beta*RP;
//   * products and sums may fuse (FMA).
// Reference (OpenMp_Multicore/): RESU equations.f90:2-116, RESV :305-420, RESZ :723-765,
// RESC :823-867, solve_P :607-665.
#pragma once
#include <cuda_runtime.h>
#include "acs_dev.cuh"

namespace acs {

// per-column table MX[i] = {x(i)-x(i-1), 1/(x(i)-x(i-1)), xm(i+1)-xm(i), 1/(xm(i+1)-xm(i))}
// per-row    table MY[j] = {y(j)-y(j-1), 1/(y(j)-y(j-1)), ym(j+1)-ym(j), 1/(ym(j+1)-ym(j))}
struct Met { double d, rd, dm, rdm; };

// Entry k of a metric table (4 doubles) from global memory through the read-only path.
__device__ __forceinline__ Met met_ldg(const double* t, int k) {
  const double2 a = __ldg(reinterpret_cast<const double2*>(t) + 2 * k);
  const double2 b = __ldg(reinterpret_cast<const double2*>(t) + 2 * k + 1);
  return {a.x, a.y, b.x, b.y};
}
__device__ __forceinline__ Met mx(const CaseDev& d, int i) { return met_ldg(d.mx, i); }
__device__ __forceinline__ Met my(const CaseDev& d, int j) { return met_ldg(d.my, j); }

// Load policies: ld() reads a field, met() an entry of a metric table.
// Loads of arrays written by other CTAs of the cluster: from L2 (.cg) or through L1 (.ca); the
// cluster barrier's release/acquire pair orders the writes before the reads in both cases.
struct LdL2 {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return __ldcg(a + q); }
  static __device__ __forceinline__ Met met(const double* t, int k) { return met_ldg(t, k); }
};
struct LdL1 {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return __ldca(a + q); }
  static __device__ __forceinline__ Met met(const double* t, int k) { return met_ldg(t, k); }
};
// Generic loads: the staged engine reads its stencil arrays from shared memory and the rest from
// global memory written by this CTA or before the cluster barrier.
struct LdGen {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return a[q]; }
  static __device__ __forceinline__ Met met(const double* t, int k) { return met_ldg(t, k); }
};
// Everything from shared memory: the tile engine stages the fields and slices of the metric
// tables before it computes.  A slice holds the four components of S consecutive table entries
// one after the other (component c of entry k at t[k + c*S], where CaseDev::mx/my point k0
// words before a slice that starts at entry k0), so the lanes of a warp, on consecutive columns,
// read consecutive words.
template <int S>
struct LdShared {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return a[q]; }
  static __device__ __forceinline__ Met met(const double* t, int k) { return {t[k], t[k + S], t[k + 2 * S], t[k + 3 * S]}; }
};

// QUICK face value seen from the face's upstream side (equations.f90:27-70 rearranged):
// flux > 0 takes 0.75 of the upwind node, 0.375 of the downwind node, -0.125 of the far upwind.
__device__ __forceinline__ double quick_face(double f, double up2, double up, double dn, double dn2) {
  return f > 0.0 ? fma(0.75, up, fma(0.375, dn, -0.125 * up2)) : fma(0.75, dn, fma(0.375, up, -0.125 * dn2));
}
__device__ __forceinline__ double upw_face(double f, double up, double dn) { return f > 0.0 ? up : dn; }

template <class L>
struct PtFastT {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return L::ld(a, q); }
  static __device__ __forceinline__ double F(const double* a, long long q) { return L::ld(a, q); }
  static __device__ __forceinline__ Met MX(const CaseDev& d, int i) { return L::met(d.mx, i); }
  static __device__ __forceinline__ Met MY(const CaseDev& d, int j) { return L::met(d.my, j); }

  // u-momentum residual RU at node (i,j)
  static __device__ __forceinline__ double ru(const CaseDev& d, const double* um, const double* vm,
                                              const double* p, int i, int j) {
    const long long q = lin(i, j, d.pitch);
    return ru_at(d, um, vm, p, d.pitch, q, d.mask[q] != 0, i, j);
  }
  // Same, with the fields indexed by q and row stride P (a shared-memory tile, or the case array
  // itself) and the node's porous flag given.
  static __device__ __forceinline__ double ru_at(const CaseDev& d, const double* um, const double* vm,
                                                 const double* p, int P, long long q, bool por, int i, int j) {
    const double e = por ? d.phi : 1.0, ie = por ? d.fc[FC_IPHI] : 1.0;
    const Met X = MX(d, i), Y = MY(d, j), Yn = MY(d, j + 1);
    const double uP = F(um, q), uW = F(um, q - 1), uE = F(um, q + 1), uS = F(um, q - P), uN = F(um, q + P);
    const double hx = 0.5 * X.d * ie, hy = 0.5 * Y.dm * ie;
    const double fn = (F(vm, q + P) + F(vm, q + P - 1)) * hx;
    const double fs = (F(vm, q) + F(vm, q - 1)) * hx;
    const double fe = (uE + uP) * hy;
    const double fw = (uP + uW) * hy;
    const bool quick = d.scheme == 0 && j >= 3 && j <= d.ny - 2;
    double conv;
    if (quick) {
      const double uWW = F(um, q - 2), uEE = F(um, q + 2), uSS = F(um, q - 2 * P), uNN = F(um, q + 2 * P);
      conv = fw * quick_face(fw, uWW, uW, uP, uE) - fe * quick_face(fe, uW, uP, uE, uEE) +
             fs * quick_face(fs, uSS, uS, uP, uN) - fn * quick_face(fn, uS, uP, uN, uNN);
    } else {
      conv = fw * upw_face(fw, uW, uP) - fe * upw_face(fe, uP, uE) + fs * upw_face(fs, uS, uP) - fn * upw_face(fn, uP, uN);
    }
    const double Xw = MX(d, i - 1).rdm;  // 1/(xm(i)-xm(i-1))
    const double diff = e * d.fc[FC_IRE] *
                        (X.d * (Yn.rd * (uN - uP) - Y.rd * (uP - uS)) + Y.dm * (X.rdm * (uE - uP) - Xw * (uP - uW)));
    double r = X.rd * Y.rd * (conv + diff) - e * (F(p, q) - F(p, q - 1)) * X.rd;
    if (d.flags & F_BART) {
      const double dudxdx = Y.dm * (uE - uP) * X.rdm - Y.dm * (uP - uW) * Xw;
      const double dxdvdy = Y.dm * (F(vm, q + P) - F(vm, q)) * Y.rdm - Y.dm * (F(vm, q + P - 1) - F(vm, q - 1)) * Y.rdm;
      r += d.b_art * (dudxdx + dxdvdy);
    }
    if (por) {
      const double vP = F(vm, q);
      r -= e * uP * (d.fc[FC_IREDA] + d.fc[FC_CFS] * sqrt(fma(uP, uP, vP * vP)));
    }
    return r - d.g * e;
  }

  // v-momentum residual RV at node (i,j)
  static __device__ __forceinline__ double rv(const CaseDev& d, const double* um, const double* vm,
                                              const double* p, const double* T, int i, int j) {
    const long long q = lin(i, j, d.pitch);
    const double T0 = (d.flags & F_BUOY) ? F(T, q) : 1.0, T1 = (d.flags & F_BUOY) ? F(T, q - d.pitch) : 1.0;
    return rv_at(d, um, vm, p, T0, T1, d.pitch, q, d.mask[q] != 0, i, j);
  }
  // Same, fields indexed by q with row stride P; T0 = T(i,j), T1 = T(i,j-1) (read only with
  // buoyancy) and the node's porous flag given.
  static __device__ __forceinline__ double rv_at(const CaseDev& d, const double* um, const double* vm,
                                                 const double* p, double T0, double T1, int P, long long q,
                                                 bool por, int i, int j) {
    const double w = (d.flags & F_BUOY) ? 1.0 - 2.0 / (T0 + T1) : 0.0;
    return rv_at_w(d, um, vm, p, w, P, q, por, i, j);
  }
  // Same, with the buoyancy factor w = 1 - 2/(T(i,j) + T(i,j-1)) given (read only with buoyancy):
  // T is the physical-step temperature, so w changes only between physical steps.
  static __device__ __forceinline__ double rv_at_w(const CaseDev& d, const double* um, const double* vm,
                                                   const double* p, double w, int P, long long q, bool por, int i,
                                                   int j) {
    const double e = por ? d.phi : 1.0, ie = por ? d.fc[FC_IPHI] : 1.0;
    const Met X = MX(d, i), Xe = MX(d, i + 1), Y = MY(d, j), Ys = MY(d, j - 1);
    const double vP = F(vm, q), vW = F(vm, q - 1), vE = F(vm, q + 1), vS = F(vm, q - P), vN = F(vm, q + P);
    const double hx = 0.5 * X.dm * ie, hy = 0.5 * Y.d * ie;
    const double fn = (vP + vN) * hx;
    const double fs = (vP + vS) * hx;
    const double fe = (F(um, q + 1) + F(um, q + 1 - P)) * hy;
    const double fw = (F(um, q) + F(um, q - P)) * hy;
    const bool quick = d.scheme == 0 && i >= 3 && i <= d.nx - 2;
    double conv;
    if (quick) {
      const double vWW = F(vm, q - 2), vEE = F(vm, q + 2), vSS = F(vm, q - 2 * P), vNN = F(vm, q + 2 * P);
      conv = fw * quick_face(fw, vWW, vW, vP, vE) - fe * quick_face(fe, vW, vP, vE, vEE) +
             fs * quick_face(fs, vSS, vS, vP, vN) - fn * quick_face(fn, vS, vP, vN, vNN);
    } else {
      conv = fw * upw_face(fw, vW, vP) - fe * upw_face(fe, vP, vE) + fs * upw_face(fs, vS, vP) - fn * upw_face(fn, vP, vN);
    }
    const double diff = e * d.fc[FC_IRE] *
                        (X.dm * (Y.rdm * (vN - vP) - Ys.rdm * (vP - vS)) + Y.d * (Xe.rd * (vE - vP) - X.rd * (vP - vW)));
    double r = X.rd * Y.rd * (conv + diff) - e * (F(p, q) - F(p, q - P)) * Y.rd;
    if (d.flags & F_BART) {
      const double dvdydy = X.dm * (vN - vP) * Y.rdm - X.dm * (vP - vS) * Ys.rdm;
      const double dydudx = X.dm * (F(um, q + 1) - F(um, q)) * X.rdm - X.dm * (F(um, q + 1 - P) - F(um, q - P)) * X.rdm;
      r += d.b_art * (dydudx + dvdydy);
    }
    if (d.flags & F_BUOY) r += d.InvFr2 * w;
    if (por) {
      const double uP = F(um, q);
      r -= e * vP * (d.fc[FC_IREDA] + d.fc[FC_CFS] * sqrt(fma(uP, uP, vP * vP)));
    }
    return r;
  }

  // RESZ (IS_C = false, diffusion 1/Pe) / RESC (IS_C = true, diffusion 1/(Re Sc))
  template <bool IS_C>
  static __device__ __forceinline__ double rs(const CaseDev& d, const double* un, const double* vn,
                                              const double* z, int i, int j) {
    const long long q = lin(i, j, d.pitch);
    return rs_at<IS_C>(d, un, vn, d.pitch, q, z, d.pitch, q, d.mask[q] != 0, i, j);
  }
  // Same, un/vn indexed by qu with row stride Pu, z by qz with row stride Pz, the node's porous
  // flag given.
  template <bool IS_C>
  static __device__ __forceinline__ double rs_at(const CaseDev& d, const double* un, const double* vn, int Pu,
                                                 long long qu, const double* z, int Pz, long long qz, bool por,
                                                 int i, int j) {
    const Met X = MX(d, i), Xe = MX(d, i + 1), Y = MY(d, j), Yn = MY(d, j + 1);
    const double zp = F(z, qz), ze = F(z, qz + 1), zw = F(z, qz - 1), zn = F(z, qz + Pz), zs = F(z, qz - Pz);
    const double conv = 0.5 * (Y.dm * ((ze + zp) * F(un, qu + 1) - (zw + zp) * F(un, qu)) +
                               X.dm * ((zn + zp) * F(vn, qu + Pu) - (zs + zp) * F(vn, qu)));
    const double k = IS_C ? d.fc[FC_IRESC] : d.fc[FC_IPE];
    const double diff = k * (Y.dm * (Xe.rd * (ze - zp) - X.rd * (zp - zw)) + X.dm * (Yn.rd * (zn - zp) - Y.rd * (zp - zs)));
    const double icap = por ? d.fc[FC_IPHI] : 1.0;
    const double s = IS_C ? diff - conv * icap : (diff - (por ? 0.0 : conv)) * icap;
    return X.rdm * Y.rdm * s;
  }

  // solve_P at one node: with RP frozen the three stages give pn = p + dtau*beta*RP
  static __device__ __forceinline__ double p_update(const CaseDev& d, const double* p, const double* un,
                                                    const double* vn, int i, int j, double* r) {
    const long long q = lin(i, j, d.pitch);
    return F(p, q) + p_incr_at(d, un, vn, d.pitch, q, i, j, r);
  }
  // dtau*beta*RP at (i,j) with un, vn indexed by q and row stride P (also returned in *r)
  static __device__ __forceinline__ double p_incr_at(const CaseDev& d, const double* un, const double* vn, int P,
                                                     long long q, int i, int j, double* r) {
    const Met X = MX(d, i), Y = MY(d, j);
    double RP = -((F(un, q + 1) - F(un, q)) * Y.dm + (F(vn, q + P) - F(vn, q)) * X.dm);
    if (d.continuity == 1) RP *= X.rdm * Y.rdm;
    *r = d.fc[FC_DTB] * RP;
    return *r;
  }
};

// Read-only loads: in a per-stage kernel no array it reads is written during the launch.
struct LdRO {
  static __device__ __forceinline__ double ld(const double* a, long long q) { return __ldg(a + q); }
  static __device__ __forceinline__ Met met(const double* t, int k) { return met_ldg(t, k); }
};

}  // namespace acs
