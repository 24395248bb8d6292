// Host-side memory and undefined-behaviour checks (test infrastructure).
//
// Built by tests/test_sanitizers.py with AddressSanitizer and UndefinedBehaviorSanitizer together
// with the product's host mesh code (solver-cfd_b200/csrc/mesh.cpp) and the CPU oracle
// (oracle/acs_oracle.cpp).  Every array is a std::vector of exactly the size the C ABI documents,
// so a read or write one element past an edge is reported.  For each geometry (reference domain
// at several imax, channels with odd sizes and one or two porous blocks) it
//   * builds the mesh with the product and with the oracle and requires identical output,
//   * calls every per-routine entry point of the oracle once on seeded fields,
//   * runs two physical steps of the pseudo-time loop (a few iterations each),
// and exits non-zero on the first mismatch or non-finite value.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/acs.h"

extern "C" {
struct orc_case;
int orc_reference_jmax(int imax);
int orc_mesh_reference(int imax, double porosity, double* x, double* y, double* xm, double* ym, int* flag,
                       double* eps, double* liga);
int orc_mesh_channel(int nx, int ny, double Lx, double Ly, double s, double bx0, double bx1, double by0,
                     double by1, double cx0, double cx1, double cy0, double cy1, double porosity, double* x,
                     double* y, double* xm, double* ym, int* flag, double* eps, double* liga);
double orc_noise(uint64_t seed, uint64_t case_id, uint64_t field, uint64_t index, double amp);
orc_case* orc_create(const acs_params* prm, const double* x, const double* y, const double* xm, const double* ym,
                     const double* eps, const double* liga);
void orc_destroy(orc_case* h);
double orc_solve_u(orc_case* h, const double* um, const double* um_tau, double* vm_tau, const double* p,
                   double* um_n_tau);
double orc_solve_v(orc_case* h, const double* vm, double* um_tau, const double* vm_tau, const double* p,
                   const double* T, double* vm_n_tau);
double orc_solve_p(orc_case* h, const double* p, const double* um_n, const double* vm_n, double* pn);
void orc_solve_z(orc_case* h, const double* um_n, const double* vm_n, const double* Z, double* Z_n_tau,
                 const double* Z_tau);
void orc_solve_c(orc_case* h, const double* um_n, const double* vm_n, const double* C, double* C_n_tau,
                 const double* C_tau);
void orc_bc_uv(orc_case* h, double* um, double* vm);
void orc_bc_p(orc_case* h, double* p);
void orc_bc_z(orc_case* h, double* z);
void orc_bc_c(orc_case* h, double* z);
struct orc_state {
  double *um, *vm, *um_tau, *vm_tau, *um_n_tau, *vm_n_tau;
  double *p, *pn;
  double *T, *T_tau, *T_n_tau, *C, *C_tau, *C_n_tau;
};
long orc_run(orc_case* h, orc_state* s, int n_steps, int* itc_io, int* iters, double* err);
}

namespace {

int g_failures = 0;

void check(bool ok, const char* what, const char* geometry) {
  if (!ok) {
    std::fprintf(stderr, "FAIL %s: %s\n", geometry, what);
    ++g_failures;
  }
}

struct Mesh {
  int nx, ny;
  std::vector<double> x, y, xm, ym, eps, liga;
  std::vector<int> flag;
  Mesh(int nx_, int ny_)
      : nx(nx_), ny(ny_), x(nx_), y(ny_), xm(nx_ + 1), ym(ny_ + 1), eps((size_t)nx_ * ny_),
        liga((size_t)nx_ * ny_), flag((size_t)nx_ * ny_) {}
  bool same(const Mesh& o) const {
    return x == o.x && y == o.y && xm == o.xm && ym == o.ym && eps == o.eps && liga == o.liga && flag == o.flag;
  }
};

struct State {
  std::vector<double> um, vm, um_tau, vm_tau, um_n_tau, vm_n_tau, p, pn, T, T_tau, T_n_tau, C, C_tau, C_n_tau;
  State(int nx, int ny) {
    const size_t nu = (size_t)(nx + 1) * ny, nv = (size_t)nx * (ny + 1), np = (size_t)nx * ny;
    for (auto* a : {&um, &um_tau, &um_n_tau}) a->assign(nu, 0.0);
    for (auto* a : {&vm, &vm_tau, &vm_n_tau}) a->assign(nv, 0.0);
    for (auto* a : {&p, &pn, &T, &T_tau, &T_n_tau, &C, &C_tau, &C_n_tau}) a->assign(np, 0.0);
  }
  void seed(uint64_t s) {
    uint64_t f = 0;
    for (auto* a : {&um, &vm, &um_tau, &vm_tau, &p, &pn, &T, &T_tau, &C, &C_tau}) {
      for (size_t k = 0; k < a->size(); ++k) (*a)[k] = 0.1 * orc_noise(s, 0, f, k, 1.0);
      ++f;
    }
    for (auto* a : {&T, &T_tau}) for (double& v : *a) v += 1.0;  // T near 1: buoyancy divides by it
  }
  orc_state view() {
    return {um.data(), vm.data(), um_tau.data(), vm_tau.data(), um_n_tau.data(), vm_n_tau.data(), p.data(),
            pn.data(), T.data(), T_tau.data(), T_n_tau.data(), C.data(), C_tau.data(), C_n_tau.data()};
  }
  bool finite() const {
    for (auto* a : {&um, &vm, &um_tau, &vm_tau, &um_n_tau, &vm_n_tau, &p, &pn, &T, &C})
      for (double v : *a)
        if (!std::isfinite(v)) return false;
    return true;
  }
};

// 0.85 x the three-stage Runge-Kutta limit for the artificial-compressibility mode
double stable_dtau(const Mesh& m, double beta, double dt) {
  double dx = 1e300, dy = 1e300;
  for (int i = 1; i < m.nx; ++i) dx = std::fmin(dx, m.x[i] - m.x[i - 1]);
  for (int j = 1; j < m.ny; ++j) dy = std::fmin(dy, m.y[j] - m.y[j - 1]);
  return 0.85 * std::sqrt(3.0) / (std::sqrt(beta * dt) * 2.0 * std::sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy)));
}

void exercise(const acs_params& prm, const Mesh& m, const char* geometry) {
  orc_case* h = orc_create(&prm, m.x.data(), m.y.data(), m.xm.data(), m.ym.data(), m.eps.data(), m.liga.data());
  State s(m.nx, m.ny);
  s.seed(7);
  // every per-routine entry point once (the order of main.f90:122-132)
  orc_solve_u(h, s.um.data(), s.um_tau.data(), s.vm_tau.data(), s.pn.data(), s.um_n_tau.data());
  orc_solve_v(h, s.vm.data(), s.um_tau.data(), s.vm_tau.data(), s.pn.data(), s.T.data(), s.vm_n_tau.data());
  orc_solve_p(h, s.p.data(), s.um_n_tau.data(), s.vm_n_tau.data(), s.pn.data());
  orc_solve_z(h, s.um_n_tau.data(), s.vm_n_tau.data(), s.T.data(), s.T_n_tau.data(), s.T_tau.data());
  orc_solve_c(h, s.um_n_tau.data(), s.vm_n_tau.data(), s.C.data(), s.C_n_tau.data(), s.C_tau.data());
  orc_bc_uv(h, s.um.data(), s.vm.data());
  orc_bc_p(h, s.p.data());
  orc_bc_z(h, s.T.data());
  orc_bc_c(h, s.C.data());
  check(s.finite(), "per-routine outputs finite", geometry);
  // two physical steps of the loop
  State r(m.nx, m.ny);
  r.seed(11);
  orc_state v = r.view();
  int itc = 1, iters[2] = {0, 0};
  double err[2] = {0.0, 0.0};
  const long total = orc_run(h, &v, 2, &itc, iters, err);
  check(total == (long)iters[0] + iters[1] && iters[0] >= 2 && iters[1] >= 1, "iteration counts", geometry);
  check(r.finite(), "loop state finite", geometry);
  orc_destroy(h);
}

void reference_geometry(int imax, int scheme) {
  char name[64];
  std::snprintf(name, sizeof(name), "reference imax=%d scheme=%d", imax, scheme);
  const int jmax = acs_reference_jmax(imax);
  check(jmax == orc_reference_jmax(imax), "jmax", name);
  Mesh a(imax, jmax), b(imax, jmax);
  check(acs_mesh_reference(imax, 0.5, a.x.data(), a.y.data(), a.xm.data(), a.ym.data(), a.flag.data(),
                           a.eps.data(), a.liga.data()) == ACS_OK, "acs_mesh_reference", name);
  check(orc_mesh_reference(imax, 0.5, b.x.data(), b.y.data(), b.xm.data(), b.ym.data(), b.flag.data(),
                           b.eps.data(), b.liga.data()) == jmax, "orc_mesh_reference", name);
  check(a.same(b), "product mesh == oracle mesh", name);
  acs_params p{};
  p.imax = imax; p.jmax = jmax; p.scheme = scheme; p.bc = ACS_BC_REFERENCE; p.solve_scalars = 1;
  p.itc_max = 12; p.Re = 1.0; p.Pe = 1.0; p.Sc = 1.0; p.Da = 1e-2; p.Cf = 1.75 / std::sqrt(150.0 * 0.125);
  p.g = 9.80665; p.InvFr2 = 1.0; p.v_in = 0.5; p.T_in = 1.0; p.C_in = 0.0; p.b_art = 0.3; p.beta = 1300.0;
  p.dt = 5e-3; p.dtau = 5e-5; p.eps = 1e-4; p.arith = ACS_ARITH_EXACT; p.continuity = 0;
  exercise(p, a, name);
}

void channel_geometry(int nx, int ny, int blocks, int scheme) {
  char name[64];
  std::snprintf(name, sizeof(name), "channel %dx%d blocks=%d scheme=%d", nx, ny, blocks, scheme);
  const double box1[4] = {0.6, 1.0, 0.3, 0.7}, box2[4] = {1.3, 1.6, 0.1, 0.5}, none[4] = {1.0, 0.0, 0.0, 0.0};
  const double* b1 = blocks >= 1 ? box1 : nullptr;
  const double* b2 = blocks >= 2 ? box2 : nullptr;
  Mesh a(nx, ny), b(nx, ny);
  check(acs_mesh_channel(nx, ny, 2.0, 1.0, 1.5, b1, b2, 0.4, a.x.data(), a.y.data(), a.xm.data(), a.ym.data(),
                         a.flag.data(), a.eps.data(), a.liga.data()) == ACS_OK, "acs_mesh_channel", name);
  const double* o1 = b1 ? b1 : none;
  const double* o2 = b2 ? b2 : none;
  orc_mesh_channel(nx, ny, 2.0, 1.0, 1.5, o1[0], o1[1], o1[2], o1[3], o2[0], o2[1], o2[2], o2[3], 0.4,
                   b.x.data(), b.y.data(), b.xm.data(), b.ym.data(), b.flag.data(), b.eps.data(), b.liga.data());
  check(a.same(b), "product mesh == oracle mesh", name);
  acs_params p{};
  p.imax = nx; p.jmax = ny; p.scheme = scheme; p.bc = ACS_BC_CHANNEL; p.solve_scalars = 1; p.itc_max = 12;
  p.Re = 200.0; p.Pe = 140.0; p.Sc = 1.0; p.Da = 1e-3; p.Cf = 0.55; p.g = 0.0; p.InvFr2 = 1.0; p.v_in = 1.0;
  p.T_in = 1.0; p.C_in = 1.0; p.b_art = 0.0; p.beta = 1.0; p.dt = 1e-3; p.eps = 1e-6;
  p.arith = ACS_ARITH_EXACT; p.continuity = 1;
  p.dtau = stable_dtau(a, p.beta, p.dt);
  exercise(p, a, name);
}

}  // namespace

int main() {
  for (int imax : {6, 7, 10, 12, 23}) {
    reference_geometry(imax, ACS_SCHEME_QUICK);
    reference_geometry(imax, ACS_SCHEME_UPWIND);
  }
  channel_geometry(6, 6, 0, ACS_SCHEME_QUICK);
  channel_geometry(13, 9, 1, ACS_SCHEME_QUICK);
  channel_geometry(17, 11, 2, ACS_SCHEME_QUICK);
  channel_geometry(24, 7, 1, ACS_SCHEME_UPWIND);
  // the noise generator and its array form
  std::vector<uint64_t> idx(97);
  std::vector<double> out(97);
  for (size_t k = 0; k < idx.size(); ++k) idx[k] = k * 7919u;
  check(acs_noise_array(3, 5, 2, idx.data(), (long long)idx.size(), 1e-3, out.data()) == ACS_OK, "noise_array",
        "noise");
  for (size_t k = 0; k < idx.size(); ++k)
    check(out[k] == orc_noise(3, 5, 2, idx[k], 1e-3) && std::fabs(out[k]) <= 1e-3, "noise value", "noise");
  check(acs_noise_array(3, 5, 2, nullptr, 4, 1e-3, out.data()) == ACS_E_ARG, "noise null index", "noise");
  check(acs_mesh_reference(5, 0.5, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == ACS_E_ARG,
        "mesh too small", "reference");
  if (g_failures) {
    std::fprintf(stderr, "%d check(s) failed\n", g_failures);
    return 1;
  }
  std::printf("host checks passed\n");
  return 0;
}
