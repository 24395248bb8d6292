// fast_tables.cu -- per-case tables of the FAST arithmetic (see engine_fast.cu).
//
// MX[i] = {x(i)-x(i-1), 1/(x(i)-x(i-1)), xm(i+1)-xm(i), 1/(xm(i+1)-xm(i))} for i = 1..imax+1 and
// MY[j] likewise from y and ym; entries whose neighbours do not exist are zero.  The
// reciprocals are computed once here instead of once per node and stage.
#include <cmath>
#include <vector>

#include "fast.h"

namespace acs {

struct FastPlan {
  double* tables = nullptr;
};

int fast_create(std::vector<CaseDev>& cases, const acs_grid* grids, const acs_params* params, FastPlan** out) {
  const int n = (int)cases.size();
  std::vector<size_t> off(n);
  size_t total = 0;
  for (int c = 0; c < n; ++c) {
    if (!(cases[c].flags & F_BINARY))
      return fail(ACS_E_UNSUPPORTED, "FAST arithmetic needs epsilon1/liga_poros in {(1,0),(phi,1)} for every case");
    off[c] = total;
    total += 4 * (size_t)(cases[c].nx + 2) + 4 * (size_t)(cases[c].ny + 2);
  }
  std::vector<double> h(total, 0.0);
  for (int c = 0; c < n; ++c) {
    const acs_grid& g = grids[c];
    const int nx = g.imax, ny = g.jmax;
    auto X = [&](int i) { return g.x[i - 1]; };
    auto Y = [&](int j) { return g.y[j - 1]; };
    auto XM = [&](int i) { return g.xm[i - 1]; };
    auto YM = [&](int j) { return g.ym[j - 1]; };
    double* mx = h.data() + off[c];
    double* my = mx + 4 * (size_t)(nx + 2);
    for (int i = 1; i <= nx + 1; ++i) {
      double* e = mx + 4 * i;
      if (i >= 2 && i <= nx) { e[0] = X(i) - X(i - 1); e[1] = 1.0 / e[0]; }
      if (i <= nx) { e[2] = XM(i + 1) - XM(i); e[3] = 1.0 / e[2]; }
    }
    for (int j = 1; j <= ny + 1; ++j) {
      double* e = my + 4 * j;
      if (j >= 2 && j <= ny) { e[0] = Y(j) - Y(j - 1); e[1] = 1.0 / e[0]; }
      if (j <= ny) { e[2] = YM(j + 1) - YM(j); e[3] = 1.0 / e[2]; }
    }
    CaseDev& d = cases[c];
    const acs_params& p = params[c];
    d.fc[FC_IPHI] = 1.0 / d.phi;
    d.fc[FC_IRE] = 1.0 / p.Re;
    d.fc[FC_IREDA] = 1.0 / (p.Re * p.Da);
    d.fc[FC_CFS] = p.Cf / std::sqrt(d.phi * p.Da);
    d.fc[FC_IRESC] = 1.0 / p.Re / p.Sc;
    d.fc[FC_IPE] = 1.0 / p.Pe;
    d.fc[FC_DTB] = p.dtau * p.beta;
  }
  FastPlan* f = new FastPlan();
  if (cudaMalloc(&f->tables, sizeof(double) * total) != cudaSuccess ||
      cudaMemcpy(f->tables, h.data(), sizeof(double) * total, cudaMemcpyHostToDevice) != cudaSuccess) {
    delete f;
    return fail(ACS_E_NOMEM, "FAST table allocation failed");
  }
  for (int c = 0; c < n; ++c) {
    cases[c].mx = f->tables + off[c];
    cases[c].my = f->tables + off[c] + 4 * (size_t)(cases[c].nx + 2);
  }
  *out = f;
  return ACS_OK;
}

void fast_destroy(FastPlan* f) {
  if (!f) return;
  if (f->tables) cudaFree(f->tables);
  delete f;
}

}  // namespace acs
