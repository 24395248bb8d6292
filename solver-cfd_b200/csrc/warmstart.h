// warmstart.h -- device side of the learned warm start (warmstart.cu), called by solver.cu.
//
// Canvas: every case of a batch is drawn on a common H x W canvas; node (i, j) of any field
// (um, vm, p, T, C; 1-based, staggered) sits at pixel (y, x) = (j-1, i-1), so the staggered
// arrays share one (nx+1) x (ny+1) grid with no interpolation.  Pixels outside a field's own
// shape hold 0.
#pragma once
#include <cuda_runtime.h>
#include "acs_dev.cuh"

namespace acs {

constexpr int WS_FIELDS = 5;     // u, v, p, T, C
constexpr int WS_IN = 11;        // u, v, p, T, C, porous mask, previous increment of the 5 fields
constexpr int WS_OUT = 8;        // 5 increment channels, padded to 8

struct WsCase {
  double* prev[WS_FIELDS];  // fields at the previous feature call (physical step start)
  double* inc[WS_FIELDS];   // their increment over the last physical step
  double* incp[WS_FIELDS];  // the increment over the step before (for the quadratic start)
};

// History (incp = inc, inc = fields - prev, prev = fields), the per-case, per-field RMS of inc into sc[c*8+f]
// (1 where it is 0; ss is scratch of the same size; scale_out, if not null, receives sc as FP32)
// and X[c][y][x][11] (FP32): fields, porous indicator, inc / sc.
void launch_ws_features(const CaseDev* dc, const CaseCtl* dk, const WsCase* dw, int n, int H, int W, int has_prev,
                        double* ss, double* sc, float* X, float* scale_out, cudaStream_t s);
// T[c][y][x][8] = ((fields - prev) - inc) / sc (the increment's change over the step just run,
// relative to the increment's size), Wt = 1 where the node exists in that field, else 0.
void launch_ws_target(const CaseDev* dc, const CaseCtl* dk, const WsCase* dw, int n, int H, int W, const double* sc,
                      float* T, float* Wt, cudaStream_t s);
// Candidates plain / extrapolated / learned (Y may be null: no learned candidate), initial
// residuals into res[3c + k], choice[c] = k of the committed start (policy 0: smallest residual,
// 1: the prediction, 2: plain).  order 1: the extrapolated candidate is x + inc (linear);
// order 2: x + (2 inc - incp) (quadratic through the last three step starts).
void launch_ws_start(const CaseDev* dc, CaseCtl* dk, const WsCase* dw, int n, int H, int W, const double* sc,
                     const float* Y, int ldy, const float* scale, int policy, int order, unsigned long long* res,
                     int* choice, cudaStream_t s);

}  // namespace acs
