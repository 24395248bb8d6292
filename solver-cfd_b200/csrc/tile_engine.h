// tile_engine.h -- host interface of the tile engine (tile_engine.cu).
//
// One pseudo-iteration of every active case of a batch is four stage kernels over a table of
// 32 x 32-node tiles covering all cases -- three Runge-Kutta stages of U and V side by side, then
// P with the three stages of T and of C -- plus the bcUV side effects for cases whose tau arrays
// were uploaded (after stage 1) and the loop control of control.cu.  Each stage kernel loads
// its tiles' stencil inputs into shared memory with TMA (2-D tensor maps over the case arrays,
// zero fill outside), computes the stage, applies the boundary passes to the tile in shared
// memory and stores the whole tile.  FAST arithmetic only.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "acs_dev.cuh"

namespace acs {

constexpr int TE_TILE = 32;     // tile edge in nodes
constexpr int TE_BOX_UV = 36;   // TMA box of the U/V stage kernels: tile + 2-node halo per side
constexpr int TE_BOX_PTC = 40;  // TMA box of the P/T/C kernel: tile + 4 (three fused T/C stages)
constexpr int TE_THREADS = 256;

// Buffers of a case that have a tensor map: U[3], V[3], P[2], T[3], C[3], S[4].
enum TeBuf { TE_U = 0, TE_V = 3, TE_P = 6, TE_T = 8, TE_C = 11, TE_S = 14, TE_NBUF = 18 };

struct TeMaps {
  CUtensorMap uv[TE_NBUF];   // 36 x 36 boxes (stencil inputs of U/V; T, C at the P/T/C kernel)
  CUtensorMap ptc[TE_NBUF];  // 40 x 40 boxes (un, vn, T_tau, C_tau at the P/T/C kernel)
  CUtensorMap pt[TE_NBUF];   // 32 x 32 boxes (pointwise inputs: um, vm, p)
  CUtensorMap t33[3];        // 32 x 33 boxes of T[0..2] (buoyancy reads T(i,j) and T(i,j-1))
  CUtensorMap liga32, liga36;  // the porosity indicator liga (1 in the porous block, else 0)
  CUtensorMap buoyw;         // 32 x 32 boxes of the buoyancy factor (CaseDev::S2[3])
};

// Tile origins of one case, 1-based node (i0, j0): x = i-1 in [0, pitch), y = j-1 in [0, ny+1)
// walked in steps of 32; the last tile of a row or column starts at extent - 32, so it may overlap
// its neighbour.  Every boundary node of a case then lies in a tile that also holds the nodes its
// boundary pass copies from (at most three nodes further in), so a tile can finish its boundary
// itself.  Overlapping tiles compute identical values.
void te_case_tiles(int c, int pitch, int ny, std::vector<Tile>& out);

// Encodes the tensor maps of every buffer of every case (host memory, `maps` holds n entries).
int te_encode_maps(const std::vector<CaseDev>& cases, TeMaps* maps);

// Launches of one pseudo-iteration (without the control kernel).  err: device word set to a
// nonzero code when a TMA wait times out.
void te_launch_uv(int stage, const CaseDev* cs, CaseCtl* ctl, const Tile* tiles, int ntiles, const TeMaps* maps,
                  int* err, cudaStream_t s);
void te_launch_ptc(const CaseDev* cs, CaseCtl* ctl, const Tile* tiles, int ntiles, const TeMaps* maps, int* err,
                   cudaStream_t s);
// The bcUV side effects on um_tau / vm_tau after stage 1 of an iteration that follows an upload
// (cases with CaseCtl::tau_dirty set).
void te_launch_tau_bc(const CaseDev* cs, CaseCtl* ctl, int ncases, cudaStream_t s);
// One-time kernel attributes (dynamic shared memory sizes); returns the first error.
cudaError_t te_prepare();

}  // namespace acs
