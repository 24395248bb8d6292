// mesh.cpp -- driver-side helpers exported through the C ABI: the reference mesh
// (nonsymetric_mesh.f90:1-218 for the domain compiled into comum.f90:29-46), the channel mesh
// used by the synthetic configurations, and the seeded noise generator.
//
// These run on the host once per case (the reference driver calls `mesh` once before the loop)
// and are not part of the timed loop.  Their arithmetic follows the Fortran expression order so
// the metric arrays are bit-identical to the reference's (pinned against its grid_u.dat and
// grid_v.dat outputs).
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/acs.h"

namespace {

constexpr int kFluid = 0, kBoundary = 1, kInterior = 2, kBoundarySide = 3;  // comum.f90:75

// Staggered mid-points xm, ym (nonsymetric_mesh.f90:48-60); all arrays 1-based.
void staggered(int nx, int ny, const double* X, const double* Y, double* XM, double* YM) {
  XM[1] = -(X[2] + X[1]) * 0.5;
  XM[nx + 1] = (X[nx] + X[nx - 1]) * 0.5 + (X[nx] - X[nx - 1]);
  for (int i = 2; i <= nx; ++i) XM[i] = (X[i] + X[i - 1]) * 0.5;
  YM[1] = Y[1] - (Y[2] - Y[1]) * 0.5;
  YM[ny + 1] = (Y[ny] + Y[ny - 1]) * 0.5 + (Y[ny] - Y[ny - 1]);
  for (int j = 2; j <= ny; ++j) YM[j] = (Y[j] + Y[j - 1]) * 0.5;
}

// Porous flag (nonsymetric_mesh.f90:166-218).  `flag` is column-major nx x ny, pre-filled with
// kInterior inside the block(s) and kFluid elsewhere.  The last sweep of the reference reads one
// word before each column (flag(0,j)), which in column-major storage is flag(nx,j-1); reads
// before the first word count as "not boundary".
void dilate(int nx, int ny, std::vector<int>& flag) {
  auto at = [&](int i, int j) -> int& { return flag[(size_t)(i - 1) + (size_t)(j - 1) * nx]; };
  auto word = [&](int i, int j) -> int {
    const long w = (long)(i - 1) + (long)(j - 1) * nx;
    return (w >= 0 && w < (long)nx * ny) ? flag[w] : -1;
  };
  for (int j = 2; j < ny; ++j)
    for (int i = 2; i < nx; ++i)
      if (at(i, j) == kInterior &&
          (at(i - 1, j) == kFluid || at(i, j - 1) == kFluid || at(i + 1, j) == kFluid || at(i, j + 1) == kFluid))
        at(i, j) = kBoundary;
  for (int j = 2; j < ny; ++j)
    if (at(1, j) == kInterior && (at(1, j - 1) == kFluid || at(1, j + 1) == kFluid)) at(1, j) = kBoundary;
  for (int j = 1; j < ny; ++j)
    for (int i = 1; i < nx; ++i)
      if (at(i, j) == kFluid && (word(i - 1, j) == kBoundary || word(i, j - 1) == kBoundary ||
                                 word(i + 1, j) == kBoundary || word(i, j + 1) == kBoundary))
        at(i, j) = kBoundarySide;
}

void porous_fields(int nx, int ny, const std::vector<int>& flag, double porosity, int* flag_out,
                   double* eps, double* liga) {
  for (size_t q = 0; q < (size_t)nx * ny; ++q) {
    const bool porous = flag[q] != kFluid;
    eps[q] = porous ? porosity : 1.0;
    liga[q] = porous ? 1.0 : 0.0;
    if (flag_out) flag_out[q] = flag[q];
  }
}

// s(eta) of the reference stretching (nonsymetric_mesh.f90:22-23)
inline double stretch(double P, double Q, double eta) {
  return P * eta + (1.0 - P) * (1.0 - (std::tanh(Q * (1.0 - eta))) / std::tanh(Q));
}

}  // namespace

extern "C" {

int acs_reference_jmax(int imax) {
  const double Lhori = 12.0, Hvert = 15.0 + 5.0;
  const double dx_c = Lhori / (imax - 1);
  return (int)(Hvert / dx_c + 1.0);
}

int acs_mesh_reference(int imax, double porosity, double* x, double* y, double* xm, double* ym,
                       int* flag_out, double* epsilon1, double* liga_poros) {
  if (imax < 6 || !x || !y || !xm || !ym || !epsilon1 || !liga_poros) return ACS_E_ARG;
  const double Lhori = 12.0, y_down = 5.0;
  const double Px = 1.0, Py = 1.6, Q = 1.0;
  const double dx_c = Lhori / (imax - 1);
  const int nx = imax, ny = acs_reference_jmax(imax);
  double* X = x - 1;  // 1-based views
  double* Y = y - 1;
  for (int i = 1; i <= nx; ++i) X[i] = ((double)i - 1.0) * dx_c - Lhori / 2.0;
  for (int j = 1; j <= ny; ++j) Y[j] = ((double)j - 1.0) * dx_c - y_down;
  const int ic = nx / 2 + 1;
  for (int i = ic; i <= nx; ++i) X[i] = X[nx] - stretch(Px, Q, (X[i] - X[nx]) / (X[ic] - X[nx])) * (X[nx] - X[ic]);
  for (int i = ic; i >= 1; --i) X[i] = -X[nx] - stretch(Px, Q, (X[i] + X[nx]) / (X[ic] + X[nx])) * (-X[nx] - X[ic]);
  const int jc = (int)(y_down / dx_c) + 1;
  for (int j = jc; j <= ny; ++j) Y[j] = Y[ny] - stretch(Py, Q, (Y[j] - Y[ny]) / (Y[jc] - Y[ny])) * (Y[ny] - Y[jc]);
  for (int j = jc; j >= 1; --j) Y[j] = -Y[ny] - stretch(Py, Q, (Y[j] + Y[ny]) / (Y[jc] + Y[ny])) * (-Y[ny] - Y[jc]);
  staggered(nx, ny, X, Y, xm - 1, ym - 1);
  std::vector<int> flag((size_t)nx * ny);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      flag[(size_t)(i - 1) + (size_t)(j - 1) * nx] = (X[i] <= -4.0 && Y[j] >= 0.5) ? kInterior : kFluid;
  dilate(nx, ny, flag);
  porous_fields(nx, ny, flag, porosity, flag_out, epsilon1, liga_poros);
  return ACS_OK;
}

}  // extern "C"

// The channel mesh's 1-D arrays (x, y, xm, ym; 0-based storage of the 1-based arrays), shared by
// acs_mesh_channel and the device generator of mesh_device.cu.
void acs_channel_axes(int nx, int ny, double Lx, double Ly, double s, double* x, double* y, double* xm, double* ym) {
  double* X = x - 1;
  double* Y = y - 1;
  for (int i = 1; i <= nx; ++i) X[i] = Lx * ((double)(i - 1) / (double)(nx - 1));
  for (int j = 1; j <= ny; ++j) {
    const double xi = (double)(j - 1) / (double)(ny - 1);
    Y[j] = s > 0.0 ? 0.5 * Ly * (1.0 + std::tanh(s * (2.0 * xi - 1.0)) / std::tanh(s)) : Ly * xi;
  }
  staggered(nx, ny, X, Y, xm - 1, ym - 1);
}

extern "C" {

int acs_mesh_channel(int imax, int jmax, double Lx, double Ly, double s, const double* box1,
                     const double* box2, double porosity, double* x, double* y, double* xm,
                     double* ym, int* flag_out, double* epsilon1, double* liga_poros) {
  if (imax < 6 || jmax < 6 || !x || !y || !xm || !ym || !epsilon1 || !liga_poros) return ACS_E_ARG;
  const int nx = imax, ny = jmax;
  acs_channel_axes(nx, ny, Lx, Ly, s, x, y, xm, ym);
  const double* X = x - 1;
  const double* Y = y - 1;
  auto inside = [](const double* b, double px, double py) {
    return b && b[0] <= b[1] && px >= b[0] && px <= b[1] && py >= b[2] && py <= b[3];
  };
  std::vector<int> flag((size_t)nx * ny);
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i)
      flag[(size_t)(i - 1) + (size_t)(j - 1) * nx] =
          (inside(box1, X[i], Y[j]) || inside(box2, X[i], Y[j])) ? kInterior : kFluid;
  dilate(nx, ny, flag);
  porous_fields(nx, ny, flag, porosity, flag_out, epsilon1, liga_poros);
  return ACS_OK;
}

double acs_noise(uint64_t seed, uint64_t case_id, uint64_t field, uint64_t index, double amp) {
  uint64_t z = (seed + 1) * 0x9E3779B97F4A7C15ULL + case_id * 0xD1B54A32D192ED03ULL +
               field * 0x8CB92BA72F3D8DD7ULL + index * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * 0x1.0p-53;
  return amp * (2.0 * u - 1.0);
}

int acs_noise_array(uint64_t seed, uint64_t case_id, uint64_t field, const uint64_t* index, long long n,
                    double amp, double* out) {
  if (n < 0 || (n > 0 && (!index || !out))) return ACS_E_ARG;
  for (long long k = 0; k < n; ++k) out[k] = acs_noise(seed, case_id, field, index[k], amp);
  return ACS_OK;
}

}  // extern "C"
