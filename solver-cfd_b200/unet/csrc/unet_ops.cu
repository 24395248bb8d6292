// unet_ops.cu -- data-movement and elementwise kernels of the U-Net (everything but the GEMMs).
//
// Layouts: activations are NHWC, i.e. a [pixels][channels] matrix with the channel index
// fastest, pixels ordered (b, y, x); BF16 for forward activations and GEMM operands, FP32 for
// gradients.  A 3x3 "same" convolution is the GEMM  Y = col(X) W^T  with
//   col(X)[m][k],  m = (b, y, x),  k = (ky*3 + kx)*C + c  ->  X[b][y+ky-1][x+kx-1][c] (0 outside),
// K padded with zeros to a multiple of 8 (row stride Kp).  Its gradients are
//   dW = dZ^T col(X)   (dZ^T and col(X)^T are produced by transpose kernels),
//   dX = col2im(dZ W)  (col2im gathers the 9 taps of every input pixel).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../../include/unet.h"

namespace unet {
namespace {

using bf16 = __nv_bfloat16;

constexpr int T = 256;
inline unsigned blocks(long long n) { return (unsigned)((n + T - 1) / T < 65535LL * 64 ? (n + T - 1) / T : 65535LL * 64); }

__global__ void k_im2col(const bf16* __restrict__ X, int B, int H, int W, int C, int Kp, bf16* __restrict__ col) {
  const long long n = (long long)B * H * W * Kp;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % Kp);
    const long long m = q / Kp;
    bf16 v = __float2bfloat16_rn(0.f);
    if (k < 9 * C) {
      const int tap = k / C, c = k - tap * C;
      const int ky = tap / 3, kx = tap - ky * 3;
      const int x = (int)(m % W), y = (int)((m / W) % H), b = (int)(m / ((long long)W * H));
      const int yy = y + ky - 1, xx = x + kx - 1;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[(((long long)b * H + yy) * W + xx) * C + c];
    }
    col[q] = v;
  }
}

// C a multiple of 8 (then Kp = 9C): one thread per 16-byte vector of 8 channels of one tap of one
// pixel, consecutive threads on consecutive vectors (coalesced loads and stores)
__global__ void k_im2col_v8(const uint4* __restrict__ X, int B, int H, int W, int C, uint4* __restrict__ col) {
  const int C8 = C >> 3;
  const long long n = (long long)B * H * W * 9 * C8;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(q % (9 * C8));
    const long long m = q / (9 * C8);
    const int tap = r / C8, c8 = r - tap * C8;
    const int ky = tap / 3, kx = tap - ky * 3;
    const int x = (int)(m % W), y = (int)((m / W) % H), b = (int)(m / ((long long)W * H));
    const int yy = y + ky - 1, xx = x + kx - 1;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[(((long long)b * H + yy) * W + xx) * C8 + c8];
    col[q] = v;
  }
}

__global__ void k_col2im(const float* __restrict__ dcol, int B, int H, int W, int C, int Kp, float* __restrict__ dX) {
  const long long n = (long long)B * H * W * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    float s = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky)
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int yo = y - ky + 1, xo = x - kx + 1;  // output pixel that read X[y][x] through tap (ky,kx)
        if (yo >= 0 && yo < H && xo >= 0 && xo < W)
          s += dcol[(((long long)b * H + yo) * W + xo) * Kp + (ky * 3 + kx) * C + c];
      }
    dX[q] = s;
  }
}

// dst[c][r] = src[r][c] for r < rows, c < cols (32 x 32 shared-memory tiles)
template <class Ty>
__global__ void k_transpose(const Ty* __restrict__ src, int rows, int cols, int lds, Ty* __restrict__ dst, int ldd) {
  __shared__ Ty tile[32][33];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int r = r0 + dy, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[dy][threadIdx.x] = src[(long long)r * lds + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int c = c0 + dy, r = r0 + threadIdx.x;
    if (c < cols && r < rows) dst[(long long)c * ldd + r] = tile[threadIdx.x][dy];
  }
}

__global__ void k_pool_fwd(const bf16* __restrict__ X, int B, int H, int W, int C, bf16* __restrict__ Y) {
  const int h = H / 2, w = W / 2;
  const long long n = (long long)B * h * w * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((long long)w * h));
    const long long i0 = (((long long)b * H + 2 * y) * W + 2 * x) * C + c;
    const float s = __bfloat162float(X[i0]) + __bfloat162float(X[i0 + C]) + __bfloat162float(X[i0 + (long long)W * C]) +
                    __bfloat162float(X[i0 + (long long)W * C + C]);
    Y[q] = __float2bfloat16_rn(0.25f * s);
  }
}

// dX[fine] = dY[coarse] / 4 (+= when accumulate)
__global__ void k_pool_bwd(const float* __restrict__ dY, int B, int H, int W, int C, float* __restrict__ dX, int acc) {
  const long long n = (long long)B * H * W * C;
  const int w = W / 2, h = H / 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    const float g = 0.25f * dY[(((long long)b * h + y / 2) * w + x / 2) * C + c];
    dX[q] = acc ? dX[q] + g : g;
  }
}

// nearest 2x upsampling of X (B, h, w, C) into channels [cofs, cofs+C) of Y (B, 2h, 2w, ldy)
__global__ void k_up_fwd(const bf16* __restrict__ X, int B, int h, int w, int C, bf16* __restrict__ Y, int ldy, int cofs) {
  const int H = 2 * h, W = 2 * w;
  const long long n = (long long)B * H * W * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    Y[p * ldy + cofs + c] = X[(((long long)b * h + y / 2) * w + x / 2) * C + c];
  }
}

// dX (B, h, w, C) = sum of the 4 children of dY channels [cofs, cofs+C)
__global__ void k_up_bwd(const float* __restrict__ dY, int ldy, int cofs, int B, int h, int w, int C, float* __restrict__ dX) {
  const long long n = (long long)B * h * w * C;
  const int W = 2 * w, H = 2 * h;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % w), y = (int)((p / w) % h), b = (int)(p / ((long long)w * h));
    const long long f = ((long long)b * H + 2 * y) * W + 2 * x;
    dX[q] = dY[f * ldy + cofs + c] + dY[(f + 1) * ldy + cofs + c] + dY[(f + W) * ldy + cofs + c] +
            dY[(f + W + 1) * ldy + cofs + c];
  }
}

// Y[:, cofs:cofs+C] = X  (M pixels)
__global__ void k_copy_ch(const bf16* __restrict__ X, long long M, int C, bf16* __restrict__ Y, int ldy, int cofs) {
  const long long n = M * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    Y[(q / C) * ldy + cofs + q % C] = X[q];
}

// dX (+)= dY[:, cofs:cofs+C]
__global__ void k_take_ch(const float* __restrict__ dY, int ldy, int cofs, long long M, int C, float* __restrict__ dX, int acc) {
  const long long n = M * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float g = dY[(q / C) * ldy + cofs + q % C];
    dX[q] = acc ? dX[q] + g : g;
  }
}

// dZ = dY * [Y > 0] (relu) or dY, as BF16
__global__ void k_act_bwd(const float* __restrict__ dY, const bf16* __restrict__ Y, long long n, int relu, bf16* __restrict__ dZ) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float g = dY[q];
    dZ[q] = __float2bfloat16_rn(relu ? (__bfloat162float(Y[q]) > 0.f ? g : 0.f) : g);
  }
}

// db[c] += sum_m dZ[m][c]
__global__ void k_colsum(const bf16* __restrict__ dZ, long long M, int C, float* __restrict__ db) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (long long m = blockIdx.x; m < M; m += gridDim.x) s += __bfloat162float(dZ[m * C + c]);
  atomicAdd(db + c, s);
}

__global__ void k_f2bf(const float* __restrict__ a, long long n, bf16* __restrict__ b) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    b[q] = __float2bfloat16_rn(a[q]);
}

// masked mean-square error over n values: w = per-value weight (0 excludes), norm = sum of w
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ tgt, const float* __restrict__ w, long long n,
                      float inv_norm, float* __restrict__ dout, float* __restrict__ loss) {
  float s = 0.f;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float d = out[q] - tgt[q];
    const float ww = w[q];
    s += ww * d * d;
    dout[q] = 2.f * ww * d * inv_norm;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_norm);
}

// masked mean-square error plus lam x the squared first differences of the error along x and y
// (a difference counts where both nodes have weight): the residual of a predicted start is a
// differential operator of its error, so the loss also asks for accurate differences.
// One thread per (pixel, channel) of an NHWC [B][H][W][C] tensor.
__global__ void k_mse_grad(const float* __restrict__ out, const float* __restrict__ tgt, const float* __restrict__ w,
                           int B, int H, int W, int C, float lam, float inv_norm, float* __restrict__ dout,
                           float* __restrict__ loss) {
  const long long n = (long long)B * H * W * C;
  float s = 0.f;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const long long p = q / C;
    const int x = (int)(p % W), y = (int)((p / W) % H);
    const float wq = w[q];
    const float e = wq > 0.f ? out[q] - tgt[q] : 0.f;
    float g = 2.f * wq * e;
    s += wq * e * e;
    if (wq > 0.f) {
      const long long qe = q + C, qw = q - C, qn = q + (long long)W * C, qs = q - (long long)W * C;
      if (x + 1 < W && w[qe] > 0.f) { const float d = (out[qe] - tgt[qe]) - e; s += lam * d * d; g -= 2.f * lam * d; }
      if (x > 0 && w[qw] > 0.f) { const float d = e - (out[qw] - tgt[qw]); g += 2.f * lam * d; }
      if (y + 1 < H && w[qn] > 0.f) { const float d = (out[qn] - tgt[qn]) - e; s += lam * d * d; g -= 2.f * lam * d; }
      if (y > 0 && w[qs] > 0.f) { const float d = e - (out[qs] - tgt[qs]); g += 2.f * lam * d; }
    }
    dout[q] = g * inv_norm;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_norm);
}

// 3 x 3 box mean of every channel over the canvas (edges average the neighbours that exist)
__global__ void k_smooth3(const float* __restrict__ X, int B, int H, int W, int C, float* __restrict__ Y) {
  const long long n = (long long)B * H * W * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const long long p = q / C;
    const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((long long)W * H));
    float s = 0.f;
    int k = 0;
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int yy = y + dy, xx = x + dx;
        if (yy < 0 || yy >= H || xx < 0 || xx >= W) continue;
        s += X[(((long long)b * H + yy) * W + xx) * C + c];
        ++k;
      }
    Y[q] = s / (float)k;
  }
}

// Adam on FP32 master parameters, refreshing the BF16 copy used by the GEMMs
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float bc1, float bc2, bf16* __restrict__ pb) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float upd = lr * (mq / bc1) / (sqrtf(vq / bc2) + eps);
    const float pq = p[q] - upd;
    p[q] = pq;
    if (pb) pb[q] = __float2bfloat16_rn(pq);
  }
}

// y = (x - shift[c]) * mul[c] over M pixels of C channels, to BF16 and/or FP32 (in place allowed)
__global__ void k_normalize(const float* X, long long M, int C, const float* __restrict__ shift,
                            const float* __restrict__ mul, bf16* Yb, float* Yf) {
  const long long n = M * C;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % C);
    const float y = (X[q] - shift[c]) * mul[c];
    if (Yb) Yb[q] = __float2bfloat16_rn(y);
    if (Yf) Yf[q] = y;
  }
}

inline int ret(cudaStream_t) { return cudaGetLastError() == cudaSuccess ? 0 : 3; }

}  // namespace
}  // namespace unet

using namespace unet;
#define S_ static_cast<cudaStream_t>(stream)

extern "C" {

int unet_im2col(const void* X, int B, int H, int W, int C, int Kp, void* col, void* stream) {
  if (!X || !col || Kp < 9 * C || (Kp & 7)) return 1;
  if ((C & 7) == 0 && Kp == 9 * C && !(reinterpret_cast<uintptr_t>(X) & 15) && !(reinterpret_cast<uintptr_t>(col) & 15)) {
    k_im2col_v8<<<blocks((long long)B * H * W * 9 * (C >> 3)), T, 0, S_>>>((const uint4*)X, B, H, W, C, (uint4*)col);
    return ret(S_);
  }
  k_im2col<<<blocks((long long)B * H * W * Kp), T, 0, S_>>>((const bf16*)X, B, H, W, C, Kp, (bf16*)col);
  return ret(S_);
}
int unet_col2im(const float* dcol, int B, int H, int W, int C, int Kp, float* dX, void* stream) {
  if (!dcol || !dX) return 1;
  k_col2im<<<blocks((long long)B * H * W * C), T, 0, S_>>>(dcol, B, H, W, C, Kp, dX);
  return ret(S_);
}
int unet_transpose_bf16(const void* src, int rows, int cols, int lds, void* dst, int ldd, void* stream) {
  if (!src || !dst) return 1;
  dim3 g((cols + 31) / 32, (rows + 31) / 32), b(32, 8);
  k_transpose<bf16><<<g, b, 0, S_>>>((const bf16*)src, rows, cols, lds, (bf16*)dst, ldd);
  return ret(S_);
}
int unet_pool_fwd(const void* X, int B, int H, int W, int C, void* Y, void* stream) {
  if (!X || !Y || (H & 1) || (W & 1)) return 1;
  k_pool_fwd<<<blocks((long long)B * H * W * C / 4), T, 0, S_>>>((const bf16*)X, B, H, W, C, (bf16*)Y);
  return ret(S_);
}
int unet_pool_bwd(const float* dY, int B, int H, int W, int C, float* dX, int accumulate, void* stream) {
  if (!dY || !dX || (H & 1) || (W & 1)) return 1;
  k_pool_bwd<<<blocks((long long)B * H * W * C), T, 0, S_>>>(dY, B, H, W, C, dX, accumulate);
  return ret(S_);
}
int unet_up_fwd(const void* X, int B, int h, int w, int C, void* Y, int ldy, int cofs, void* stream) {
  if (!X || !Y || cofs + C > ldy) return 1;
  k_up_fwd<<<blocks((long long)B * 4 * h * w * C), T, 0, S_>>>((const bf16*)X, B, h, w, C, (bf16*)Y, ldy, cofs);
  return ret(S_);
}
int unet_up_bwd(const float* dY, int ldy, int cofs, int B, int h, int w, int C, float* dX, void* stream) {
  if (!dY || !dX || cofs + C > ldy) return 1;
  k_up_bwd<<<blocks((long long)B * h * w * C), T, 0, S_>>>(dY, ldy, cofs, B, h, w, C, dX);
  return ret(S_);
}
int unet_copy_channels(const void* X, long long M, int C, void* Y, int ldy, int cofs, void* stream) {
  if (!X || !Y || cofs + C > ldy) return 1;
  k_copy_ch<<<blocks(M * C), T, 0, S_>>>((const bf16*)X, M, C, (bf16*)Y, ldy, cofs);
  return ret(S_);
}
int unet_take_channels(const float* dY, int ldy, int cofs, long long M, int C, float* dX, int accumulate, void* stream) {
  if (!dY || !dX || cofs + C > ldy) return 1;
  k_take_ch<<<blocks(M * C), T, 0, S_>>>(dY, ldy, cofs, M, C, dX, accumulate);
  return ret(S_);
}
int unet_act_bwd(const float* dY, const void* Y, long long n, int relu, void* dZ, void* stream) {
  if (!dY || !dZ || (relu && !Y)) return 1;
  k_act_bwd<<<blocks(n), T, 0, S_>>>(dY, (const bf16*)Y, n, relu, (bf16*)dZ);
  return ret(S_);
}
int unet_bias_grad(const void* dZ, long long M, int C, float* db, void* stream) {
  if (!dZ || !db) return 1;
  dim3 g((unsigned)(M < 1024 ? M : 1024), (C + 63) / 64);
  k_colsum<<<g, 64, 0, S_>>>((const bf16*)dZ, M, C, db);
  return ret(S_);
}
int unet_f32_to_bf16(const float* a, long long n, void* b, void* stream) {
  if (!a || !b) return 1;
  k_f2bf<<<blocks(n), T, 0, S_>>>(a, n, (bf16*)b);
  return ret(S_);
}
int unet_mse(const float* out, const float* tgt, const float* w, long long n, float inv_norm, float* dout, float* loss,
             void* stream) {
  if (!out || !tgt || !w || !dout || !loss) return 1;
  k_mse<<<blocks(n) < 4096 ? blocks(n) : 4096, T, 0, S_>>>(out, tgt, w, n, inv_norm, dout, loss);
  return ret(S_);
}
int unet_mse_grad(const float* out, const float* tgt, const float* w, int B, int H, int W, int C, float lam,
                  float inv_norm, float* dout, float* loss, void* stream) {
  if (!out || !tgt || !w || !dout || !loss || B <= 0 || H <= 0 || W <= 0 || C <= 0) return 1;
  const long long n = (long long)B * H * W * C;
  k_mse_grad<<<blocks(n) < 4096 ? blocks(n) : 4096, T, 0, S_>>>(out, tgt, w, B, H, W, C, lam, inv_norm, dout, loss);
  return ret(S_);
}
int unet_smooth3(const float* X, int B, int H, int W, int C, float* Y, void* stream) {
  if (!X || !Y || X == Y || B <= 0 || H <= 0 || W <= 0 || C <= 0) return 1;
  k_smooth3<<<blocks((long long)B * H * W * C), T, 0, S_>>>(X, B, H, W, C, Y);
  return ret(S_);
}
int unet_normalize(const float* X, long long M, int C, const float* shift, const float* mul, void* Y_bf16,
                   float* Y_f32, void* stream) {
  if (!X || !shift || !mul || (!Y_bf16 && !Y_f32)) return 1;
  k_normalize<<<blocks(M * C), T, 0, S_>>>(X, M, C, shift, mul, (bf16*)Y_bf16, Y_f32);
  return ret(S_);
}
int unet_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps, int t,
              void* p_bf16, void* stream) {
  if (!p || !g || !m || !v || t < 1) return 1;
  float bc1 = 1.f, bc2 = 1.f;
  for (int i = 0; i < t && i < 100000; ++i) { bc1 *= b1; bc2 *= b2; }
  k_adam<<<blocks(n), T, 0, S_>>>(p, g, m, v, n, lr, b1, b2, eps, 1.f - bc1, 1.f - bc2, (bf16*)p_bf16);
  return ret(S_);
}

}  // extern "C"
