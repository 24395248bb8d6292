// unet_gemm.cu -- host launcher of the tcgen05 GEMM (gemm_tc.cuh) behind the C ABI in unet.h.
#include <cuda_runtime.h>

#include "../../../include/unet.h"
#include "gemm_tc.cuh"

namespace unet {
namespace {

template <int BN, int EPI, bool CONV = false>
cudaError_t go(const GemmArgs& a, int splits, cudaStream_t s) {
  constexpr int smem = TC_STAGES * (TC_BM * TC_BK * 2 + BN * TC_BK * 2) + 64;
  auto k = k_gemm_tc<BN, EPI, CONV>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.M + TC_BM - 1) / TC_BM, (a.N + BN - 1) / BN, splits);
  k<<<grid, TC_THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

template <int EPI, bool CONV = false>
cudaError_t by_bn(const GemmArgs& a, int bn, int splits, cudaStream_t s) {
  switch (bn) {
    case 16: return go<16, EPI, CONV>(a, splits, s);
    case 32: return go<32, EPI, CONV>(a, splits, s);
    case 64: return go<64, EPI, CONV>(a, splits, s);
    case 128: return go<128, EPI, CONV>(a, splits, s);
    default: return go<256, EPI, CONV>(a, splits, s);
  }
}

}  // namespace
}  // namespace unet

extern "C" int unet_gemm(const void* A, int lda, const void* B, int ldb, int M, int N, int K, int epilogue,
                         float* C, void* Y, int ldc, const float* bias, int relu, int splits, int* err,
                         void* stream) {
  using namespace unet;
  if (!A || !B || M <= 0 || N <= 0 || K <= 0 || (K & 7) || (lda & 7) || (ldb & 7) || lda < K || ldb < K)
    return 1;
  if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15)) return 1;
  if (epilogue < 0 || epilogue > 3 || splits < 1) return 1;
  if ((epilogue == EPI_BIAS_BF16 && !Y) || (epilogue != EPI_BIAS_BF16 && !C)) return 1;
  int bn = 16;
  while (bn < N && bn < 256) bn *= 2;
  const int kt = (K + TC_BK - 1) / TC_BK;
  if (splits > kt) splits = kt;
  GemmArgs a;
  a.A = static_cast<const __nv_bfloat16*>(A);
  a.B = static_cast<const __nv_bfloat16*>(B);
  a.M = M; a.N = N; a.K = K; a.lda = lda; a.ldb = ldb;
  a.C = C; a.Y = static_cast<__nv_bfloat16*>(Y); a.ldc = ldc; a.bias = bias; a.relu = relu;
  a.k_tiles_per_split = (kt + splits - 1) / splits;
  a.cH = a.cW = a.cC = 0;
  splits = (kt + a.k_tiles_per_split - 1) / a.k_tiles_per_split;
  a.err = err;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  switch (epilogue) {
    case EPI_STORE_F32: e = by_bn<EPI_STORE_F32>(a, bn, splits, s); break;
    case EPI_ATOMIC_F32: e = by_bn<EPI_ATOMIC_F32>(a, bn, splits, s); break;
    case EPI_BIAS_BF16: e = by_bn<EPI_BIAS_BF16>(a, bn, splits, s); break;
    default: e = by_bn<EPI_BIAS_F32>(a, bn, splits, s); break;
  }
  return e == cudaSuccess ? 0 : 3;
}

extern "C" int unet_conv3x3(const void* X, int B, int H, int W, int C, const void* Wt, int ldw, int Cout, int epilogue,
                            float* Cf, void* Y, int ldc, const float* bias, int relu, int* err, void* stream) {
  using namespace unet;
  if (!X || !Wt || B <= 0 || H <= 0 || W <= 0 || C <= 0 || (C & 7) || Cout <= 0 || (ldw & 7) || ldw < 9 * C)
    return 1;
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(Wt) & 15)) return 1;
  if (epilogue != EPI_STORE_F32 && epilogue != EPI_BIAS_BF16 && epilogue != EPI_BIAS_F32) return 1;
  if ((epilogue == EPI_BIAS_BF16 && !Y) || (epilogue != EPI_BIAS_BF16 && !Cf)) return 1;
  const long long M = (long long)B * H * W;
  if (M > 0x7fffffffLL) return 1;
  int bn = 16;
  while (bn < Cout && bn < 256) bn *= 2;
  GemmArgs a;
  a.A = static_cast<const __nv_bfloat16*>(X);
  a.B = static_cast<const __nv_bfloat16*>(Wt);
  a.M = (int)M; a.N = Cout; a.K = 9 * C; a.lda = C; a.ldb = ldw;
  a.C = Cf; a.Y = static_cast<__nv_bfloat16*>(Y); a.ldc = ldc; a.bias = bias; a.relu = relu;
  a.k_tiles_per_split = (a.K + TC_BK - 1) / TC_BK;
  a.err = err;
  a.cH = H; a.cW = W; a.cC = C;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  switch (epilogue) {
    case EPI_STORE_F32: e = by_bn<EPI_STORE_F32, true>(a, bn, 1, s); break;
    case EPI_BIAS_BF16: e = by_bn<EPI_BIAS_BF16, true>(a, bn, 1, s); break;
    default: e = by_bn<EPI_BIAS_F32, true>(a, bn, 1, s); break;
  }
  return e == cudaSuccess ? 0 : 3;
}
