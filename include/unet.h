/*
 * unet.h -- C ABI of the learned warm start: BF16 U-Net kernels on the B200 tensor cores.
 *
 * No counterpart in the reference (the warm start is new).  All pointers are device pointers;
 * tensors are BF16 (`void*`) or FP32 (`float*`).  Return value 0 = OK, 1 = bad argument,
 * 3 = CUDA error.  `stream` is a cudaStream_t (NULL = legacy default stream).
 */
#ifndef UNET_H
#define UNET_H
#ifdef __cplusplus
extern "C" {
#endif

/* D[m][n] = sum_k A[m][k] B[n][k] on tcgen05 tensor cores (BF16 in, FP32 accumulation).
 * A: M x K row-major (lda >= K), B: N x K row-major (ldb >= K); K, lda, ldb multiples of 8,
 * A and B 16-byte aligned.  epilogue: 0 C = D (FP32), 1 C += D (FP32 atomics, for split-K),
 * 2 Y = bf16(act(D + bias)) with act = ReLU when relu != 0, 3 C = D + bias (FP32); row stride ldc.
 * splits > 1 divides K over blockIdx.z (epilogue 1).  *err (may be NULL) is set to 1 when an
 * internal wait timed out. */
int unet_gemm(const void* A, int lda, const void* B, int ldb, int M, int N, int K, int epilogue,
              float* C, void* Y, int ldc, const float* bias, int relu, int splits, int* err, void* stream);

#ifdef __cplusplus
}
#endif
#endif
