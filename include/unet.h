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

/* 3x3 "same" convolution as an implicit GEMM (no col matrix in memory): D = col(X) Wt^T with
 * X NHWC BF16 [B*H*W][C] (C a multiple of 8), col as for unet_im2col with Kp = 9C, Wt [Cout][ldw]
 * BF16 (ldw >= 9C, multiple of 8).  epilogue 0 (C = D, FP32), 2 (Y = bf16(act(D + bias))) or
 * 3 (C = D + bias, FP32), row stride ldc.  Same results as unet_im2col + unet_gemm. */
int unet_conv3x3(const void* X, int B, int H, int W, int C, const void* Wt, int ldw, int Cout, int epilogue,
                 float* Cf, void* Y, int ldc, const float* bias, int relu, int* err, void* stream);

/* Layer kernels.  Activations are NHWC ([pixels][channels], pixels ordered batch, row, column).
 * A 3x3 "same" convolution is the GEMM col(X) W^T with col(X)[m][(ky*3+kx)*C + c] =
 * X[b][y+ky-1][x+kx-1][c] (zero outside the canvas and for k >= 9C; Kp = padded K, multiple of 8). */
int unet_im2col(const void* X, int B, int H, int W, int C, int Kp, void* col, void* stream);
/* dX[b][y][x][c] = sum over taps of dcol at the output pixels that read X[b][y][x][c] (FP32) */
int unet_col2im(const float* dcol, int B, int H, int W, int C, int Kp, float* dX, void* stream);
/* dst[c][r] = src[r][c] (BF16), r < rows, c < cols, row strides lds / ldd */
int unet_transpose_bf16(const void* src, int rows, int cols, int lds, void* dst, int ldd, void* stream);
/* 2x2 average pooling (H, W even), and its gradient (accumulate != 0 adds into dX) */
int unet_pool_fwd(const void* X, int B, int H, int W, int C, void* Y, void* stream);
int unet_pool_bwd(const float* dY, int B, int H, int W, int C, float* dX, int accumulate, void* stream);
/* nearest 2x upsampling of X (B,h,w,C) into channels [cofs, cofs+C) of Y (B,2h,2w, row stride ldy),
 * and its gradient (sum of the 4 children) */
int unet_up_fwd(const void* X, int B, int h, int w, int C, void* Y, int ldy, int cofs, void* stream);
int unet_up_bwd(const float* dY, int ldy, int cofs, int B, int h, int w, int C, float* dX, void* stream);
/* channel-slice copies for the skip concatenations: Y[:, cofs:cofs+C] = X, dX (+)= dY[:, cofs:cofs+C] */
int unet_copy_channels(const void* X, long long M, int C, void* Y, int ldy, int cofs, void* stream);
int unet_take_channels(const float* dY, int ldy, int cofs, long long M, int C, float* dX, int accumulate,
                       void* stream);
/* dZ = bf16(relu ? dY * [Y > 0] : dY) over n values */
int unet_act_bwd(const float* dY, const void* Y, long long n, int relu, void* dZ, void* stream);
/* db[c] += sum_m dZ[m][c] (db must be zeroed by the caller) */
int unet_bias_grad(const void* dZ, long long M, int C, float* db, void* stream);
int unet_f32_to_bf16(const float* a, long long n, void* b, void* stream);
/* *loss += sum w (out - tgt)^2 * inv_norm, dout = 2 w (out - tgt) inv_norm (loss zeroed by the caller) */
int unet_mse(const float* out, const float* tgt, const float* w, long long n, float inv_norm, float* dout,
             float* loss, void* stream);
/* as unet_mse on an NHWC [B][H][W][C] tensor, plus lam x the squared differences of the error
 * between x- and y-neighbours that both have weight (loss and gradient) */
int unet_mse_grad(const float* out, const float* tgt, const float* w, int B, int H, int W, int C, float lam,
                  float inv_norm, float* dout, float* loss, void* stream);
/* Y = 3 x 3 box mean of X per channel (NHWC FP32; edges average the existing neighbours; Y != X) */
int unet_smooth3(const float* X, int B, int H, int W, int C, float* Y, void* stream);
/* y = (x - shift[c]) * mul[c] over M pixels x C channels (FP32 in) to Y_bf16 and/or Y_f32 (either may be
 * NULL, not both; Y_f32 may alias X) */
int unet_normalize(const float* X, long long M, int C, const float* shift, const float* mul, void* Y_bf16,
                   float* Y_f32, void* stream);
/* Adam step t (>= 1) on FP32 master parameters p; p_bf16 (may be NULL) receives bf16(p) */
int unet_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
              int t, void* p_bf16, void* stream);

#ifdef __cplusplus
}
#endif
#endif
