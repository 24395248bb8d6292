// gemm_tc.cuh -- BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05).
//
//   D[m][n] = sum_k A[m][k] * B[n][k]        A: M x K, B: N x K, both row-major (K contiguous)
//
// One CTA (4 warps) computes a 128 x BN tile.  K is walked in slabs of 64: every slab of A and B
// is copied to shared memory with 16-byte cp.async (zero fill outside the matrix) in the
// canonical K-major, no-swizzle UMMA layout -- 8-row x 16-byte core matrices, the 8 K-chunks of
// 16 bytes of a slab stored one after the other, each holding all rows -- so one shared-memory
// descriptor per 16-wide K step addresses it (leading byte offset = distance between the two
// K-chunks of a step, stride byte offset = 128 bytes between 8-row groups).  Thread 0 issues
// tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = BN, K = 16) with the accumulator in tensor
// memory and commits to an mbarrier per stage.  Three stages: the copies of slabs s+1 and s+2
// (cp.async groups) are in flight while the MMAs of slab s run, and a stage is refilled once the
// commit of the MMAs that read it has arrived.  The epilogue reads the accumulator with tcgen05.ld (32 lanes x 32 bit,
// 16 columns per load): warp w owns TMEM lanes 32w..32w+31, i.e. tile rows 32w..32w+31.
//
// Every wait on an mbarrier is bounded; on a timeout the kernel waits (bounded again) for the
// commit of the last MMAs it issued, records the failure in *err, frees its tensor memory and
// returns.  After *err is set the output is not valid and the caller should stop using the GEMM.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace unet {

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;
constexpr int TC_THREADS = 128;
constexpr int TC_STAGES = 3;
constexpr long long TC_WAIT_LIMIT = 1ll << 26;

enum Epilogue {
  EPI_STORE_F32 = 0,   // C[m*ldc+n] = acc
  EPI_ATOMIC_F32 = 1,  // C[m*ldc+n] += acc (split-K partial sums)
  EPI_BIAS_BF16 = 2,   // Y[m*ldc+n] = bf16(act(acc + bias[n])), act = ReLU when relu != 0
  EPI_BIAS_F32 = 3,    // C[m*ldc+n] = acc + bias[n]
};

struct GemmArgs {
  const __nv_bfloat16* A;
  const __nv_bfloat16* B;
  int M, N, K;           // K: multiple of 8 (16-byte rows), lda/ldb in elements
  int lda, ldb;
  float* C;              // EPI_STORE_F32 / EPI_ATOMIC_F32 / EPI_BIAS_F32
  __nv_bfloat16* Y;      // EPI_BIAS_BF16
  int ldc;
  const float* bias;
  int relu;
  int k_tiles_per_split; // split-K: blockIdx.z covers this many 64-wide K slabs
  int* err;              // set to 1 when an mbarrier wait times out
  // implicit 3x3 convolution (k_gemm_tc<..., true>): A is the NHWC activation X [M = batch*H*W
  // pixels][cH channels], row m of the virtual A is col(X)[m][(ky*3+kx)*cC + c] (zero outside the
  // image), K = 9*cC with cC a multiple of 8
  int cH, cW, cC;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (tcgen05): start address, leading/stride byte offsets (all >> 4),
// version 1, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long long it = 0; it < TC_WAIT_LIMIT; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Thread 0 waits (bounded) and the CTA learns the outcome together, so every thread takes the
// same branch afterwards.
__device__ __forceinline__ bool cta_wait(uint32_t bar, uint32_t parity, int* flag) {
  if (threadIdx.x == 0) *flag = mbar_wait(bar, parity) ? 1 : 0;
  __syncthreads();
  const bool ok = *flag != 0;
  __syncthreads();  // every thread has read the flag before thread 0 can write the next one
  return ok;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(n) : "memory");
}

// Copy one 64-wide K slab of `rows` rows starting at (r0, k0) into the UMMA layout at `sbase`.
__device__ __forceinline__ void load_slab(uint32_t sbase, const __nv_bfloat16* G, int ld, int r0, int nrows_total,
                                          int k0, int K, int rows) {
  const int vecs = rows * (TC_BK / 8);
  for (int v = threadIdx.x; v < vecs; v += TC_THREADS) {
    const int r = v >> 3, c = v & 7;
    const int gr = r0 + r, gk = k0 + c * 8;
    const bool ok = gr < nrows_total && gk < K;
    const __nv_bfloat16* src = ok ? G + (long long)gr * ld + gk : G;
    cp_async16(sbase + (uint32_t)(c * rows * 16 + r * 16), src, ok);
  }
}

// A slab of the virtual col(X) matrix: each 16-byte chunk is 8 channels of one tap of one pixel
// (cC is a multiple of 8, so a chunk never straddles two taps), copied straight from X.
__device__ __forceinline__ void load_slab_conv(uint32_t sbase, const GemmArgs& a, int r0, int k0) {
  const int vecs = TC_BM * (TC_BK / 8);
  for (int v = threadIdx.x; v < vecs; v += TC_THREADS) {
    const int r = v >> 3, c = v & 7;
    const int m = r0 + r, k = k0 + c * 8;
    bool ok = m < a.M && k < a.K;
    const __nv_bfloat16* src = a.A;
    if (ok) {
      const int tap = k / a.cC, ch = k - tap * a.cC;
      const int ky = tap / 3, kx = tap - ky * 3;
      const int x = m % a.cW, y = (m / a.cW) % a.cH, b = m / (a.cW * a.cH);
      const int yy = y + ky - 1, xx = x + kx - 1;
      ok = yy >= 0 && yy < a.cH && xx >= 0 && xx < a.cW;
      if (ok) src = a.A + (((long long)b * a.cH + yy) * a.cW + xx) * a.cC + ch;
    }
    cp_async16(sbase + (uint32_t)(c * TC_BM * 16 + r * 16), src, ok);
  }
}

template <int BN, int EPI, bool CONV = false>
__global__ void __launch_bounds__(TC_THREADS) k_gemm_tc(GemmArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  // layout: [TC_STAGES][A: 128 x 64][B: BN x 64] bf16, then one mbarrier per stage, the TMEM
  // address and the wait flag
  constexpr int S = TC_STAGES;
  constexpr int A_BYTES = TC_BM * TC_BK * 2;
  constexpr int B_BYTES = BN * TC_BK * 2;
  constexpr int STAGE = A_BYTES + B_BYTES;
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + S * STAGE);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(smem + S * STAGE + 8 * S);
  int* wait_flag = reinterpret_cast<int*>(smem + S * STAGE + 8 * S + 4);
  const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
  const int kt_total = (a.K + TC_BK - 1) / TC_BK;
  const int kt0 = blockIdx.z * a.k_tiles_per_split;
  const int kt1 = min(kt_total, kt0 + a.k_tiles_per_split);
  const int nk = kt1 > kt0 ? kt1 - kt0 : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int q = 0; q < S; ++q) mbar_init(smem_u32(&bars[q]), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_holder;
  constexpr uint32_t idesc = umma_idesc(TC_BM, BN);
  bool ok = true;
  uint32_t phase = 0u;  // bit q: parity of the next completion of stage q's mbarrier
  int last_commit = -1;  // the last slab whose MMAs thread 0 committed (same value in every thread)

  // slab t of this split goes to stage t % S; cp.async group g holds slab g
  auto load_tile = [&](int t) {
    const uint32_t sa = smem_u32(smem + (t % S) * STAGE), sb = sa + A_BYTES;
    if (CONV) load_slab_conv(sa, a, m0, (kt0 + t) * TC_BK);
    else load_slab(sa, a.A, a.lda, m0, a.M, (kt0 + t) * TC_BK, a.K, TC_BM);
    load_slab(sb, a.B, a.ldb, n0, a.N, (kt0 + t) * TC_BK, a.K, BN);
  };
  for (int t = 0; t < S - 1; ++t) {
    if (t < nk) load_tile(t);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int i = 0; i < nk; ++i) {
    const int st = i % S;
    const uint32_t sa = smem_u32(smem + st * STAGE), sb = sa + A_BYTES;
    // slabs 0..i have landed (at most S-2 newer groups are still in flight)
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int ks = 0; ks < TC_BK / 16; ++ks) {
        const uint64_t da = umma_desc(sa + ks * 2 * TC_BM * 16, TC_BM * 16, 128);
        const uint64_t db = umma_desc(sb + ks * 2 * BN * 16, BN * 16, 128);
        const uint32_t acc = (i > 0 || ks > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   ::"r"(smem_u32(&bars[st])) : "memory");
    }
    last_commit = i;
    // refill: slab i+S-1 goes to the stage the MMAs of slab i-1 read
    const int j = i + S - 1;
    if (j < nk) {
      if (i >= 1) {
        const int sp = (i - 1) % S;
        ok = cta_wait(smem_u32(&bars[sp]), (phase >> sp) & 1u, wait_flag);
        phase ^= 1u << sp;
        if (!ok) break;
      }
      load_tile(j);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  // the commits of the last min(nk, S) slabs have not been waited for yet (one per stage)
  for (int t = nk > S ? nk - S : 0; ok && t < nk; ++t) {
    const int sp = t % S;
    ok = cta_wait(smem_u32(&bars[sp]), (phase >> sp) & 1u, wait_flag);
    phase ^= 1u << sp;
  }
  if (!ok && last_commit >= 0) {
    // A wait timed out while MMAs may still run.  A tcgen05.commit arrives once every MMA this
    // thread issued before it has completed, so one more bounded wait on the last commit (slab L
    // is the (L / S)-th use of stage L % S) drains them all before the tensor memory is freed.
    // If this wait times out too, nothing more can be done here: the error word tells the caller
    // that the output, and the state of this context, are no longer reliable.
    const int L = last_commit;
    cta_wait(smem_u32(&bars[L % S]), (uint32_t)((L / S) & 1), wait_flag);
  }
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (!ok) {
    if (threadIdx.x == 0 && a.err) atomicExch(a.err, 1);
  } else if (nk > 0) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int nb = n0 + c0;
      const long long o0 = (long long)row * a.ldc + nb;
      if (EPI == EPI_BIAS_BF16 && row < a.M && nb + 16 <= a.N && (a.ldc & 7) == 0 &&
          !(reinterpret_cast<uintptr_t>(a.Y) & 15)) {
        // 16 consecutive columns of one row: two 16-byte stores
        uint32_t pk[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          float v0 = __uint_as_float(r[j]) + (a.bias ? a.bias[nb + j] : 0.f);
          float v1 = __uint_as_float(r[j + 1]) + (a.bias ? a.bias[nb + j + 1] : 0.f);
          if (a.relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
          const __nv_bfloat162 h = __floats2bfloat162_rn(v0, v1);
          pk[j >> 1] = *reinterpret_cast<const uint32_t*>(&h);
        }
        uint4* dst = reinterpret_cast<uint4*>(a.Y + o0);
        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
      } else if ((EPI == EPI_STORE_F32 || EPI == EPI_BIAS_F32) && row < a.M && nb + 16 <= a.N &&
                 (a.ldc & 3) == 0 && !(reinterpret_cast<uintptr_t>(a.C) & 15)) {
        float4* dst = reinterpret_cast<float4*>(a.C + o0);
#pragma unroll
        for (int j = 0; j < 16; j += 4) {
          float4 v = make_float4(__uint_as_float(r[j]), __uint_as_float(r[j + 1]), __uint_as_float(r[j + 2]),
                                 __uint_as_float(r[j + 3]));
          if (EPI == EPI_BIAS_F32 && a.bias) {
            v.x += a.bias[nb + j]; v.y += a.bias[nb + j + 1]; v.z += a.bias[nb + j + 2]; v.w += a.bias[nb + j + 3];
          }
          dst[j >> 2] = v;
        }
      } else if (row < a.M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c0 + j;
          if (n >= a.N) break;
          float v = __uint_as_float(r[j]);
          const long long o = (long long)row * a.ldc + n;
          if (EPI == EPI_STORE_F32) a.C[o] = v;
          else if (EPI == EPI_ATOMIC_F32) atomicAdd(a.C + o, v);
          else if (EPI == EPI_BIAS_F32) a.C[o] = v + (a.bias ? a.bias[n] : 0.f);
          else {
            v += a.bias ? a.bias[n] : 0.f;
            if (a.relu) v = fmaxf(v, 0.f);
            a.Y[o] = __float2bfloat16_rn(v);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

}  // namespace unet
