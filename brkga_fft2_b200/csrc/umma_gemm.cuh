// umma_gemm.cuh — bf16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[M, N] (fp32, row-major, ldc) = sum_k A[m, k] * B[n, k]
//   A: bf16 [M, K] K-major (row-major, lda), B: bf16 [N, K] K-major (ldb).
//   M % 128 == 0, N % BN == 0 (BN = 64 or 128), K % 64 == 0 (callers pad with zeros).
//
// One CTA of 128 threads per 128 x BN output tile.  Per 64-wide K step the
// threads copy the A and B tiles with cp.async (six buffers in dynamic shared
// memory: four steps of copies in flight, two of MMAs) in the canonical K-major
// "interleaved" layout (8 x 16-byte core matrices; core (row block, k chunk)
// at (row_block * kChunks + k_chunk) * 128 bytes, so the descriptor's leading
// byte offset — next k chunk — is 128 B and its stride byte offset — next
// 8-row block — is 128 x kChunks B, 1024 B for the 64-wide K tile), one elected thread issues four K=16
// tcgen05.mma.cta_group::1.kind::f16 with the fp32 accumulator in tensor
// memory (BN columns), and tcgen05.commit signals an mbarrier the CTA waits on.
// The epilogue reads the accumulator with tcgen05.ld.32x32b (warp w owns
// lanes 32w..32w+31 = output rows) and stores fp32.
//
// The epilogue (Epilogue below) either stores the fp32 tile, or applies the
// surrogate's elementwise step in registers before anything leaves the SM:
// bias + ReLU, or the ReLU derivative of a forward activation, then any of
// an fp32 store, a bf16 row-major copy, a bf16 transposed copy (the lanes of
// a warp own consecutive rows, so those stores coalesce) and one partial dot
// product per row with a weight vector (the 256 -> 1 output layer; each CTA
// writes the partial of its BN columns, summed later in a fixed order).
//
// Every wait is bounded: after kSpinLimit polls the kernel records
// BRKGA_ERR_CUDA in *err, skips its epilogue, frees its tensor memory and
// returns.  No TMA and no multicast are used.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace umma {

constexpr int kTileM = 128;
constexpr int kTileK = 64;
constexpr int kChunks = kTileK / 8;  // 16-byte chunks of K per row in one stage
constexpr long long kSpinLimit = 20000000;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, SWIZZLE_NONE, K-major.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor: D fp32, A and B bf16, both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void commit_to(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait; false after kSpinLimit polls
__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (try_wait(bar, parity)) return true;
  return false;
}

constexpr int kStages = 6;  // shared-memory buffers
constexpr int kAhead = 4;   // K steps of copies in flight; the MMAs of kStages - kAhead steps may still run

// Dynamic shared memory of gemm_bf16_kernel<BN>: kStages stages of A and B tiles.
template <int BN>
constexpr int gemm_smem_bytes() {
  return kStages * (kTileM * kTileK + BN * kTileK) * 2;
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// What the epilogue does with an output tile (see the file comment).
//   kind kStore:     C[row, col] = acc                                  (fp32)
//   kind kBiasRelu:  v = max(acc + bias[col], 0)
//   kind kReluMask:  v = ref[row, col] > 0 ? acc : 0   (ref: the forward activation)
// then, where the pointer is set: C[row, col] = v, out[row, col] = bf16(v),
// outT[col, row] = bf16(v), part[tile_n, row] = sum over the tile's columns of v * dotw[col].
enum EpiKind { kStore = 0, kBiasRelu = 1, kReluMask = 2 };
struct Epilogue {
  int kind = kStore;
  float* C = nullptr;
  int ldc = 0;
  const float* bias = nullptr;
  const float* ref = nullptr;
  int ld_ref = 0;
  __nv_bfloat16* out = nullptr;
  int ld_out = 0;
  __nv_bfloat16* outT = nullptr;
  int ld_outT = 0;
  const float* dotw = nullptr;
  float* part = nullptr;
  int ld_part = 0;
};

// Pipeline: the threads keep kAhead K steps of tiles in flight as
// asynchronous copies (cp.async, straight into shared memory) while one
// thread issues the MMAs of the oldest complete step; a buffer is refilled
// only after the MMAs that read it (kStages - kAhead steps earlier) have
// signalled their mbarrier, so the MMAs of the last steps keep running.
template <int BN>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __nv_bfloat16* __restrict__ A, int lda,
                                                        const __nv_bfloat16* __restrict__ B, int ldb,
                                                        const __grid_constant__ Epilogue ep, int K, int* err) {
  static_assert(BN == 64 || BN == 128, "BN must be 64 or 128");
  constexpr int kCols = BN;                    // tensor-memory columns (power of two >= 32)
  constexpr int kAWords = kTileM * kTileK / 8;  // uint4 per A stage
  constexpr int kBWords = BN * kTileK / 8;
  extern __shared__ __align__(1024) uint4 smem_tiles[];
  __shared__ __align__(8) uint64_t bar[kStages];
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * BN;
  // stage b: A tile at b * (kAWords + kBWords), B tile right after it
  auto tileA = [&](int b) { return smem_tiles + b * (kAWords + kBWords); };
  auto tileB = [&](int b) { return smem_tiles + b * (kAWords + kBWords) + kAWords; };

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    s_fail = 0;
    for (int b = 0; b < kStages; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar[b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = instr_desc_bf16(kTileM, BN);

  // copy a 128 x kTileK A tile and a BN x kTileK B tile of step kt into stage
  // buf: chunk (r, c) of 8 bf16 -> core ((r/8)*kChunks + c), row r%8.  Eight
  // consecutive lanes fill the 8 rows of one core matrix (128 contiguous
  // bytes: no bank conflict), the next eight the next chunk of the same rows,
  // so a warp reads 64 contiguous bytes of each of 8 rows (whole sectors).
  auto stage = [&](int buf, int kt) {
#pragma unroll
    for (int j = 0; j < kTileM * kChunks / 128; ++j) {
      const int i = tid + 128 * j, ri = i & 7, c = (i >> 3) % kChunks, r = ((i >> 3) / kChunks) * 8 + ri;
      cp_async16(tileA(buf) + ((r >> 3) * kChunks + c) * 8 + ri, A + (size_t)(m0 + r) * lda + kt * kTileK + c * 8);
    }
#pragma unroll
    for (int j = 0; j < BN * kChunks / 128; ++j) {
      const int i = tid + 128 * j, ri = i & 7, c = (i >> 3) % kChunks, r = ((i >> 3) / kChunks) * 8 + ri;
      cp_async16(tileB(buf) + ((r >> 3) * kChunks + c) * 8 + ri, B + (size_t)(n0 + r) * ldb + kt * kTileK + c * 8);
    }
  };

  const int ksteps = K / kTileK;
#pragma unroll
  for (int p = 0; p < kAhead; ++p) {
    if (p < ksteps) stage(p, p);
    cp_async_commit();  // one group per step, empty ones included, so the group count stays uniform
  }
  int last = -1;  // last k step whose MMAs were committed
  for (int kt = 0; kt < ksteps; ++kt) {
    const int buf = kt % kStages;
    cp_async_wait<kAhead - 1>();  // this thread's copies of step kt have landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(tileA(buf)), b0 = smem_u32(tileB(buf));
#pragma unroll
      for (int s = 0; s < kTileK / 16; ++s) {
        // K = 16 is two 8-wide chunks: chunk 2s at +256*s bytes, the next one +128 B (LBO)
        const uint64_t ad = smem_desc(a0 + 256u * s, 128u, 128u * kChunks);
        const uint64_t bd = smem_desc(b0 + 256u * s, 128u, 128u * kChunks);
        mma_bf16(tmem, ad, bd, idesc, (kt > 0 || s > 0) ? 1u : 0u);
      }
      commit_to(&bar[buf]);
    }
    last = kt;
    const int nk = kt + kAhead;  // the step to prefetch, into the buffer of step kt - (kStages - kAhead)
    constexpr int kLag = kStages - kAhead;
    if (nk < ksteps) {
      if (kt >= kLag) {
        const int pb = (kt - kLag) % kStages;
        if (!wait_parity(&bar[pb], (uint32_t)(((kt - kLag) / kStages) & 1))) {
          if (lane == 0) atomicExch(&s_fail, 1);
        }
        __syncthreads();
        if (s_fail) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      }
      stage(nk % kStages, nk);
    }
    cp_async_commit();
  }
  // the MMAs of one thread complete in order: the last commit covers them all
  if (!s_fail && last >= 0) {
    if (!wait_parity(&bar[last % kStages], (uint32_t)((last / kStages) & 1))) {
      if (lane == 0) atomicExch(&s_fail, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
  }

  if (!s_fail) {
    const int row = m0 + warp * 32 + lane;
    float dot = 0.f;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 32) {
      uint32_t v[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
            "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
            "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int col0 = n0 + c0;
      float x[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) x[j] = __uint_as_float(v[j]);
      if (ep.kind == kBiasRelu) {
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = fmaxf(x[j] + ep.bias[col0 + j], 0.f);
      } else if (ep.kind == kReluMask) {
        const float4* r4 = reinterpret_cast<const float4*>(ep.ref + (size_t)row * ep.ld_ref + col0);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float4 r = r4[q];
          if (!(r.x > 0.f)) x[4 * q] = 0.f;
          if (!(r.y > 0.f)) x[4 * q + 1] = 0.f;
          if (!(r.z > 0.f)) x[4 * q + 2] = 0.f;
          if (!(r.w > 0.f)) x[4 * q + 3] = 0.f;
        }
      }
      if (ep.C) {
        float4* dst = reinterpret_cast<float4*>(ep.C + (size_t)row * ep.ldc + col0);
#pragma unroll
        for (int q = 0; q < 8; ++q) dst[q] = make_float4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
      }
      if (ep.out) {
        uint4* dst = reinterpret_cast<uint4*>(ep.out + (size_t)row * ep.ld_out + col0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint32_t w[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const __nv_bfloat162 pr = __floats2bfloat162_rn(x[8 * q + 2 * e], x[8 * q + 2 * e + 1]);
            w[e] = *reinterpret_cast<const uint32_t*>(&pr);
          }
          dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
        }
      }
      if (ep.outT) {
#pragma unroll
        for (int j = 0; j < 32; ++j) ep.outT[(size_t)(col0 + j) * ep.ld_outT + row] = __float2bfloat16(x[j]);
      }
      if (ep.dotw) {
#pragma unroll
        for (int j = 0; j < 32; ++j) dot += x[j] * ep.dotw[col0 + j];
      }
    }
    if (ep.dotw) ep.part[(size_t)blockIdx.y * ep.ld_part + row] = dot;
  } else if (tid == 0) {
    atomicExch(err, 3 /* BRKGA_ERR_CUDA */);
    // let the MMAs still in flight finish before the tensor memory is released
    if (last >= 0) wait_parity(&bar[last % kStages], (uint32_t)((last / kStages) & 1));
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // no copy may land after the CTA is gone
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

}  // namespace umma
