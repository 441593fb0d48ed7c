// umma_gemm.cuh — bf16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   C[M, N] (fp32, row-major, ldc) = sum_k A[m, k] * B[n, k]
//   A: bf16 [M, K] K-major (row-major, lda), B: bf16 [N, K] K-major (ldb).
//   M % 128 == 0, N % BN == 0 (BN = 64 or 128), K % 64 == 0 (callers pad with zeros).
//
// One CTA of 128 threads per 128 x BN output tile.  Per 64-wide K step one
// thread loads the A and B tiles with TMA (cp.async.bulk.tensor, tensor maps
// built on the host, 128-byte swizzle: rows of 64 bf16, the layout the MMA's
// K-major SWIZZLE_128B descriptor reads) into a ring of stages in dynamic
// shared memory, counted on one mbarrier per stage; a second thread issues
// four K = 16 tcgen05.mma.cta_group::1.kind::f16 per step with the fp32
// accumulator in tensor memory (BN columns) and frees the stage with
// tcgen05.commit.  All copies of a small GEMM are in flight at once; the
// tensor core never waits for a CTA-wide barrier.  The epilogue reads the
// accumulator with tcgen05.ld.32x32b (warp w owns lanes 32w..32w+31 = output
// rows).
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
// returns, after waiting (bounded) for the copies it issued.  No multicast.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "umma_core.cuh"

namespace umma {

constexpr int kTileM = 128;
constexpr int kTileK = 64;

// Shared-memory matrix descriptor, K-major with the 128-byte swizzle that
// the TMA copies write: rows of 128 bytes (64 bf16), 8-row groups 1024 bytes
// apart (stride byte offset); the leading byte offset is unused for this
// layout.  A K = 16 slice of the row starts 32 bytes further.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;              // leading byte offset (16 B, ignored)
  d |= (uint64_t)(1024u >> 4) << 32;   // stride byte offset
  d |= (uint64_t)1 << 46;              // descriptor version for sm_100
  d |= (uint64_t)2 << 61;              // layout: 128-byte swizzle
  return d;
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

// Stages of A and B tiles in shared memory (24 KB per stage at BN = 64,
// 32 KB at BN = 128): enough that the copies of every K step of the
// surrogate's GEMMs (K <= 640) are in flight at once.
template <int BN>
__host__ __device__ constexpr int gemm_stages() {
  return BN == 128 ? 5 : 6;
}

// Dynamic shared memory of gemm_bf16_kernel<BN>: the stages plus 1 KB to
// align them on the swizzle's 1024-byte period.
template <int BN>
__host__ __device__ constexpr int gemm_smem_bytes() {
  return gemm_stages<BN>() * (kTileM * kTileK + BN * kTileK) * 2 + 1024;
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the kernel before it in the stream is still
// running; pdl_wait() blocks until that kernel has completed and its memory
// is visible, so it comes before the first global access of any kernel
// launched that way.  pdl_trigger() lets the next such kernel start
// launching (its CTAs then wait in their own pdl_wait).  Both are no-ops for
// a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// One arrival that also announces `bytes` of asynchronous copies to come.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// TMA tile load (no multicast): box at (x = K element, y = row) of the
// tensor map into shared memory, completion counted on `bar`.  x is a
// multiple of 64 elements (128 bytes), so every copy starts 16-byte aligned.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
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

// Pipeline (warp-specialised, one CTA of 128 threads per 128 x BN tile):
//   thread 0   (producer) loads the A and B tiles of each 64-wide K step with
//              two TMA copies (cp.async.bulk.tensor.2d, 128-byte swizzle)
//              into stage kt % kSt; the stage's "full" mbarrier counts the
//              bytes (expect_tx), and a stage is refilled only after its
//              "empty" mbarrier reports that the MMAs reading it are done;
//   thread 32  (MMA issuer) waits for "full", issues the step's four K = 16
//              tcgen05.mma and commits them to the stage's "empty" barrier;
//              after the last step one more commit signals "acc";
//   all warps  wait for "acc" and run the epilogue from tensor memory.
// No multicast; every wait is bounded (the error path is in the kernel).
template <int BN>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __grid_constant__ CUtensorMap tmA,
                                                        const __grid_constant__ CUtensorMap tmB,
                                                        const __grid_constant__ Epilogue ep, int K, int* err) {
  static_assert(BN == 64 || BN == 128, "BN must be 64 or 128");
  constexpr int kSt = gemm_stages<BN>();
  constexpr int kCols = BN;  // tensor-memory columns (power of two >= 32)
  constexpr uint32_t kABytes = kTileM * kTileK * 2, kBBytes = BN * kTileK * 2, kStageBytes = kABytes + kBBytes;
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[kSt];
  __shared__ __align__(8) uint64_t empty[kSt];
  __shared__ __align__(8) uint64_t accb;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail, s_issued, s_consumed;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * BN;
  // the 128-byte swizzle repeats every 1024 bytes: stages start on that boundary
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 32) {
    s_fail = 0;
    s_issued = 0;
    s_consumed = 0;
    for (int b = 0; b < kSt; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], 1);
    }
    mbar_init(&accb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid == 64) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = instr_desc_bf16(kTileM, BN);
  const int ksteps = K / kTileK;
  // the set-up above touched no global memory: from here on the operands of
  // the kernel before this one must be complete
  pdl_wait();
  pdl_trigger();

  if (tid == 0) {  // producer
    int kt = 0;
    for (; kt < ksteps; ++kt) {
      const int b = kt % kSt;
      if (kt >= kSt && !wait_parity(&empty[b], (uint32_t)((kt / kSt - 1) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      if (*(volatile int*)&s_fail) break;
      const uint32_t a_dst = base + (uint32_t)b * kStageBytes;
      mbar_expect_tx(&full[b], kStageBytes);
      tma_load_2d(a_dst, &tmA, kt * kTileK, m0, &full[b]);
      tma_load_2d(a_dst + kABytes, &tmB, kt * kTileK, n0, &full[b]);
    }
    s_issued = kt;
  } else if (tid == 32) {  // MMA issuer
    int kt = 0;
    for (; kt < ksteps; ++kt) {
      const int b = kt % kSt;
      if (!wait_parity(&full[b], (uint32_t)((kt / kSt) & 1))) {
        atomicExch(&s_fail, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = base + (uint32_t)b * kStageBytes, b0 = a0 + kABytes;
#pragma unroll
      for (int s = 0; s < kTileK / 16; ++s)  // K = 16 is 32 bytes along the swizzled 128-byte row
        mma_bf16(tmem, smem_desc_sw128(a0 + 32u * s), smem_desc_sw128(b0 + 32u * s), idesc,
                 (kt > 0 || s > 0) ? 1u : 0u);
      commit_to(&empty[b]);
    }
    s_consumed = kt;
    commit_to(&accb);  // tracks every MMA this thread issued, whether the loop finished or not
  }
  __syncwarp();
  const bool acc_ok = wait_parity(&accb, 0u);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!acc_ok && lane == 0) atomicExch(&s_fail, 1);
  __syncthreads();

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
    // no copy may land after the CTA is gone: wait (bounded) for every stage
    // the producer issued and the MMA thread did not consume
    for (int kt = s_consumed; kt < s_issued; ++kt) wait_parity(&full[kt % kSt], (uint32_t)((kt / kSt) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
  }
}

}  // namespace umma
