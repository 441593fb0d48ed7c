// corr_i8.cuh — the collision test of one 32-row candidate chunk as an INT8
// tensor-core correlation (tcgen05.mma kind::i8, INT32 accumulators in
// tensor memory).  Included by brkga_decoder.cu, which owns the plate and
// rotation tables and the bit-packed search it is measured against.
//
// What it computes.  For a plate G (L x W cells), a rotated part mask R
// (h x w) and the candidate top rows ty_n = ty_hi - n, n = 0..31, the overlap
// count of every placement in the chunk:
//
//   C[x, n] = sum_{i < h, j < w} R[i, j] * G[ty_n + i, x + j],   0 <= x <= W - w,
//
// and the placement is collision-free iff C == 0 — the reference's test
// (collision_backend.py:109-128: an FFT correlation of the plate with the
// mask, rounded, == 0), evaluated exactly in integers here.
//
// As a GEMM.  With y = ty_n + i the plate row, i = y - ty_hi + n, so
//   C[x, n] = sum_y sum_j A_y[x, j] * B_y[n, j],
//   A_y[x, j] = G[y, x + j]                (im2col of plate row y: M = x, K = j)
//   B_y[n, j] = R[y - ty_hi + n, j]        (mask rows, zero outside 0..h-1)
// summed over the h + 31 plate rows y = ty_hi - 31 .. ty_hi + h - 1 of the
// chunk.  One CTA (128 threads) owns 128 consecutive x (one M = 128 tile) and
// all 32 candidate rows (N = 32); the accumulator is 128 lanes x 32 int32
// columns of tensor memory.
//
// Operand layouts (shared memory, K-major, no swizzle; a core matrix is 8
// rows of 16 bytes).  Both operands put 8-row groups back to back (stride
// byte offset 128 B), so row r of a K chunk sits at 16 r bytes and K chunks
// sit one leading byte offset apart:
// * S, the mask with 32 zero rows above and below: S[k, j] = R[k - 32, j],
//   k < h + 64, chunk c at c * 16 (h + 64) bytes.  B_y is then just rows
//   (y - ty_hi + 32) .. +31 of S: its descriptor starts 16 (y - ty_hi + 32)
//   bytes in, so the mask is staged once and never copied per row.
// * A_y, rebuilt for every plate row (the im2col has no such shift: row x
//   needs the plate bits from x + 16c, a one-byte step): 128 rows x Kp bytes,
//   chunk c at c * 2048 bytes, each 16-byte piece 16 plate bits expanded to
//   0/1 bytes.  Two A buffers: the threads build row y + 1 while the tensor
//   core multiplies row y.
// K per row is w rounded up to 32 (the K of one kind::i8 MMA); S is zero in
// the padded columns, so whatever A holds there adds nothing.
//
// Every wait is bounded (the decoder's tensor-core waits: kSpinLimit polls),
// after which the CTA raises BRKGA_ERR_CUDA, waits once more for its MMAs in
// flight, frees its tensor memory and returns.  No TMA, no multicast.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "umma_core.cuh"

namespace corr {

constexpr int kThreads = 128;   // one thread per candidate column x of the tile
constexpr int kTileM = 128;     // candidate columns per CTA
constexpr int kN = 32;          // candidate top rows: one chunk of the decoder
constexpr int kMaxSide = 256;   // mask rows and columns this path takes
constexpr int kWinWords = 16;   // plate window per row: bits x0 .. x0 + 511
constexpr int kTmemCols = 32;   // accumulator columns (kN int32)

// 0/1 bytes of the 16 bits of v (bit b -> byte b), as one uint4.
__device__ __forceinline__ uint4 expand16(uint32_t v) {
  // n * 0x00204081 puts bit k of a nibble n at bit 8k (the shifted copies
  // n, n << 7, n << 14, n << 21 do not overlap), & 0x01010101 keeps those.
  return make_uint4(((v & 0xFu) * 0x00204081u) & 0x01010101u, (((v >> 4) & 0xFu) * 0x00204081u) & 0x01010101u,
                    (((v >> 8) & 0xFu) * 0x00204081u) & 0x01010101u, (((v >> 12) & 0xFu) * 0x00204081u) & 0x01010101u);
}

// Instruction descriptor, kind::i8: D s32 (2 << 4), A and B u8 (0), both K-major, M x N.
__host__ __device__ constexpr uint32_t instr_desc_u8(int M, int N) {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// Dynamic shared memory of one CTA for a mask of h rows and Kp (w rounded up
// to 32) columns: S, two A buffers, the plate window.
__host__ __device__ constexpr int smem_bytes(int h, int Kp) {
  return Kp * (h + 64) + 2 * kTileM * Kp + (h + kN - 1) * kWinWords * 4;
}

// One chunk test: the plate (L rows of RS words, bit c = column c, zero past
// column W), the rotation's bit-packed rows (mw words per row), the chunk's
// bottom-most candidate top row ty_hi, and the output: 32 rows (candidate
// ty_hi - n) of nwo = ceil((W - w + 1) / 32) words, bit b of word k set when
// the placement at x = 32k + b is collision-free.
struct ChunkArgs {
  const uint32_t* plate;
  int L, W, RS;
  const uint32_t* mask;
  int h, w, mw;
  int ty_hi;
  uint32_t* out;
};

// The CTA's share of one chunk test: candidate columns x0 .. x0 + 127, where
// x0 = 128 * tile.  Called by all 128 threads (contains __syncthreads); the
// caller checked h, w <= kMaxSide, ty_hi <= L - h and that x0 <= W - w.
__device__ __forceinline__ void chunk_tile(const ChunkArgs& a, int tile, unsigned char* smem, uint64_t* bar,
                                           uint32_t* tmem_slot, int* fail, int32_t* status) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int x0 = tile * kTileM;
  const int Kp = (a.w + 31) & ~31, nck = Kp >> 4;
  const int nrows = a.h + kN - 1;  // plate rows ty_hi - 31 .. ty_hi + h - 1
  const uint32_t lbo_s = 16u * (uint32_t)(a.h + 64);
  unsigned char* S = smem;
  unsigned char* Abuf = smem + (size_t)nck * lbo_s;
  uint32_t* win = reinterpret_cast<uint32_t*>(Abuf + 2 * kTileM * Kp);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(umma::smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    *fail = 0;
    for (int b = 0; b < 2; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(umma::smem_u32(&bar[b])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // S: mask row k - 32 (zero outside 0..h-1), 16 columns per piece
  for (int i = tid; i < nck * (a.h + 64); i += kThreads) {
    const int c = i / (a.h + 64), k = i - c * (a.h + 64), r = k - 32, wd = c >> 1;
    uint32_t v = 0u;
    if (r >= 0 && r < a.h && wd < a.mw) v = (a.mask[(size_t)r * a.mw + wd] >> ((c & 1) << 4)) & 0xFFFFu;
    *reinterpret_cast<uint4*>(S + (size_t)c * lbo_s + 16 * k) = expand16(v);
  }
  // the plate window: rows ty_hi - 31 .. ty_hi + h - 1 (zero outside the
  // plate), words x0/32 .. x0/32 + 15 of each (zero past the row's words)
  for (int i = tid; i < nrows * kWinWords; i += kThreads) {
    const int rr = i / kWinWords, q = i - rr * kWinWords;
    const int y = a.ty_hi - (kN - 1) + rr, wd = (x0 >> 5) + q;
    win[i] = (y >= 0 && y < a.L && wd < a.RS) ? a.plate[(size_t)y * a.RS + wd] : 0u;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  constexpr uint32_t idesc = instr_desc_u8(kTileM, kN);
  const uint32_t s0 = umma::smem_u32(S), a0 = umma::smem_u32(Abuf);

  int last = -1;  // last plate row whose MMAs were committed
  for (int rr = 0; rr < nrows; ++rr) {
    const int buf = rr & 1;
    if (rr >= 2) {  // the MMAs of row rr - 2 read this buffer
      if (tid == 0 && !umma::wait_parity(&bar[buf], (uint32_t)(((rr - 2) >> 1) & 1))) *fail = 1;
      __syncthreads();
      if (*fail) break;
    }
    // A_y row x = x0 + tid: plate bits x + 16c .. x + 16c + 15 of the window row
    {
      const uint32_t* wr = win + rr * kWinWords;
      unsigned char* dst = Abuf + (size_t)buf * kTileM * Kp + 16 * tid;
      for (int c = 0; c < nck; ++c) {
        const int p = tid + 16 * c;  // <= 127 + 16 * 15 = 367: words <= 12 of 16
        const uint32_t v = __funnelshift_r(wr[p >> 5], wr[(p >> 5) + 1], p & 31) & 0xFFFFu;
        *reinterpret_cast<uint4*>(dst + (size_t)c * 2048) = expand16(v);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ab = a0 + (uint32_t)(buf * kTileM * Kp);
      const uint32_t bb = s0 + 16u * (uint32_t)(rr + 1);  // S row y - ty_hi + 32 = rr + 1
      for (int s = 0; s < Kp / 32; ++s) {
        const uint64_t ad = umma::smem_desc(ab + 4096u * s, 2048u, 128u);
        const uint64_t bd = umma::smem_desc(bb + 2u * lbo_s * s, lbo_s, 128u);
        mma_u8(tmem, ad, bd, idesc, (rr > 0 || s > 0) ? 1u : 0u);
      }
      umma::commit_to(&bar[buf]);
    }
    last = rr;
  }
  if (!*fail && last >= 0) {  // the commits of one thread complete in order: the last covers all
    if (tid == 0 && !umma::wait_parity(&bar[last & 1], (uint32_t)((last >> 1) & 1))) *fail = 1;
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!*fail) {
    uint32_t v[32];
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
          "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
          "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    const int x = x0 + warp * 32 + lane, nx = a.W - a.w + 1, nwo = (nx + 31) >> 5, k = (x0 >> 5) + warp;
#pragma unroll
    for (int n = 0; n < kN; ++n) {
      const unsigned word = __ballot_sync(0xFFFFFFFFu, v[n] == 0u && x < nx && a.ty_hi - n >= 0);
      if (lane == 0 && k < nwo) a.out[(size_t)n * nwo + k] = word;
    }
  } else if (tid == 0) {
    atomicCAS(status, 0, 3 /* BRKGA_ERR_CUDA */);
    if (last >= 0) umma::wait_parity(&bar[last & 1], (uint32_t)((last >> 1) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

}  // namespace corr
