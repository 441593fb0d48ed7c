// brkga_surrogate.cu — online-trained MLP that ranks chromosomes by predicted
// makespan (C ABI in include/brkga_b200.h).  No counterpart in the reference:
// its GA decodes every offspring exactly (BRKGA_alg3.py:119-123).
//
// Network: features (3 per part in decode order + 2 per machine, padded to a
// multiple of 64) -> 512 -> 256 -> 1, ReLU; bf16 weights and activations on
// the tensor cores (umma_gemm.cuh, tcgen05) with fp32 accumulation, fp32
// master weights and Adam state.  Every matrix product of the forward and
// backward pass is one tcgen05 GEMM:
//   Z1  = X   W1^T      dW2 = dZ2^T H1      dH1 = dZ2 W2      dW1 = dZ1^T X
//   Z2  = H1  W2^T
// (transposed bf16 copies of X, H1, dZ2, dZ1 and W2 are written by the
// elementwise kernels so that every operand is K-major).  The last layer,
// biases, the loss and Adam run on the CUDA cores.
//
// Features of a chromosome: parts sorted as the decoder visits them (by
// machine, then sequencing key, placement.py:118-135); for part slot p:
// machine / (M-1), proc_time / max proc_time, proc_time_height / max
// proc_time_height; then per machine: assigned area / plate area and
// assigned proc_time / max.  Targets: makespan standardised with the mean and
// standard deviation of the first observed batch; infeasible chromosomes
// (1e16) are not learned from.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/brkga_b200.h"
#include "umma_gemm.cuh"

// access to the decoder's device tables (brkga_decoder.cu)
extern "C" int brkga_internal_problem_tables(const BrkgaProblem* pb, int* N, int* M, int* T, int* mode,
                                             const double** thr, const int32_t** gene_type, const double** part_area,
                                             const double** pt, const double** pth, const double** bin_area);

namespace {

constexpr int kH1 = 512;
constexpr int kH2 = 256;
constexpr int kMaxGenes = 8192;
constexpr int kMaxTrainBatch = 16384;  // rows of one gradient step (sizes the backward pass's row-block partials)

struct U4 {
  uint32_t x, y, z, w;
};

__device__ inline uint32_t mulhi32(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

// Philox4x32-10 (Salmon et al., SC'11), as in brkga_ga.cu
__device__ inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = mulhi32(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = mulhi32(0xCD9E8D57u, c.z);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  return c;
}

__device__ inline float unit_float(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

__device__ inline unsigned ordered_bits(float v) {
  unsigned u = __float_as_uint(v);
  if (v == 0.0f) u = 0u;
  if (v != v) u = 0x7FC00000u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ inline int machine_of(float mv, const double* thr, int M, int mode) {
  if (M <= 1) return 0;
  if (mv != mv) return M;
  int m = 0;
  if (mode == BRKGA_THRESH_F32) {
    while (m < M - 1 && !(mv <= (float)thr[m])) ++m;
  } else {
    while (m < M - 1 && !((double)mv <= thr[m])) ++m;
  }
  return m;
}

struct FeatParams {
  const float* chrom;
  int P, N, M, T, mode, in_pad;
  int kind;               // BRKGA_SURROGATE_FEATURES_DECODE or _ORDER
  float inv_area;         // 1 / largest part area (order features)
  const double* thr;
  const int32_t* gene_type;
  const double* part_area;
  const double* pt;
  const double* pth;
  const double* bin_area;
  float inv_pt, inv_pth;  // 1 / max proc time, 1 / max height time
  __nv_bfloat16* X;       // [rows, in_pad]
  int row_offset;
};

// One CTA per chromosome: sort (machine, key, gene) like the decoder, write the
// feature row.  Per-machine sums run in decode order, so features are deterministic.
// Order features (kind BRKGA_SURROGATE_FEATURES_ORDER): the parts sorted by
// sequencing key alone, machine keys ignored, and per part its key, its area
// over the largest part area and its height time on machine 0 over the largest.
__global__ void features_kernel(FeatParams p) {
  umma::pdl_wait();
  umma::pdl_trigger();
  extern __shared__ unsigned long long keys[];
  __shared__ float s_area[256], s_pt[256];
  __shared__ int s_cnt[257], s_start[257];
  const int c = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  int S2 = 1;
  while (S2 < p.N) S2 <<= 1;
  const float* ch = p.chrom + (size_t)c * 2 * p.N;
  for (int m = tid; m <= p.M; m += nt) s_cnt[m] = 0;
  __syncthreads();
  for (int i = tid; i < S2; i += nt) {
    unsigned long long key = ~0ull;
    if (i < p.N) {
      const int m = p.kind == BRKGA_SURROGATE_FEATURES_ORDER ? 0 : machine_of(ch[p.N + i], p.thr, p.M, p.mode);
      key = ((unsigned long long)m << 48) | ((unsigned long long)ordered_bits(ch[i]) << 16) | (unsigned long long)i;
      atomicAdd(&s_cnt[m], 1);
    }
    keys[i] = key;
  }
  __syncthreads();
  for (int k = 2; k <= S2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S2; i += nt) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = keys[i], b = keys[ixj];
          if ((a > b) == ((i & k) == 0)) {
            keys[i] = b;
            keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  if (tid == 0) {
    int acc = 0;
    for (int m = 0; m < p.M; ++m) {
      s_start[m] = acc;
      acc += s_cnt[m];
    }
  }
  // Each part's share of its machine's loads, all parts at once (the table
  // reads overlap); the per-machine sums below then add them in decode order
  // from shared memory.
  float* c_area = reinterpret_cast<float*>(keys + S2);  // [N]
  float* c_load = c_area + p.N;                         // [N]
  if (p.kind != BRKGA_SURROGATE_FEATURES_ORDER) {
    for (int q = tid; q < p.N; q += nt) {
      const unsigned long long key = keys[q];
      const int m = (int)(key >> 48);
      float av = 0.f, lv = 0.f;
      if (m < p.M) {
        const int t = p.gene_type[(int)(key & 0xFFFFu)];
        av = (float)(p.part_area[t] / p.bin_area[m]);
        lv = (float)p.pt[(size_t)m * p.T + t] * p.inv_pt;
      }
      c_area[q] = av;
      c_load[q] = lv;
    }
  }
  __syncthreads();
  for (int m = tid; m < p.M && p.kind != BRKGA_SURROGATE_FEATURES_ORDER; m += nt) {
    float area = 0.f, load = 0.f;
    for (int q = s_start[m]; q < s_start[m] + s_cnt[m]; ++q) {
      area += c_area[q];
      load += c_load[q];
    }
    s_area[m] = area;
    s_pt[m] = load;
  }
  __syncthreads();
  __nv_bfloat16* row = p.X + (size_t)(p.row_offset + c) * p.in_pad;
  if (p.kind == BRKGA_SURROGATE_FEATURES_ORDER) {
    for (int i = tid; i < p.in_pad; i += nt) {
      float v = 0.f;
      if (i < 3 * p.N) {
        const int g = (int)(keys[i / 3] & 0xFFFFu), f = i % 3;
        const int t = p.gene_type[g];
        v = f == 0 ? ch[g] : f == 1 ? (float)p.part_area[t] * p.inv_area : (float)p.pth[t] * p.inv_pth;
      }
      row[i] = __float2bfloat16(v);
    }
    return;
  }
  const float mscale = p.M > 1 ? 1.f / (float)(p.M - 1) : 0.f;
  for (int i = tid; i < p.in_pad; i += nt) {
    float v = 0.f;
    if (i < 3 * p.N) {
      const unsigned long long key = keys[i / 3];
      const int m = (int)(key >> 48);
      if (m < p.M) {
        const int t = p.gene_type[(int)(key & 0xFFFFu)];
        const int f = i % 3;
        v = f == 0 ? (float)m * mscale
                   : f == 1 ? (float)p.pt[(size_t)m * p.T + t] * p.inv_pt : (float)p.pth[(size_t)m * p.T + t] * p.inv_pth;
      }
    } else if (i < 3 * p.N + 2 * p.M) {
      const int q = i - 3 * p.N;
      v = (q & 1) ? s_pt[q >> 1] : s_area[q >> 1];
    }
    row[i] = __float2bfloat16(v);
  }
}

// The same features with one warp per chromosome, for N <= 32 E parts and at
// most 32 machines: the warp sorts the (machine, key, gene) keys in
// registers (E per lane, bitonic network, partners in other lanes exchanged
// by shuffles; no CTA barrier), then works from its own slice of shared
// memory.  Same keys, same order of the per-machine sums, same values as
// features_kernel: the rows are identical.
constexpr int kFeatWarps = 8;  // warps (chromosomes) per CTA
__host__ __device__ constexpr size_t feat_warp_bytes(int E) {
  return (size_t)32 * E * 8 + (size_t)32 * E * 12 + 4 * 33 * 4;  // keys, shares + types, per-machine arrays
}
template <int E>
__global__ void __launch_bounds__(32 * kFeatWarps) features_warp_kernel(FeatParams p) {
  umma::pdl_wait();
  umma::pdl_trigger();
  extern __shared__ __align__(16) unsigned char fsm[];
  constexpr int S2 = 32 * E;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * kFeatWarps + warp;
  if (c >= p.P) return;
  unsigned char* base = fsm + (size_t)warp * feat_warp_bytes(E);
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(base);
  float* c_area = reinterpret_cast<float*>(keys + S2);
  float* c_load = c_area + S2;
  int* c_type = reinterpret_cast<int*>(c_load + S2);
  int* m_start = c_type + S2;  // [33]
  float* m_area = reinterpret_cast<float*>(m_start + 33);
  float* m_load = m_area + 33;
  const float* ch = p.chrom + (size_t)c * 2 * p.N;
  const bool order = p.kind == BRKGA_SURROGATE_FEATURES_ORDER;
  unsigned long long k[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = lane * E + e;
    k[e] = ~0ull;
    if (i < p.N) {
      const int m = order ? 0 : machine_of(ch[p.N + i], p.thr, p.M, p.mode);
      k[e] = ((unsigned long long)m << 48) | ((unsigned long long)ordered_bits(ch[i]) << 16) | (unsigned long long)i;
    }
  }
  // bitonic sort of S2 keys, element i = lane * E + e
#pragma unroll 1
  for (int kk = 2; kk <= S2; kk <<= 1) {
#pragma unroll 1
    for (int j = kk >> 1; j > 0; j >>= 1) {
      if (j >= E) {  // partner in lane ^ (j / E), same register
        const int dl = j / E;
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int i = lane * E + e;
          const unsigned long long o = __shfl_xor_sync(0xFFFFFFFFu, k[e], dl);
          const bool asc = (i & kk) == 0, lower = (i & j) == 0;
          k[e] = (asc == lower) ? (k[e] < o ? k[e] : o) : (k[e] > o ? k[e] : o);
        }
      } else {  // partner in the same lane
#pragma unroll
        for (int e = 0; e < E; ++e) {
#pragma unroll
          for (int jj = 1; jj < E; jj <<= 1) {
            if (jj == j && (e & jj) == 0) {
              const int i = lane * E + e;
              const bool asc = (i & kk) == 0;
              const unsigned long long a = k[e], b = k[e | jj];
              if ((a > b) == asc) {
                k[e] = b;
                k[e | jj] = a;
              }
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) keys[lane * E + e] = k[e];
  __syncwarp();
  // first sorted position of each machine 0..M (the keys are ordered by machine)
  for (int m = lane; m <= p.M && m <= 32; m += 32) {
    int lo = 0, hi = S2;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((int)(keys[mid] >> 48) < m) lo = mid + 1;
      else hi = mid;
    }
    m_start[m] = lo;
  }
  for (int q = lane; q < p.N; q += 32) {
    const unsigned long long key = keys[q];
    const int m = (int)(key >> 48);
    float av = 0.f, lv = 0.f;
    int t = -1;
    if (m < p.M) {
      t = p.gene_type[(int)(key & 0xFFFFu)];
      if (!order) {
        av = (float)(p.part_area[t] / p.bin_area[m]);
        lv = (float)p.pt[(size_t)m * p.T + t] * p.inv_pt;
      }
    }
    c_area[q] = av;
    c_load[q] = lv;
    c_type[q] = t;
  }
  __syncwarp();
  if (!order && lane < p.M) {  // per machine, in decode order
    float area = 0.f, load = 0.f;
    for (int q = m_start[lane]; q < m_start[lane + 1]; ++q) {
      area += c_area[q];
      load += c_load[q];
    }
    m_area[lane] = area;
    m_load[lane] = load;
  }
  __syncwarp();
  __nv_bfloat16* row = p.X + (size_t)(p.row_offset + c) * p.in_pad;
  if (order) {
    for (int i = lane; i < p.in_pad; i += 32) {
      float v = 0.f;
      if (i < 3 * p.N) {
        const int q = i / 3, f = i - 3 * q, g = (int)(keys[q] & 0xFFFFu), t = c_type[q];
        v = f == 0 ? ch[g] : f == 1 ? (float)p.part_area[t] * p.inv_area : (float)p.pth[t] * p.inv_pth;
      }
      row[i] = __float2bfloat16(v);
    }
    return;
  }
  const float mscale = p.M > 1 ? 1.f / (float)(p.M - 1) : 0.f;
  for (int i = lane; i < p.in_pad; i += 32) {
    float v = 0.f;
    if (i < 3 * p.N) {
      const int q = i / 3, f = i - 3 * q;
      const int m = (int)(keys[q] >> 48);
      if (m < p.M) {
        const int t = c_type[q];
        v = f == 0 ? (float)m * mscale
                   : f == 1 ? (float)p.pt[(size_t)m * p.T + t] * p.inv_pt : (float)p.pth[(size_t)m * p.T + t] * p.inv_pth;
      }
    } else if (i < 3 * p.N + 2 * p.M) {
      const int q = i - 3 * p.N;
      v = (q & 1) ? m_load[q >> 1] : m_area[q >> 1];
    }
    row[i] = __float2bfloat16(v);
  }
}

// Launch with programmatic stream serialisation: the kernel may begin while
// the one before it in the stream finishes; it waits for that kernel's
// results in pdl_wait() (see umma_gemm.cuh).  In a captured graph the
// dependency becomes a programmatic edge.  A failed launch is reported by
// the next cudaGetLastError().
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// out[h] = sum_b A[b, h] * (scale ? scale[b] : 1) * (mask ? (mask[b, h] > 0) : 1) * (colscale ? colscale[h] : 1)
// 32 columns per CTA (threadIdx.x, coalesced rows), the rows split over
// kColRows thread rows and summed in shared memory in a fixed order, so the
// result does not depend on scheduling.
constexpr int kColRows = 16;
__global__ void __launch_bounds__(32 * kColRows) col_reduce_kernel(const float* A, const float* scale,
                                                                   const float* mask, const float* colscale, int B,
                                                                   int H, float* out) {
  umma::pdl_wait();
  umma::pdl_trigger();
  __shared__ float part[kColRows][33];
  const int h = blockIdx.x * 32 + threadIdx.x;
  float s = 0.f;
  if (h < H) {
    for (int b = threadIdx.y; b < B; b += kColRows) {
      const size_t i = (size_t)b * H + h;
      float v = A ? A[i] : 1.f;
      if (scale) v *= scale[b];
      if (mask && !(mask[i] > 0.f)) v = 0.f;
      s += v;
    }
  }
  part[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && h < H) {
    float t = 0.f;
#pragma unroll
    for (int y = 0; y < kColRows; ++y) t += part[y][threadIdx.x];
    out[h] = colscale ? t * colscale[h] : t;
  }
}

void col_reduce(const float* A, const float* scale, const float* mask, const float* colscale, int B, int H,
                float* out, cudaStream_t st) {
  launch_pdl(col_reduce_kernel, (H + 31) / 32, dim3(32, kColRows), 0, st, A, scale, mask, colscale, B, H, out);
}

// The output layer's backward pass and the loss, from the partial dot
// products the Z2 GEMM's epilogue left per column tile, on tiles of 32 rows x
// 32 columns (grid kH2 / 32 x B / 32, all independent): y = sum of the
// partials + b3; e = y - t and dy = 2 e / n on the n valid rows (MSE), 0 on
// padding; dZ2 = (Z2 > 0) dy w3 as bf16, row-major and — through a
// shared-memory tile, so the stores coalesce — transposed.  Each tile leaves
// its column sums of Z2 dy (for gw3) and dZ2 (for gb2) over its 32 rows, and
// the tiles of the first column block the row sums of dy (for gb3) and e^2
// (the loss); out_grads() adds those row blocks in a fixed order.  Tile (0, 0)
// also advances the minibatch and Adam step counters when `bump`.
__global__ void __launch_bounds__(256) out_backward_kernel(
    const float* part, int n_tiles, int ld_part, const float* b3, const float* t, const int* n_valid, const float* Z2,
    const float* w3, int B, float* y, __nv_bfloat16* dZ, __nv_bfloat16* dZT, float* pw3, float* pb2, float* pb3,
    float* ploss, long long* step, long long* adam_t, int bump) {
  umma::pdl_wait();
  umma::pdl_trigger();
  __shared__ float s_dy[32], s_e[32];
  __shared__ __nv_bfloat16 s_t[32][34];  // [column][row], padded
  __shared__ float s_w[8][33], s_b[8][33];
  const int tx = threadIdx.x, ty = threadIdx.y, h = blockIdx.x * 32 + tx, r0 = blockIdx.y * 32;
  const int n = *n_valid;
  if (ty == 0) {
    const int b = r0 + tx;
    float v = b3[0];
    for (int q = 0; q < n_tiles; ++q) v += part[(size_t)q * ld_part + b];
    const float e = b < n ? v - t[b] : 0.f;
    s_e[tx] = e;
    s_dy[tx] = 2.f * e / (float)n;
    if (blockIdx.x == 0) y[b] = v;
  }
  __syncthreads();
  const float wh = w3[h];
  float aw = 0.f, ab = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int rr = ty + 8 * k, b = r0 + rr;
    const float z = Z2[(size_t)b * kH2 + h], d = s_dy[rr];
    const float g = z > 0.f ? d * wh : 0.f;
    const __nv_bfloat16 q = __float2bfloat16(g);
    dZ[(size_t)b * kH2 + h] = q;
    s_t[tx][rr] = q;
    aw += z * d;
    ab += g;
  }
  s_w[ty][tx] = aw;
  s_b[ty][tx] = ab;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = ty + 8 * k;
    dZT[(size_t)(blockIdx.x * 32 + c) * B + r0 + tx] = s_t[c][tx];
  }
  if (ty == 0) {
    float sw = 0.f, sb = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      sw += s_w[j][tx];
      sb += s_b[j][tx];
    }
    pw3[(size_t)blockIdx.y * kH2 + h] = sw;
    pb2[(size_t)blockIdx.y * kH2 + h] = sb;
    if (blockIdx.x == 0 && tx == 0) {
      float sd = 0.f, l = 0.f;
      for (int j = 0; j < 32; ++j) {
        sd += s_dy[j];
        l += s_e[j] * s_e[j];
      }
      pb3[blockIdx.y] = sd;
      ploss[blockIdx.y] = l;
      if (bump && blockIdx.y == 0) {
        *step += 1;
        *adam_t += 1;
      }
    }
  }
}

// Where the output layer's row-block partials live and how many there are.
struct OutPartials {
  const float *w3, *b2, *b3, *loss;  // [nrb * kH2], [nrb * kH2], [nrb], [nrb]
  int nrb;
  const int* n_valid;
  float* loss_out;
};

// Gradient of parameter i of the flat vector if it belongs to the output
// layer's w3, b2 or b3 (row blocks added in order; b3 also writes the loss),
// else g.  off_b2: first index of b2 (w3 and b3 follow it).
__device__ __forceinline__ float out_grad(int i, float g, int off_b2, const OutPartials& op) {
  if (i < off_b2) return g;
  const int j = i - off_b2;
  if (j < 2 * kH2) {  // b2 then w3
    const float* src = j < kH2 ? op.b2 : op.w3;
    const int h = j < kH2 ? j : j - kH2;
    float acc = 0.f;
    for (int r = 0; r < op.nrb; ++r) acc += src[(size_t)r * kH2 + h];
    return acc;
  }
  float acc = 0.f, l = 0.f;  // b3
  for (int r = 0; r < op.nrb; ++r) {
    acc += op.b3[r];
    l += op.loss[r];
  }
  *op.loss_out = l / (float)*op.n_valid;
  return acc;
}

// The output layer's gradients and the loss into the flat gradient vector
// (the gradients entry point, which runs no Adam).
__global__ void out_grads_kernel(float* grads, int off_b2, OutPartials op) {
  umma::pdl_wait();
  umma::pdl_trigger();
  for (int j = threadIdx.x; j < 2 * kH2 + 1; j += blockDim.x) grads[off_b2 + j] = out_grad(off_b2 + j, 0.f, off_b2, op);
}

// Predictions: y = sum of the output layer's partials + b3, in makespan units
// once the target scaling is set.
__global__ void predict_out_kernel(const float* part, int n_tiles, int ld_part, const float* b3, int P,
                                   const double* norm, float* y, double* out) {
  umma::pdl_wait();
  umma::pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P) return;
  float v = b3[0];
  for (int q = 0; q < n_tiles; ++q) v += part[(size_t)q * ld_part + i];
  y[i] = v;
  out[i] = norm[2] != 0.0 ? (double)v * norm[1] + norm[0] : (double)v;
}

// Adam (Kingma & Ba) on every parameter, then the bf16 copies the GEMMs read
// (W1; W2 row-major and transposed) from the updated values; the step count
// t is read from device memory so graph replays stay correct.
// With `op` set (the training loop), the output layer's gradients are added
// up from the backward kernel's row-block partials here, and written to g too.
__global__ void adam_cast_kernel(float* w, float* g, float* m, float* v, int n, float lr, float b1, float b2,
                                 float eps, const long long* t_ptr, int nW1, int offW2, int nW2, __nv_bfloat16* W1b,
                                 __nv_bfloat16* W2b, __nv_bfloat16* W2Tb, int off_b2, OutPartials op) {
  umma::pdl_wait();
  umma::pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = (float)(*t_ptr);
  const float bc1 = 1.f - powf(b1, t), bc2 = 1.f - powf(b2, t);
  float gi = g[i];
  if (op.nrb > 0 && i >= off_b2) {
    gi = out_grad(i, gi, off_b2, op);
    g[i] = gi;
  }
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  w[i] = wi;
  if (i < nW1) {
    W1b[i] = __float2bfloat16(wi);
  } else if (i >= offW2 && i < offW2 + nW2) {
    const int j = i - offW2, r = j / kH1, c = j - r * kH1;
    const __nv_bfloat16 q = __float2bfloat16(wi);
    W2b[j] = q;
    W2Tb[(size_t)c * kH2 + r] = q;
  }
}

__global__ void cast_kernel(const float* W, int rows, int cols, __nv_bfloat16* out, __nv_bfloat16* outT) {
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i - (long long)r * cols);
    const __nv_bfloat16 q = __float2bfloat16(W[i]);
    if (out) out[i] = q;
    if (outT) outT[(size_t)c * rows + r] = q;
  }
}

// uniform(-a, a) with a = sqrt(6 / fan_in) (He-uniform), Philox stream `tag`
__global__ void init_weights_kernel(float* W, int n, int fan_in, int valid_cols, int cols, uint32_t k0, uint32_t k1,
                                    uint32_t tag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const U4 r = philox(U4{(uint32_t)i, 0u, 0u, 0x5300u + tag}, k0, k1);
  const float a = sqrtf(6.f / (float)fan_in);
  W[i] = (cols > 0 && (i % cols) >= valid_cols) ? 0.f : (2.f * unit_float(r.x) - 1.f) * a;
}

struct ObsParams {
  const double* makespan;
  int P;
  const __nv_bfloat16* Xsrc;  // [P, in_pad] features of the observed rows
  int in_pad;
  __nv_bfloat16* bufX;        // [cap, in_pad]
  float* bufY;                // [cap]
  int cap;
  double* norm;               // [mu, sigma, set]
};

// Standardisation from the first observed batch (feasible rows only).
__global__ void set_norm_kernel(const double* ms, int P, double* norm) {
  umma::pdl_wait();
  umma::pdl_trigger();
  if (norm[2] != 0.0) return;
  __shared__ double s1[256], s2[256], sn[256];
  const int tid = threadIdx.x;
  double a = 0, b = 0, n = 0;
  for (int i = tid; i < P; i += blockDim.x) {
    const double v = ms[i];
    if (v < 1e15 && v == v) {
      a += v;
      b += v * v;
      n += 1;
    }
  }
  s1[tid] = a;
  s2[tid] = b;
  sn[tid] = n;
  __syncthreads();
  for (int h = blockDim.x >> 1; h; h >>= 1) {
    if (tid < h) {
      s1[tid] += s1[tid + h];
      s2[tid] += s2[tid + h];
      sn[tid] += sn[tid + h];
    }
    __syncthreads();
  }
  if (tid == 0 && sn[0] >= 2) {
    const double mu = s1[0] / sn[0];
    const double var = fmax(s2[0] / sn[0] - mu * mu, 1e-12 * mu * mu + 1e-12);
    norm[0] = mu;
    norm[1] = sqrt(var);
    norm[2] = 1.0;
  }
}

// Ring-buffer slots of the feasible rows, in row order: one CTA of 1024
// threads takes 1024 rows per pass and numbers the feasible ones by a prefix
// count (ballots within a warp, then a scan of the 32 warp totals), so the
// slots are those of a walk over the rows in order.
constexpr int kObsThreads = 1024;
__global__ void __launch_bounds__(kObsThreads) observe_slots_kernel(const double* ms, int P, const double* norm,
                                                                    long long* count, int cap, int* slot) {
  umma::pdl_wait();
  umma::pdl_trigger();
  __shared__ int warp_sum[kObsThreads / 32];
  __shared__ long long base;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) base = *count;
  const bool ready = norm[2] != 0.0;
  __syncthreads();
  for (int r0 = 0; r0 < P; r0 += kObsThreads) {
    const int r = r0 + tid;
    bool ok = false;
    if (r < P) {
      const double v = ms[r];
      ok = ready && v < 1e15 && v == v;
    }
    const unsigned bal = __ballot_sync(0xFFFFFFFFu, ok);
    if (lane == 0) warp_sum[wid] = __popc(bal);
    __syncthreads();
    if (wid == 0) {  // inclusive scan of the warp totals
      int v = warp_sum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= o) v += u;
      }
      warp_sum[lane] = v;
    }
    __syncthreads();
    const long long idx = base + (wid ? warp_sum[wid - 1] : 0) + __popc(bal & ((1u << lane) - 1u));
    if (r < P) slot[r] = ok ? (int)(idx % cap) : -1;
    __syncthreads();
    if (tid == 0) base += warp_sum[kObsThreads / 32 - 1];
    __syncthreads();
  }
  if (tid == 0) *count = base;
}

// Append feasible rows (features + standardised target) to their slots.
__global__ void observe_kernel(ObsParams p, const int* slot) {
  umma::pdl_wait();
  umma::pdl_trigger();
  const int r = blockIdx.x;
  if (r >= p.P) return;
  const int sl = slot[r];
  if (sl < 0) return;
  for (int i = threadIdx.x; i < p.in_pad; i += blockDim.x)
    p.bufX[(size_t)sl * p.in_pad + i] = p.Xsrc[(size_t)r * p.in_pad + i];
  if (threadIdx.x == 0) p.bufY[sl] = (float)((p.makespan[r] - p.norm[0]) / p.norm[1]);
}

// Minibatch: uniform rows of the filled part of the ring buffer.
__global__ void gather_kernel(const __nv_bfloat16* bufX, const float* bufY, const long long* count, int cap, int B,
                              int n_valid_max, int in_pad, uint32_t k0, uint32_t k1, const long long* step,
                              __nv_bfloat16* X, __nv_bfloat16* XT, float* y, int* n_valid) {
  umma::pdl_wait();
  umma::pdl_trigger();
  const int b = blockIdx.x;
  const long long filled = min((long long)cap, *count);
  const int nv = (int)min((long long)n_valid_max, filled);
  if (b == 0 && threadIdx.x == 0) *n_valid = nv;
  const bool real = b < nv && filled > 0;
  int src = 0;
  if (real) {
    const U4 r = philox(U4{(uint32_t)b, (uint32_t)(*step), 0x6A7u, 0u}, k0, k1);
    src = (int)mulhi32(r.x, (uint32_t)filled);
  }
  for (int i = threadIdx.x; i < in_pad; i += blockDim.x) {
    const __nv_bfloat16 q = real ? bufX[(size_t)src * in_pad + i] : __float2bfloat16(0.f);
    X[(size_t)b * in_pad + i] = q;
    XT[(size_t)i * B + b] = q;
  }
  if (threadIdx.x == 0) y[b] = real ? bufY[src] : 0.f;
}

__global__ void bump_kernel(long long* step) { *step += 1; }

__global__ void set_int_kernel(int* p, int v) { *p = v; }

__global__ void transpose_bf16_kernel(const __nv_bfloat16* X, int B, int I, __nv_bfloat16* XT) {
  const long long n = (long long)B * I;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / I), c = (int)(i - (long long)b * I);
    XT[(size_t)c * B + b] = X[i];
  }
}

int grid_for(long long n, int block = 256) {
  long long g = (n + block - 1) / block;
  return (int)std::max(1LL, std::min(g, 148LL * 32));
}

int round_up(int v, int a) { return (v + a - 1) / a * a; }

}  // namespace

struct BrkgaSurrogate {
  const BrkgaProblem* problem = nullptr;
  int N = 0, M = 0, T = 0, mode = 0;
  int in = 0, in_pad = 0, max_batch = 0, cap = 0;
  uint64_t seed = 0;
  float inv_pt = 1.f, inv_pth = 1.f;
  const double* thr = nullptr;
  const int32_t* gene_type = nullptr;
  const double* part_area = nullptr;
  const double* pt = nullptr;
  const double* pth = nullptr;
  const double* bin_area = nullptr;
  std::vector<void*> allocs;
  // parameters (fp32 master), gradients, Adam moments: one flat block each
  float *W1, *b1, *W2, *b2, *w3, *b3;
  float *gW1, *gb1, *gW2, *gb2, *gw3, *gb3;
  float *mom, *vel, *params, *grads;
  long long n_params = 0;
  __nv_bfloat16 *W1b, *W2b, *W2Tb;
  // activations for up to max_batch rows
  __nv_bfloat16 *X, *XT, *H1b, *H1Tb, *dZ2b, *dZ2Tb, *dZ1Tb;
  float *Z1, *Z2, *y, *t, *dH1, *loss;
  float* part;  // [4, max_batch]: the output layer's partial dot per Z2 column tile
  int last_nrb = 0;  // row blocks of the last backward pass
  float* outp;  // row-block partials of the output layer's gradients: w3, b2 [nrb, kH2], b3, loss [nrb]
  int features_kind = BRKGA_SURROGATE_FEATURES_DECODE;
  float inv_area = 1.f;
  int* n_valid;
  int* slot;
  int* err;
  long long *count, *step, *adam_t;
  double* norm;
  __nv_bfloat16* bufX;
  float* bufY;
};

namespace {

template <typename T>
int dalloc(BrkgaSurrogate* s, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return BRKGA_ERR_CUDA;
  s->allocs.push_back(q);
  if (cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) return BRKGA_ERR_CUDA;
  *p = static_cast<T*>(q);
  return BRKGA_OK;
}

// The GEMM's two-stage tiles exceed the default 48 KB of shared memory: opt
// in once per device (at surrogate creation or the first brkga_gemm_bf16,
// so never inside a stream capture).
int prepare_gemm() {
  static int ready[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BRKGA_ERR_CUDA;
  if (ready[dev]) return BRKGA_OK;
  if (cudaFuncSetAttribute(umma::gemm_bf16_kernel<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           umma::gemm_smem_bytes<128>()) != cudaSuccess ||
      cudaFuncSetAttribute(umma::gemm_bf16_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           umma::gemm_smem_bytes<64>()) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  ready[dev] = 1;
  return BRKGA_OK;
}

// 128 x 128 tiles when they alone fill the GPU twice over, else 128 x 64
// (these GEMMs are small: more CTAs matter more than tile reuse).
int tile_n(int M, int N) { return (N % 128 == 0 && (long long)(M / 128) * (N / 128) >= 2 * 148) ? 128 : 64; }

// cuTensorMapEncodeTiled from the driver, looked up once per process through
// the runtime (no link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

// Tensor map of a bf16 [rows, K] K-major operand with row stride ld
// elements: boxes of 64 K elements (128 bytes) x box_rows rows, 128-byte
// swizzle.  The base must be 16-byte aligned and ld a multiple of 8.
int tile_map(CUtensorMap* map, const __nv_bfloat16* ptr, int rows, int K, int ld, int box_rows) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return BRKGA_ERR_CUDA;
  if (reinterpret_cast<uintptr_t>(ptr) % 16 || ld % 8) return BRKGA_ERR_INVALID_ARGUMENT;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)umma::kTileK, (cuuint32_t)box_rows};
  const cuuint32_t elem[2] = {1, 1};
  const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims, strides,
                         box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? BRKGA_OK : BRKGA_ERR_INVALID_ARGUMENT;
}

int gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, const umma::Epilogue& ep, int M, int N,
         int K, int* err, cudaStream_t st) {
  if (M % 128 || K % 64 || N % 64) return BRKGA_ERR_INVALID_ARGUMENT;
  const int bn = tile_n(M, N);
  CUtensorMap ta, tb;
  int r;
  if ((r = tile_map(&ta, A, M, K, lda, umma::kTileM)) || (r = tile_map(&tb, B, N, K, ldb, bn))) return r;
  if (bn == 128) {
    launch_pdl(umma::gemm_bf16_kernel<128>, dim3(M / 128, N / 128), 128, umma::gemm_smem_bytes<128>(), st, ta, tb,
               ep, K, err);
  } else {
    launch_pdl(umma::gemm_bf16_kernel<64>, dim3(M / 128, N / 64), 128, umma::gemm_smem_bytes<64>(), st, ta, tb, ep,
               K, err);
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

umma::Epilogue store_to(float* C, int ldc) {
  umma::Epilogue e;
  e.kind = umma::kStore;
  e.C = C;
  e.ldc = ldc;
  return e;
}

// Dynamic shared memory of features_kernel: the sort keys, then each part's
// area and time shares of its machine.
size_t features_smem(int S2, int N) { return (size_t)S2 * 8 + (size_t)N * 8; }

int features(BrkgaSurrogate* s, const float* d_chrom, int P, __nv_bfloat16* X, cudaStream_t st) {
  FeatParams fp;
  fp.chrom = d_chrom;
  fp.P = P;
  fp.N = s->N;
  fp.M = s->M;
  fp.T = s->T;
  fp.mode = s->mode;
  fp.in_pad = s->in_pad;
  fp.thr = s->thr;
  fp.gene_type = s->gene_type;
  fp.part_area = s->part_area;
  fp.pt = s->pt;
  fp.pth = s->pth;
  fp.bin_area = s->bin_area;
  fp.inv_pt = s->inv_pt;
  fp.inv_pth = s->inv_pth;
  fp.kind = s->features_kind;
  fp.inv_area = s->inv_area;
  fp.X = X;
  fp.row_offset = 0;
  int S2 = 1;
  while (S2 < s->N) S2 <<= 1;
  if (s->M <= 32 && S2 <= 256) {  // one warp per chromosome
    const dim3 grid((P + kFeatWarps - 1) / kFeatWarps), block(32 * kFeatWarps);
    if (S2 <= 32) launch_pdl(features_warp_kernel<1>, grid, block, kFeatWarps * feat_warp_bytes(1), st, fp);
    else if (S2 <= 64) launch_pdl(features_warp_kernel<2>, grid, block, kFeatWarps * feat_warp_bytes(2), st, fp);
    else if (S2 <= 128) launch_pdl(features_warp_kernel<4>, grid, block, kFeatWarps * feat_warp_bytes(4), st, fp);
    else launch_pdl(features_warp_kernel<8>, grid, block, kFeatWarps * feat_warp_bytes(8), st, fp);
  } else {
    launch_pdl(features_kernel, P, std::min(1024, std::max(64, S2 / 2)), features_smem(S2, s->N), st, fp);
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// First index of b2 in the flat parameter vector (w3 and b3 follow it).
int off_b2(const BrkgaSurrogate* s) { return (int)((long long)kH1 * s->in_pad + kH1 + (long long)kH2 * kH1); }

OutPartials out_partials(const BrkgaSurrogate* s, int nrb) {
  OutPartials op;
  op.nrb = nrb;
  op.w3 = s->outp;
  op.b2 = s->outp + (size_t)nrb * kH2;
  op.b3 = s->outp + (size_t)2 * nrb * kH2;
  op.loss = op.b3 + nrb;
  op.n_valid = s->n_valid;
  op.loss_out = s->loss;
  return op;
}

// Forward pass on s->X [B, in_pad] (B % 128 == 0), two GEMMs: Z1 = X W1^T
// with bias + ReLU in its epilogue -> H1 (bf16; with `train` also Z1 fp32 and
// H1 transposed for the backward pass), Z2 = H1 W2^T with bias + ReLU and the
// output layer's dot with w3 per column tile -> s->part (with `train` also Z2
// fp32).  *n_tiles: the partials per row, summed by the next kernel.
int forward(BrkgaSurrogate* s, int B, bool train, int* n_tiles, cudaStream_t st) {
  int r;
  umma::Epilogue e1;
  e1.kind = umma::kBiasRelu;
  e1.bias = s->b1;
  e1.out = s->H1b;
  e1.ld_out = kH1;
  if (train) {
    e1.C = s->Z1;
    e1.ldc = kH1;
    e1.outT = s->H1Tb;
    e1.ld_outT = B;
  }
  if ((r = gemm(s->X, s->in_pad, s->W1b, s->in_pad, e1, B, kH1, s->in_pad, s->err, st))) return r;
  umma::Epilogue e2;
  e2.kind = umma::kBiasRelu;
  e2.bias = s->b2;
  e2.dotw = s->w3;
  e2.part = s->part;
  e2.ld_part = s->max_batch;
  if (train) {
    e2.C = s->Z2;
    e2.ldc = kH2;
  }
  if ((r = gemm(s->H1b, kH1, s->W2b, kH1, e2, B, kH2, kH1, s->err, st))) return r;
  *n_tiles = kH2 / tile_n(B, kH2);
  return BRKGA_OK;
}

int cast_weights(BrkgaSurrogate* s, cudaStream_t st) {
  cast_kernel<<<grid_for((long long)kH1 * s->in_pad), 256, 0, st>>>(s->W1, kH1, s->in_pad, s->W1b, nullptr);
  cast_kernel<<<grid_for((long long)kH2 * kH1), 256, 0, st>>>(s->W2, kH2, kH1, s->W2b, s->W2Tb);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// Gradients of the MSE on the minibatch in the activation buffers (forward
// pass included): the output layer's backward pass in one kernel, then
// dW2 = dZ2^T H1, dH1 = dZ2 W2 with the ReLU derivative (Z1 > 0) in its
// epilogue (-> dH1 fp32 and dZ1 transposed bf16), gb1 = column sums of dH1,
// dW1 = dZ1^T X.  With `bump` the step counters advance (training loop).
int gradients(BrkgaSurrogate* s, int B, int bump, cudaStream_t st) {
  int r, n_tiles = 0;
  const int I = s->in_pad;
  if ((r = forward(s, B, true, &n_tiles, st))) return r;
  const int nrb = B / 32;
  float* pw3 = s->outp;
  float* pb2 = pw3 + (size_t)nrb * kH2;
  float* pb3 = pb2 + (size_t)nrb * kH2;
  launch_pdl(out_backward_kernel, dim3(kH2 / 32, nrb), dim3(32, 8), 0, st,
      s->part, n_tiles, s->max_batch, s->b3, s->t, s->n_valid, s->Z2, s->w3, B, s->y, s->dZ2b, s->dZ2Tb, pw3, pb2,
      pb3, pb3 + nrb, s->step, s->adam_t, bump);
  s->last_nrb = nrb;
  if (!bump) launch_pdl(out_grads_kernel, 1, 256, 0, st, s->grads, off_b2(s), out_partials(s, nrb));
  if ((r = gemm(s->dZ2Tb, B, s->H1Tb, B, store_to(s->gW2, kH1), kH2, kH1, B, s->err, st))) return r;
  umma::Epilogue eh;
  eh.kind = umma::kReluMask;
  eh.ref = s->Z1;
  eh.ld_ref = kH1;
  eh.C = s->dH1;
  eh.ldc = kH1;
  eh.outT = s->dZ1Tb;
  eh.ld_outT = B;
  if ((r = gemm(s->dZ2b, kH2, s->W2Tb, kH2, eh, B, kH1, kH2, s->err, st))) return r;
  col_reduce(s->dH1, nullptr, nullptr, nullptr, B, kH1, s->gb1, st);
  if ((r = gemm(s->dZ1Tb, B, s->XT, B, store_to(s->gW1, I), kH1, I, B, s->err, st))) return r;
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// Adam on every parameter; `fused_out`: the output layer's gradients are
// still row-block partials of the last backward pass (the training loop).
int adam_cast(BrkgaSurrogate* s, float lr, bool fused_out, cudaStream_t st) {
  const long long nW1 = (long long)kH1 * s->in_pad;
  OutPartials op = out_partials(s, fused_out ? s->last_nrb : 0);
  launch_pdl(adam_cast_kernel, grid_for(s->n_params), 256, 0, st, s->params, s->grads, s->mom, s->vel,
             (int)s->n_params, lr, 0.9f, 0.999f, 1e-8f, s->adam_t, (int)nW1, (int)(nW1 + kH1), kH2 * kH1, s->W1b,
             s->W2b, s->W2Tb, off_b2(s), op);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

}  // namespace

extern "C" {

// Back to the state right after creation: initial weights, zero biases and
// Adam moments, empty example buffer, target scaling unset.  Synchronous.
int brkga_surrogate_reset(BrkgaSurrogate* s) {
  if (!s) return BRKGA_ERR_INVALID_ARGUMENT;
  const int I = s->in_pad;
  const long long nW1 = (long long)kH1 * I, nW2 = (long long)kH2 * kH1;
  if (cudaMemset(s->params, 0, s->n_params * 4) != cudaSuccess || cudaMemset(s->mom, 0, s->n_params * 4) ||
      cudaMemset(s->vel, 0, s->n_params * 4) || cudaMemset(s->grads, 0, s->n_params * 4) ||
      cudaMemset(s->count, 0, 8) || cudaMemset(s->step, 0, 8) || cudaMemset(s->adam_t, 0, 8) ||
      cudaMemset(s->norm, 0, 24))
    return BRKGA_ERR_CUDA;
  const uint32_t k0 = (uint32_t)s->seed, k1 = (uint32_t)(s->seed >> 32);
  init_weights_kernel<<<grid_for(nW1), 256>>>(s->W1, (int)nW1, s->in, s->in, I, k0, k1, 1);
  init_weights_kernel<<<grid_for(nW2), 256>>>(s->W2, (int)nW2, kH1, kH1, kH1, k0, k1, 2);
  init_weights_kernel<<<1, 256>>>(s->w3, kH2, kH2, kH2, kH2, k0, k1, 3);
  const int st = cast_weights(s, nullptr);
  if (st) return st;
  return cudaDeviceSynchronize() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_gemm_bf16(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, float* d_C, int32_t ldc, int32_t M,
                    int32_t N, int32_t K, int32_t* d_err, void* stream) {
  if (!d_A || !d_B || !d_C || !d_err || M < 0 || N < 0 || K < 0 || lda < K || ldb < K || ldc < N || lda % 8 ||
      ldb % 8 || ldc % 4)
    return BRKGA_ERR_INVALID_ARGUMENT;
  if (M == 0 || N == 0 || K == 0) return BRKGA_OK;
  const int st = prepare_gemm();
  if (st) return st;
  return gemm(static_cast<const __nv_bfloat16*>(d_A), lda, static_cast<const __nv_bfloat16*>(d_B), ldb,
              store_to(d_C, ldc), M, N, K, d_err, static_cast<cudaStream_t>(stream));
}

void brkga_surrogate_destroy(BrkgaSurrogate* s) {
  if (!s) return;
  for (void* p : s->allocs) cudaFree(p);
  delete s;
}

int brkga_surrogate_create(const BrkgaProblem* problem, int32_t max_batch, int32_t buffer_capacity, uint64_t seed,
                           BrkgaSurrogate** out) {
  return brkga_surrogate_create_ex(problem, max_batch, buffer_capacity, seed, BRKGA_SURROGATE_FEATURES_DECODE, out);
}

int brkga_surrogate_create_ex(const BrkgaProblem* problem, int32_t max_batch, int32_t buffer_capacity, uint64_t seed,
                              int32_t features, BrkgaSurrogate** out) {
  if (!problem || !out || max_batch < 128 || max_batch % 128 || buffer_capacity < 1 ||
      (features != BRKGA_SURROGATE_FEATURES_DECODE && features != BRKGA_SURROGATE_FEATURES_ORDER))
    return BRKGA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  BrkgaSurrogate* s = new BrkgaSurrogate();
  s->problem = problem;
  s->features_kind = features;
  const double* bin_area = nullptr;
  if (brkga_internal_problem_tables(problem, &s->N, &s->M, &s->T, &s->mode, &s->thr, &s->gene_type, &s->part_area,
                                    &s->pt, &s->pth, &bin_area) != BRKGA_OK || s->N > kMaxGenes || s->M > 256) {
    delete s;
    return BRKGA_ERR_INVALID_ARGUMENT;
  }
  s->bin_area = bin_area;
  s->in = features == BRKGA_SURROGATE_FEATURES_ORDER ? 3 * s->N : 3 * s->N + 2 * s->M;
  s->in_pad = round_up(s->in, 64);
  s->max_batch = max_batch;
  s->cap = buffer_capacity;
  s->seed = seed;
  // feature scales from the host copies of the time tables
  {
    std::vector<double> pt((size_t)s->M * s->T), pth((size_t)s->M * s->T);
    if (cudaMemcpy(pt.data(), s->pt, pt.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(pth.data(), s->pth, pth.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      delete s;
      return BRKGA_ERR_CUDA;
    }
    std::vector<double> area(s->T);
    if (cudaMemcpy(area.data(), s->part_area, area.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
      delete s;
      return BRKGA_ERR_CUDA;
    }
    const double mp = *std::max_element(pt.begin(), pt.end()), mh = *std::max_element(pth.begin(), pth.end());
    const double ma = *std::max_element(area.begin(), area.end());
    s->inv_pt = mp > 0 ? (float)(1.0 / mp) : 1.f;
    s->inv_pth = mh > 0 ? (float)(1.0 / mh) : 1.f;
    s->inv_area = ma > 0 ? (float)(1.0 / ma) : 1.f;
  }
  if (cudaFuncSetAttribute(features_warp_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kFeatWarps * feat_warp_bytes(8))) != cudaSuccess ||
      cudaFuncSetAttribute(features_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)features_smem(kMaxGenes, kMaxGenes)) !=
          cudaSuccess ||
      prepare_gemm() != BRKGA_OK) {
    delete s;
    return BRKGA_ERR_CUDA;
  }
  const int B = max_batch, I = s->in_pad;
  const long long nW1 = (long long)kH1 * I, nW2 = (long long)kH2 * kH1;
  s->n_params = nW1 + kH1 + nW2 + kH2 + kH2 + 1;
  int st = BRKGA_OK;
  if ((st = dalloc(s, &s->params, s->n_params)) || (st = dalloc(s, &s->grads, s->n_params)) ||
      (st = dalloc(s, &s->mom, s->n_params)) || (st = dalloc(s, &s->vel, s->n_params)) ||
      (st = dalloc(s, &s->W1b, nW1)) || (st = dalloc(s, &s->W2b, nW2)) || (st = dalloc(s, &s->W2Tb, nW2)) ||
      (st = dalloc(s, &s->X, (size_t)B * I)) || (st = dalloc(s, &s->XT, (size_t)B * I)) ||
      (st = dalloc(s, &s->H1b, (size_t)B * kH1)) || (st = dalloc(s, &s->H1Tb, (size_t)B * kH1)) ||
      (st = dalloc(s, &s->dZ2b, (size_t)B * kH2)) || (st = dalloc(s, &s->dZ2Tb, (size_t)B * kH2)) ||
      (st = dalloc(s, &s->dZ1Tb, (size_t)B * kH1)) || (st = dalloc(s, &s->Z1, (size_t)B * kH1)) ||
      (st = dalloc(s, &s->Z2, (size_t)B * kH2)) || (st = dalloc(s, &s->y, B)) || (st = dalloc(s, &s->t, B)) ||
      (st = dalloc(s, &s->part, (size_t)4 * B)) ||
      (st = dalloc(s, &s->outp, (size_t)(kMaxTrainBatch / 32) * (2 * kH2 + 2))) || (st = dalloc(s, &s->dH1, (size_t)B * kH1)) || (st = dalloc(s, &s->loss, 1)) ||
      (st = dalloc(s, &s->n_valid, 1)) || (st = dalloc(s, &s->slot, B)) || (st = dalloc(s, &s->err, 1)) || (st = dalloc(s, &s->count, 1)) ||
      (st = dalloc(s, &s->step, 1)) || (st = dalloc(s, &s->adam_t, 1)) || (st = dalloc(s, &s->norm, 3)) ||
      (st = dalloc(s, &s->bufX, (size_t)s->cap * I)) || (st = dalloc(s, &s->bufY, s->cap))) {
    brkga_surrogate_destroy(s);
    return st;
  }
  float* q = s->params;
  s->W1 = q; q += nW1; s->b1 = q; q += kH1; s->W2 = q; q += nW2; s->b2 = q; q += kH2; s->w3 = q; q += kH2; s->b3 = q;
  q = s->grads;
  s->gW1 = q; q += nW1; s->gb1 = q; q += kH1; s->gW2 = q; q += nW2; s->gb2 = q; q += kH2; s->gw3 = q; q += kH2;
  s->gb3 = q;
  if ((st = brkga_surrogate_reset(s)) != BRKGA_OK) {
    brkga_surrogate_destroy(s);
    return st ? st : BRKGA_ERR_CUDA;
  }
  *out = s;
  return BRKGA_OK;
}

int brkga_surrogate_dims(const BrkgaSurrogate* s, int32_t* in_features, int32_t* in_padded, int64_t* n_params) {
  if (!s) return BRKGA_ERR_INVALID_ARGUMENT;
  if (in_features) *in_features = s->in;
  if (in_padded) *in_padded = s->in_pad;
  if (n_params) *n_params = s->n_params;
  return BRKGA_OK;
}

int brkga_surrogate_buffers(const BrkgaSurrogate* s, float** params, float** grads, void** X, float** y,
                            int32_t** err, int64_t** count, double** norm) {
  if (!s) return BRKGA_ERR_INVALID_ARGUMENT;
  if (params) *params = s->params;
  if (grads) *grads = s->grads;
  if (X) *X = s->X;
  if (y) *y = s->y;
  if (err) *err = s->err;
  if (count) *count = reinterpret_cast<int64_t*>(s->count);
  if (norm) *norm = s->norm;
  return BRKGA_OK;
}

int brkga_surrogate_predict(BrkgaSurrogate* s, const float* d_chrom, int32_t P, double* d_pred, void* stream) {
  if (!s || P < 0 || (P > 0 && (!d_chrom || !d_pred))) return BRKGA_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int r;
  for (int off = 0; off < P; off += s->max_batch) {
    const int n = std::min(s->max_batch, P - off);
    const int B = round_up(n, 128);
    if (B > n && cudaMemsetAsync(s->X + (size_t)n * s->in_pad, 0, (size_t)(B - n) * s->in_pad * 2, st) != cudaSuccess)
      return BRKGA_ERR_CUDA;
    if ((r = features(s, d_chrom + (size_t)off * 2 * s->N, n, s->X, st))) return r;
    int n_tiles = 0;
    if ((r = forward(s, B, false, &n_tiles, st))) return r;
    launch_pdl(predict_out_kernel, (n + 255) / 256, 256, 0, st, s->part, n_tiles, s->max_batch, s->b3, n, s->norm,
               s->y, d_pred + off);
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_surrogate_observe(BrkgaSurrogate* s, const float* d_chrom, const double* d_makespan, int32_t P,
                            void* stream) {
  if (!s || P < 0 || (P > 0 && (!d_chrom || !d_makespan))) return BRKGA_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int r;
  launch_pdl(set_norm_kernel, 1, 256, 0, st, d_makespan, P, s->norm);
  for (int off = 0; off < P; off += s->max_batch) {
    const int n = std::min(s->max_batch, P - off);
    if ((r = features(s, d_chrom + (size_t)off * 2 * s->N, n, s->X, st))) return r;
    ObsParams op;
    op.makespan = d_makespan + off;
    op.P = n;
    op.Xsrc = s->X;
    op.in_pad = s->in_pad;
    op.bufX = s->bufX;
    op.bufY = s->bufY;
    op.cap = s->cap;
    op.norm = s->norm;
    launch_pdl(observe_slots_kernel, 1, kObsThreads, 0, st, op.makespan, n, s->norm, s->count, s->cap, s->slot);
    launch_pdl(observe_kernel, n, 128, 0, st, op, s->slot);
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_surrogate_gradients(BrkgaSurrogate* s, int32_t B, void* stream) {
  // gradients of the MSE on the rows already in the activation buffers
  // (s->X, s->XT, s->t, *n_valid) — used by tests and by brkga_surrogate_train
  if (!s || B < 128 || B % 128 || B > s->max_batch || B > kMaxTrainBatch) return BRKGA_ERR_INVALID_ARGUMENT;
  return gradients(s, B, 0, static_cast<cudaStream_t>(stream));
}

int brkga_surrogate_adam(BrkgaSurrogate* s, float lr, void* stream) {
  if (!s) return BRKGA_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  bump_kernel<<<1, 1, 0, st>>>(s->adam_t);
  return adam_cast(s, lr, false, st);
}

int brkga_surrogate_train(BrkgaSurrogate* s, int32_t steps, int32_t batch, float lr, void* stream) {
  if (!s || steps < 0 || batch < 128 || batch % 128 || batch > s->max_batch || batch > kMaxTrainBatch)
    return BRKGA_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int r;
  // one step = 9 launches: minibatch gather, two forward GEMMs, the output
  // layer's backward pass (which also advances the step counters), three
  // backward GEMMs, one column reduction, Adam with the bf16 casts
  for (int i = 0; i < steps; ++i) {
    launch_pdl(gather_kernel, batch, 128, 0, st, s->bufX, s->bufY, s->count, s->cap, batch, batch, s->in_pad,
               (uint32_t)s->seed, (uint32_t)(s->seed >> 32), s->step, s->X, s->XT, s->t, s->n_valid);
    if ((r = gradients(s, batch, 1, st))) return r;
    if ((r = adam_cast(s, lr, true, st))) return r;
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// Put a caller-chosen minibatch in the activation buffers: X [B, in_pad] bf16
// (device), targets t [B] (device), the first n_valid rows real.  Tests use it
// to compare gradients with the CPU oracle.
int brkga_surrogate_load_batch(BrkgaSurrogate* s, const void* d_X, const float* d_t, int32_t B, int32_t n_valid,
                               void* stream) {
  if (!s || !d_X || !d_t || B < 128 || B % 128 || B > s->max_batch || n_valid < 1 || n_valid > B)
    return BRKGA_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(s->X, d_X, (size_t)B * s->in_pad * 2, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(s->t, d_t, (size_t)B * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  set_int_kernel<<<1, 1, 0, st>>>(s->n_valid, n_valid);
  transpose_bf16_kernel<<<grid_for((long long)B * s->in_pad), 256, 0, st>>>(s->X, B, s->in_pad, s->XT);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// Features of P chromosomes into the first rows of the activation buffer X (tests).
int brkga_surrogate_features(BrkgaSurrogate* s, const float* d_chrom, int32_t P, void* stream) {
  if (!s || !d_chrom || P < 1 || P > s->max_batch) return BRKGA_ERR_INVALID_ARGUMENT;
  return features(s, d_chrom, P, s->X, static_cast<cudaStream_t>(stream));
}

// Copy one of the surrogate's device arrays to or from host memory (tests,
// checkpoints): 0 = parameters (fp32, flat), 1 = gradients, 2 = activations X
// (bf16 [max_batch, in_pad]), 3 = predictions y (fp32 [max_batch]), 4 = loss
// (fp32 [1]), 5 = target standardisation (float64 mean, std, set flag),
// 6 = Adam moments m and v (fp32, 2 x parameters), 7 = Adam step (int64),
// 8 = the example ring's standardised targets (fp32 [capacity]), 9 = examples
// observed so far (int64).
int brkga_surrogate_io(BrkgaSurrogate* s, int32_t what, void* host, int64_t bytes, int32_t to_device) {
  if (!s || !host || bytes < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  void* dev = nullptr;
  int64_t size = 0;
  switch (what) {
    case 0: dev = s->params; size = s->n_params * 4; break;
    case 1: dev = s->grads; size = s->n_params * 4; break;
    case 2: dev = s->X; size = (int64_t)s->max_batch * s->in_pad * 2; break;
    case 3: dev = s->y; size = (int64_t)s->max_batch * 4; break;
    case 4: dev = s->loss; size = 4; break;
    case 5: dev = s->norm; size = 24; break;
    case 6: dev = s->mom; size = s->n_params * 8; break;  // mom and vel are separate allocations
    case 7: dev = s->adam_t; size = 8; break;
    case 8: dev = s->bufY; size = (int64_t)s->cap * 4; break;
    case 9: dev = s->count; size = 8; break;
    default: return BRKGA_ERR_INVALID_ARGUMENT;
  }
  if (bytes > size) return BRKGA_ERR_INVALID_ARGUMENT;
  if (what == 6) {
    const int64_t half = s->n_params * 4;
    char* h = static_cast<char*>(host);
    const int64_t b1 = std::min(bytes, half), b2 = std::max<int64_t>(0, bytes - half);
    cudaError_t e1 = to_device ? cudaMemcpy(s->mom, h, b1, cudaMemcpyHostToDevice)
                               : cudaMemcpy(h, s->mom, b1, cudaMemcpyDeviceToHost);
    cudaError_t e2 = b2 == 0 ? cudaSuccess
                     : to_device ? cudaMemcpy(s->vel, h + half, b2, cudaMemcpyHostToDevice)
                                 : cudaMemcpy(h + half, s->vel, b2, cudaMemcpyDeviceToHost);
    return (e1 == cudaSuccess && e2 == cudaSuccess) ? BRKGA_OK : BRKGA_ERR_CUDA;
  }
  const cudaError_t e = to_device ? cudaMemcpy(dev, host, bytes, cudaMemcpyHostToDevice)
                                  : cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return BRKGA_ERR_CUDA;
  if (to_device && what == 0) {
    const int r = cast_weights(s, nullptr);
    if (r) return r;
    return cudaDeviceSynchronize() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
  }
  return BRKGA_OK;
}

}  // extern "C"
