// brkga_ga.cu — the BRKGA generation step on the GPU (C ABI in include/brkga_b200.h).
//
// One generation of the reference's GA loop (BRKGA_alg3.py:229-265):
//   rank      sort the population by fitness (partition, :178-186): elites are
//             the n_elites best, in ascending fitness; ties keep the lower index
//   breed     new population = [elites | mutants | offspring] (:246-250):
//             mutants are uniform [0,1) keys (:207-208); each offspring takes
//             one random elite and one random non-elite parent and copies each
//             key from the elite with probability rho (:188-205)
//   decode    (brkga_decode on rows n_elites..P-1; elites keep their fitness)
//   track     per-generation min and mean fitness (:255-262), best-so-far
//             chromosome, generation counter
// Randomness is counter-based Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), keyed by the run
// seed and indexed by (gene block, row, generation, stream tag), so every
// kernel is deterministic and replayable inside a CUDA graph: the generation
// number is read from device memory, not baked into the launch.

#include <cuda_runtime.h>

#include <mutex>

#include <cstdint>

#include "../../include/brkga_b200.h"

namespace {

constexpr int kMaxRank = 8192;         // single-CTA bitonic sort: 8192 x 12 B in shared memory
constexpr int kMaxRankCount = 65536;   // larger populations: rank by counting (P^2 key comparisons)
constexpr int kRankTile = 2048;

enum Tag : uint32_t { kTagInit = 0, kTagMutant = 1, kTagMask = 2, kTagParents = 3 };

struct U4 {
  uint32_t x, y, z, w;
};

__host__ __device__ inline uint32_t mulhi32(uint32_t a, uint32_t b) {
  return (uint32_t)(((uint64_t)a * b) >> 32);
}

// Philox4x32 with 10 rounds: round(c, k) = (hi(M1*c2) ^ c1 ^ k0, lo(M1*c2),
// hi(M0*c0) ^ c3 ^ k1, lo(M0*c0)); the key is bumped by the Weyl constants
// between rounds.
__host__ __device__ inline U4 philox(U4 c, uint32_t k0, uint32_t k1) {
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

// 24 random bits -> float in [0, 1), exactly representable
__device__ inline float unit_float(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

__device__ inline unsigned long long ordered_f64(double v) {
  unsigned long long u = (unsigned long long)__double_as_longlong(v);
  if (v == 0.0) u = 0ull;
  if (v != v) u = 0x7FF8000000000000ull;  // NaN (a failed decode) ranks last
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

__global__ void init_population_kernel(float* pop, int P, int K, uint32_t k0, uint32_t k1, int skip_rows) {
  const int blocks = (K + 3) >> 2;
  const long long n = (long long)P * blocks;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(i / blocks), b = (int)(i - (long long)row * blocks);
    if (row < skip_rows) continue;
    const U4 r = philox(U4{(uint32_t)b, (uint32_t)row, 0u, kTagInit}, k0, k1);
    const uint32_t v[4] = {r.x, r.y, r.z, r.w};
    for (int q = 0; q < 4 && 4 * b + q < K; ++q) pop[(size_t)row * K + 4 * b + q] = unit_float(v[q]);
  }
}

__global__ void rank_kernel(const double* fit, int P, int S2, int32_t* order) {
  extern __shared__ unsigned long long sm[];
  unsigned long long* key = sm;
  int* idx = reinterpret_cast<int*>(sm + S2);
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int i = tid; i < S2; i += nt) {
    key[i] = i < P ? ordered_f64(fit[i]) : ~0ull;
    idx[i] = i < P ? i : 0x7FFFFFFF;
  }
  __syncthreads();
  for (int k = 2; k <= S2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S2; i += nt) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = key[i], b = key[ixj];
          const int ia = idx[i], ib = idx[ixj];
          const bool gt = a > b || (a == b && ia > ib);
          if (gt == ((i & k) == 0)) {
            key[i] = b;
            key[ixj] = a;
            idx[i] = ib;
            idx[ixj] = ia;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < P; i += nt) order[i] = idx[i];
}

// Rank by counting for populations above the single-CTA sort: the rank of row
// i is the number of rows j with (key_j, j) < (key_i, i), the keys of all rows
// streamed through shared memory tile by tile (every thread reads the same
// entry: broadcast).  Same order as rank_kernel; O(P^2) comparisons, about
// 0.1 ms at P = 20,000.
__global__ void rank_count_kernel(const double* fit, int P, int32_t* order) {
  __shared__ unsigned long long tile[kRankTile];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long ki = i < P ? ordered_f64(fit[i]) : 0ull;
  int rank = 0;
  for (int base = 0; base < P; base += kRankTile) {
    const int n = min(kRankTile, P - base);
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) tile[t] = ordered_f64(fit[base + t]);
    __syncthreads();
    if (i < P) {
      for (int t = 0; t < n; ++t) {
        const unsigned long long kj = tile[t];
        rank += (kj < ki) | ((kj == ki) & (base + t < i));
      }
    }
  }
  if (i < P) order[rank] = i;
}

// One thread per (row, 4-key block) of the new population.  Offspring come
// in families of `family` consecutive rows that share one parent pair: the
// pair of family f is drawn from the Philox stream of row ne + nm + f, the
// stream the plain GA uses for that offspring row, so family = 1 is the plain
// breed and family k > 1 gives every plain offspring slot k siblings; each
// child's crossover mask comes from its own row.
__global__ void breed_kernel(const float* pop, const double* fit, const int32_t* order, int P, int out_rows, int K,
                             int ne, int nm, int family, float rho, uint32_t k0, uint32_t k1,
                             const long long* generation, float* next, double* next_fit) {
  const uint32_t gen = (uint32_t)(*generation);
  const int blocks = (K + 3) >> 2;
  const long long n = (long long)out_rows * blocks;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int row = (int)(i / blocks), b = (int)(i - (long long)row * blocks);
    float* dst = next + (size_t)row * K + 4 * b;
    const int nk = min(4, K - 4 * b);
    if (row < ne) {  // elites, best first
      const float* src = pop + (size_t)order[row] * K + 4 * b;
      for (int q = 0; q < nk; ++q) dst[q] = src[q];
      if (b == 0) next_fit[row] = fit[order[row]];
    } else if (row < ne + nm) {  // mutants
      const U4 r = philox(U4{(uint32_t)b, (uint32_t)row, gen, kTagMutant}, k0, k1);
      const uint32_t v[4] = {r.x, r.y, r.z, r.w};
      for (int q = 0; q < nk; ++q) dst[q] = unit_float(v[q]);
    } else {  // offspring of one elite and one non-elite parent
      const int prow = ne + nm + (row - ne - nm) / family;
      const U4 pr = philox(U4{0u, (uint32_t)prow, gen, kTagParents}, k0, k1);
      const int e = order[(int)mulhi32(pr.x, (uint32_t)ne)];
      const int o = order[ne + (int)mulhi32(pr.y, (uint32_t)(P - ne))];  // non-elites of the parent population
      const U4 r = philox(U4{(uint32_t)b, (uint32_t)row, gen, kTagMask}, k0, k1);
      const uint32_t v[4] = {r.x, r.y, r.z, r.w};
      for (int q = 0; q < nk; ++q) {
        const int g = 4 * b + q;
        dst[q] = unit_float(v[q]) < rho ? pop[(size_t)e * K + g] : pop[(size_t)o * K + g];
      }
    }
  }
}

// Per family of `family` consecutive candidates, the index of the one with the
// smallest prediction (ties: the first; NaN never wins over a number).
__global__ void select_families_kernel(const double* pred, int n_families, int family, int32_t* out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n_families) return;
  const double* p = pred + (size_t)f * family;
  int best = 0;
  for (int j = 1; j < family; ++j)
    if (p[j] < p[best] || (p[best] != p[best] && p[j] == p[j])) best = j;
  out[f] = f * family + best;
}

__global__ void gather_rows_kernel(const float* src, const int32_t* idx, int n, int K, float* dst) {
  const long long total = (long long)n * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / K), k = (int)(i - (long long)r * K);
    dst[i] = src[(size_t)idx[r] * K + k];
  }
}

// Audit sample: rows idx[0..n) of the population and their makespans into
// slot g = *generation of the audit arrays (nothing when g >= slots).
__global__ void audit_kernel(const float* pop, const double* fit, const int32_t* idx, int n, int K,
                             const long long* generation, int slots, float* audit_pop, double* audit_fit) {
  const long long g = *generation;
  if (g < 0 || g >= slots) return;
  const long long total = (long long)n * K;
  float* dst = audit_pop + (size_t)g * n * K;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / K), k = (int)(i - (long long)r * K);
    dst[i] = pop[(size_t)idx[r] * K + k];
  }
  if (blockIdx.x == 0)
    for (int r = threadIdx.x; r < n; r += blockDim.x) audit_fit[(size_t)g * n + r] = fit[idx[r]];
}

// Surrogate quality on the rows decoded this generation: Spearman correlation
// of predicted and exact makespans (ranks from the two orderings; feasible
// rows only) and the mean absolute error; stats[2g], stats[2g+1].
__global__ void screen_stats_kernel(const double* pred, const double* exact, const int32_t* order_pred,
                                    const int32_t* order_exact, int n, const long long* generation, double* stats,
                                    int stats_len, int* rank_scratch) {
  __shared__ double s_a[1024], s_b[1024], s_c[1024], s_m[1024], s_n[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  int* rp = rank_scratch;
  int* re = rank_scratch + n;
  for (int i = tid; i < n; i += nt) {
    rp[order_pred[i]] = i;
    re[order_exact[i]] = i;
  }
  __syncthreads();
  // feasible rows keep their order among themselves; infeasible exact values rank last
  double sa = 0, sb = 0, sab = 0, mae = 0, cnt = 0;
  for (int i = tid; i < n; i += nt) {
    const double e = exact[i];
    if (e < 1e15 && e == e) {
      sa += rp[i];
      sb += re[i];
      sab += (double)rp[i] * re[i];
      mae += fabs(pred[i] - e);
      cnt += 1;
    }
  }
  s_a[tid] = sa;
  s_b[tid] = sb;
  s_c[tid] = sab;
  s_m[tid] = mae;
  s_n[tid] = cnt;
  __syncthreads();
  for (int h = nt >> 1; h; h >>= 1) {
    if (tid < h) {
      s_a[tid] += s_a[tid + h];
      s_b[tid] += s_b[tid + h];
      s_c[tid] += s_c[tid + h];
      s_m[tid] += s_m[tid + h];
      s_n[tid] += s_n[tid + h];
    }
    __syncthreads();
  }
  // second pass for the variances (ranks are permutations only when all rows are feasible)
  double va = 0, vb = 0;
  const double k = s_n[0];
  const double ma = k > 0 ? s_a[0] / k : 0, mb = k > 0 ? s_b[0] / k : 0;
  for (int i = tid; i < n; i += nt) {
    const double e = exact[i];
    if (e < 1e15 && e == e) {
      va += (rp[i] - ma) * (rp[i] - ma);
      vb += (re[i] - mb) * (re[i] - mb);
    }
  }
  __syncthreads();
  s_a[tid] = va;
  s_b[tid] = vb;
  __syncthreads();
  for (int h = nt >> 1; h; h >>= 1) {
    if (tid < h) {
      s_a[tid] += s_a[tid + h];
      s_b[tid] += s_b[tid + h];
    }
    __syncthreads();
  }
  if (tid == 0) {
    const long long g = *generation;
    if (g >= 0 && g < stats_len) {
      const double cov = s_c[0] / fmax(k, 1.0) - ma * mb;
      const double den = sqrt(s_a[0] / fmax(k, 1.0) * s_b[0] / fmax(k, 1.0));
      stats[2 * g] = (k >= 2 && den > 0) ? cov / den : nan("");
      stats[2 * g + 1] = k > 0 ? s_m[0] / k : nan("");
    }
  }
}

// Min and mean of the fitness (history), best-so-far chromosome, generation++.
__global__ void track_kernel(const double* fit, const float* pop, int P, int K, long long* generation,
                             double* history, int history_len, double* best_fit, float* best_sol) {
  __shared__ double s_min[1024], s_sum[1024];
  __shared__ int s_arg[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  double mn = INFINITY, sum = 0.0;
  int arg = 0x7FFFFFFF;
  // fixed per-thread order, then a fixed tree: the mean does not depend on scheduling
  for (int i = tid; i < P; i += nt) {
    const double v = fit[i];
    sum += v;
    if (v < mn || (v == mn && i < arg)) {
      mn = v;
      arg = i;
    }
  }
  s_min[tid] = mn;
  s_sum[tid] = sum;
  s_arg[tid] = arg;
  __syncthreads();
  for (int h = nt >> 1; h > 0; h >>= 1) {
    if (tid < h) {
      s_sum[tid] += s_sum[tid + h];
      const double a = s_min[tid], b = s_min[tid + h];
      if (b < a || (b == a && s_arg[tid + h] < s_arg[tid])) {
        s_min[tid] = b;
        s_arg[tid] = s_arg[tid + h];
      }
    }
    __syncthreads();
  }
  const long long g = *generation;
  const bool better = s_arg[0] < P && s_min[0] < *best_fit;
  __syncthreads();
  if (better)
    for (int k = tid; k < K; k += nt) best_sol[k] = pop[(size_t)s_arg[0] * K + k];
  if (tid == 0) {
    if (g >= 0 && g < history_len) {
      history[2 * g] = s_min[0];
      history[2 * g + 1] = s_sum[0] / (double)P;
    }
    if (better) *best_fit = s_min[0];
    *generation = g + 1;
  }
}

// rank_kernel's opt-in to more than 48 KB of dynamic shared memory, once per
// device: std::call_once makes concurrent first calls from several host
// threads wait for the one that sets the attribute.
constexpr int kMaxDevices = 64;
std::once_flag g_rank_once[kMaxDevices];
int g_rank_opt_status[kMaxDevices];

int rank_opt_in(int dev) {
  std::call_once(g_rank_once[dev], [dev] {
    g_rank_opt_status[dev] =
        cudaFuncSetAttribute(rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kMaxRank * (int)(sizeof(unsigned long long) + sizeof(int))) == cudaSuccess
            ? BRKGA_OK
            : BRKGA_ERR_CUDA;
  });
  return g_rank_opt_status[dev];
}

int grid_for(long long n) {
  long long g = (n + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return (int)(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

int brkga_ga_breed_pool(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                        int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, float rho,
                        uint64_t seed, const int64_t* d_generation, float* d_next_pop, double* d_next_fitness,
                        void* stream);
int brkga_ga_breed_families(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                            int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, int32_t family,
                            float rho, uint64_t seed, const int64_t* d_generation, float* d_next_pop,
                            double* d_next_fitness, void* stream);

int brkga_ga_init_population(float* d_pop, int32_t P, int32_t n_keys, uint64_t seed, int32_t skip_rows,
                             void* stream) {
  if (P < 0 || n_keys < 1 || skip_rows < 0 || (P > 0 && !d_pop)) return BRKGA_ERR_INVALID_ARGUMENT;
  if (P == 0) return BRKGA_OK;
  init_population_kernel<<<grid_for((long long)P * ((n_keys + 3) / 4)), 256, 0, (cudaStream_t)stream>>>(
      d_pop, P, n_keys, (uint32_t)seed, (uint32_t)(seed >> 32), skip_rows);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_rank(const double* d_fitness, int32_t P, int32_t* d_order, void* stream) {
  if (P < 0 || P > kMaxRankCount || (P > 0 && (!d_fitness || !d_order))) return BRKGA_ERR_INVALID_ARGUMENT;
  if (P == 0) return BRKGA_OK;
  if (P > kMaxRank) {
    rank_count_kernel<<<(P + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_fitness, P, d_order);
    return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
  }
  int S2 = 1;
  while (S2 < P) S2 <<= 1;
  const size_t smem = (size_t)S2 * (sizeof(unsigned long long) + sizeof(int));
  if (smem > 48 * 1024) {  // above the default limit: opt in once per device (first call outside capture)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return BRKGA_ERR_CUDA;
    const int st = rank_opt_in(dev);
    if (st) return st;
  }
  rank_kernel<<<1, 1024, smem, (cudaStream_t)stream>>>(d_fitness, P, S2, d_order);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_breed(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P, int32_t n_keys,
                   int32_t n_elites, int32_t n_mutants, float rho, uint64_t seed, const int64_t* d_generation,
                   float* d_next_pop, double* d_next_fitness, void* stream) {
  if (P < 1 || n_keys < 1 || n_elites < 1 || n_mutants < 0 || n_elites + n_mutants > P || !d_pop || !d_fitness ||
      !d_order || !d_generation || !d_next_pop || !d_next_fitness || d_pop == d_next_pop)
    return BRKGA_ERR_INVALID_ARGUMENT;
  return brkga_ga_breed_pool(d_pop, d_fitness, d_order, P, P, n_keys, n_elites, n_mutants, rho, seed, d_generation,
                             d_next_pop, d_next_fitness, stream);
}

int brkga_ga_breed_pool(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                        int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, float rho,
                        uint64_t seed, const int64_t* d_generation, float* d_next_pop, double* d_next_fitness,
                        void* stream) {
  return brkga_ga_breed_families(d_pop, d_fitness, d_order, P, out_rows, n_keys, n_elites, n_mutants, 1, rho, seed,
                                 d_generation, d_next_pop, d_next_fitness, stream);
}

int brkga_ga_breed_families(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                            int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, int32_t family,
                            float rho, uint64_t seed, const int64_t* d_generation, float* d_next_pop,
                            double* d_next_fitness, void* stream) {
  if (P < 1 || out_rows < n_elites || n_keys < 1 || n_elites < 1 || n_elites > P || n_mutants < 0 || family < 1 ||
      n_elites + n_mutants > out_rows || (n_elites + n_mutants < out_rows && n_elites >= P) || !d_pop ||
      !d_fitness || !d_order || !d_generation || !d_next_pop || !d_next_fitness || d_pop == d_next_pop)
    return BRKGA_ERR_INVALID_ARGUMENT;
  breed_kernel<<<grid_for((long long)out_rows * ((n_keys + 3) / 4)), 256, 0, (cudaStream_t)stream>>>(
      d_pop, d_fitness, d_order, P, out_rows, n_keys, n_elites, n_mutants, family, rho, (uint32_t)seed,
      (uint32_t)(seed >> 32), reinterpret_cast<const long long*>(d_generation), d_next_pop, d_next_fitness);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_select_families(const double* d_pred, int32_t n_families, int32_t family, int32_t* d_index,
                             void* stream) {
  if (n_families < 0 || family < 1 || (n_families > 0 && (!d_pred || !d_index))) return BRKGA_ERR_INVALID_ARGUMENT;
  if (n_families == 0) return BRKGA_OK;
  select_families_kernel<<<(n_families + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_pred, n_families, family,
                                                                                     d_index);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_gather(const float* d_src, const int32_t* d_index, int32_t n, int32_t n_keys, float* d_dst,
                    void* stream) {
  if (n < 0 || n_keys < 1 || (n > 0 && (!d_src || !d_index || !d_dst))) return BRKGA_ERR_INVALID_ARGUMENT;
  if (n == 0) return BRKGA_OK;
  gather_rows_kernel<<<grid_for((long long)n * n_keys), 256, 0, (cudaStream_t)stream>>>(d_src, d_index, n, n_keys,
                                                                                      d_dst);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_audit(const float* d_pop, const double* d_fitness, const int32_t* d_index, int32_t n, int32_t n_keys,
                   const int64_t* d_generation, int32_t slots, float* d_audit_pop, double* d_audit_fit,
                   void* stream) {
  if (n < 0 || n_keys < 1 || slots < 0 ||
      (n > 0 && (!d_pop || !d_fitness || !d_index || !d_generation || !d_audit_pop || !d_audit_fit)))
    return BRKGA_ERR_INVALID_ARGUMENT;
  if (n == 0 || slots == 0) return BRKGA_OK;
  audit_kernel<<<grid_for((long long)n * n_keys), 256, 0, (cudaStream_t)stream>>>(
      d_pop, d_fitness, d_index, n, n_keys, reinterpret_cast<const long long*>(d_generation), slots, d_audit_pop,
      d_audit_fit);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_screen_stats(const double* d_pred, const double* d_exact, const int32_t* d_order_pred,
                          const int32_t* d_order_exact, int32_t n, const int64_t* d_generation, double* d_stats,
                          int32_t stats_len, int32_t* d_scratch, void* stream) {
  if (n < 1 || !d_pred || !d_exact || !d_order_pred || !d_order_exact || !d_generation || !d_stats || !d_scratch)
    return BRKGA_ERR_INVALID_ARGUMENT;
  screen_stats_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(d_pred, d_exact, d_order_pred, d_order_exact, n,
                                                           reinterpret_cast<const long long*>(d_generation),
                                                           d_stats, stats_len, d_scratch);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_ga_track(const double* d_fitness, const float* d_pop, int32_t P, int32_t n_keys, int64_t* d_generation,
                   double* d_history, int32_t history_len, double* d_best_fitness, float* d_best_solution,
                   void* stream) {
  if (P < 1 || n_keys < 1 || !d_fitness || !d_pop || !d_generation || (history_len > 0 && !d_history) ||
      !d_best_fitness || !d_best_solution)
    return BRKGA_ERR_INVALID_ARGUMENT;
  track_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(d_fitness, d_pop, P, n_keys,
                                                     reinterpret_cast<long long*>(d_generation), d_history,
                                                     history_len, d_best_fitness, d_best_solution);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

}  // extern "C"
