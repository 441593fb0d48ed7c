// brkga_decoder.cu — B200 (sm_100a) BRKGA chromosome decoder behind the C ABI
// of include/brkga_b200.h.
//
// Semantics: the reference's sequential decoder (paulonasc7/BRKGA_FFT2
// placement.py:94-165, binClassNew.py:45-174, numba_utils.py:50-188,
// collision_backend.py:109-213).  The reference finds collision-free
// positions with a float FFT correlation; here the correlation is evaluated
// exactly on bit-packed rows, which yields the same feasible set.
//
// A problem holds K >= 1 independent instances (own parts, machines, plate
// sizes).  Their tables are merged into one set of device arrays: part types,
// rotations, mask rows and machines get absolute indices, and each instance
// records its bases (InstDev).  A launch decodes P_k chromosomes of every
// instance k; the per-launch row/item offsets travel in the kernel
// parameters (InstRun), so one launch of each kernel serves all instances.
//
// Pipeline per launch (three kernels on one stream, no host sync):
//   1. assign_sort_kernel  one CTA per chromosome: machine of every gene from
//      the machine keys, then a bitonic sort of (machine, sequencing key,
//      gene) 64-bit keys in shared memory -> per-(chromosome, machine) part
//      order (placement.py:118-135).  order_items_kernel then sorts the
//      (chromosome, machine) items of all instances by part count.
//   2. decode_kernel       persistent CTAs of 1, 2 or 4 warps (the launch
//      shape), one (chromosome, machine) item at a time, longest first, from
//      a device counter.  A plate is L rows of ceil(W/32)+2 32-bit words (bit
//      x of a row = cell x); the first S plates of an item live in shared
//      memory, further ones in a global pool.  For each part: first-fit over
//      plates (area filter, then the collision search), else a new plate with
//      the best rotation at (0, L-1).  The collision search splits (rotation,
//      32 candidate rows) chunks over the warps, skipping chunks that cannot
//      beat the best position found so far; a lane runs the vacancy
//      filter of one candidate top row, then the (surviving candidate,
//      32-column word) pairs are dealt to the lanes for the exact
//      run-dilation test, mask rows coarse to fine from the bottom: each lane
//      walks the first runs of its pair alone, the pairs still open are
//      finished in order by the whole warp (a lane per run, results ANDed);
//      the first pair with a free column gives the bottom-most candidate and
//      its leftmost x.  Results are merged with a 64-bit lexicographic key
//      (newLen, -y, x, rotation) by atomicMin in shared memory, which is the
//      reference's rotation rule (binClassNew.py:101-117) — see key_of().
//   3. reduce_kernel       max over machines, 1e16 for infeasible chromosomes.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/brkga_b200.h"
#include "corr_i8.cuh"

namespace {

constexpr int kMaxMachines = 255;
constexpr int kMaxGenes = 8192;     // bitonic sort buffer: 8192 x 8 B = 64 KB shared memory
constexpr int kMaxSide = 8191;      // 13-bit fields of the selection key
constexpr int kMaxItemWarps = 4;   // decode CTAs have 1, 2 or 4 warps (one item per CTA)
constexpr int kGreedyThreads = 128;
constexpr int kResidentWarps = 32;  // automatic shape: 32 warps per SM (the register limit at 64 per thread)
constexpr int kMaxInst = BRKGA_MAX_INSTANCES;
constexpr int kMaxCtasPerSm = 32;
constexpr int kMaxSmemPlates = 8;
constexpr int kDefaultTaskMax = 8192;
// Latency launches (the 4-warp shape: few waves of items) end with their
// longest items, each sharing its SM with seven other CTAs until the queue
// drains.  The CTA that takes one of the first kCritItems items of the
// longest-first queue marks its SM, and the other CTAs there take no new
// item while the mark stands, so that SM empties and the long item gets its
// issue slots; the other SMs absorb the queue.  Measured at P100M4
// population 500: 2-4 % faster with 8 or 16 items; on throughput launches
// (2- and 1-warp shapes) draining SMs costs 2-7 %, so it is off there.
constexpr int kCritItems = 16;
constexpr int kCritSlots = 1024;  // per-SM marks, indexed by %smid
constexpr int kMaxTaskMax = 32 * 256;  // 32 candidates x the output words of the widest plate
constexpr unsigned long long kKeyNone = ~0ull;
constexpr unsigned kFull = 0xFFFFFFFFu;

struct RotDev {
  int h, w, mw;      // rows, columns, 32-bit words per mask row
  int vt;            // first entry in vtest[]: h (row << 16 | longest run of the row), collision-test order
  int trun, ntrun;   // runs of ones of all rows in test order: truns[trun .. trun + ntrun)
  int mask_base;     // first word in maskbits[] (h * mw words)
  int imax, dmax;    // row with the longest run of ones and that length
};

// The rotations of one part type that fit one machine's plate
// (numba_utils.py:82-84), fixed per (type, machine) and so built once at
// problem creation: in rotation order and by height (stable; the order of
// CTAs with fewer than four warps), the smallest height, and the words one
// read of the plate and of each rotated mask takes (the scan-bytes counter).
struct RotList {
  unsigned char nr;
  unsigned char r[4];   // rotation order
  unsigned char rs[4];  // by height, ties in rotation order
  unsigned char pad[3];
  int hmin;
  unsigned int scan_words;
};
static_assert(sizeof(RotList) == 20, "RotList layout");

struct MachDev {
  int L, W, NW, RS;  // plate rows, columns, words per row, row stride (NW + 2 zero pad words)
  double area;       // MachineData.bin_area
  double setup;      // MachineData.setup_time
};

struct BinScal {     // per-plate scalars of binClassNew.BuildingPlate
  double area, pt, pth;
  int minrow, maxrow, enc, pool;
};

// Where instance k's entries start in the merged tables.
struct InstDev {
  int N, M, T, mode;
  int gbase;    // gene_type[gbase + j]: absolute part type of gene j
  int tbase;    // first absolute part type
  int mbase;    // mach[mbase + m]
  int thrbase;  // thr[thrbase + m], M - 1 entries
  int tmbase;   // pt/pth[tmbase + m*T + t], newbin_ok/fits[tmbase + t*M + m] (t local)
};

// Merged device tables of all instances of a problem.
struct Tables {
  const InstDev* inst;
  const int32_t* gene_type;
  const double* thr;
  const MachDev* mach;
  const double* pt;
  const double* pth;
  const double* part_area;  // [absolute type]
  const int32_t* nrot;
  const int32_t* best_rot;
  const RotDev* rot;        // [absolute type * 4 + rotation]
  const uint32_t* vtest;
  const uint2* truns;       // (start | length << 16, row) per run of ones
  const uint32_t* maskbits;
  const uint8_t* newbin_ok;
  const uint8_t* fits;
  const RotList* rl;        // [(type, machine)], indexed like fits
};

// One instance's slice of a launch.
struct InstRun {
  int P;               // chromosomes of this instance in the launch
  int crow0;           // first row in chrom / makespan / infeas
  int item0;           // first (chromosome, machine) item
  int S2;              // bitonic sort width (power of two >= N)
  long long chrom_off; // first float of its chromosomes
  long long out_off;   // first makespan
  long long seq0;      // first entry of its part orders (and log entries), N per item
};

// Everything a launch needs besides the tables.
struct Run {
  int K, n_rows, n_items, Nmax;
  const float* chrom;
  double* out;
  uint16_t* seq;
  int32_t* cnt;
  int32_t* infeas;
  int32_t* order;
  double* mk;
  BrkgaPlacement* log;
  int32_t* status;
  unsigned int* item_ctr;
  unsigned int* pool_ctr;
  int* crit;           // kCritSlots marks: CTAs busy with a critical item, per SM
  int crit_items;      // items at the head of the queue that mark their SM (0 = off)
  unsigned long long* counters;
  BinScal* binscal;  // Nmax per resident CTA
  uint32_t* pool;
  long long pool_bins;
  int S, slot_words, slot_vac_off;
  int task_max;  // most (survivor, word) pairs of a chunk dealt across lanes
  InstRun r[kMaxInst];
};
static_assert(sizeof(Tables) + sizeof(Run) <= 4096, "kernel parameters must stay within 4 KB");

// ---------------------------------------------------------------- device helpers

__device__ __forceinline__ unsigned ordered_bits(float v) {
  unsigned u = __float_as_uint(v);
  if (v == 0.0f) u = 0u;               // -0 and +0 compare equal in the reference's sort
  if (v != v) u = 0x7FC00000u;         // NaN sorts after every number (np.argsort)
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// placement.py:122-127 for ascending thresholds: the first machine whose
// upper threshold is >= the key, else the last; a NaN key matches no mask.
__device__ __forceinline__ int machine_of(float mv, const double* thr, int M, int mode) {
  if (M <= 1) return 0;
  if (mv != mv) return M;
  int m = 0;
  if (mode == BRKGA_THRESH_F32) {
    while (m < M - 1 && !(mv <= (float)thr[m])) ++m;
  } else {
    const double v = (double)mv;
    while (m < M - 1 && !(v <= thr[m])) ++m;
  }
  return m;
}

// Selection key, smaller is better.  Within one plate the reference keeps the
// rotation of largest packing density (area + a) / (newLen * W); numerator and
// W are shared and newLen * W are distinct integers <= 2^26, so the float64
// quotients are strictly ordered by newLen: max density == min newLen.  Ties
// go to the larger bottom row y, then the smaller x, then the first rotation.
__device__ __forceinline__ unsigned long long key_of(int newlen, int y, int x, int r) {
  return ((unsigned long long)newlen << 28) | ((unsigned long long)(kMaxSide - y) << 15) |
         ((unsigned long long)x << 2) | (unsigned long long)r;
}

// bits [p, p + 32) of a row (p >= 0; reads words p>>5 and p>>5 + 1)
__device__ __forceinline__ uint32_t bits32(const uint32_t* row, int p) {
  const int wi = p >> 5;
  return __funnelshift_r(row[wi], row[wi + 1], p & 31);
}

__device__ __forceinline__ bool range_any(const uint32_t* row, int lo, int hi) {
  const int wl = lo >> 5, wh = (hi - 1) >> 5;
  const uint32_t ml = 0xFFFFFFFFu << (lo & 31);
  const uint32_t mh = 0xFFFFFFFFu >> (31 - ((hi - 1) & 31));
  if (wl == wh) return (row[wl] & ml & mh) != 0u;
  if (row[wl] & ml) return true;
  for (int w = wl + 1; w < wh; ++w)
    if (row[w]) return true;
  return (row[wh] & mh) != 0u;
}

// For the 32 placements x' = 0..31 (absolute x = p0 - a + x'), bit x' is set
// when a run of d mask cells starting at plate column p0 + x' covers an
// occupied cell: OR of row bits [p0 + x', p0 + x' + d).
__device__ __forceinline__ uint32_t blocked(const uint32_t* row, int p0, int d) {
  if (d <= 32) {
    uint32_t lo = bits32(row, p0), hi = bits32(row, p0 + 32);
    int s = 1;
    while (2 * s <= d) {  // doubling: after a step lo bit j = OR of 2s bits from j
      lo |= __funnelshift_r(lo, hi, s);
      hi |= hi >> s;
      s <<= 1;
    }
    if (d > s) lo |= __funnelshift_r(lo, hi, d - s);
    return lo;
  }
  // d > 32: every window contains [p0 + 31, p0 + d)
  if (range_any(row, p0 + 31, p0 + d)) return 0xFFFFFFFFu;
  uint32_t res = 0u;
  const uint32_t left = bits32(row, p0) & 0x7FFFFFFFu;       // cell p0+j blocks x' <= j
  if (left) res |= (2u << (31 - __clz(left))) - 1u;
  const uint32_t right = bits32(row, p0 + d) & 0x7FFFFFFFu;  // cell p0+d+j blocks x' > j
  if (right) res |= ~((2u << (__ffs(right) - 1)) - 1u);
  return res;
}

constexpr int kTestIlp = 2;  // independent run dilations per step of the exact test
constexpr int kVacIlp = 4;   // vacancy rows compared per step of the filter
// Runs a lane walks alone before the pairs still open share the warp: a
// sixth of the rotation's runs, between 8 and 20 (measured best on the
// 50- to 400-part workloads).
__device__ __forceinline__ int solo_runs(int n_runs) { return min(n_runs, min(20, max(8, n_runs / 6))); }

// Necessary condition for the rotation to fit with its top row at ty: the
// plate rows it covers have free runs at least as long as the mask rows'
// longest runs (numba_utils.py:50-94).  The first kVacRows rows of the
// collision-test order (widest row, then coarse to fine from the bottom)
// are checked, kVacIlp per step so their loads overlap: a candidate
// that fails the filter fails within them almost always, and one that slips
// through is rejected by the exact test (24 rows measured 1 % faster than
// 32 on the 100- to 400-part workloads, 16 rows up to 3.5 % slower).
constexpr int kVacRows = 24;
__device__ __forceinline__ bool vacancy_ok(const uint16_t* vac, int ty, const RotDev& rd,
                                           const uint32_t* vtest) {
  const uint32_t* v = vtest + rd.vt;
  const uint16_t* row = vac + ty;
  const int h = min(rd.h, kVacRows);
  int i = 0;
  for (; i + kVacIlp <= h; i += kVacIlp) {
    bool bad = false;
#pragma unroll
    for (int u = 0; u < kVacIlp; ++u) {
      const uint32_t e = __ldg(v + i + u);
      bad |= row[e >> 16] < (e & 0xFFFFu);
    }
    if (bad) return false;
  }
  for (; i < h; ++i) {
    const uint32_t e = __ldg(v + i);
    if (row[e >> 16] < (e & 0xFFFFu)) return false;
  }
  return true;
}

// The bits of F (candidate columns base .. base + 31) at which the rotation
// fits with its top row at plate row g0: every run of ones of the mask, in
// collision-test order (widest row, then the rows coarse to fine from the
// bottom), clears the columns it would overlap; kTestIlp independent
// runs per step, stop when F is empty.
__device__ __forceinline__ uint32_t word_free(const uint32_t* g0, int RS, int base, uint32_t F, const RotDev& rd,
                                              const uint2* truns) {
  const uint2* e = truns + rd.trun;
  const int n = rd.ntrun;
  int q = 0;
  for (; q + kTestIlp <= n && F; q += kTestIlp) {
    uint32_t bl = 0u;
#pragma unroll
    for (int u = 0; u < kTestIlp; ++u) {
      const uint2 r = __ldg(e + q + u);
      bl |= blocked(g0 + (int)r.y * RS, base + (int)(r.x & 0xFFFFu), (int)(r.x >> 16));
    }
    F &= ~bl;
  }
  for (; q < n && F; ++q) {
    const uint2 r = __ldg(e + q);
    F &= ~blocked(g0 + (int)r.y * RS, base + (int)(r.x & 0xFFFFu), (int)(r.x >> 16));
  }
  return F;
}

// Leftmost x at which the rotation fits with its top row at ty, or -1
// (output words of 32 candidate columns tried left to right).
__device__ __forceinline__ int first_free_x(const uint32_t* grid, int RS, int W, int ty, const RotDev& rd,
                                            const uint2* truns) {
  const int nx = W - rd.w + 1;
  const int nwo = (nx + 31) >> 5;
  const uint32_t* g0 = grid + (size_t)ty * RS;
  for (int k = 0; k < nwo; ++k) {
    const uint32_t F0 = (k == nwo - 1 && (nx & 31)) ? ((1u << (nx & 31)) - 1u) : 0xFFFFFFFFu;
    const uint32_t F = word_free(g0, RS, k << 5, F0, rd, truns);
    if (F) return (k << 5) + __ffs(F) - 1;
  }
  return -1;
}

// Longest run of ones in x, branch-free: p_s marks the starts of runs of at
// least s ones (s = 1, 2, 4, 8, 16); descending, cur marks the starts of runs
// of at least n + s ones when cur & (p_s >> n) is not empty.
__device__ __forceinline__ int longest_ones(uint32_t x) {
  if (x == 0xFFFFFFFFu) return 32;
  const uint32_t p1 = x, p2 = p1 & (p1 >> 1), p4 = p2 & (p2 >> 2), p8 = p4 & (p4 >> 4), p16 = p8 & (p8 >> 8);
  const uint32_t p[5] = {p16, p8, p4, p2, p1};
  uint32_t cur = 0xFFFFFFFFu;
  int n = 0;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const uint32_t c = cur & (p[i] >> n);
    if (c) {
      cur = c;
      n += 16 >> i;
    }
  }
  return n;
}

// longest run of empty cells in a plate row (numba_utils.py:160-188)
__device__ int max_zero_run(const uint32_t* row, int W, int NW) {
  int run = 0, best = 0;
  for (int w = 0; w < NW; ++w) {
    uint32_t v = row[w];
    const int valid = W - 32 * w;
    if (valid < 32) v |= 0xFFFFFFFFu << valid;
    if (v == 0u) {
      run += 32;
      continue;
    }
    const int tz = __ffs(v) - 1;
    run += tz;
    best = max(best, run);
    const int hb = 31 - __clz(v);
    if (hb > tz + 1) best = max(best, longest_ones(~v & ((1u << hb) - 1u) & ~((2u << tz) - 1u)));
    run = __clz(v);
  }
  return max(best, run);
}

__device__ __forceinline__ void raise_status(int32_t* status, int code) {
  atomicCAS(status, 0, code);
}

// The window a (candidate, output word) pair of the exact test reads: plate
// rows row0 .. row0 + h - 1 and, in each, the words that the dilations of the
// mask's runs touch for the 32 columns base .. base + 31 — at most word
// ((base + w + 31) >> 5) + 1 (a run starts at s >= 0 with s + d <= w, a table
// invariant of the rotation's run list).  Checked once per pair, so the runs
// inside need no check of their own.
__device__ __forceinline__ bool pair_in_plate(int row0, int base, const RotDev& rd, const MachDev& md) {
  return row0 >= 0 && row0 + rd.h <= md.L && base >= 0 && ((base + rd.w + 31) >> 5) + 1 < md.RS;
}

// Instance of a launch row / item: the last instance starting at or before v
// (instances with no rows share their start with the next one, which wins).
__device__ __forceinline__ int inst_of_row(const Run& run, int v) {
  int lo = 0, hi = run.K - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (run.r[mid].crow0 <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int inst_of_item(const Run& run, int v) {
  int lo = 0, hi = run.K - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (run.r[mid].item0 <= v) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// ---------------------------------------------------------------- kernels

__global__ void assign_sort_kernel(const __grid_constant__ Tables tb, const __grid_constant__ Run run) {
  extern __shared__ unsigned long long keys[];
  __shared__ int s_cnt[kMaxMachines + 1];
  __shared__ int s_start[kMaxMachines + 1];
  __shared__ int s_inf;
  const int row = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const int k = inst_of_row(run, row);
  const InstRun& ir = run.r[k];
  const InstDev id = tb.inst[k];
  const int N = id.N, M = id.M, S2 = ir.S2, c = row - ir.crow0;
  if (row == 0)
    for (int i = tid; i < kCritSlots; i += nt) run.crit[i] = 0;
  if (row == 0 && tid == 0) {
    *run.item_ctr = 0u;
    *run.pool_ctr = 0u;
    run.counters[0] = run.counters[1] = run.counters[2] = run.counters[3] = 0ull;
    *run.status = 0;
  }
  for (int i = tid; i <= M; i += nt) s_cnt[i] = 0;
  if (tid == 0) s_inf = 0;
  __syncthreads();
  const float* ch = run.chrom + ir.chrom_off + (long long)c * 2 * N;
  const double* thr = tb.thr + id.thrbase;
  for (int i = tid; i < S2; i += nt) {
    unsigned long long key = ~0ull;
    if (i < N) {
      const int m = machine_of(ch[N + i], thr, M, id.mode);
      atomicAdd(&s_cnt[m], 1);
      const int t = tb.gene_type[id.gbase + i] - id.tbase;
      if (m < M && !tb.fits[id.tmbase + t * M + m]) s_inf = 1;  // placement.py:47-53
      key = ((unsigned long long)m << 48) | ((unsigned long long)ordered_bits(ch[i]) << 16) |
            (unsigned long long)i;
    }
    keys[i] = key;
  }
  __syncthreads();
  for (int kk = 2; kk <= S2; kk <<= 1) {
    for (int j = kk >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < S2; i += nt) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = keys[i], b = keys[ixj];
          const bool up = (i & kk) == 0;
          if ((a > b) == up) {
            keys[i] = b;
            keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  if (tid == 0) {
    int acc = 0;
    for (int m = 0; m < M; ++m) {
      s_start[m] = acc;
      acc += s_cnt[m];
    }
  }
  __syncthreads();
  uint16_t* seq = run.seq + ir.seq0 + (long long)c * M * N;
  for (int i = tid; i < N; i += nt) {
    const unsigned long long key = keys[i];
    const int m = (int)(key >> 48);
    if (m < M) seq[(long long)m * N + (i - s_start[m])] = (uint16_t)(key & 0xFFFFu);
  }
  for (int m = tid; m < M; m += nt) run.cnt[ir.item0 + c * M + m] = s_cnt[m];
  if (tid == 0) run.infeas[row] = s_inf;
}

// Weight of an item for the longest-first order: its part count, 0 when the
// chromosome is infeasible (nothing to decode).
__device__ __forceinline__ int item_weight(const Tables& tb, const Run& run, int item) {
  const int k = inst_of_item(run, item);
  const int row = run.r[k].crow0 + (item - run.r[k].item0) / tb.inst[k].M;
  return run.infeas[row] ? 0 : run.cnt[item];
}

// Items of all instances in decreasing part count: the persistent CTAs pull
// them in this order, so the longest decodes start first.
__global__ void order_items_kernel(const __grid_constant__ Tables tb, const __grid_constant__ Run run) {
  extern __shared__ int start[];  // Nmax + 1 weights
  const int tid = threadIdx.x, nt = blockDim.x, Nw = run.Nmax;
  for (int i = tid; i <= Nw; i += nt) start[i] = 0;
  __syncthreads();
  for (int i = tid; i < run.n_items; i += nt) atomicAdd(&start[item_weight(tb, run, i)], 1);
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int w = Nw; w >= 0; --w) {
      const int h = start[w];
      start[w] = acc;
      acc += h;
    }
  }
  __syncthreads();
  for (int i = tid; i < run.n_items; i += nt) run.order[atomicAdd(&start[item_weight(tb, run, i)], 1)] = i;
}

// Shared state of one CTA-cooperative plate search.
struct SearchShared {
  unsigned long long best;
  int chunk, total, nr;
  int rlist[4];
  int rh[4];      // heights of the rotations in rlist
  RotDev rd[4];   // their descriptors, read by every chunk
  unsigned char surv[kMaxItemWarps][32];  // per warp: lanes whose candidate passed the vacancy filter
};

// Best placement key of part type t (absolute) on one plate (kKeyNone if it
// does not fit): the CTA's warps pull (rotation, 32 candidate top rows)
// chunks from a shared counter (rotations interleaved, bottom rows first),
// skip chunks that cannot beat the best key found so far, stop once no
// rotation can at the current level, and merge with atomicMin.  Called by
// all threads of the CTA; contains __syncthreads.
__device__ __forceinline__ unsigned long long search_plate(const Tables& tb, const MachDev& md,
                                                           const uint32_t* grid, const uint16_t* vac, int enc,
                                                           int t, const RotList* rlp, int task_max, int32_t* status,
                                                           SearchShared& sh,
                                                           unsigned long long& c_tests,
                                                           unsigned long long& c_chunks,
                                                           unsigned long long& c_bytes) {
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid < 4) {  // one thread per rotation: the list was built at problem creation
    const int nr0 = rlp->nr;
    // With fewer than four warps a level's chunks are taken one after another:
    // the shortest rotation first has the smallest best-case key and prunes
    // the others sooner (measured 4.5 % off the 2-warp P200M6 launch; with
    // four warps every rotation of a level starts at once and the order only
    // cost time).
    if (tid < nr0) {
      const int r = blockDim.x < 128 ? rlp->rs[tid] : rlp->r[tid];
      const RotDev rd = tb.rot[t * 4 + r];
      sh.rlist[tid] = r;
      sh.rh[tid] = rd.h;
      sh.rd[tid] = rd;
    }
    if (tid == 0) {
      sh.nr = nr0;
      sh.total = nr0 ? nr0 * ((md.L - rlp->hmin + 1 + 31) >> 5) : 0;
      sh.best = kKeyNone;
      sh.chunk = 0;
      c_tests += nr0;
      c_bytes += 4ull * rlp->scan_words;
    }
  }
  __syncthreads();
  const int nr = sh.nr, total = sh.total;
  for (int guard = 0; guard < total; ++guard) {
    int ci = 0;
    if (lane == 0) ci = atomicAdd(&sh.chunk, 1);
    ci = __shfl_sync(kFull, ci, 0);
    if (ci >= total) break;
    const int level = nr == 4 ? ci >> 2 : nr == 2 ? ci >> 1 : nr == 1 ? ci : ci / 3;
    const int slot = ci - level * nr;
    const int r = sh.rlist[slot];
    const RotDev rd = sh.rd[slot];
    const int ty_hi = md.L - rd.h - 32 * level;
    if (ty_hi < 0) continue;
    unsigned long long cur = 0;
    if (lane == 0) cur = *(volatile unsigned long long*)&sh.best;
    cur = __shfl_sync(kFull, cur, 0);
    if (key_of(max(enc, md.L - ty_hi), ty_hi + rd.h - 1, 0, r) >= cur) {
      // The best key a chunk can give only grows with its level, and the best
      // found only shrinks: when no rotation can beat it at this level, no
      // later chunk (same level or higher) can, and the warp is done.
      bool beat = false;
      for (int j = 0; j < nr; ++j) {
        const int tyj = md.L - sh.rh[j] - 32 * level;
        beat |= tyj >= 0 && key_of(max(enc, md.L - tyj), tyj + sh.rh[j] - 1, 0, sh.rlist[j]) < cur;
      }
      if (!beat) break;
      continue;
    }
    const int ty = ty_hi - lane;
    if (lane == 0) ++c_chunks;
    // Vacancy filter one candidate per lane.  Then, when there are few enough
    // (survivor, output word) pairs, they are dealt to the lanes in rounds of
    // 32, bottom-most survivor and leftmost word first, so lanes whose
    // candidate failed the filter take part in the exact test of the others;
    // in a round each lane first walks a few runs of its pair alone, then the
    // pairs still open are finished by the whole warp in order, and the first
    // pair with a free column is the bottom-most candidate's leftmost x.
    // Otherwise each lane tests its own candidate's words left to right.
    const bool pass = ty >= 0 && vacancy_ok(vac, ty, rd, tb.vtest);
    const unsigned S = __ballot_sync(kFull, pass);
    if (!S) continue;
    const int nx = md.W - rd.w + 1, nwo = (nx + 31) >> 5;
    const int ntask = __popc(S) * nwo;
    if (ntask <= task_max) {
      unsigned char* surv = sh.surv[tid >> 5];
      if (pass) surv[__popc(S & ((1u << lane) - 1u))] = (unsigned char)lane;
      __syncwarp();
      const uint32_t Flast = (nx & 31) ? ((1u << (nx & 31)) - 1u) : kFull;
      const uint2* runs = tb.truns + rd.trun;
      const int n_runs = rd.ntrun, qsolo = solo_runs(n_runs);
      for (int t0 = 0; t0 < ntask; t0 += 32) {
        {  // the round's first pair has the smallest key left in the chunk: stop when it cannot win
          unsigned long long cur = 0;
          if (lane == 0) cur = *(volatile unsigned long long*)&sh.best;
          cur = __shfl_sync(kFull, cur, 0);
          const int si0 = t0 / nwo, k0 = t0 - si0 * nwo;
          const int ty0 = ty_hi - surv[si0];
          if (key_of(max(enc, md.L - ty0), ty0 + rd.h - 1, k0 << 5, r) >= cur) break;
        }
        // Solo phase: each lane walks the first runs of its own pair, two per
        // step; most blocked words close within them.
        const int t = t0 + lane;
        uint32_t F = 0u;
        int k = 0, sl = 0, q = 0;
        if (t < ntask) {
          const int si = t / nwo;
          k = t - si * nwo;
          sl = surv[si];
          F = k == nwo - 1 ? Flast : kFull;
          const int row0 = ty_hi - sl, base = k << 5;
          if (!pair_in_plate(row0, base, rd, md)) {  // never on consistent tables: skip the pair, flag the launch
            raise_status(status, BRKGA_ERR_INTERNAL);
            F = 0u;
          }
          const uint32_t* g0 = grid + (size_t)row0 * md.RS;
          for (; q < qsolo && F; q += 2) {
            const uint2 e0 = __ldg(runs + q);
            uint32_t bl = blocked(g0 + (int)e0.y * md.RS, base + (int)(e0.x & 0xFFFFu), (int)(e0.x >> 16));
            if (q + 1 < qsolo) {
              const uint2 e1 = __ldg(runs + q + 1);
              bl |= blocked(g0 + (int)e1.y * md.RS, base + (int)(e1.x & 0xFFFFu), (int)(e1.x >> 16));
            }
            F &= ~bl;
          }
          q = min(q, qsolo);
        }
        // Shared phase: a pair with runs left and columns open is walked by the
        // whole warp, in task order, up to the first pair already proven free
        // (pairs after it cannot win): every lane takes every 32nd remaining
        // run on its own, then the lanes AND their open columns.  The first
        // pair that stays free is the bottom-most candidate's leftmost x.
        const unsigned open = __ballot_sync(kFull, F != 0u && q < n_runs);
        const unsigned done_free = __ballot_sync(kFull, F != 0u && q >= n_runs);
        unsigned rem = open & (done_free ? ((done_free & (0u - done_free)) - 1u) : kFull);
        int win = done_free ? __ffs(done_free) - 1 : -1;
        uint32_t Fw = __shfl_sync(kFull, F, win < 0 ? 0 : win);
        while (rem) {
          const int l = __ffs(rem) - 1;
          rem &= rem - 1u;
          uint32_t Fp = __shfl_sync(kFull, F, l);
          const int ql = __shfl_sync(kFull, q, l);
          const int kl = __shfl_sync(kFull, k, l);
          const int sll = __shfl_sync(kFull, sl, l);
          const int row0 = ty_hi - sll, base = kl << 5;
          {  // pairs come in key order: stop when this one cannot beat the best found
            unsigned long long cur = 0;
            if (lane == 0) cur = *(volatile unsigned long long*)&sh.best;
            cur = __shfl_sync(kFull, cur, 0);
            if (key_of(max(enc, md.L - row0), row0 + rd.h - 1, base + __ffs(Fp) - 1, r) >= cur) {
              win = -1;
              break;
            }
          }
          if (!pair_in_plate(row0, base, rd, md)) {  // warp-uniform: the pair's values came from shuffles
            if (lane == 0) raise_status(status, BRKGA_ERR_INTERNAL);
            continue;
          }
          const uint32_t* g0 = grid + (size_t)row0 * md.RS;
          for (int qq = ql + lane; qq < n_runs && Fp; qq += 32) {
            const uint2 e = __ldg(runs + qq);
            Fp &= ~blocked(g0 + (int)e.y * md.RS, base + (int)(e.x & 0xFFFFu), (int)(e.x >> 16));
          }
          for (int o = 1; o < 32; o <<= 1) Fp &= __shfl_xor_sync(kFull, Fp, o);
          if (Fp) {
            win = l;
            Fw = Fp;
            break;
          }
        }
        if (win >= 0) {
          const int kb = __shfl_sync(kFull, k, win);
          const int slb = __shfl_sync(kFull, sl, win);
          if (lane == 0) {
            const int tyb = ty_hi - slb;
            atomicMin(&sh.best, key_of(max(enc, md.L - tyb), tyb + rd.h - 1, (kb << 5) + __ffs(Fw) - 1, r));
          }
          break;
        }
      }
      __syncwarp();
    } else {
      const int x = pass ? first_free_x(grid, md.RS, md.W, ty, rd, tb.truns) : -1;
      const unsigned fm = __ballot_sync(kFull, x >= 0);
      if (fm) {
        const int l = __ffs(fm) - 1;
        const int xb = __shfl_sync(kFull, x, l);
        if (lane == 0) {
          const int tyb = ty_hi - l;
          atomicMin(&sh.best, key_of(max(enc, md.L - tyb), tyb + rd.h - 1, xb, r));
        }
      }
    }
  }
  __syncthreads();
  return sh.best;
}

// Insert rotation r of part type t (absolute) with its top row at ty and left
// column x (binClassNew.py:155-174): OR the mask rows into the plate words,
// recompute the vacancy of the touched rows (numba_utils.py:160-188); thread 0
// updates the plate scalars with the part's area and times on this machine.
// One thread per mask row does both the OR of its row and that plate row's
// vacancy (a plate row is touched by one mask row only), so no barrier
// separates them.  All threads of the CTA; ends with __syncthreads.
__device__ __forceinline__ void place_part(const Tables& tb, const MachDev& md, uint32_t* grid, uint16_t* vac,
                                           BinScal* scal, int t, int r, int x, int ty, double a, double ptv,
                                           double pthv) {
  const int tid = threadIdx.x;
  const RotDev rd = tb.rot[t * 4 + r];
  const int sx = x & 31, wx = x >> 5, mw = rd.mw;
  const uint32_t* mb = tb.maskbits + rd.mask_base;
  for (int i = tid; i < rd.h; i += blockDim.x) {
    uint32_t* row = grid + (size_t)(ty + i) * md.RS;
    const uint32_t* m = mb + (size_t)i * mw;
    uint32_t* dst = row + wx;
    if (mw <= 8) {  // all loads first, so their latencies overlap
      uint32_t w[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) w[j] = j < mw ? __ldg(m + j) : 0u;
      uint32_t prev = 0u;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (j < mw) {
          const uint32_t v = __funnelshift_l(prev, w[j], sx);
          if (v) dst[j] |= v;
          prev = w[j];
        }
      }
      const uint32_t v = __funnelshift_l(prev, 0u, sx);
      if (v) dst[mw] |= v;
    } else {
      uint32_t prev = 0u;
      for (int j = 0; j < mw; ++j) {
        const uint32_t cur = __ldg(m + j);
        const uint32_t v = __funnelshift_l(prev, cur, sx);
        if (v) dst[j] |= v;
        prev = cur;
      }
      const uint32_t v = __funnelshift_l(prev, 0u, sx);
      if (v) dst[mw] |= v;
    }
    vac[ty + i] = (uint16_t)max_zero_run(row, md.W, md.NW);
  }
  if (tid == 0) {
    BinScal s = *scal;
    s.area += a;
    s.minrow = min(s.minrow, ty);
    s.maxrow = max(s.maxrow, ty + rd.h - 1);
    s.enc = (s.minrow > s.maxrow) ? 0 : md.L - s.minrow;  // binClassNew.py:147-152
    s.pt += ptv;
    if (pthv > s.pth) s.pth = pthv;
    *scal = s;
  }
  __syncthreads();
}

// Empty plate: zero words, vacancy W (binClassNew.py:18-20), fresh scalars.
__device__ __forceinline__ void open_plate(const MachDev& md, uint32_t* grid, uint16_t* vac, BinScal* scal,
                                           int pool_index) {
  const int tid = threadIdx.x;
  for (int i = tid; i < md.L * md.RS; i += blockDim.x) grid[i] = 0u;
  for (int i = tid; i < md.L; i += blockDim.x) vac[i] = (uint16_t)md.W;
  if (tid == 0) {
    BinScal z;
    z.area = 0.0;
    z.pt = 0.0;
    z.pth = 0.0;
    z.minrow = md.L;
    z.maxrow = -1;
    z.enc = 0;
    z.pool = pool_index;
    *scal = z;
  }
  __syncthreads();
}

__device__ __forceinline__ void decode_key(unsigned long long key, int* r, int* x, int* y) {
  *r = (int)(key & 3ull);
  *x = (int)((key >> 2) & 0x1FFFull);
  *y = kMaxSide - (int)((key >> 15) & 0x1FFFull);
}

// The item a CTA is decoding, set up by thread 0.
struct ItemCtx {
  int item;      // global item index, -1 when the queue is empty
  int row;       // chromosome row of the launch
  int m, M, T;   // machine (local), machines and part types of the instance
  int n;         // parts on this machine
  int N;         // genes of the instance (log entries per item)
  int gbase, tbase, tmbase;
  int infeas;
  long long seq; // first entry of its part order / log
  MachDev md;
};

// The tables go by value (every access has a fixed parameter offset); only
// the per-launch instance array, which is searched, is a grid constant.
// kThreads = 32, 64 or 128 (1, 2 or 4 warps per item); 32 resident warps
// per SM cap the kernel at 64 registers, which it fits without spilling.
template <int kThreads>
__global__ void __launch_bounds__(kThreads, kResidentWarps * 32 / kThreads)
    decode_kernel(const Tables tb, const __grid_constant__ Run run) {
  extern __shared__ __align__(16) uint32_t smem[];
  // Two search states, used by alternate searches: the state a search returns
  // from is not written again until the search after next, by which time every
  // thread has passed the next search's barriers — so a search needs no
  // barrier after reading its result.
  __shared__ SearchShared sh2[2];
  __shared__ ItemCtx ctx;
  int sh_par = 0;
  __shared__ int s_fail, s_pool;
  const int tid = threadIdx.x, lane = tid & 31;
  BinScal* bs = run.binscal + (size_t)blockIdx.x * run.Nmax;
  unsigned long long c_tests = 0, c_chunks = 0, c_bins = 0, c_bytes = 0;
  unsigned my_sm = 0;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(my_sm));
  my_sm &= (unsigned)(kCritSlots - 1);
  bool crit = false;  // thread 0: this CTA holds a critical item and marked its SM

  for (;;) {
    if (tid == 0) {
      if (crit) {
        atomicSub(&run.crit[my_sm], 1);
        crit = false;
      }
      ctx.item = -1;
      // While another CTA of this SM decodes a critical item, take none: the
      // CTA that holds the mark keeps pulling, so every item is still taken.
      const bool leave = run.crit_items > 0 && *(volatile int*)&run.crit[my_sm] > 0;
      const int q = leave ? run.n_items : (int)atomicAdd(run.item_ctr, 1u);
      if (q < run.crit_items && q < run.n_items) {
        crit = true;
        atomicAdd(&run.crit[my_sm], 1);
      }
      if (q < run.n_items) {
        const int item = run.order[q];
        const int k = inst_of_item(run, item);
        const InstDev id = tb.inst[k];
        const int li = item - run.r[k].item0, c = li / id.M;
        ctx.item = item;
        ctx.row = run.r[k].crow0 + c;
        ctx.m = li - c * id.M;
        ctx.M = id.M;
        ctx.T = id.T;
        ctx.n = run.cnt[item];
        ctx.N = id.N;
        ctx.gbase = id.gbase;
        ctx.tbase = id.tbase;
        ctx.tmbase = id.tmbase;
        ctx.infeas = run.infeas[ctx.row];
        ctx.seq = run.r[k].seq0 + (long long)li * id.N;
        ctx.md = tb.mach[id.mbase + ctx.m];
      }
    }
    __syncthreads();
    const int item = ctx.item;
    if (item < 0) break;
    const MachDev md = ctx.md;
    const int n = ctx.n;
    BrkgaPlacement* lg = run.log ? run.log + ctx.seq : nullptr;
    const uint16_t* seq = run.seq + ctx.seq;
    const int N = ctx.N;
    if (ctx.infeas) {  // any part too large for its machine: the whole chromosome scores 1e16
      if (lg)
        for (int k = tid; k < N; k += kThreads) lg[k] = BrkgaPlacement{-1, -1, -1, -1, -1};
      if (tid == 0) run.mk[item] = 0.0;
      __syncthreads();
      continue;
    }
    if (lg)
      for (int k = n + tid; k < N; k += kThreads) lg[k] = BrkgaPlacement{-1, -1, -1, -1, -1};

    int nb = 0;
    bool failed = false;
    for (int k = 0; k < n && !failed; ++k) {
      const int gene = seq[k];
      const int t = tb.gene_type[ctx.gbase + gene];
      const double a = tb.part_area[t];
      int pb = -1;
      unsigned long long key = kKeyNone;

      // ---- first fit over the open plates (placement.py:56-64)
      for (int b = 0; b < nb; ++b) {
        if (bs[b].area + a > md.area) continue;  // placement.py:57-59
        const uint32_t* grid = b < run.S ? smem + (size_t)b * run.slot_words
                                         : run.pool + (size_t)bs[b].pool * run.slot_words;
        const uint16_t* vac = reinterpret_cast<const uint16_t*>(grid + run.slot_vac_off);
        key = search_plate(tb, md, grid, vac, bs[b].enc, t,
                           tb.rl + ctx.tmbase + (size_t)(t - ctx.tbase) * ctx.M + ctx.m, run.task_max, run.status,
                           sh2[sh_par], c_tests,
                           c_chunks, c_bytes);
        sh_par ^= 1;
        if (key != kKeyNone) {
          pb = b;
          break;
        }
      }

      int r, x, ty;
      if (pb < 0) {
        // ---- new plate, best rotation at column 0, bottom row L-1 (placement.py:66-83)
        r = tb.best_rot[t];
        if (tid == 0) {
          s_fail = 0;
          s_pool = -1;
          if (!tb.newbin_ok[ctx.tmbase + (t - ctx.tbase) * ctx.M + ctx.m]) {
            s_fail = BRKGA_ERR_NEW_BIN_UNFIT;
          } else if (nb >= run.S) {
            const unsigned idx = atomicAdd(run.pool_ctr, 1u);
            if ((long long)idx >= run.pool_bins) s_fail = BRKGA_ERR_CAPACITY;
            else s_pool = (int)idx;
          }
        }
        __syncthreads();
        if (s_fail) {
          if (tid == 0) {
            raise_status(run.status, s_fail);
            run.mk[item] = nan("");
          }
          failed = true;
          break;
        }
        pb = nb++;
        uint32_t* grid = pb < run.S ? smem + (size_t)pb * run.slot_words : run.pool + (size_t)s_pool * run.slot_words;
        open_plate(md, grid, reinterpret_cast<uint16_t*>(grid + run.slot_vac_off), &bs[pb], s_pool);
        if (tid == 0) ++c_bins;
        x = 0;
        ty = md.L - tb.rot[t * 4 + r].h;
      } else {
        int y;
        decode_key(key, &r, &x, &y);
        ty = y - tb.rot[t * 4 + r].h + 1;
      }

      // ---- insert (binClassNew.py:155-174)
      uint32_t* grid = pb < run.S ? smem + (size_t)pb * run.slot_words : run.pool + (size_t)bs[pb].pool * run.slot_words;
      const size_t tm = (size_t)ctx.tmbase + (size_t)ctx.m * ctx.T + (t - ctx.tbase);
      place_part(tb, md, grid, reinterpret_cast<uint16_t*>(grid + run.slot_vac_off), &bs[pb], t, r, x, ty, a,
                 tb.pt[tm], tb.pth[tm]);
      if (tid == 0 && lg) lg[k] = BrkgaPlacement{gene, pb, x, ty + tb.rot[t * 4 + r].h - 1, r};
    }
    if (!failed && tid == 0) {  // placement.py:86-89
      double ms = 0.0;
      for (int b = 0; b < nb; ++b) ms += (bs[b].pt + bs[b].pth) + md.setup;
      run.mk[item] = ms;
    }
    __syncthreads();
  }
  if (tid == 0) {
    atomicAdd(&run.counters[0], c_tests);
    atomicAdd(&run.counters[2], c_bins);
    atomicAdd(&run.counters[3], c_bytes);
  }
  if (lane == 0) atomicAdd(&run.counters[1], c_chunks);
}

__global__ void reduce_kernel(const __grid_constant__ Tables tb, const __grid_constant__ Run run) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= run.n_rows) return;
  const int k = inst_of_row(run, row);
  double* out = run.out + run.r[k].out_off + (row - run.r[k].crow0);
  if (run.infeas[row]) {
    *out = 1e16;  // placement.py:9,151-153
    return;
  }
  const int M = tb.inst[k].M;
  const double* mk = run.mk + run.r[k].item0 + (long long)(row - run.r[k].crow0) * M;
  double worst = 0.0;
  bool bad = false;
  for (int m = 0; m < M; ++m) {
    const double v = mk[m];
    if (v != v) bad = true;
    else if (v > worst) worst = v;  // placement.py:154-156
  }
  *out = bad ? nan("") : worst;
}

// Greedy initial solution (BRKGA_alg3.py:445-603 with binClassInitialSol.py):
// one CTA walks the parts in the given order; each part goes where the
// system makespan after placing it is smallest (ties: the later option wins
// over an earlier one on another machine or a new plate, the first existing
// plate wins within a machine): a new plate on some machine (best rotation at
// column 0, bottom row L-1) or any existing plate of the machine that can take
// it (every plate is tested, no area filter).  Plates live in the global pool.
// Single-instance problems only, so every table base is 0.
struct GreedyArgs {
  int N, M, T;
  int32_t* status;
  unsigned long long* counters;
  BinScal* binscal;
  uint32_t* pool;
  int slot_words, slot_vac_off;
  const int32_t* order;
  int n;
  int32_t* out_machine;  // [n]
  BrkgaPlacement* out;   // [n]: gene, plate index within its machine, x, bottom row y, rotation
  int32_t* plate_machine;
  int32_t* plate_index;  // index of the plate within its machine
  double* machine_makespan;  // [M]
};

__global__ void __launch_bounds__(kGreedyThreads) greedy_kernel(const __grid_constant__ Tables tb,
                                                                const __grid_constant__ GreedyArgs g) {
  __shared__ SearchShared sh2[2];  // alternate searches, as in decode_kernel
  __shared__ int s_fail;
  int sh_par = 0;
  const int tid = threadIdx.x;
  BinScal* bs = g.binscal;
  unsigned long long c_tests = 0, c_chunks = 0, c_bytes = 0;
  int nplates = 0;
  double cw = 0.0;  // current_worst_makespan
  for (int m = tid; m < g.M; m += kGreedyThreads) g.machine_makespan[m] = 0.0;
  __syncthreads();
  for (int k = 0; k < g.n; ++k) {
    const int gene = g.order[k];
    const int t = tb.gene_type[gene];
    const double a = tb.part_area[t];
    double best = INFINITY;
    int kind = -1, cm = -1, cb = -1;  // kind 0 = new plate, 1 = existing plate
    unsigned long long ckey = kKeyNone;
    double ccand = 0.0;
    for (int m = 0; m < g.M; ++m) {
      bool placed_in_exist = false;
      if (!tb.fits[t * g.M + m]) continue;  // BRKGA_alg3.py:465-470
      const MachDev md = tb.mach[m];
      const double mm = g.machine_makespan[m];
      const double ptm = tb.pt[(size_t)m * g.T + t], pthm = tb.pth[(size_t)m * g.T + t];
      const double cand = ((mm + md.setup) + ptm) + pthm;  // :472
      const double nm = cw > cand ? cw : cand;
      if (nm <= best) {
        best = nm;
        kind = 0;
        cm = m;
        ccand = cand;
      }
      for (int b = 0; b < nplates; ++b) {
        if (g.plate_machine[b] != m) continue;
        const uint32_t* grid = g.pool + (size_t)bs[b].pool * g.slot_words;
        const unsigned long long key =
            search_plate(tb, md, grid, reinterpret_cast<const uint16_t*>(grid + g.slot_vac_off), bs[b].enc, t,
                         tb.rl + (size_t)t * g.M + m, kDefaultTaskMax, g.status, sh2[sh_par], c_tests, c_chunks,
                         c_bytes);
        sh_par ^= 1;
        if (key == kKeyNone) continue;
        const double bpth = bs[b].pth;
        const double cand2 = bpth < pthm ? ((mm - bpth) + pthm) + ptm : mm + ptm;  // :486-489
        const double nm2 = cw > cand2 ? cw : cand2;
        if (nm2 <= best) {
          if (placed_in_exist && nm2 == best) continue;
          placed_in_exist = true;
          best = nm2;
          kind = 1;
          cm = m;
          cb = b;
          ckey = key;
          ccand = cand2;
        }
      }
    }
    if (kind < 0) {  // fits no machine: the reference crashes here (bestBatch == [])
      if (tid == 0) raise_status(g.status, BRKGA_ERR_BAD_INSTANCE);
      return;
    }
    const MachDev md = tb.mach[cm];
    int r, x, ty, b;
    if (kind == 0) {
      r = tb.best_rot[t];
      if (tid == 0) s_fail = (!tb.newbin_ok[t * g.M + cm] || nplates >= g.n) ? 1 : 0;
      __syncthreads();
      if (s_fail) {
        if (tid == 0) raise_status(g.status, BRKGA_ERR_NEW_BIN_UNFIT);
        return;
      }
      b = nplates++;
      uint32_t* grid = g.pool + (size_t)b * g.slot_words;
      open_plate(md, grid, reinterpret_cast<uint16_t*>(grid + g.slot_vac_off), &bs[b], b);
      if (tid == 0) {
        int idx = 0;
        for (int q = 0; q < b; ++q) idx += g.plate_machine[q] == cm;
        g.plate_machine[b] = cm;
        g.plate_index[b] = idx;
      }
      x = 0;
      ty = md.L - tb.rot[t * 4 + r].h;
    } else {
      int y;
      decode_key(ckey, &r, &x, &y);
      ty = y - tb.rot[t * 4 + r].h + 1;
      b = cb;
    }
    uint32_t* grid = g.pool + (size_t)bs[b].pool * g.slot_words;
    place_part(tb, md, grid, reinterpret_cast<uint16_t*>(grid + g.slot_vac_off), &bs[b], t, r, x, ty, a,
               tb.pt[(size_t)cm * g.T + t], tb.pth[(size_t)cm * g.T + t]);
    if (tid == 0) {
      g.out_machine[k] = cm;
      g.out[k] = BrkgaPlacement{gene, g.plate_index[b], x, ty + tb.rot[t * 4 + r].h - 1, r};
      g.machine_makespan[cm] = ccand;  // :541, :565
    }
    cw = cw > ccand ? cw : ccand;
    __syncthreads();
  }
  if (tid == 0) {
    atomicAdd(&g.counters[0], c_tests);
    atomicAdd(&g.counters[3], c_bytes);
  }
}

// ---------------------------------------------------------------- chunk tests
// The collision test of one 32-row candidate chunk by either path, for the
// measurement that decides between them (brkga_chunk_free): the bit-packed
// run-dilation search the decode kernel uses (word_free, every word tested
// to the end, no early stop) and the INT8 tensor-core correlation
// (corr_i8.cuh).  Both write the same words: row n = candidate top row
// ty_hi - n, bit b of word k = placement at x = 32k + b is collision-free.

// The item's plate geometry and rotation, checked against the tables; false
// (and BRKGA_ERR_INVALID_ARGUMENT raised) when the item is malformed.
__device__ __forceinline__ bool chunk_item(const Tables& tb, const BrkgaChunkTest& it, int M, int T, int max_side,
                                           corr::ChunkArgs* a, RotDev* rdo, int32_t* status) {
  bool ok = it.plate && it.out && it.machine >= 0 && it.machine < M && it.part_type >= 0 && it.part_type < T &&
            it.rot >= 0 && it.rot < tb.nrot[it.part_type];
  if (ok) {
    const MachDev md = tb.mach[it.machine];
    const RotDev rd = tb.rot[it.part_type * 4 + it.rot];
    ok = rd.h <= md.L && rd.w <= md.W && rd.h <= max_side && rd.w <= max_side && it.ty_hi >= 0 &&
         it.ty_hi <= md.L - rd.h;
    a->plate = it.plate;
    a->L = md.L;
    a->W = md.W;
    a->RS = md.RS;
    a->mask = tb.maskbits + rd.mask_base;
    a->h = rd.h;
    a->w = rd.w;
    a->mw = rd.mw;
    a->ty_hi = it.ty_hi;
    a->out = it.out;
    *rdo = rd;
  }
  if (!ok && threadIdx.x == 0 && blockIdx.y == 0) raise_status(status, BRKGA_ERR_INVALID_ARGUMENT);
  return ok;
}

__global__ void __launch_bounds__(128, 8) chunk_free_bitset_kernel(const Tables tb, const BrkgaChunkTest* items, int M,
                                                                int T, int32_t* status) {
  const BrkgaChunkTest it = items[blockIdx.x];
  corr::ChunkArgs a;
  RotDev rd;
  if (!chunk_item(tb, it, M, T, kMaxSide, &a, &rd, status)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nx = a.W - a.w + 1, nwo = (nx + 31) >> 5;
  for (int n = warp; n < corr::kN; n += 4) {
    const int ty = a.ty_hi - n;
    for (int k = lane; k < nwo; k += 32) {
      uint32_t F = 0u;
      if (ty >= 0) {
        const uint32_t F0 = (k == nwo - 1 && (nx & 31)) ? ((1u << (nx & 31)) - 1u) : kFull;
        F = word_free(a.plate + (size_t)ty * a.RS, a.RS, k << 5, F0, rd, tb.truns);
      }
      a.out[(size_t)n * nwo + k] = F;
    }
  }
}

// grid (items, candidate-column tiles of 128); one CTA per SM (its shared memory)
__global__ void __launch_bounds__(corr::kThreads, 1) chunk_free_i8_kernel(const Tables tb,
                                                                          const BrkgaChunkTest* items, int M, int T,
                                                                          int32_t* status) {
  extern __shared__ __align__(1024) unsigned char csmem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int fail;
  const BrkgaChunkTest it = items[blockIdx.x];
  corr::ChunkArgs a;
  RotDev rd;
  if (!chunk_item(tb, it, M, T, corr::kMaxSide, &a, &rd, status)) return;
  if ((int)blockIdx.y * corr::kTileM > a.W - a.w) return;  // no candidate column in this tile
  corr::chunk_tile(a, (int)blockIdx.y, csmem, bar, &tmem_slot, &fail, status);
}

// ---------------------------------------------------------------- host side

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Layout {
  size_t off_ctr, off_crit, off_seq, off_cnt, off_inf, off_ord, off_mk, off_bins, off_pool, total;
};

// Sizes of one launch: chromosome rows, (chromosome, machine) items, part-order entries.
struct LaunchCounts {
  int64_t rows = 0, items = 0, seq = 0;
};

// One launch shape of the decode kernel.
struct Shape {
  int warps = 4;     // per CTA (one item per CTA)
  int ctas = 0;      // resident CTAs per SM
  int S = 0;         // plates per item in shared memory
  size_t smem = 0;   // dynamic shared memory per CTA
  int n_slots = 0;   // resident CTAs on the GPU (the persistent grid)
};

}  // namespace

// Fixed device scratch for brkga_decode_noalloc: every GPU that loads this
// library reserves it until the process exits.  Host code must not use the
// symbol as an address; brkga_problem_create looks up its device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[BRKGA_NOALLOC_SCRATCH_BYTES];

struct BrkgaProblem {
  int device = 0;
  void* noalloc_scratch = nullptr;  // device address of g_noalloc_scratch on `device`
  int K = 0;                        // instances
  std::vector<InstDev> inst;
  std::vector<int> s2;              // bitonic sort width per instance
  int S2max = 1, Nmax = 0;
  int N = 0, M = 0, T = 0, mode = 0;  // instance 0 (the single-instance entry points)
  int sm_count = 0;
  int req_warps = 0, req_ctas = 0, req_plates = -1;  // requested launch shape (0 / 0 / -1 = automatic)
  int task_max = kDefaultTaskMax;
  Shape shape[3];      // 4, 2 and 1 warps per item
  int min_S = 0;       // fewest plates in shared memory of the three shapes (pool sizing)
  int slot_words = 0, slot_vac_off = 0;
  std::vector<MachDev> mach;
  std::vector<void*> allocations;
  Tables tb{};
  InstDev* d_inst = nullptr;
  int32_t* d_gene_type = nullptr;
  double* d_thr = nullptr;
  MachDev* d_mach = nullptr;
  double* d_pt = nullptr;
  double* d_pth = nullptr;
  double* d_area = nullptr;
  int32_t* d_nrot = nullptr;
  int32_t* d_best = nullptr;
  RotDev* d_rot = nullptr;
  uint32_t* d_vtest = nullptr;
  uint2* d_truns = nullptr;
  uint32_t* d_maskbits = nullptr;
  uint8_t* d_fits = nullptr;
  uint8_t* d_newbin_ok = nullptr;
  RotList* d_rl = nullptr;
  double* d_bin_area = nullptr;
  // brkga_evaluate_host state
  std::mutex mu;
  cudaStream_t stream = nullptr;
  float* e_chrom = nullptr;
  double* e_out = nullptr;
  int32_t* e_status = nullptr;
  BrkgaPlacement* e_log = nullptr;
  // page-locked staging of a call's results: status at 0, counters at 8,
  // makespans from 64, so the three copies back are queued without a
  // staging round trip each and waited for once
  unsigned char* e_host = nullptr;
  void* e_ws = nullptr;
  size_t e_ws_bytes = 0;
  int e_cap_P = 0;
  bool e_cap_log = false;
  int64_t e_pool_bins = 0;
  int64_t last_counters[4] = {0, 0, 0, 0};
};

namespace {

int counts_of(const BrkgaProblem* pb, const int32_t* pops, LaunchCounts* lc) {
  LaunchCounts c;
  for (int k = 0; k < pb->K; ++k) {
    if (pops[k] < 0) return BRKGA_ERR_INVALID_ARGUMENT;
    c.rows += pops[k];
    c.items += (int64_t)pops[k] * pb->inst[k].M;
    c.seq += (int64_t)pops[k] * pb->inst[k].M * pb->inst[k].N;
  }
  if (c.rows >= ((int64_t)1 << 31) || c.items >= ((int64_t)1 << 31)) return BRKGA_ERR_INVALID_ARGUMENT;
  *lc = c;
  return BRKGA_OK;
}

// The shape a launch of `items` items uses: the requested CTA size, else
// 4 warps per item while the items fill at most three waves of resident
// 4-warp CTAs (per-item latency dominates), 2 warps up to sixteen waves of
// 2-warp CTAs, 1 warp beyond (throughput dominates; no CTA barriers).
const Shape& pick_shape(const BrkgaProblem* pb, int64_t items) {
  if (pb->req_warps == 4) return pb->shape[0];
  if (pb->req_warps == 2) return pb->shape[1];
  if (pb->req_warps == 1) return pb->shape[2];
  if (items <= 3 * (int64_t)pb->shape[0].n_slots) return pb->shape[0];
  if (items <= 16 * (int64_t)pb->shape[1].n_slots) return pb->shape[1];
  return pb->shape[2];
}

// CTAs whose plate scalars the workspace of a launch of `items` items holds:
// the most resident CTAs of any shape a launch of at most `items` items can
// use, so that a workspace sized for the largest population serves every
// smaller launch too.
int scratch_slots(const BrkgaProblem* pb, int64_t items) {
  if (pb->req_warps) return pick_shape(pb, items).n_slots;
  int n = pb->shape[0].n_slots;
  if (items > 3 * (int64_t)pb->shape[0].n_slots) n = std::max(n, pb->shape[1].n_slots);
  if (items > 16 * (int64_t)pb->shape[1].n_slots) n = std::max(n, pb->shape[2].n_slots);
  return n;
}

Layout layout_of(const BrkgaProblem* pb, const LaunchCounts& lc, int64_t pool_bins) {
  Layout l;
  size_t o = 0;
  l.off_ctr = o;
  o += 64;
  l.off_crit = o = align_up(o, 256);
  o += (size_t)kCritSlots * sizeof(int);
  l.off_seq = o = align_up(o, 256);
  o += (size_t)lc.seq * sizeof(uint16_t);
  l.off_cnt = o = align_up(o, 256);
  o += (size_t)lc.items * sizeof(int32_t);
  l.off_inf = o = align_up(o, 256);
  o += (size_t)lc.rows * sizeof(int32_t);
  l.off_ord = o = align_up(o, 256);
  o += (size_t)lc.items * sizeof(int32_t);
  l.off_mk = o = align_up(o, 256);
  o += (size_t)lc.items * sizeof(double);
  l.off_bins = o = align_up(o, 256);
  o += (size_t)scratch_slots(pb, lc.items) * std::max(pb->Nmax, 1) * sizeof(BinScal);
  l.off_pool = o = align_up(o, 256);
  o += (size_t)pool_bins * pb->slot_words * sizeof(uint32_t);
  l.total = align_up(o, 256);
  return l;
}

int64_t default_pool_bins(const BrkgaProblem* pb, int64_t items) {
  return std::max<int64_t>(256, items * (pb->min_S > 0 ? 2 : 4));
}

template <typename T>
int upload(BrkgaProblem* pb, T** dst, const std::vector<T>& src) {
  const size_t bytes = std::max<size_t>(1, src.size()) * sizeof(T);
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return BRKGA_ERR_CUDA;
  pb->allocations.push_back(p);
  if (!src.empty() && cudaMemcpy(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  *dst = static_cast<T*>(p);
  return BRKGA_OK;
}

class DeviceGuard {
 public:
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev_);
    if (prev_ != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() { cudaSetDevice(prev_); }

 private:
  int prev_ = 0;
};

template <int kThreads>
int prepare_kernel(size_t dyn_max) {
  return cudaFuncSetAttribute(decode_kernel<kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn_max) ==
                 cudaSuccess
             ? BRKGA_OK
             : BRKGA_ERR_CUDA;
}

int occupancy(int warps, size_t smem, int* occ) {
  const cudaError_t e =
      warps == 1   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, decode_kernel<32>, 32, smem)
      : warps == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, decode_kernel<64>, 64, smem)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, decode_kernel<128>, 128, smem);
  return e == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

// Launch shapes of the decode kernel, one per CTA size (4, 2 and 1 warps per
// item): resident CTAs per SM and plates per item kept in shared memory.
// For the requested CTA size (warps_req), ctas_req = 0 picks the CTAs
// automatically (32 resident warps per SM, the register limit) and
// plates_req = -1 keeps as many plates as fit in their share (at most 4);
// the other CTA size, or both when warps_req = 0, gets the automatic shape.
// A requested shape that cannot be resident is refused.
int configure(BrkgaProblem* pb, int warps_req, int ctas_req, int plates_req) {
  if (warps_req == 0 && (ctas_req != 0 || plates_req != -1)) return BRKGA_ERR_INVALID_ARGUMENT;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, pb->device) != cudaSuccess) return BRKGA_ERR_CUDA;
  pb->sm_count = prop.multiProcessorCount;
  // A plate of machine m uses its own L x RS words, then L vacancy entries:
  // a slot holds the largest plate of any machine (not Lmax x RSmax, which
  // for a tall plate beside a wide one is far more than either needs).
  int Lmax = 0, slot_vac_off = 0;
  for (const MachDev& m : pb->mach) {
    Lmax = std::max(Lmax, m.L);
    slot_vac_off = std::max(slot_vac_off, m.L * m.RS);
  }
  const int slot_words = (int)align_up((size_t)slot_vac_off + (size_t)(Lmax + 1) / 2, 4);
  const size_t slot_bytes = (size_t)slot_words * 4;
  cudaFuncAttributes fa4, fa2, fa1;
  if (cudaFuncGetAttributes(&fa4, decode_kernel<128>) != cudaSuccess ||
      cudaFuncGetAttributes(&fa2, decode_kernel<64>) != cudaSuccess ||
      cudaFuncGetAttributes(&fa1, decode_kernel<32>) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  const size_t static_smem = std::max({fa4.sharedSizeBytes, fa2.sharedSizeBytes, fa1.sharedSizeBytes});
  const size_t per_sm = prop.sharedMemPerMultiprocessor;
  const size_t per_block_max = prop.sharedMemPerBlockOptin - static_smem;  // dynamic part
  const size_t reserve = 1024 + static_smem;  // per-block system reservation + static shared variables
  const int max_fit = (int)std::min<size_t>(kMaxSmemPlates, per_block_max / slot_bytes);
  int st;
  if ((st = prepare_kernel<128>(per_block_max)) || (st = prepare_kernel<64>(per_block_max)) ||
      (st = prepare_kernel<32>(per_block_max)))
    return st;
  if (cudaFuncSetAttribute(assign_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxGenes * 8) !=
      cudaSuccess)
    return BRKGA_ERR_CUDA;
  if (cudaFuncSetAttribute(order_items_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (kMaxGenes + 1) * (int)sizeof(int)) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  if (cudaFuncSetAttribute(chunk_free_i8_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           corr::smem_bytes(corr::kMaxSide, corr::kMaxSide)) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  auto fit_for = [&](int ctas) {  // plates per item that fit when `ctas` CTAs share an SM
    const size_t share = per_sm / ctas;
    if (share <= reserve) return 0;
    return (int)std::min<size_t>((share - reserve) / slot_bytes, (size_t)max_fit);
  };
  Shape shapes[3];
  for (int v = 0; v < 3; ++v) {
    const int warps = 4 >> v;
    const int auto_ctas = kResidentWarps / warps;
    const bool req = warps_req == warps;
    const int creq = req ? ctas_req : 0, preq = req ? plates_req : -1;
    int S, ctas;
    if (creq == 0) {
      ctas = auto_ctas;
      if (preq >= 0) {
        S = preq;
        while (ctas > 1 && fit_for(ctas) < S) --ctas;
        if (fit_for(ctas) < S) return BRKGA_ERR_INVALID_ARGUMENT;
      } else {
        // Resident warps matter far more than where the plates live (the
        // pool stays in L2): as many plates per item in shared memory as
        // their share holds, none for large plates.
        S = std::min(fit_for(ctas), 4);
      }
    } else {
      ctas = creq;
      S = preq >= 0 ? preq : std::min(fit_for(ctas), 4);
    }
    if (S > max_fit) return BRKGA_ERR_INVALID_ARGUMENT;
    const size_t smem = (size_t)S * slot_bytes;
    int occ = 0;
    if ((st = occupancy(warps, smem, &occ))) return st;
    if (occ < 1 || (creq > 0 && occ < creq)) return BRKGA_ERR_INVALID_ARGUMENT;
    shapes[v].warps = warps;
    shapes[v].S = S;
    shapes[v].smem = smem;
    shapes[v].ctas = std::max(1, std::min(occ, ctas));
    shapes[v].n_slots = pb->sm_count * shapes[v].ctas;
  }
  pb->slot_vac_off = slot_vac_off;
  pb->slot_words = slot_words;
  pb->min_S = shapes[0].S;
  for (int v = 0; v < 3; ++v) {
    pb->shape[v] = shapes[v];
    pb->min_S = std::min(pb->min_S, shapes[v].S);
  }
  pb->req_warps = warps_req;
  pb->req_ctas = ctas_req;
  pb->req_plates = plates_req;
  return BRKGA_OK;
}

int validate(const BrkgaProblemDesc* d) {
  if (!d) return BRKGA_ERR_INVALID_ARGUMENT;
  if (d->n_genes < 1 || d->n_genes > kMaxGenes || d->n_machines < 1 || d->n_machines > kMaxMachines ||
      d->n_types < 1 || (d->threshold_mode != BRKGA_THRESH_F32 && d->threshold_mode != BRKGA_THRESH_F64))
    return BRKGA_ERR_INVALID_ARGUMENT;
  if (!d->gene_type || (!d->thresholds && d->n_machines > 1) || !d->bin_length || !d->bin_width ||
      !d->bin_area || !d->setup_time || !d->proc_time || !d->proc_time_height || !d->part_area ||
      !d->part_nrot || !d->part_best_rot || !d->rot_h || !d->rot_w || !d->rot_mask_offset || !d->masks)
    return BRKGA_ERR_INVALID_ARGUMENT;
  for (int j = 0; j < d->n_genes; ++j)
    if (d->gene_type[j] < 0 || d->gene_type[j] >= d->n_types) return BRKGA_ERR_BAD_INSTANCE;
  for (int m = 0; m + 1 < d->n_machines; ++m) {
    if (!std::isfinite(d->thresholds[m])) return BRKGA_ERR_BAD_INSTANCE;
    if (m > 0 && d->thresholds[m] < d->thresholds[m - 1]) return BRKGA_ERR_BAD_INSTANCE;
  }
  for (int m = 0; m < d->n_machines; ++m) {
    if (d->bin_length[m] < 1 || d->bin_length[m] > kMaxSide || d->bin_width[m] < 1 ||
        d->bin_width[m] > kMaxSide || !std::isfinite(d->bin_area[m]) || !std::isfinite(d->setup_time[m]))
      return BRKGA_ERR_BAD_INSTANCE;
  }
  for (int t = 0; t < d->n_types; ++t) {
    if (!(d->part_area[t] > 0.0) || !std::isfinite(d->part_area[t])) return BRKGA_ERR_BAD_INSTANCE;
    const int nrot = d->part_nrot[t];
    if (nrot != 2 && nrot != 4) return BRKGA_ERR_BAD_INSTANCE;
    if (d->part_best_rot[t] < 0 || d->part_best_rot[t] >= nrot) return BRKGA_ERR_BAD_INSTANCE;
    for (int r = 0; r < nrot; ++r) {
      const int k = t * 4 + r;
      const int h = d->rot_h[k], w = d->rot_w[k];
      if (h < 1 || w < 1 || h > kMaxSide || w > kMaxSide) return BRKGA_ERR_BAD_INSTANCE;
      const int64_t off = d->rot_mask_offset[k];
      if (off < 0 || off + (int64_t)h * w > d->masks_bytes) return BRKGA_ERR_BAD_INSTANCE;
      for (int64_t i = 0; i < (int64_t)h * w; ++i)
        if (d->masks[off + i] > 1) return BRKGA_ERR_BAD_INSTANCE;
    }
    for (int m = 0; m < d->n_machines; ++m) {
      const size_t i = (size_t)m * d->n_types + t;
      if (!std::isfinite(d->proc_time[i]) || !std::isfinite(d->proc_time_height[i])) return BRKGA_ERR_BAD_INSTANCE;
    }
  }
  return BRKGA_OK;
}

// Host copies of the merged tables while a problem is built.
struct Merged {
  std::vector<InstDev> inst;
  std::vector<int32_t> gene_type, nrot, best;
  std::vector<double> thr, pt, pth, area, bin_area;
  std::vector<RotDev> rot;
  std::vector<uint32_t> vtest;
  std::vector<uint2> truns;
  std::vector<uint32_t> maskbits;
  std::vector<uint8_t> fits, newbin_ok;
  std::vector<RotList> rl;
  std::vector<MachDev> mach;
};

// Append one instance: derived part tables (densities, runs of ones,
// bit-packed rows) with absolute indices, machines, times, flags.
void merge_instance(const BrkgaProblemDesc* d, Merged& g) {
  const int N = d->n_genes, M = d->n_machines, T = d->n_types;
  InstDev id;
  id.N = N;
  id.M = M;
  id.T = T;
  id.mode = d->threshold_mode;
  id.gbase = (int)g.gene_type.size();
  id.tbase = (int)g.area.size();
  id.mbase = (int)g.mach.size();
  id.thrbase = (int)g.thr.size();
  id.tmbase = (int)g.pt.size();
  for (int t = 0; t < T; ++t) {
    for (int r = 0; r < 4; ++r) {
      RotDev rd{};
      if (r < d->part_nrot[t]) {
        const int k = t * 4 + r, h = d->rot_h[k], w = d->rot_w[k];
        const uint8_t* mk = d->masks + d->rot_mask_offset[k];
        rd.h = h;
        rd.w = w;
        rd.mw = (w + 31) / 32;
        rd.mask_base = (int)g.maskbits.size();
        rd.imax = 0;
        rd.dmax = 0;
        std::vector<std::vector<uint32_t>> row_runs(h);
        std::vector<int> dens(h, 0);
        for (int i = 0; i < h; ++i) {
          int best = 0, j = 0;
          while (j < w) {
            if (mk[(size_t)i * w + j]) {
              const int s = j;
              while (j < w && mk[(size_t)i * w + j]) ++j;
              row_runs[i].push_back((uint32_t)s | ((uint32_t)(j - s) << 16));
              best = std::max(best, j - s);
            } else {
              ++j;
            }
          }
          dens[i] = best;
          if (best > rd.dmax) {
            rd.dmax = best;
            rd.imax = i;
          }
          for (int wd = 0; wd < rd.mw; ++wd) {
            uint32_t v = 0;
            for (int bit = 0; bit < 32 && wd * 32 + bit < w; ++bit)
              if (mk[(size_t)i * w + wd * 32 + bit]) v |= 1u << bit;
            g.maskbits.push_back(v);
          }
        }
        // collision-test order: the widest row, then the rows coarse to fine
        // from the bottom (every 16th, then every 8th, 4th, 2nd, the rest).
        // Plates fill from the bottom, so low rows reject a blocked candidate
        // soonest; spreading the first tests over the part's height catches
        // a collision higher up without walking every row below it.
        rd.trun = (int)g.truns.size();
        {
          std::vector<int> order;
          std::vector<char> used(h, 0);
          order.push_back(rd.imax);
          used[rd.imax] = 1;
          for (int st = 16; st >= 1; st >>= 1)
            for (int i = h - 1; i >= 0; i -= st)
              if (!used[i]) {
                order.push_back(i);
                used[i] = 1;
              }
          for (int i : order)
            for (uint32_t r : row_runs[i]) g.truns.push_back(make_uint2(r, (unsigned)i));
          rd.vt = (int)g.vtest.size();
          for (int i : order) g.vtest.push_back(((uint32_t)i << 16) | (uint32_t)dens[i]);
        }
        rd.ntrun = (int)g.truns.size() - rd.trun;
      }
      g.rot.push_back(rd);
    }
    g.area.push_back(d->part_area[t]);
    g.nrot.push_back(d->part_nrot[t]);
    g.best.push_back(d->part_best_rot[t]);
  }
  std::vector<uint8_t> fits((size_t)T * M), newbin_ok((size_t)T * M);
  for (int m = 0; m < M; ++m) {
    MachDev md;
    md.L = d->bin_length[m];
    md.W = d->bin_width[m];
    md.NW = (md.W + 31) / 32;
    md.RS = md.NW + 2;
    md.area = d->bin_area[m];
    md.setup = d->setup_time[m];
    g.mach.push_back(md);
    g.bin_area.push_back(d->bin_area[m]);
    for (int t = 0; t < T; ++t) {
      const int h0 = d->rot_h[t * 4], w0 = d->rot_w[t * 4];
      fits[(size_t)t * M + m] = !((h0 > md.L || w0 > md.W) && (w0 > md.L || h0 > md.W));
      const int rb = d->part_best_rot[t];
      newbin_ok[(size_t)t * M + m] = d->rot_h[t * 4 + rb] <= md.L && d->rot_w[t * 4 + rb] <= md.W;
    }
  }
  g.fits.insert(g.fits.end(), fits.begin(), fits.end());
  g.newbin_ok.insert(g.newbin_ok.end(), newbin_ok.begin(), newbin_ok.end());
  for (int t = 0; t < T; ++t)
    for (int m = 0; m < M; ++m) {
      const MachDev& md = g.mach[id.mbase + m];
      RotList l{};
      int rh[4];
      l.hmin = kMaxSide + 1;
      for (int r = 0; r < d->part_nrot[t]; ++r) {
        const int h = d->rot_h[t * 4 + r], w = d->rot_w[t * 4 + r];
        if (h <= md.L && w <= md.W) {  // numba_utils.py:82-84
          rh[l.nr] = h;
          l.r[l.nr] = l.rs[l.nr] = (unsigned char)r;
          ++l.nr;
          l.hmin = std::min(l.hmin, h);
          l.scan_words += (unsigned)(md.L * md.NW + h * ((w + 31) / 32));
        }
      }
      for (int i = 1; i < l.nr; ++i)  // stable insertion sort by height
        for (int j = i; j > 0 && rh[j] < rh[j - 1]; --j) {
          std::swap(rh[j], rh[j - 1]);
          std::swap(l.rs[j], l.rs[j - 1]);
        }
      g.rl.push_back(l);
    }
  for (int m = 0; m + 1 < M; ++m)
    g.thr.push_back(d->threshold_mode == BRKGA_THRESH_F32 ? (double)(float)d->thresholds[m] : d->thresholds[m]);
  for (int j = 0; j < N; ++j) g.gene_type.push_back(id.tbase + d->gene_type[j]);
  g.pt.insert(g.pt.end(), d->proc_time, d->proc_time + (size_t)M * T);
  g.pth.insert(g.pth.end(), d->proc_time_height, d->proc_time_height + (size_t)M * T);
  g.inst.push_back(id);
}

// chrom_offs / out_offs (host [K], may be NULL): where each instance's
// chromosomes (in floats) and makespans start; NULL = packed one after another.
int fill_run(const BrkgaProblem* pb, const int32_t* pops, const int64_t* chrom_offs, const int64_t* out_offs,
             const LaunchCounts& lc, const Layout& l, char* ws, const float* d_chrom, double* d_out,
             BrkgaPlacement* d_log, int32_t* d_status, int64_t pool_bins, Run* run) {
  std::memset(run, 0, sizeof(Run));
  run->K = pb->K;
  run->n_rows = (int)lc.rows;
  run->n_items = (int)lc.items;
  run->Nmax = pb->Nmax;
  run->chrom = d_chrom;
  run->out = d_out;
  run->seq = reinterpret_cast<uint16_t*>(ws + l.off_seq);
  run->cnt = reinterpret_cast<int32_t*>(ws + l.off_cnt);
  run->infeas = reinterpret_cast<int32_t*>(ws + l.off_inf);
  run->order = reinterpret_cast<int32_t*>(ws + l.off_ord);
  run->mk = reinterpret_cast<double*>(ws + l.off_mk);
  run->log = d_log;
  run->status = d_status;
  unsigned int* ctr = reinterpret_cast<unsigned int*>(ws + l.off_ctr);
  run->item_ctr = ctr;
  run->pool_ctr = ctr + 1;
  run->counters = reinterpret_cast<unsigned long long*>(ws + l.off_ctr + 8);
  run->crit = reinterpret_cast<int*>(ws + l.off_crit);
  run->crit_items = pick_shape(pb, lc.items).warps == 4 ? kCritItems : 0;
  run->binscal = reinterpret_cast<BinScal*>(ws + l.off_bins);
  run->pool = reinterpret_cast<uint32_t*>(ws + l.off_pool);
  run->pool_bins = pool_bins;
  run->S = pick_shape(pb, lc.items).S;
  run->slot_words = pb->slot_words;
  run->slot_vac_off = pb->slot_vac_off;
  run->task_max = pb->task_max;
  int64_t row = 0, item = 0, seq = 0, chrom = 0;
  for (int k = 0; k < pb->K; ++k) {
    const InstDev& id = pb->inst[k];
    InstRun& r = run->r[k];
    r.P = pops[k];
    r.crow0 = (int)row;
    r.item0 = (int)item;
    r.S2 = pb->s2[k];
    r.chrom_off = chrom_offs ? chrom_offs[k] : chrom;
    r.out_off = out_offs ? out_offs[k] : row;
    r.seq0 = seq;
    row += pops[k];
    item += (int64_t)pops[k] * id.M;
    seq += (int64_t)pops[k] * id.M * id.N;
    chrom += (int64_t)pops[k] * 2 * id.N;
  }
  return BRKGA_OK;
}

int launch(const BrkgaProblem* pb, int stage, const Run& run, cudaStream_t s) {
  if (run.n_rows == 0) return BRKGA_OK;
  if (stage == 0 || stage == 1) {
    const int at = std::min(1024, std::max(64, pb->S2max / 2));
    assign_sort_kernel<<<run.n_rows, at, (size_t)pb->S2max * 8, s>>>(pb->tb, run);
    order_items_kernel<<<1, 1024, (size_t)(pb->Nmax + 1) * sizeof(int), s>>>(pb->tb, run);
  }
  if (stage == 0 || stage == 2) {
    const Shape& sh = pick_shape(pb, run.n_items);
    const int grid = (int)std::min<int64_t>(sh.n_slots, run.n_items);
    if (sh.warps == 1) decode_kernel<32><<<grid, 32, sh.smem, s>>>(pb->tb, run);
    else if (sh.warps == 2) decode_kernel<64><<<grid, 64, sh.smem, s>>>(pb->tb, run);
    else decode_kernel<128><<<grid, 128, sh.smem, s>>>(pb->tb, run);
  }
  if (stage == 0 || stage == 3) reduce_kernel<<<(run.n_rows + 255) / 256, 256, 0, s>>>(pb->tb, run);
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

}  // namespace

extern "C" {

int brkga_abi_version(void) { return BRKGA_ABI_VERSION; }

#ifndef BRKGA_BUILD_ID
#define BRKGA_BUILD_ID "unstamped"
#endif
const char* brkga_build_id(void) { return BRKGA_BUILD_ID; }

// Device tables for the surrogate (same library, not part of the public ABI;
// single-instance problems, whose table bases are all 0).
__attribute__((visibility("hidden"))) int brkga_internal_problem_tables(
    const BrkgaProblem* pb, int* N, int* M, int* T, int* mode, const double** thr, const int32_t** gene_type,
    const double** part_area, const double** pt, const double** pth, const double** bin_area) {
  if (!pb || pb->K != 1) return BRKGA_ERR_INVALID_ARGUMENT;
  *N = pb->N;
  *M = pb->M;
  *T = pb->T;
  *mode = pb->mode;
  *thr = pb->d_thr;
  *gene_type = pb->d_gene_type;
  *part_area = pb->d_area;
  *pt = pb->d_pt;
  *pth = pb->d_pth;
  *bin_area = pb->d_bin_area;
  return BRKGA_OK;
}

const char* brkga_status_string(int status) {
  switch (status) {
    case BRKGA_OK: return "ok";
    case BRKGA_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BRKGA_ERR_BAD_INSTANCE: return "bad instance";
    case BRKGA_ERR_CUDA: return "CUDA error";
    case BRKGA_ERR_WORKSPACE: return "workspace too small";
    case BRKGA_ERR_CAPACITY: return "bin pool exhausted";
    case BRKGA_ERR_NEW_BIN_UNFIT: return "new plate received a rotation that does not fit";
    case BRKGA_ERR_NO_DEVICE: return "no CUDA device";
    case BRKGA_ERR_INTERNAL: return "device consistency check failed";
    default: return "unknown status";
  }
}

void brkga_problem_destroy(BrkgaProblem* pb) {
  if (!pb) return;
  {
    DeviceGuard g(pb->device);
    for (void* p : pb->allocations) cudaFree(p);
    if (pb->e_chrom) cudaFree(pb->e_chrom);
    if (pb->e_out) cudaFree(pb->e_out);
    if (pb->e_status) cudaFree(pb->e_status);
    if (pb->e_log) cudaFree(pb->e_log);
    if (pb->e_ws) cudaFree(pb->e_ws);
    if (pb->e_host) cudaFreeHost(pb->e_host);
    if (pb->stream) cudaStreamDestroy(pb->stream);
  }
  delete pb;
}

int brkga_problem_create_multi(const BrkgaProblemDesc* descs, int32_t K, BrkgaProblem** out) {
  if (!out) return BRKGA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!descs || K < 1 || K > kMaxInst) return BRKGA_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < K; ++k) {
    const int st = validate(&descs[k]);
    if (st) return st;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return BRKGA_ERR_NO_DEVICE;
  }
  Merged g;
  for (int k = 0; k < K; ++k) merge_instance(&descs[k], g);
  if (g.maskbits.size() >= ((size_t)1 << 31) || g.truns.size() >= ((size_t)1 << 31)) return BRKGA_ERR_BAD_INSTANCE;
  BrkgaProblem* pb = new BrkgaProblem();
  cudaGetDevice(&pb->device);
  pb->K = K;
  pb->inst = g.inst;
  pb->mach = g.mach;
  for (const InstDev& id : g.inst) {
    int s2 = 1;
    while (s2 < id.N) s2 <<= 1;
    pb->s2.push_back(s2);
    pb->S2max = std::max(pb->S2max, s2);
    pb->Nmax = std::max(pb->Nmax, id.N);
  }
  pb->N = g.inst[0].N;
  pb->M = g.inst[0].M;
  pb->T = g.inst[0].T;
  pb->mode = g.inst[0].mode;

  int st;
  if ((st = upload(pb, &pb->d_inst, g.inst)) || (st = upload(pb, &pb->d_gene_type, g.gene_type)) ||
      (st = upload(pb, &pb->d_thr, g.thr)) || (st = upload(pb, &pb->d_mach, g.mach)) ||
      (st = upload(pb, &pb->d_pt, g.pt)) || (st = upload(pb, &pb->d_pth, g.pth)) ||
      (st = upload(pb, &pb->d_area, g.area)) || (st = upload(pb, &pb->d_nrot, g.nrot)) ||
      (st = upload(pb, &pb->d_best, g.best)) || (st = upload(pb, &pb->d_rot, g.rot)) ||
      (st = upload(pb, &pb->d_vtest, g.vtest)) || (st = upload(pb, &pb->d_truns, g.truns)) ||
      (st = upload(pb, &pb->d_maskbits, g.maskbits)) ||
      (st = upload(pb, &pb->d_fits, g.fits)) || (st = upload(pb, &pb->d_newbin_ok, g.newbin_ok)) ||
      (st = upload(pb, &pb->d_rl, g.rl)) ||
      (st = upload(pb, &pb->d_bin_area, g.bin_area)) || (st = configure(pb, 0, 0, -1))) {
    brkga_problem_destroy(pb);
    return st;
  }
  Tables& tb = pb->tb;
  tb.inst = pb->d_inst;
  tb.gene_type = pb->d_gene_type;
  tb.thr = pb->d_thr;
  tb.mach = pb->d_mach;
  tb.pt = pb->d_pt;
  tb.pth = pb->d_pth;
  tb.part_area = pb->d_area;
  tb.nrot = pb->d_nrot;
  tb.best_rot = pb->d_best;
  tb.rot = pb->d_rot;
  tb.vtest = pb->d_vtest;
  tb.truns = pb->d_truns;
  tb.maskbits = pb->d_maskbits;
  tb.newbin_ok = pb->d_newbin_ok;
  tb.fits = pb->d_fits;
  tb.rl = pb->d_rl;
  if (cudaGetSymbolAddress(&pb->noalloc_scratch, g_noalloc_scratch) != cudaSuccess) {
    brkga_problem_destroy(pb);
    return BRKGA_ERR_CUDA;
  }
  *out = pb;
  return BRKGA_OK;
}

int brkga_problem_create(const BrkgaProblemDesc* d, BrkgaProblem** out) {
  if (!out) return BRKGA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (!d) return BRKGA_ERR_INVALID_ARGUMENT;
  return brkga_problem_create_multi(d, 1, out);
}

int brkga_problem_instances(const BrkgaProblem* pb, int32_t* K) {
  if (!pb || !K) return BRKGA_ERR_INVALID_ARGUMENT;
  *K = pb->K;
  return BRKGA_OK;
}

int brkga_set_launch_config(BrkgaProblem* pb, int32_t warps_per_item, int32_t ctas_per_sm, int32_t smem_plates,
                            int32_t task_max) {
  if (!pb || (warps_per_item != 0 && warps_per_item != 1 && warps_per_item != 2 && warps_per_item != 4) ||
      ctas_per_sm < 0 ||
      ctas_per_sm > kMaxCtasPerSm || smem_plates < -1 || smem_plates > kMaxSmemPlates || task_max < -1 ||
      task_max > kMaxTaskMax)
    return BRKGA_ERR_INVALID_ARGUMENT;
  DeviceGuard g(pb->device);
  const int old_warps = pb->req_warps, old_ctas = pb->req_ctas, old_plates = pb->req_plates;
  const int st = configure(pb, warps_per_item, ctas_per_sm, smem_plates);
  if (st) {
    configure(pb, old_warps, old_ctas, old_plates);
    return st;
  }
  pb->task_max = task_max < 0 ? kDefaultTaskMax : task_max;
  return BRKGA_OK;
}

int brkga_get_launch_config(const BrkgaProblem* pb, int64_t items, int32_t* warps_per_item, int32_t* ctas_per_sm,
                            int32_t* smem_plates, int32_t* resident_ctas, int32_t* task_max) {
  if (!pb || items < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  const Shape& sh = pick_shape(pb, items);
  if (warps_per_item) *warps_per_item = sh.warps;
  if (ctas_per_sm) *ctas_per_sm = sh.ctas;
  if (smem_plates) *smem_plates = sh.S;
  if (resident_ctas) *resident_ctas = sh.n_slots;
  if (task_max) *task_max = pb->task_max;
  return BRKGA_OK;
}

int brkga_workspace_bytes_multi(const BrkgaProblem* pb, const int32_t* pops, int64_t pool_bins, size_t* bytes) {
  if (!pb || !pops || !bytes || pool_bins < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  LaunchCounts lc;
  const int st = counts_of(pb, pops, &lc);
  if (st) return st;
  if (pool_bins == 0) pool_bins = default_pool_bins(pb, lc.items);
  *bytes = layout_of(pb, lc, pool_bins).total;
  return BRKGA_OK;
}

int brkga_workspace_bytes(const BrkgaProblem* pb, int32_t P, int64_t pool_bins, size_t* bytes) {
  if (!pb || pb->K != 1) return BRKGA_ERR_INVALID_ARGUMENT;
  return brkga_workspace_bytes_multi(pb, &P, pool_bins, bytes);
}

int brkga_decode_multi_at(int32_t stage, const BrkgaProblem* pb, const float* d_chrom, const int64_t* chrom_offsets,
                          const int32_t* pops, double* d_makespan, const int64_t* makespan_offsets,
                          BrkgaPlacement* d_log, int32_t* d_status, void* d_ws, size_t ws_bytes, int64_t pool_bins,
                          void* stream) {
  if (!pb || !pops || pool_bins < 0 || stage < 0 || stage > 3) return BRKGA_ERR_INVALID_ARGUMENT;
  LaunchCounts lc;
  int st = counts_of(pb, pops, &lc);
  if (st) return st;
  for (int k = 0; k < pb->K; ++k)
    if ((chrom_offsets && chrom_offsets[k] < 0) || (makespan_offsets && makespan_offsets[k] < 0))
      return BRKGA_ERR_INVALID_ARGUMENT;
  if (lc.rows == 0) return BRKGA_OK;
  if (!d_chrom || !d_makespan || !d_status || !d_ws) return BRKGA_ERR_INVALID_ARGUMENT;
  if (pool_bins == 0) pool_bins = default_pool_bins(pb, lc.items);
  const Layout l = layout_of(pb, lc, pool_bins);
  if (ws_bytes < l.total) return BRKGA_ERR_WORKSPACE;
  DeviceGuard g(pb->device);
  Run run;
  fill_run(pb, pops, chrom_offsets, makespan_offsets, lc, l, static_cast<char*>(d_ws), d_chrom, d_makespan, d_log,
           d_status, pool_bins, &run);
  return launch(pb, stage, run, static_cast<cudaStream_t>(stream));
}

int brkga_decode_multi_stage(int32_t stage, const BrkgaProblem* pb, const float* d_chrom, const int32_t* pops,
                             double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status, void* d_ws,
                             size_t ws_bytes, int64_t pool_bins, void* stream) {
  return brkga_decode_multi_at(stage, pb, d_chrom, nullptr, pops, d_makespan, nullptr, d_log, d_status, d_ws,
                               ws_bytes, pool_bins, stream);
}

int brkga_decode_multi(const BrkgaProblem* pb, const float* d_chrom, const int32_t* pops, double* d_makespan,
                       BrkgaPlacement* d_log, int32_t* d_status, void* d_ws, size_t ws_bytes, int64_t pool_bins,
                       void* stream) {
  return brkga_decode_multi_stage(0, pb, d_chrom, pops, d_makespan, d_log, d_status, d_ws, ws_bytes, pool_bins,
                                  stream);
}

int brkga_decode_stage(int32_t stage, const BrkgaProblem* pb, const float* d_chrom, int32_t P,
                       double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status, void* d_ws,
                       size_t ws_bytes, int64_t pool_bins, void* stream) {
  if (!pb || pb->K != 1 || P < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  return brkga_decode_multi_stage(stage, pb, d_chrom, &P, d_makespan, d_log, d_status, d_ws, ws_bytes, pool_bins,
                                  stream);
}

int brkga_decode(const BrkgaProblem* pb, const float* d_chrom, int32_t P, double* d_makespan,
                 BrkgaPlacement* d_log, int32_t* d_status, void* d_ws, size_t ws_bytes, int64_t pool_bins,
                 void* stream) {
  return brkga_decode_stage(0, pb, d_chrom, P, d_makespan, d_log, d_status, d_ws, ws_bytes, pool_bins, stream);
}

// Decode without allocating: the workspace is the library's fixed device
// array (address resolved when the problem was created), the bin pool takes
// whatever that array has left after the per-population tables.
int brkga_decode_noalloc(const BrkgaProblem* pb, const float* d_chrom, int32_t P, double* d_makespan,
                         BrkgaPlacement* d_log, int32_t* d_status, void* stream) {
  if (!pb || pb->K != 1 || P < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  if (P == 0) return BRKGA_OK;
  if (!pb->noalloc_scratch) return BRKGA_ERR_INVALID_ARGUMENT;
  const size_t cap = (size_t)BRKGA_NOALLOC_SCRATCH_BYTES;
  LaunchCounts lc;
  if (counts_of(pb, &P, &lc)) return BRKGA_ERR_INVALID_ARGUMENT;
  const Layout fixed = layout_of(pb, lc, 0);  // offsets up to the pool do not depend on the pool size
  if (fixed.off_pool >= cap) return BRKGA_ERR_WORKSPACE;
  int64_t pool_bins = (int64_t)((cap - fixed.off_pool) / ((size_t)pb->slot_words * sizeof(uint32_t)));
  while (pool_bins > 0 && layout_of(pb, lc, pool_bins).total > cap) --pool_bins;  // 256-byte rounding
  if (pool_bins < 1) return BRKGA_ERR_WORKSPACE;
  return brkga_decode_stage(0, pb, d_chrom, P, d_makespan, d_log, d_status, pb->noalloc_scratch, cap,
                            pool_bins, stream);
}

int brkga_evaluate_host(BrkgaProblem* pb, const float* h_chrom, int32_t P, double* h_makespan,
                        BrkgaPlacement* h_log) {
  if (!pb || pb->K != 1 || P < 0 || (P > 0 && (!h_chrom || !h_makespan))) return BRKGA_ERR_INVALID_ARGUMENT;
  if (P == 0) return BRKGA_OK;
  std::lock_guard<std::mutex> lock(pb->mu);
  DeviceGuard g(pb->device);
  if (!pb->stream && cudaStreamCreateWithFlags(&pb->stream, cudaStreamNonBlocking) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  const bool want_log = h_log != nullptr;
  if (P > pb->e_cap_P || (want_log && !pb->e_cap_log)) {
    const int cap = std::max(P, pb->e_cap_P);
    cudaFree(pb->e_chrom);
    cudaFree(pb->e_out);
    cudaFree(pb->e_status);
    cudaFree(pb->e_log);
    if (pb->e_host) cudaFreeHost(pb->e_host);
    pb->e_host = nullptr;
    pb->e_chrom = nullptr;
    pb->e_out = nullptr;
    pb->e_status = nullptr;
    pb->e_log = nullptr;
    pb->e_cap_P = 0;
    if (cudaMalloc(&pb->e_chrom, (size_t)cap * 2 * pb->N * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&pb->e_out, (size_t)cap * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&pb->e_status, sizeof(int32_t)) != cudaSuccess ||
        cudaHostAlloc(&pb->e_host, 64 + (size_t)cap * sizeof(double), cudaHostAllocDefault) != cudaSuccess)
      return BRKGA_ERR_CUDA;
    if ((want_log || pb->e_cap_log) &&
        cudaMalloc(&pb->e_log, (size_t)cap * pb->M * pb->N * sizeof(BrkgaPlacement)) != cudaSuccess)
      return BRKGA_ERR_CUDA;
    pb->e_cap_log = want_log || pb->e_cap_log;
    pb->e_cap_P = cap;
  }
  LaunchCounts lc;
  if (counts_of(pb, &P, &lc)) return BRKGA_ERR_INVALID_ARGUMENT;
  if (pb->e_pool_bins < default_pool_bins(pb, lc.items)) pb->e_pool_bins = default_pool_bins(pb, lc.items);
  if (cudaMemcpyAsync(pb->e_chrom, h_chrom, (size_t)P * 2 * pb->N * sizeof(float), cudaMemcpyHostToDevice,
                      pb->stream) != cudaSuccess)
    return BRKGA_ERR_CUDA;
  for (int attempt = 0; attempt < 12; ++attempt) {
    const Layout l = layout_of(pb, lc, pb->e_pool_bins);
    if (l.total > pb->e_ws_bytes) {
      if (cudaStreamSynchronize(pb->stream) != cudaSuccess) return BRKGA_ERR_CUDA;
      cudaFree(pb->e_ws);
      pb->e_ws = nullptr;
      pb->e_ws_bytes = 0;
      if (cudaMalloc(&pb->e_ws, l.total) != cudaSuccess) return BRKGA_ERR_CUDA;
      pb->e_ws_bytes = l.total;
    }
    int st = brkga_decode(pb, pb->e_chrom, P, pb->e_out, want_log ? pb->e_log : nullptr, pb->e_status, pb->e_ws,
                          pb->e_ws_bytes, pb->e_pool_bins, pb->stream);
    if (st) return st;
    unsigned char* hs = pb->e_host;
    if (cudaMemcpyAsync(hs, pb->e_status, sizeof(int32_t), cudaMemcpyDeviceToHost, pb->stream) != cudaSuccess ||
        cudaMemcpyAsync(hs + 8, static_cast<char*>(pb->e_ws) + l.off_ctr + 8, 4 * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost, pb->stream) != cudaSuccess ||
        cudaMemcpyAsync(hs + 64, pb->e_out, (size_t)P * sizeof(double), cudaMemcpyDeviceToHost, pb->stream) !=
            cudaSuccess)
      return BRKGA_ERR_CUDA;
    if (cudaStreamSynchronize(pb->stream) != cudaSuccess) return BRKGA_ERR_CUDA;
    int32_t status = 0;
    unsigned long long counters[4];
    std::memcpy(&status, hs, sizeof(status));
    std::memcpy(counters, hs + 8, sizeof(counters));
    std::memcpy(h_makespan, hs + 64, (size_t)P * sizeof(double));
    for (int i = 0; i < 4; ++i) pb->last_counters[i] = (int64_t)counters[i];
    if (status == BRKGA_ERR_CAPACITY) {
      pb->e_pool_bins *= 2;
      continue;
    }
    if (status) return status;
    if (want_log &&
        cudaMemcpy(h_log, pb->e_log, (size_t)P * pb->M * pb->N * sizeof(BrkgaPlacement), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
      return BRKGA_ERR_CUDA;
    return BRKGA_OK;
  }
  return BRKGA_ERR_CAPACITY;
}

int brkga_initial_solution_host(BrkgaProblem* pb, const int32_t* h_order, int32_t n, int32_t* h_machine,
                                BrkgaPlacement* h_place, double* h_machine_makespan) {
  if (!pb || pb->K != 1 || n < 0 || (n > 0 && (!h_order || !h_machine || !h_place)) || !h_machine_makespan)
    return BRKGA_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < n; ++k)
    if (h_order[k] < 0 || h_order[k] >= pb->N) return BRKGA_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(pb->mu);
  DeviceGuard guard(pb->device);
  const int nn = std::max(n, 1);
  // one allocation: order, outputs, plate tables, scalars, counters, status, pool (one plate per part at most)
  size_t o = 0;
  const size_t off_order = o;
  o = align_up(o + (size_t)nn * 4, 256);
  const size_t off_mach = o;
  o = align_up(o + (size_t)nn * 4, 256);
  const size_t off_out = o;
  o = align_up(o + (size_t)nn * sizeof(BrkgaPlacement), 256);
  const size_t off_pm = o;
  o = align_up(o + (size_t)nn * 4, 256);
  const size_t off_pi = o;
  o = align_up(o + (size_t)nn * 4, 256);
  const size_t off_mk = o;
  o = align_up(o + (size_t)pb->M * 8, 256);
  const size_t off_bs = o;
  o = align_up(o + (size_t)nn * sizeof(BinScal), 256);
  const size_t off_ctr = o;
  o = align_up(o + 64, 256);
  const size_t off_pool = o;
  o = align_up(o + (size_t)nn * pb->slot_words * 4, 256);
  char* d = nullptr;
  if (cudaMalloc(&d, o) != cudaSuccess) return BRKGA_ERR_CUDA;
  int st = BRKGA_OK;
  do {
    if (cudaMemset(d, 0, off_pool) != cudaSuccess ||
        (n > 0 && cudaMemcpy(d + off_order, h_order, (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess)) {
      st = BRKGA_ERR_CUDA;
      break;
    }
    GreedyArgs g;
    std::memset(&g, 0, sizeof(g));
    g.N = pb->N;
    g.M = pb->M;
    g.T = pb->T;
    g.status = reinterpret_cast<int32_t*>(d + off_ctr + 40);
    g.counters = reinterpret_cast<unsigned long long*>(d + off_ctr + 8);
    g.binscal = reinterpret_cast<BinScal*>(d + off_bs);
    g.pool = reinterpret_cast<uint32_t*>(d + off_pool);
    g.slot_words = pb->slot_words;
    g.slot_vac_off = pb->slot_vac_off;
    g.order = reinterpret_cast<const int32_t*>(d + off_order);
    g.n = n;
    g.out_machine = reinterpret_cast<int32_t*>(d + off_mach);
    g.out = reinterpret_cast<BrkgaPlacement*>(d + off_out);
    g.plate_machine = reinterpret_cast<int32_t*>(d + off_pm);
    g.plate_index = reinterpret_cast<int32_t*>(d + off_pi);
    g.machine_makespan = reinterpret_cast<double*>(d + off_mk);
    greedy_kernel<<<1, kGreedyThreads>>>(pb->tb, g);
    int32_t status = 0;
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&status, g.status, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      st = BRKGA_ERR_CUDA;
      break;
    }
    if (status) {
      st = status;
      break;
    }
    if ((n > 0 && (cudaMemcpy(h_machine, g.out_machine, (size_t)n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
                   cudaMemcpy(h_place, g.out, (size_t)n * sizeof(BrkgaPlacement), cudaMemcpyDeviceToHost) !=
                       cudaSuccess)) ||
        cudaMemcpy(h_machine_makespan, g.machine_makespan, (size_t)pb->M * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = BRKGA_ERR_CUDA;
  } while (false);
  cudaFree(d);
  return st;
}

int brkga_chunk_free(const BrkgaProblem* pb, int32_t path, const BrkgaChunkTest* d_items, int32_t n_items,
                     int32_t* d_status, void* stream) {
  if (!pb || pb->K != 1 || n_items < 0 || (path != BRKGA_COLLISION_BITSET && path != BRKGA_COLLISION_INT8_TC))
    return BRKGA_ERR_INVALID_ARGUMENT;
  if (n_items == 0) return BRKGA_OK;
  if (!d_items || !d_status) return BRKGA_ERR_INVALID_ARGUMENT;
  DeviceGuard g(pb->device);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (path == BRKGA_COLLISION_BITSET) {
    chunk_free_bitset_kernel<<<n_items, 128, 0, s>>>(pb->tb, d_items, pb->M, pb->T, d_status);
  } else {
    int wmax = 1;
    for (const MachDev& m : pb->mach) wmax = std::max(wmax, m.W);
    const dim3 grid((unsigned)n_items, (unsigned)((wmax + corr::kTileM - 1) / corr::kTileM));
    chunk_free_i8_kernel<<<grid, corr::kThreads, corr::smem_bytes(corr::kMaxSide, corr::kMaxSide), s>>>(
        pb->tb, d_items, pb->M, pb->T, d_status);
  }
  return cudaGetLastError() == cudaSuccess ? BRKGA_OK : BRKGA_ERR_CUDA;
}

int brkga_last_counters(const BrkgaProblem* pb, int64_t* tests, int64_t* chunks, int64_t* bins,
                        int64_t* scan_bytes) {
  if (!pb) return BRKGA_ERR_INVALID_ARGUMENT;
  if (tests) *tests = pb->last_counters[0];
  if (chunks) *chunks = pb->last_counters[1];
  if (bins) *bins = pb->last_counters[2];
  if (scan_bytes) *scan_bytes = pb->last_counters[3];
  return BRKGA_OK;
}

}  // extern "C"
