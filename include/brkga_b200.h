/*
 * brkga_b200.h — C ABI of the B200 BRKGA chromosome decoder.
 *
 * The decoder maps a population of random-key chromosomes (float32, P rows of
 * 2N keys: N sequencing keys then N machine keys) to one makespan per
 * chromosome, with the placement rule of the reference's sequential decoder
 * (placement.py:94-165, binClassNew.py:45-174).  Plain pointers and sizes
 * only; no exception crosses this boundary; every entry point returns a
 * BrkgaStatus code.
 *
 * Reference interfaces replaced (paths inside paulonasc7/BRKGA_FFT2):
 *   brkga_problem_create   NativeFullDecoder::NativeFullDecoder  full_native_decoder.py:408-533
 *                          + _pack_problem_data                  full_native_decoder.py:2788-2926
 *   brkga_problem_destroy  NativeFullDecoder destructor (pybind11-owned object)
 *   brkga_evaluate_host    NativeFullDecoder::evaluate_batch     full_native_decoder.py:563-641
 *                          (host float32 [P,2N] in, host float64 [P] out)
 *   brkga_decode           the device part of evaluate_batch: process_machine_batch
 *                          full_native_decoder.py:1290-1431, stream-ordered, caller-owned buffers
 *   brkga_workspace_bytes  workspace sizing (reference: grow_grid_storage :2102-2153)
 */
#ifndef BRKGA_B200_H
#define BRKGA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BRKGA_ABI_VERSION 1

/* Machine-assignment comparison: placement.py:122-127 compares float32 keys
 * against Python-float thresholds, which NumPy >= 2 evaluates in float32;
 * full_native_decoder.py:961-973 compares in float64.  The two differ only
 * for thresholds that are not exactly representable in float32 (M = 3, 5, 6...). */
#define BRKGA_THRESH_F32 0
#define BRKGA_THRESH_F64 1

typedef enum BrkgaStatus {
  BRKGA_OK = 0,
  BRKGA_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, P < 0 ...            */
  BRKGA_ERR_BAD_INSTANCE = 2,     /* inconsistent tables (e.g. mask larger than 1024) */
  BRKGA_ERR_CUDA = 3,             /* a CUDA runtime call failed                      */
  BRKGA_ERR_WORKSPACE = 4,        /* workspace too small for this P                  */
  BRKGA_ERR_CAPACITY = 5,         /* device bin pool exhausted (retry with more)      */
  BRKGA_ERR_NEW_BIN_UNFIT = 6,    /* a new plate got a best_rotation that does not fit;
                                     the reference raises in numpy slicing here      */
  BRKGA_ERR_NO_DEVICE = 7,
  BRKGA_ERR_INTERNAL = 8          /* a device-side consistency check failed: an access
                                     would have left a plate; the access was skipped
                                     and the makespans of the launch are not valid */
} BrkgaStatus;

/* Host description of one instance.  All arrays are read during
 * brkga_problem_create only (they are copied to the device). */
typedef struct BrkgaProblemDesc {
  int32_t n_genes;        /* N: parts in the instance; a chromosome has 2N keys */
  int32_t n_machines;     /* M >= 1 */
  int32_t n_types;        /* T: distinct part types */
  int32_t threshold_mode; /* BRKGA_THRESH_F32 or BRKGA_THRESH_F64 */
  const int32_t* gene_type;        /* [N]   type index 0..T-1 of gene j (instance_parts) */
  const double* thresholds;        /* [M-1] machine-key thresholds, ascending */
  const int32_t* bin_length;       /* [M]   plate rows L   (MachineData.bin_length) */
  const int32_t* bin_width;        /* [M]   plate columns W (MachineData.bin_width) */
  const double* bin_area;          /* [M]   MachineData.bin_area */
  const double* setup_time;        /* [M]   MachineData.setup_time */
  const double* proc_time;         /* [M*T] MachinePartData.proc_time */
  const double* proc_time_height;  /* [M*T] MachinePartData.proc_time_height */
  const double* part_area;         /* [T]   PartData.area (> 0) */
  const int32_t* part_nrot;        /* [T]   2 or 4 */
  const int32_t* part_best_rot;    /* [T]   index of the rotation used on a new plate */
  const int32_t* rot_h;            /* [T*4] rows of np.rot90(mask, r) */
  const int32_t* rot_w;            /* [T*4] columns of np.rot90(mask, r) */
  const int64_t* rot_mask_offset;  /* [T*4] byte offset of rotation r's row-major 0/1 mask */
  const uint8_t* masks;            /* concatenated masks */
  int64_t masks_bytes;
} BrkgaProblemDesc;

/* One placement of the audit log: gene index, plate index within the
 * machine, left column x, bottom row y and rotation — the fields of the
 * reference's golden files (create_golden.py:194-210: part_id/bin_idx/col/row/rot). */
typedef struct BrkgaPlacement {
  int32_t gene;
  int32_t bin;
  int32_t x;
  int32_t y;
  int32_t rot;
} BrkgaPlacement;

typedef struct BrkgaProblem BrkgaProblem; /* opaque, device-resident tables */

/* Library ABI version (BRKGA_ABI_VERSION). */
int brkga_abi_version(void);

/* Build identity compiled into the library: a hash of the sources, headers
 * and compiler flags it was built from ("unstamped" when built without one).
 * No reference counterpart. */
const char* brkga_build_id(void);

/* Static text for a status code. */
const char* brkga_status_string(int status);

/* Validate the tables, derive bit-packed masks, row runs and densities, and
 * copy everything to the current CUDA device.  (full_native_decoder.py:408-533) */
int brkga_problem_create(const BrkgaProblemDesc* desc, BrkgaProblem** out);

/* Free the device tables and the object.  Safe on NULL. */
void brkga_problem_destroy(BrkgaProblem* problem);

/* Device bytes a caller must provide to brkga_decode for P chromosomes with
 * a bin pool of `pool_bins` plates (0 = the library's default for P).  A
 * workspace of that size serves every population of at most P chromosomes
 * under the same launch configuration. */
int brkga_workspace_bytes(const BrkgaProblem* problem, int32_t P, int64_t pool_bins,
                          size_t* bytes);

/* Decode P chromosomes on `stream` (a cudaStream_t, NULL = legacy default).
 *   d_chrom     device float32 [P, 2N], row-major
 *   d_makespan  device float64 [P]; 1e16 for infeasible chromosomes
 *               (placement.py:9,151-153); NaN where d_status reports an error
 *   d_log       device BrkgaPlacement [P, M, N] or NULL; entries past a
 *               machine's part count hold gene = -1
 *   d_status    device int32 [1]: 0 or a BrkgaStatus raised inside the kernels
 *   d_ws        device workspace of brkga_workspace_bytes(problem, P, pool_bins)
 * Asynchronous: returns launch errors only; no allocation, no host sync. */
int brkga_decode(const BrkgaProblem* problem, const float* d_chrom, int32_t P,
                 double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status,
                 void* d_ws, size_t ws_bytes, int64_t pool_bins, void* stream);

/* One stage of brkga_decode with the same arguments: 1 = machine assignment
 * and key sort, 2 = the decode kernel, 3 = the max-over-machines reduction;
 * 0 = all three (what brkga_decode does).  Running 1, 2, 3 in order on one
 * stream equals brkga_decode; lets a caller put its own CUDA events around
 * the decode kernel.  (No reference counterpart: the reference's phases are
 * host-driven, full_native_decoder.py:1481-2097.) */
int brkga_decode_stage(int32_t stage, const BrkgaProblem* problem, const float* d_chrom, int32_t P,
                       double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status, void* d_ws,
                       size_t ws_bytes, int64_t pool_bins, void* stream);

/* Size of the library's fixed device scratch used by brkga_decode_noalloc:
 * 64 MiB, reserved on every GPU that loads the library until the process exits. */
#define BRKGA_NOALLOC_SCRATCH_BYTES (64u << 20)

/* brkga_decode for callers that must not allocate device memory — code that
 * runs under a memory manager owning every device byte (a plugin host, an
 * embedded scheduler), or a loop that must never hit cudaMalloc/cudaFree
 * because those can synchronise the device.  No reference counterpart: the
 * reference grows its workspaces as it goes.
 * Same inputs and outputs as brkga_decode, but the workspace is a fixed
 * 64 MiB array inside the library, so nothing is allocated or freed here.
 * Its device address is looked up by brkga_problem_create (set-up, with the
 * problem's device current).  The per-population tables must fit in it
 * (else BRKGA_ERR_WORKSPACE, before any launch); the plate pool gets the rest,
 * and running out of it sets *d_status = BRKGA_ERR_CAPACITY (decode a smaller
 * batch then).  All calls share the one array: calls that overlap on the GPU
 * (other streams, other problems, other threads) race and must be ordered by
 * the caller.  Nothing needs clearing between calls — each decode resets the
 * counters it uses. */
int brkga_decode_noalloc(const BrkgaProblem* problem, const float* d_chrom, int32_t P,
                         double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status, void* stream);

/* ---- Several independent instances per launch ----
 * No reference counterpart: the reference builds one evaluator per instance
 * (FullNativeDecoderEvaluator, full_native_decoder.py:2937-2981) and decodes
 * one population at a time.  Here a problem may hold up to
 * BRKGA_MAX_INSTANCES instances with their own parts, machines and plate
 * sizes; one launch decodes P_k chromosomes of each instance k, every
 * (chromosome, machine) item of every instance in one persistent decode
 * kernel, longest items first.  The single-instance entry points above
 * (brkga_decode, brkga_decode_stage, brkga_workspace_bytes,
 * brkga_decode_noalloc, brkga_evaluate_host, brkga_initial_solution_host,
 * the surrogate) refuse a problem of more than one instance with
 * BRKGA_ERR_INVALID_ARGUMENT. */
#define BRKGA_MAX_INSTANCES 64

/* brkga_problem_create for descs[0..K-1] (1 <= K <= BRKGA_MAX_INSTANCES);
 * brkga_problem_create(d) is brkga_problem_create_multi(d, 1). */
int brkga_problem_create_multi(const BrkgaProblemDesc* descs, int32_t K, BrkgaProblem** out);

/* Number of instances of a problem. */
int brkga_problem_instances(const BrkgaProblem* problem, int32_t* K);

/* Workspace bytes for pops[k] chromosomes of instance k (pops: host int32 [K]). */
int brkga_workspace_bytes_multi(const BrkgaProblem* problem, const int32_t* pops, int64_t pool_bins,
                                size_t* bytes);

/* Decode pops[k] chromosomes of every instance k in one launch of each kernel.
 *   pops        host int32 [K], read during the call (values go into the
 *               kernel parameters, so a captured graph keeps them)
 *   d_chrom     device float32: instance 0's pops[0] rows of 2*N_0 keys, then
 *               instance 1's rows of 2*N_1 keys, and so on
 *   d_makespan  device float64 [sum pops], rows in the same order
 *   d_log       NULL or device BrkgaPlacement: per row, M_k * N_k entries
 *               (machine-major, as brkga_decode), rows in order
 * Otherwise as brkga_decode (stream-ordered, no allocation, no host sync). */
int brkga_decode_multi(const BrkgaProblem* problem, const float* d_chrom, const int32_t* pops,
                       double* d_makespan, BrkgaPlacement* d_log, int32_t* d_status, void* d_ws,
                       size_t ws_bytes, int64_t pool_bins, void* stream);

/* One stage (1, 2, 3; 0 = all) of brkga_decode_multi, as brkga_decode_stage. */
int brkga_decode_multi_stage(int32_t stage, const BrkgaProblem* problem, const float* d_chrom,
                             const int32_t* pops, double* d_makespan, BrkgaPlacement* d_log,
                             int32_t* d_status, void* d_ws, size_t ws_bytes, int64_t pool_bins,
                             void* stream);

/* brkga_decode_multi_stage with each instance's rows at an explicit place:
 * instance k's pops[k] chromosomes start at float chrom_offsets[k] of d_chrom
 * and its makespans at element makespan_offsets[k] of d_makespan (host int64
 * [K]; either may be NULL = packed one after another).  Lets a GA decode the
 * non-elite rows of every instance's population block in place. */
int brkga_decode_multi_at(int32_t stage, const BrkgaProblem* problem, const float* d_chrom,
                          const int64_t* chrom_offsets, const int32_t* pops, double* d_makespan,
                          const int64_t* makespan_offsets, BrkgaPlacement* d_log, int32_t* d_status,
                          void* d_ws, size_t ws_bytes, int64_t pool_bins, void* stream);

/* Launch configuration of the decode kernel (the autotuner's knobs; no
 * reference counterpart).  Results never depend on it.
 *   warps_per_item  1, 2 or 4 warps per CTA, one (chromosome, machine) item
 *                   per CTA; 0 = automatic per launch (4 while the items fill
 *                   at most three waves of resident 4-warp CTAs, where the
 *                   latency of one item dominates; 2 up to sixteen waves of
 *                   2-warp CTAs; 1 beyond, where throughput does)
 *   ctas_per_sm     resident CTAs per SM for that size (1..32; 0 = 32
 *                   resident warps per SM, the register limit)
 *   smem_plates     plates of each item kept in shared memory (0..8, the
 *                   rest in the global pool; -1 = as many as fit, at most 4)
 *   task_max        0..8192, -1 = the default 8192: a warp that tests 32
 *                   candidate rows deals the (candidate that passed the
 *                   vacancy filter, 32-column output word) pairs across its
 *                   lanes when there are at most task_max of them, else each
 *                   lane tests its own candidate
 * ctas_per_sm and smem_plates need an explicit warps_per_item (with 0 they
 * must be 0 and -1).  A shape that cannot be resident is refused with
 * BRKGA_ERR_INVALID_ARGUMENT and the previous configuration kept.  The
 * workspace size depends on the configuration: query brkga_workspace_bytes
 * again after a change.  Not to be called while a decode of this problem is
 * being launched from another thread. */
int brkga_set_launch_config(BrkgaProblem* problem, int32_t warps_per_item, int32_t ctas_per_sm,
                            int32_t smem_plates, int32_t task_max);

/* The configuration a launch of `items` (chromosome, machine) items uses:
 * warps per item, CTAs per SM, plates per item in shared memory, the decode
 * kernel's grid (SMs x CTAs per SM) and task_max; any output may be NULL. */
int brkga_get_launch_config(const BrkgaProblem* problem, int64_t items, int32_t* warps_per_item,
                            int32_t* ctas_per_sm, int32_t* smem_plates, int32_t* resident_ctas,
                            int32_t* task_max);

/* Host-to-host evaluation, the drop-in for NativeFullDecoder::evaluate_batch
 * (full_native_decoder.py:563-641): copies h_chrom [P, 2N] float32 to the
 * device, decodes, and writes h_makespan [P] float64.  Grows its internal
 * workspace and retries on BRKGA_ERR_CAPACITY.  Synchronous.  h_log may be
 * NULL (else host BrkgaPlacement [P, M, N]). */
int brkga_evaluate_host(BrkgaProblem* problem, const float* h_chrom, int32_t P,
                        double* h_makespan, BrkgaPlacement* h_log);

/* Counters of the last brkga_evaluate_host call: placement tests (plate x
 * rotation pairs that passed the size and area filters and went to the
 * collision search), 32-row candidate chunks searched, plates opened, and
 * the algorithmic scan bytes sum over tests of 4*(L*ceil(W/32) + h*ceil(w/32))
 * (one read of the bit-packed plate and rotated mask).  The same four int64
 * values sit at byte offset 8 of a brkga_decode workspace after the run. */
int brkga_last_counters(const BrkgaProblem* problem, int64_t* tests, int64_t* chunks, int64_t* bins,
                        int64_t* scan_bytes);

/* Greedy initial solution (BRKGA_alg3.py:445-603, binClassInitialSol.py:41-111):
 * the parts (gene indices, h_order[n], the reference sorts them by height and
 * then area, both descending) are placed one by one where the largest machine
 * makespan grows least — a new plate on a machine or any existing plate of it
 * that can take the part.  Outputs per placement, in order: h_machine[k] and
 * h_place[k] = (gene, plate index within the machine, x, bottom row y,
 * rotation); h_machine_makespan[M].  Synchronous; allocates and frees its own
 * device memory.  Building the chromosome from this is host work
 * (brkga_fft2_b200.initial). */
int brkga_initial_solution_host(BrkgaProblem* problem, const int32_t* h_order, int32_t n, int32_t* h_machine,
                                BrkgaPlacement* h_place, double* h_machine_makespan);

/* ---- GA generation step (device-resident population; BRKGA_alg3.py:210-265) ----
 * Randomness: Philox4x32-10 keyed by `seed`, counters (key block, row,
 * generation, stream), so results are deterministic and independent of the
 * launch configuration.  The reference draws from NumPy's global MT19937, so
 * GA trajectories are not comparable draw for draw; the operators are. */

/* Uniform [0,1) float32 keys for rows skip_rows..P-1 of d_pop [P, n_keys]
 * (initial population, BRKGA_alg3.py:213). */
int brkga_ga_init_population(float* d_pop, int32_t P, int32_t n_keys, uint64_t seed, int32_t skip_rows,
                             void* stream);

/* d_order[P] = indices sorting d_fitness ascending, ties by index; NaN last.
 * P <= 65536 (a single-CTA sort up to 8192, ranking by counting above).
 * Replaces partition (BRKGA_alg3.py:178-186).  For 4096 < P <= 8192 the
 * first call on a device sets a kernel attribute, so make it outside graph capture. */
int brkga_ga_rank(const double* d_fitness, int32_t P, int32_t* d_order, void* stream);

/* Next population [elites | mutants | offspring] (BRKGA_alg3.py:188-208,246-250):
 * rows 0..n_elites-1 copy the best rows (and their fitness into d_next_fitness),
 * the next n_mutants rows are uniform keys, the rest are offspring of a uniform
 * elite and a uniform non-elite parent, each key taken from the elite with
 * probability rho.  The generation number is read from *d_generation. */
int brkga_ga_breed(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                   int32_t n_keys, int32_t n_elites, int32_t n_mutants, float rho, uint64_t seed,
                   const int64_t* d_generation, float* d_next_pop, double* d_next_fitness, void* stream);

/* brkga_ga_breed writing out_rows rows (>= P allowed): the parents still come
 * from the P-row population; rows past n_elites + n_mutants are offspring.
 * Builds the oversampled candidate pool that the surrogate screens. */
int brkga_ga_breed_pool(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                        int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, float rho,
                        uint64_t seed, const int64_t* d_generation, float* d_next_pop, double* d_next_fitness,
                        void* stream);

/* brkga_ga_breed_pool with offspring in families of `family` consecutive
 * rows sharing one parent pair: family f's pair is the one the plain breed
 * draws for offspring row n_elites + n_mutants + f, each child's crossover
 * mask its own; family = 1 is brkga_ga_breed_pool.  Lets a surrogate choose
 * among siblings while the parents stay those of the plain GA (no reference
 * counterpart: BRKGA_alg3.py:188-205 makes one child per pair). */
int brkga_ga_breed_families(const float* d_pop, const double* d_fitness, const int32_t* d_order, int32_t P,
                            int32_t out_rows, int32_t n_keys, int32_t n_elites, int32_t n_mutants, int32_t family,
                            float rho, uint64_t seed, const int64_t* d_generation, float* d_next_pop,
                            double* d_next_fitness, void* stream);

/* d_index[f] = f * family + the position of the smallest of d_pred[f * family
 * .. f * family + family - 1] (ties: the first; NaN loses to any number). */
int brkga_ga_select_families(const double* d_pred, int32_t n_families, int32_t family, int32_t* d_index,
                             void* stream);

/* d_dst[i, :] = d_src[d_index[i], :] for i < n (rows of n_keys float32). */
int brkga_ga_gather(const float* d_src, const int32_t* d_index, int32_t n, int32_t n_keys, float* d_dst,
                    void* stream);

/* Surrogate quality for generation g = *d_generation: d_stats[2g] = Spearman
 * correlation between predicted and exact makespans of the n decoded rows
 * (ranks taken from the two orderings d_order_pred / d_order_exact as
 * produced by brkga_ga_rank; infeasible rows excluded), d_stats[2g+1] = mean
 * absolute error.  d_scratch: int32 [2n]. */
int brkga_ga_screen_stats(const double* d_pred, const double* d_exact, const int32_t* d_order_pred,
                          const int32_t* d_order_exact, int32_t n, const int64_t* d_generation, double* d_stats,
                          int32_t stats_len, int32_t* d_scratch, void* stream);

/* Copy rows d_index[0..n) of d_pop [P, n_keys] and their d_fitness into slot
 * g = *d_generation of d_audit_pop [slots, n, n_keys] and d_audit_fit
 * [slots, n] (nothing when g >= slots): a sample of every generation's
 * exact makespans kept for verification after the run (no reference
 * counterpart). */
int brkga_ga_audit(const float* d_pop, const double* d_fitness, const int32_t* d_index, int32_t n,
                   int32_t n_keys, const int64_t* d_generation, int32_t slots, float* d_audit_pop,
                   double* d_audit_fit, void* stream);

/* After a population is scored: history[2g] = min, history[2g+1] = mean of
 * d_fitness for g = *d_generation (BRKGA_alg3.py:224-227,255-262); copies the
 * best row into d_best_solution when it beats *d_best_fitness; then ++*d_generation. */
int brkga_ga_track(const double* d_fitness, const float* d_pop, int32_t P, int32_t n_keys,
                   int64_t* d_generation, double* d_history, int32_t history_len, double* d_best_fitness,
                   float* d_best_solution, void* stream);

/* ---- bf16 GEMM on the tensor cores (tcgen05) ----
 * C[M,N] fp32 (row-major, ldc) = sum_k A[m,k] B[n,k]; A [M,K] and B [N,K]
 * bf16 row-major (K contiguous).  M % 128 == 0, N % 64 == 0, K % 64 == 0;
 * d_A and d_B 16-byte aligned, lda and ldb multiples of 8 (the operands are
 * loaded by TMA); *d_err is set to BRKGA_ERR_CUDA if a tensor-core or copy
 * wait times out.  Used by the surrogate; no reference counterpart. */
int brkga_gemm_bf16(const void* d_A, int32_t lda, const void* d_B, int32_t ldb, float* d_C, int32_t ldc,
                    int32_t M, int32_t N, int32_t K, int32_t* d_err, void* stream);

/* ---- Surrogate: MLP ranking chromosomes by predicted makespan ----
 * No counterpart in the reference (its GA decodes every offspring,
 * BRKGA_alg3.py:119-123).  Features: 3 per part in decode order (machine,
 * proc time, height time) + 2 per machine (area load, time load), padded to a
 * multiple of 64 -> 512 -> 256 -> 1 (ReLU); bf16 tensor-core GEMMs with fp32
 * accumulation, fp32 master weights, Adam.  All device memory is allocated by
 * brkga_surrogate_create; the other calls allocate nothing. */
typedef struct BrkgaSurrogate BrkgaSurrogate;
int brkga_surrogate_create(const BrkgaProblem* problem, int32_t max_batch /* % 128 == 0 */,
                           int32_t buffer_capacity, uint64_t seed, BrkgaSurrogate** out);
/* Feature sets: DECODE (the default above) = per part in decode order its
 * machine, proc time and height time, then per machine its area and time
 * load (3N + 2M values); ORDER = the parts sorted by sequencing key alone,
 * per part its key, its area over the largest part area and its height time
 * over the largest (3N values: the 600-value input of the 200-part screened
 * configuration).  A gradient step takes at most 16384 rows. */
#define BRKGA_SURROGATE_FEATURES_DECODE 0
#define BRKGA_SURROGATE_FEATURES_ORDER 1
int brkga_surrogate_create_ex(const BrkgaProblem* problem, int32_t max_batch, int32_t buffer_capacity,
                              uint64_t seed, int32_t features, BrkgaSurrogate** out);
void brkga_surrogate_destroy(BrkgaSurrogate* surrogate);
/* Initial weights again, empty example buffer, unset target scaling (synchronous). */
int brkga_surrogate_reset(BrkgaSurrogate* surrogate);
int brkga_surrogate_dims(const BrkgaSurrogate* surrogate, int32_t* in_features, int32_t* in_padded,
                         int64_t* n_params);
/* Predicted makespans (float64, makespan units) of P device chromosomes. */
int brkga_surrogate_predict(BrkgaSurrogate* surrogate, const float* d_chrom, int32_t P, double* d_pred,
                            void* stream);
/* Append the feasible rows of (chromosome features, exact makespan) to the
 * ring buffer of training examples; the first call fixes the target scaling. */
int brkga_surrogate_observe(BrkgaSurrogate* surrogate, const float* d_chrom, const double* d_makespan,
                            int32_t P, void* stream);
/* `steps` Adam steps on minibatches of `batch` rows drawn uniformly from the buffer. */
int brkga_surrogate_train(BrkgaSurrogate* surrogate, int32_t steps, int32_t batch, float lr, void* stream);
/* Lower-level pieces (tests): features into the activation rows; load a
 * minibatch; MSE gradients of the loaded minibatch; one Adam step. */
int brkga_surrogate_features(BrkgaSurrogate* surrogate, const float* d_chrom, int32_t P, void* stream);
int brkga_surrogate_load_batch(BrkgaSurrogate* surrogate, const void* d_X, const float* d_t, int32_t B,
                               int32_t n_valid, void* stream);
int brkga_surrogate_gradients(BrkgaSurrogate* surrogate, int32_t B, void* stream);
int brkga_surrogate_adam(BrkgaSurrogate* surrogate, float lr, void* stream);
/* Device addresses of internal arrays (any output may be NULL). */
int brkga_surrogate_buffers(const BrkgaSurrogate* surrogate, float** params, float** grads, void** X,
                            float** y, int32_t** err, int64_t** count, double** norm);
/* Synchronous copy of an internal array to/from host memory (see brkga_surrogate.cu). */
int brkga_surrogate_io(BrkgaSurrogate* surrogate, int32_t what, void* host, int64_t bytes, int32_t to_device);

/* ---- The collision test of one candidate chunk by either path ----
 * Replaces, for measurement and for the autotuner's choice of path, the
 * reference's FFT collision test (collision_backend.py:109-128; native
 * batch_fft_all_tests, full_native_decoder.py:1004-1234): the overlap of a
 * rotated part mask with a plate at 32 candidate top rows and every column.
 *   BRKGA_COLLISION_BITSET   the decode kernel's bit-packed run-dilation search
 *                            (every output word tested to the end)
 *   BRKGA_COLLISION_INT8_TC  an INT8 tensor-core correlation (tcgen05.mma
 *                            kind::i8, INT32 accumulators in tensor memory);
 *                            masks of at most 256 x 256 cells
 * One item: `plate` (device) holds L rows of ceil(W/32) + 2 uint32 words of
 * `machine`'s plate, bit c of a row = column c, zero past column W (the
 * decoder's plate format); `part_type` and `rot` name a rotation of the
 * problem; the candidates are top rows ty_hi - n, n = 0..31, with
 * 0 <= ty_hi <= L - h (rows below 0 come out empty); `out` (device) receives
 * 32 x ceil((W - w + 1) / 32) words, row n for candidate ty_hi - n, bit b of
 * word k set when the placement at column x = 32k + b overlaps nothing.
 * Both paths write identical words. */
#define BRKGA_COLLISION_BITSET 0
#define BRKGA_COLLISION_INT8_TC 1
typedef struct BrkgaChunkTest {
  const uint32_t* plate;
  uint32_t* out;
  int32_t machine;
  int32_t part_type;
  int32_t rot;
  int32_t ty_hi;
} BrkgaChunkTest;

/* Test n_items chunks (d_items: device array) by `path` on `stream`.  A
 * malformed item raises BRKGA_ERR_INVALID_ARGUMENT in *d_status (which the
 * caller zeroes) and writes nothing; a tensor-core wait that times out raises
 * BRKGA_ERR_CUDA.  Single-instance problems. */
int brkga_chunk_free(const BrkgaProblem* problem, int32_t path, const BrkgaChunkTest* d_items, int32_t n_items,
                     int32_t* d_status, void* stream);

/* ---- Measurement probe (no reference counterpart) ----
 * Shared-memory streaming kernel: `blocks` CTAs of `threads` threads (a
 * multiple of 32, at most 1024) each stream `iters` x 8 conflict-free 16-byte
 * ld.shared loads per thread over a 32 KB buffer.  d_sink: device uint32
 * [blocks * threads] (a fold of the loaded words, so the loads stay live);
 * d_cycles: device int64 [blocks], the clock64 cycles each CTA spent in its
 * load loop.  Bytes moved = blocks * threads * iters * 128; timed by the
 * caller, they give the shared-memory bandwidth that the decode kernel's
 * on-chip plate and mask reads are measured against. */
int brkga_probe_smem_stream(int32_t blocks, int32_t threads, int32_t iters, uint32_t* d_sink,
                            int64_t* d_cycles, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BRKGA_B200_H */
