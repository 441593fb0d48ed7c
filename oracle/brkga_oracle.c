/*
 * brkga_oracle.c — CPU oracle for the BRKGA chromosome decoder.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA decoder
 * is compared against (tests/, __graft_entry__.smoke(), and the CPU-baseline
 * leg of bench.py).  The product path never links, loads or calls it.
 *
 * It restates, statement by statement, the reference's sequential decoder
 * ("pp", paulonasc7/BRKGA_FFT2):
 *   placementProcedure            placement.py:94-165
 *   _process_single_machine       placement.py:29-91
 *   BuildingPlate.can_insert      binClassNew.py:45-144
 *   BuildingPlate.insert          binClassNew.py:155-174
 *   check_rotations_feasibility   numba_utils.py:50-94 (+ check_vacancy_fit_single :13-46)
 *   update_vacancy_vector_rows    numba_utils.py:160-188
 *   find_bottom_left_zero(_batch) collision_backend.py:109-213
 * The reference finds collision-free positions with a float FFT
 * cross-correlation rounded to the nearest integer; here the correlation is
 * evaluated exactly in integers (a position is free iff every run of ones in
 * every mask row covers only empty plate cells, checked with per-row prefix
 * counts).  The FFT error of the reference is < 0.004 at the sizes used
 * (far below the 0.5 rounding margin), so both give the same feasible set;
 * the golden vectors in tests/golden pin this.
 *
 * Two choices the reference leaves to its sort implementation are fixed:
 * equal sequencing keys keep gene order (stable sort), and machine keys are
 * compared in float32 or float64 as desc->threshold_mode says.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/brkga_b200.h"

#define INFEASIBLE_PENALTY 1e16 /* placement.py:9 */

typedef struct {
  int h, w;
  const uint8_t* mask; /* row-major h*w */
  int* dens;           /* [h] longest run of ones per row */
  int* run_off;        /* [h+1] */
  int* run_a;          /* run start column */
  int* run_d;          /* run length */
} Rot;

typedef struct {
  const BrkgaProblemDesc* d;
  Rot* rots; /* [T*4] */
} Model;

typedef struct {
  int L, W;
  uint8_t* grid;   /* L*W */
  int* pre;        /* L*(W+1) prefix counts of occupied cells per row */
  int64_t* vac;    /* L   vacancy (longest empty run) per row, init W (binClassNew.py:20) */
  double area;
  int min_row, max_row, enc;
  double pt, pth;
} Plate;

static void rot_build(Rot* r, const uint8_t* mask, int h, int w) {
  r->h = h;
  r->w = w;
  r->mask = mask;
  r->dens = (int*)calloc((size_t)h, sizeof(int));
  r->run_off = (int*)calloc((size_t)h + 1, sizeof(int));
  int cap = 16, n = 0;
  r->run_a = (int*)malloc(sizeof(int) * cap);
  r->run_d = (int*)malloc(sizeof(int) * cap);
  for (int i = 0; i < h; ++i) {
    r->run_off[i] = n;
    int j = 0, best = 0;
    while (j < w) {
      if (mask[(size_t)i * w + j]) {
        int s = j;
        while (j < w && mask[(size_t)i * w + j]) ++j;
        if (n == cap) {
          cap *= 2;
          r->run_a = (int*)realloc(r->run_a, sizeof(int) * cap);
          r->run_d = (int*)realloc(r->run_d, sizeof(int) * cap);
        }
        r->run_a[n] = s;
        r->run_d[n] = j - s;
        if (j - s > best) best = j - s;
        ++n;
      } else {
        ++j;
      }
    }
    r->dens[i] = best;
  }
  r->run_off[h] = n;
}

static void model_init(Model* m, const BrkgaProblemDesc* d) {
  m->d = d;
  m->rots = (Rot*)calloc((size_t)d->n_types * 4, sizeof(Rot));
  for (int t = 0; t < d->n_types; ++t)
    for (int r = 0; r < d->part_nrot[t]; ++r) {
      int k = t * 4 + r;
      rot_build(&m->rots[k], d->masks + d->rot_mask_offset[k], d->rot_h[k], d->rot_w[k]);
    }
}

static void model_free(Model* m) {
  for (int k = 0; k < m->d->n_types * 4; ++k) {
    free(m->rots[k].dens);
    free(m->rots[k].run_off);
    free(m->rots[k].run_a);
    free(m->rots[k].run_d);
  }
  free(m->rots);
}

static void plate_init(Plate* p, int L, int W) {
  p->L = L;
  p->W = W;
  p->grid = (uint8_t*)calloc((size_t)L * W, 1);
  p->pre = (int*)calloc((size_t)L * (W + 1), sizeof(int));
  p->vac = (int64_t*)malloc(sizeof(int64_t) * (size_t)L);
  for (int i = 0; i < L; ++i) p->vac[i] = W;
  p->area = 0.0;
  p->min_row = L;
  p->max_row = -1;
  p->enc = 0;
  p->pt = 0.0;
  p->pth = 0.0;
}

static void plate_free(Plate* p) {
  free(p->grid);
  free(p->pre);
  free(p->vac);
}

/* numba_utils.py:13-46 — some window of h rows has vac[s+i] >= dens[i]. */
static int vacancy_fit(const int64_t* vac, int n, const int* dens, int h) {
  if (h > n) return 0;
  for (int s = 0; s + h <= n; ++s) {
    int fits = 1;
    for (int i = 0; i < h; ++i)
      if (vac[s + i] < dens[i]) {
        fits = 0;
        break;
      }
    if (fits) return 1;
  }
  return 0;
}

/* Exact overlap test: part top-left at (ty, x) collides with nothing. */
static int position_free(const Plate* p, const Rot* r, int ty, int x) {
  const int W1 = p->W + 1;
  for (int i = 0; i < r->h; ++i) {
    const int* pr = p->pre + (size_t)(ty + i) * W1;
    for (int k = r->run_off[i]; k < r->run_off[i + 1]; ++k) {
      int c0 = x + r->run_a[k];
      if (pr[c0 + r->run_d[k]] - pr[c0] != 0) return 0;
    }
  }
  return 1;
}

/* collision_backend.py:109-128 semantics: among collision-free positions with
 * bottom row y in [h-1, L-1] and left column x in [0, W-w], the largest y,
 * then the smallest x.  Returns 1 and writes (x, y) if any exists. */
static int bottom_left(const Plate* p, const Rot* r, int* ox, int* oy) {
  for (int y = p->L - 1; y >= r->h - 1; --y) {
    int ty = y - r->h + 1;
    for (int x = 0; x + r->w <= p->W; ++x) {
      if (position_free(p, r, ty, x)) {
        *ox = x;
        *oy = y;
        return 1;
      }
    }
  }
  return 0;
}

/* binClassNew.py:155-174 (+ numba_utils.py:160-188 for the vacancy rows). */
static void plate_insert(Plate* p, const Rot* r, int x, int y, double part_area) {
  p->area += part_area;
  int ty = y - r->h + 1;
  for (int i = 0; i < r->h; ++i) {
    uint8_t* g = p->grid + (size_t)(ty + i) * p->W;
    for (int j = 0; j < r->w; ++j) g[x + j] += r->mask[(size_t)i * r->w + j];
    int* pr = p->pre + (size_t)(ty + i) * (p->W + 1);
    int acc = 0, cur = 0, best = 0;
    pr[0] = 0;
    for (int c = 0; c < p->W; ++c) {
      acc += g[c] != 0;
      pr[c + 1] = acc;
      if (g[c] == 0) {
        if (++cur > best) best = cur;
      } else {
        cur = 0;
      }
    }
    p->vac[ty + i] = best;
  }
  if (ty < p->min_row) p->min_row = ty;
  if (y > p->max_row) p->max_row = y;
  /* calculate_enclosure_box_length, binClassNew.py:147-152 */
  p->enc = (p->min_row > p->max_row) ? 0 : p->L - p->min_row;
}

/* The choice part of can_insert (binClassNew.py:45-117, binClassInitialSol.py:41-111):
 * returns 1 and (x, y, rotation) when some rotation fits. */
static int best_position(const Plate* p, const Model* m, int t, double part_area, int* ox, int* oy, int* orot) {
  const BrkgaProblemDesc* d = m->d;
  int nrot = d->part_nrot[t];
  double potential = p->area + part_area;
  int found = 0, have_best = 0, bx = 0, by = 0, br = 0;
  double packing_density = 0.0;
  for (int r = 0; r < nrot; ++r) {
    const Rot* R = &m->rots[t * 4 + r];
    if (R->h > p->L || R->w > p->W) continue;
    if (!vacancy_fit(p->vac, p->L, R->dens, R->h)) continue;
    int x, y;
    if (!bottom_left(p, R, &x, &y)) continue;
    found = 1;
    int top = y - R->h + 1;
    int new_len = p->enc > (p->L - top) ? p->enc : (p->L - top);
    double dens = potential / (double)((int64_t)new_len * p->W);
    if (dens > packing_density) {
      have_best = 1;
      packing_density = dens;
      bx = x;
      by = y;
      br = r;
    } else if (have_best && dens == packing_density && y > by) {
      bx = x;
      by = y;
      br = r;
    } else if (have_best && dens == packing_density && y == by && x < bx) {
      bx = x;
      by = y;
      br = r;
    }
  }
  if (!found || !have_best) return 0;
  *ox = bx;
  *oy = by;
  *orot = br;
  return 1;
}

/* binClassNew.py:45-144.  Returns 1 if the part was inserted. */
static int can_insert(Plate* p, const Model* m, int t, double part_area, double pt, double pth,
                      BrkgaPlacement* log, int gene, int bin_idx) {
  const BrkgaProblemDesc* d = m->d;
  int nrot = d->part_nrot[t];
  double potential = p->area + part_area;
  int found = 0, have_best = 0, bx = 0, by = 0, br = 0;
  double packing_density = 0.0; /* binClassNew.py:48 */
  for (int r = 0; r < nrot; ++r) {
    const Rot* R = &m->rots[t * 4 + r];
    if (R->h > p->L || R->w > p->W) continue;                /* numba_utils.py:82-84 */
    if (!vacancy_fit(p->vac, p->L, R->dens, R->h)) continue;  /* numba_utils.py:92 */
    int x, y;
    if (!bottom_left(p, R, &x, &y)) continue;
    found = 1; /* binClassNew.py:103-104 */
    int top = y - R->h + 1;
    int new_len = p->enc > (p->L - top) ? p->enc : (p->L - top);
    double dens = potential / (double)((int64_t)new_len * p->W); /* binClassNew.py:107-108 */
    if (dens > packing_density) {                                 /* binClassNew.py:110-117 */
      have_best = 1;
      packing_density = dens;
      bx = x;
      by = y;
      br = r;
    } else if (have_best && dens == packing_density && y > by) {
      bx = x;
      by = y;
      br = r;
    } else if (have_best && dens == packing_density && y == by && x < bx) {
      bx = x;
      by = y;
      br = r;
    }
  }
  if (!found || !have_best) return 0; /* area > 0 is validated, so found implies have_best */
  plate_insert(p, &m->rots[t * 4 + br], bx, by, part_area);
  p->pt += pt;
  if (pth > p->pth) p->pth = pth;
  if (log) {
    log->gene = gene;
    log->bin = bin_idx;
    log->x = bx;
    log->y = by;
    log->rot = br;
  }
  return 1;
}

typedef struct {
  float key;
  int gene;
} KeyGene;

static int cmp_keygene(const void* a, const void* b) {
  const KeyGene* x = (const KeyGene*)a;
  const KeyGene* y = (const KeyGene*)b;
  const int xn = x->key != x->key, yn = y->key != y->key; /* NaN sorts last, as in np.argsort */
  if (xn != yn) return xn - yn;
  if (!xn) {
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
  }
  return (x->gene > y->gene) - (x->gene < y->gene); /* stable: gene order on ties */
}

/* placement.py:118-127 (float32 path) / full_native_decoder.py:961-973 (float64). */
static int on_machine(const BrkgaProblemDesc* d, float mv, int m) {
  int M = d->n_machines;
  if (M <= 1) return 1;
  if (d->threshold_mode == BRKGA_THRESH_F32) {
    float lo = m > 0 ? (float)d->thresholds[m - 1] : 0.0f;
    float hi = m < M - 1 ? (float)d->thresholds[m] : 0.0f;
    if (m == 0) return mv <= hi;
    if (m == M - 1) return mv > lo;
    return mv > lo && mv <= hi;
  } else {
    double v = (double)mv;
    if (m == 0) return v <= d->thresholds[0];
    if (m == M - 1) return v > d->thresholds[m - 1];
    return v > d->thresholds[m - 1] && v <= d->thresholds[m];
  }
}

/* Decode one chromosome: placement.py:94-165.  Returns the makespan, or
 * NaN with *err set if a new plate receives a best rotation that does not
 * fit (the reference raises inside numpy there). */
static double decode_one(const Model* m, const float* chrom, BrkgaPlacement* log, KeyGene* buf,
                         Plate* plates, int* err) {
  const BrkgaProblemDesc* d = m->d;
  const int N = d->n_genes, M = d->n_machines, T = d->n_types;
  double worst = 0.0;
  int infeasible = 0;
  for (int mi = 0; mi < M; ++mi) {
    int n = 0;
    for (int j = 0; j < N; ++j)
      if (on_machine(d, chrom[N + j], mi)) {
        buf[n].key = chrom[j] == 0.0f ? 0.0f : chrom[j];
        buf[n].gene = j;
        ++n;
      }
    qsort(buf, (size_t)n, sizeof(KeyGene), cmp_keygene);
    const int L = d->bin_length[mi], W = d->bin_width[mi];
    int nb = 0;
    int machine_infeasible = 0;
    for (int k = 0; k < n; ++k) {
      int gene = buf[k].gene;
      int t = d->gene_type[gene];
      int h0 = d->rot_h[t * 4], w0 = d->rot_w[t * 4];
      if ((h0 > L || w0 > W) && (w0 > L || h0 > W)) { /* placement.py:47-53 */
        machine_infeasible = 1;
        break;
      }
      double a = d->part_area[t];
      double pt = d->proc_time[(size_t)mi * T + t];
      double pth = d->proc_time_height[(size_t)mi * T + t];
      BrkgaPlacement* lg = log ? &log[(size_t)mi * N + k] : NULL;
      int placed = 0;
      for (int b = 0; b < nb && !placed; ++b) {
        if (plates[b].area + a > d->bin_area[mi]) continue; /* placement.py:57-59 */
        placed = can_insert(&plates[b], m, t, a, pt, pth, lg, gene, b);
      }
      if (!placed) { /* placement.py:66-83 */
        int r = d->part_best_rot[t];
        const Rot* R = &m->rots[t * 4 + r];
        if (R->h > L || R->w > W) {
          *err = BRKGA_ERR_NEW_BIN_UNFIT;
          for (int b = 0; b < nb; ++b) plate_free(&plates[b]);
          return NAN;
        }
        plate_init(&plates[nb], L, W);
        plate_insert(&plates[nb], R, 0, L - 1, a);
        plates[nb].pt += pt;
        if (pth > plates[nb].pth) plates[nb].pth = pth;
        if (lg) {
          lg->gene = gene;
          lg->bin = nb;
          lg->x = 0;
          lg->y = L - 1;
          lg->rot = r;
        }
        ++nb;
      }
    }
    double ms = 0.0; /* placement.py:86-89 */
    for (int b = 0; b < nb; ++b) ms += (plates[b].pt + plates[b].pth) + d->setup_time[mi];
    for (int b = 0; b < nb; ++b) plate_free(&plates[b]);
    if (machine_infeasible) {
      infeasible = 1;
      continue;
    }
    if (ms > worst) worst = ms;
  }
  return infeasible ? INFEASIBLE_PENALTY : worst;
}

typedef struct {
  const Model* m;
  const float* chrom;
  int P;
  int* next;  /* the next row to decode, shared by the threads */
  double* out;
  BrkgaPlacement* log;
  int err;
} Job;

static void* worker(void* arg) {
  Job* jb = (Job*)arg;
  const BrkgaProblemDesc* d = jb->m->d;
  const int N = d->n_genes, M = d->n_machines;
  KeyGene* buf = (KeyGene*)malloc(sizeof(KeyGene) * (size_t)(N > 0 ? N : 1));
  Plate* plates = (Plate*)malloc(sizeof(Plate) * (size_t)(N > 0 ? N : 1));
  /* rows are taken one at a time from a shared counter, so a thread that
     drew short rows takes more of them (rows differ in cost several-fold) */
  for (int c = __atomic_fetch_add(jb->next, 1, __ATOMIC_RELAXED); c < jb->P;
       c = __atomic_fetch_add(jb->next, 1, __ATOMIC_RELAXED)) {
    BrkgaPlacement* lg = jb->log ? jb->log + (size_t)c * M * N : NULL;
    if (lg)
      for (size_t i = 0; i < (size_t)M * N; ++i) {
        lg[i].gene = -1;
        lg[i].bin = lg[i].x = lg[i].y = lg[i].rot = -1;
      }
    int err = 0;
    jb->out[c] = decode_one(jb->m, jb->chrom + (size_t)c * 2 * N, lg, buf, plates, &err);
    if (err) jb->err = err;
  }
  free(buf);
  free(plates);
  return NULL;
}

/* Decode P chromosomes (host float32 [P, 2N]) into host makespans [P] and an
 * optional placement log [P, M, N] using n_threads POSIX threads. */
int oracle_decode(const BrkgaProblemDesc* d, const float* chrom, int P, double* makespan,
                  BrkgaPlacement* log, int n_threads) {
  if (!d || (!chrom && P > 0) || (!makespan && P > 0) || P < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  if (n_threads < 1) n_threads = 1;
  if (n_threads > P && P > 0) n_threads = P;
  Model m;
  model_init(&m, d);
  Job* jobs = (Job*)calloc((size_t)n_threads, sizeof(Job));
  pthread_t* th = (pthread_t*)calloc((size_t)n_threads, sizeof(pthread_t));
  int next = 0;
  for (int i = 0; i < n_threads; ++i) {
    jobs[i].m = &m;
    jobs[i].chrom = chrom;
    jobs[i].P = P;
    jobs[i].next = &next;
    jobs[i].out = makespan;
    jobs[i].log = log;
    jobs[i].err = 0;
  }
  if (n_threads == 1) {
    worker(&jobs[0]);
  } else {
    for (int i = 0; i < n_threads; ++i) pthread_create(&th[i], NULL, worker, &jobs[i]);
    for (int i = 0; i < n_threads; ++i) pthread_join(th[i], NULL);
  }
  int err = 0;
  for (int i = 0; i < n_threads; ++i)
    if (jobs[i].err) err = jobs[i].err;
  free(jobs);
  free(th);
  model_free(&m);
  return err;
}

/* Greedy initial solution, BRKGA_alg3.py:445-566 with binClassInitialSol.BuildingPlate:
 * parts in `order` (gene indices); each goes to the option with the smallest
 * max(current worst makespan, machine makespan after placing it): a new plate
 * on a machine (checked first, replaced on <=), or an existing plate of the
 * machine (every plate tested, no area filter; within a machine an equal
 * makespan does not replace an earlier plate).  Outputs as brkga_initial_solution_host. */
int oracle_initial_solution(const BrkgaProblemDesc* d, const int32_t* order, int n, int32_t* out_machine,
                            BrkgaPlacement* out, double* machine_makespan) {
  if (!d || n < 0) return BRKGA_ERR_INVALID_ARGUMENT;
  Model m;
  model_init(&m, d);
  const int M = d->n_machines, T = d->n_types;
  Plate* plates = (Plate*)malloc(sizeof(Plate) * (size_t)(n > 0 ? n : 1));
  int* pmach = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int* pidx = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int np = 0, err = 0;
  double cw = 0.0;
  for (int q = 0; q < M; ++q) machine_makespan[q] = 0.0;
  for (int k = 0; k < n && !err; ++k) {
    int gene = order[k], t = d->gene_type[gene];
    double a = d->part_area[t];
    double best = INFINITY, ccand = 0.0;
    int kind = -1, cm = -1, cb = -1, cx = 0, cy = 0, cr = 0;
    for (int q = 0; q < M; ++q) {
      int placed_in_exist = 0;
      int L = d->bin_length[q], W = d->bin_width[q];
      int h0 = d->rot_h[t * 4], w0 = d->rot_w[t * 4];
      if ((h0 > L || w0 > W) && (w0 > L || h0 > W)) continue; /* :465-470 */
      double mm = machine_makespan[q];
      double pt = d->proc_time[(size_t)q * T + t], pth = d->proc_time_height[(size_t)q * T + t];
      double cand = ((mm + d->setup_time[q]) + pt) + pth; /* :472 */
      double nm = cw > cand ? cw : cand;
      if (nm <= best) {
        best = nm;
        kind = 0;
        cm = q;
        ccand = cand;
      }
      for (int b = 0; b < np; ++b) {
        if (pmach[b] != q) continue;
        int x, y, r;
        if (!best_position(&plates[b], &m, t, a, &x, &y, &r)) continue;
        double cand2 = plates[b].pth < pth ? ((mm - plates[b].pth) + pth) + pt : mm + pt; /* :486-489 */
        double nm2 = cw > cand2 ? cw : cand2;
        if (nm2 <= best) {
          if (placed_in_exist && nm2 == best) continue;
          placed_in_exist = 1;
          best = nm2;
          kind = 1;
          cm = q;
          cb = b;
          cx = x;
          cy = y;
          cr = r;
          ccand = cand2;
        }
      }
    }
    if (kind < 0) {
      err = BRKGA_ERR_BAD_INSTANCE;
      break;
    }
    int L = d->bin_length[cm], W = d->bin_width[cm];
    if (kind == 0) {
      cr = d->part_best_rot[t];
      const Rot* R = &m.rots[t * 4 + cr];
      if (R->h > L || R->w > W) {
        err = BRKGA_ERR_NEW_BIN_UNFIT;
        break;
      }
      cb = np++;
      plate_init(&plates[cb], L, W);
      pmach[cb] = cm;
      int idx = 0;
      for (int b = 0; b < cb; ++b) idx += pmach[b] == cm;
      pidx[cb] = idx;
      cx = 0;
      cy = L - 1;
    }
    plate_insert(&plates[cb], &m.rots[t * 4 + cr], cx, cy, a);
    plates[cb].pt += d->proc_time[(size_t)cm * T + t];
    double pthc = d->proc_time_height[(size_t)cm * T + t];
    if (pthc > plates[cb].pth) plates[cb].pth = pthc;
    out_machine[k] = cm;
    out[k].gene = gene;
    out[k].bin = pidx[cb];
    out[k].x = cx;
    out[k].y = cy;
    out[k].rot = cr;
    machine_makespan[cm] = ccand;
    if (ccand > cw) cw = ccand;
  }
  for (int b = 0; b < np; ++b) plate_free(&plates[b]);
  free(plates);
  free(pmach);
  free(pidx);
  model_free(&m);
  return err;
}

int oracle_abi_version(void) { return BRKGA_ABI_VERSION; }
