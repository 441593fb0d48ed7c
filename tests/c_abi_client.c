/* A plain C client of include/brkga_b200.h, as a C or C++ host of the
 * reference's native decoder would bind it (full_native_decoder.py:408-641).
 *
 *   c_abi_client <instance file> <population file> <output file>
 *
 * The instance file holds the BrkgaProblemDesc tables in this order, all
 * little-endian: int32 n_genes, n_machines, n_types, threshold_mode, int64
 * masks_bytes; then int32 gene_type[N], double thresholds[M-1], int32
 * bin_length[M], int32 bin_width[M], double bin_area[M], double
 * setup_time[M], double proc_time[M*T], double proc_time_height[M*T], double
 * part_area[T], int32 part_nrot[T], int32 part_best_rot[T], int32
 * rot_h[4T], int32 rot_w[4T], int64 rot_mask_offset[4T], uint8
 * masks[masks_bytes].  The population file: int32 P, then float32 [P, 2N].
 * Writes float64 makespans [P] to the output file.  Exit status: 0, or the
 * BrkgaStatus of the failing call (its text on stderr), or 100 on I/O errors.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "brkga_b200.h"

static void* read_block(FILE* f, size_t bytes) {
  void* p = malloc(bytes ? bytes : 1);
  if (!p || (bytes && fread(p, 1, bytes, f) != bytes)) {
    free(p);
    return NULL;
  }
  return p;
}

int main(int argc, char** argv) {
  if (argc != 4) {
    fprintf(stderr, "usage: %s instance population output\n", argv[0]);
    return 100;
  }
  FILE* fi = fopen(argv[1], "rb");
  if (!fi) return 100;
  int32_t hdr[4];
  int64_t masks_bytes = 0;
  if (fread(hdr, 4, 4, fi) != 4 || fread(&masks_bytes, 8, 1, fi) != 1) return 100;
  const int32_t N = hdr[0], M = hdr[1], T = hdr[2];
  BrkgaProblemDesc d;
  memset(&d, 0, sizeof(d));
  d.n_genes = N;
  d.n_machines = M;
  d.n_types = T;
  d.threshold_mode = hdr[3];
  d.gene_type = read_block(fi, (size_t)N * 4);
  d.thresholds = read_block(fi, (size_t)(M > 1 ? M - 1 : 0) * 8);
  d.bin_length = read_block(fi, (size_t)M * 4);
  d.bin_width = read_block(fi, (size_t)M * 4);
  d.bin_area = read_block(fi, (size_t)M * 8);
  d.setup_time = read_block(fi, (size_t)M * 8);
  d.proc_time = read_block(fi, (size_t)M * T * 8);
  d.proc_time_height = read_block(fi, (size_t)M * T * 8);
  d.part_area = read_block(fi, (size_t)T * 8);
  d.part_nrot = read_block(fi, (size_t)T * 4);
  d.part_best_rot = read_block(fi, (size_t)T * 4);
  d.rot_h = read_block(fi, (size_t)T * 16);
  d.rot_w = read_block(fi, (size_t)T * 16);
  d.rot_mask_offset = read_block(fi, (size_t)T * 32);
  d.masks = read_block(fi, (size_t)masks_bytes);
  d.masks_bytes = masks_bytes;
  fclose(fi);
  if (!d.gene_type || !d.bin_length || !d.masks || !d.rot_mask_offset) return 100;

  FILE* fp = fopen(argv[2], "rb");
  int32_t P = 0;
  if (!fp || fread(&P, 4, 1, fp) != 1 || P < 0) return 100;
  float* chrom = read_block(fp, (size_t)P * 2 * N * sizeof(float));
  fclose(fp);
  if (!chrom) return 100;

  if (brkga_abi_version() != BRKGA_ABI_VERSION) return 100;
  BrkgaProblem* problem = NULL;
  int st = brkga_problem_create(&d, &problem);
  if (st != BRKGA_OK) {
    fprintf(stderr, "brkga_problem_create: %s\n", brkga_status_string(st));
    return st;
  }
  double* makespan = malloc((size_t)(P ? P : 1) * sizeof(double));
  st = brkga_evaluate_host(problem, chrom, P, makespan, NULL);
  if (st != BRKGA_OK) {
    fprintf(stderr, "brkga_evaluate_host: %s\n", brkga_status_string(st));
    brkga_problem_destroy(problem);
    return st;
  }
  brkga_problem_destroy(problem);
  FILE* fo = fopen(argv[3], "wb");
  if (!fo || fwrite(makespan, sizeof(double), (size_t)P, fo) != (size_t)P) return 100;
  fclose(fo);
  printf("decoded %d chromosomes\n", P);
  return 0;
}
