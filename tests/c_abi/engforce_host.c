/* A C host program driving the engine through include/mdff_gpu.h the way the
   Fortran shim does: parameters once (mdff_gpu_create), then engforce calls
   on caller-owned host arrays, then mdff_gpu_destroy.
     engforce_host params.bin cell.bin pos.bin out.bin ncalls
   params.bin: the raw mdff_params; cell.bin: 9 doubles (row-major A); pos.bin:
   rx[natm], ry[natm], rz[natm]; out.bin: fx, fy, fz [natm] each, mu [natm][3],
   then u_bmhft, u_coul, u_pol of the last call.  Exit status: 0, or the
   first non-zero library status, or 100 + an I/O error. */
#include <stdio.h>
#include <stdlib.h>

#include "mdff_gpu.h"

static void* slurp(const char* path, size_t want) {
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  void* b = malloc(want ? want : 1);
  size_t got = b ? fread(b, 1, want, f) : 0;
  int extra = fgetc(f) != EOF;
  fclose(f);
  if (!b || got != want || extra) {
    free(b);
    return NULL;
  }
  return b;
}

int main(int argc, char** argv) {
  if (argc != 6) return 101;
  mdff_params* p = (mdff_params*)slurp(argv[1], sizeof(mdff_params));
  double* cell = (double*)slurp(argv[2], 9 * sizeof(double));
  if (!p || !cell || p->natm <= 0) return 102;
  size_t n = (size_t)p->natm;
  double* pos = (double*)slurp(argv[3], 3 * n * sizeof(double));
  int ncalls = atoi(argv[5]);
  if (!pos || ncalls < 1) return 103;
  double* out = (double*)calloc(6 * n + 3, sizeof(double));
  if (!out) return 104;
  mdff_handle h = NULL;
  int st = mdff_gpu_create(p, cell, &h);
  if (st != MDFF_OK) {
    fprintf(stderr, "create: %s (%s)\n", mdff_gpu_strerror(st), mdff_gpu_last_error(NULL));
    return st;
  }
  mdff_result r = {0};
  r.fx = out;
  r.fy = out + n;
  r.fz = out + 2 * n;
  r.mu = out + 3 * n;
  r.ef = NULL;
  for (int it = 0; it < ncalls && st == MDFF_OK; ++it)
    st = mdff_gpu_engforce(h, pos, pos + n, pos + 2 * n, it, &r);
  if (st != MDFF_OK) {
    fprintf(stderr, "engforce: %s (%s)\n", mdff_gpu_strerror(st), mdff_gpu_last_error(h));
  } else {
    out[6 * n] = r.u_bmhft;
    out[6 * n + 1] = r.u_coul;
    out[6 * n + 2] = r.u_pol;
    FILE* f = fopen(argv[4], "wb");
    if (!f || fwrite(out, sizeof(double), 6 * n + 3, f) != 6 * n + 3) st = 105;
    if (f) fclose(f);
  }
  mdff_gpu_destroy(h);
  free(out);
  free(pos);
  free(cell);
  free(p);
  return st;
}
