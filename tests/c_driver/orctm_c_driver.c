/*
 * A plain C caller of the library's ABI (include/orctm_gpu.h), the way a
 * Fortran or C host model uses it: build the descriptor from host arrays,
 * create a handle, upload the state, run hot-path steps, download results.
 *
 *   orctm_c_driver <input> <output>
 *
 * <input> (native byte order): int32 ie, je, ke, ntracers, ob_west, ob_east,
 * ob_north, ob_south, nsteps, solver; float64 dt, almzer, aulapts, aulapuv,
 * ah00, rtol; then the geometry arrays in the order of orctm_desc (dzw, di,
 * dlxp, dlyp, dtdxpo, dtdyo, dlxu, dlyu, dtdxuo, dlxv, dlyv, dpye, ddpo,
 * weto, dduo, amsuo, ddue, amsue) in the host layouts of the header; then
 * every field 0 .. ORCTM_F_THO + ntracers - 1 (orctm_field_size values each).
 * <output>: UOO, VOE, WNO, PNH and the tracers after the steps, float64.
 * Exit status 0 on success; otherwise 2 and the library's message on stderr
 * (the create status is printed as "create status N").
 */
#include <stdio.h>
#include <stdlib.h>

#include "orctm_gpu.h"

static double* read_doubles(FILE* f, size_t n) {
  double* a = (double*)malloc(sizeof(double) * (n ? n : 1));
  if (!a || fread(a, sizeof(double), n, f) != n) {
    fprintf(stderr, "short input\n");
    exit(2);
  }
  return a;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  int iv[10];
  double dv[6];
  if (fread(iv, sizeof(int), 10, f) != 10 || fread(dv, sizeof(double), 6, f) != 6) return 2;
  const int ie = iv[0], je = iv[1], ke = iv[2], ntr = iv[3], nsteps = iv[8], solver = iv[9];
  const size_t p2 = (size_t)ie * je, u2 = (size_t)(ie + 1) * je, v2 = (size_t)ie * (je + 1);
  orctm_desc d = {0};
  d.ie = ie; d.je = je; d.ke = ke; d.i_start = 0; d.j_start = 0; d.ntracers = ntr;
  d.ob_west = iv[4]; d.ob_east = iv[5]; d.ob_north = iv[6]; d.ob_south = iv[7];
  d.dt = dv[0]; d.almzer = dv[1]; d.aulapts = dv[2]; d.aulapuv = dv[3]; d.ah00 = dv[4];
  d.dzw = read_doubles(f, ke);
  d.di = read_doubles(f, ke + 1);
  d.dlxp = read_doubles(f, p2); d.dlyp = read_doubles(f, p2);
  d.dtdxpo = read_doubles(f, p2); d.dtdyo = read_doubles(f, p2);
  d.dlxu = read_doubles(f, u2); d.dlyu = read_doubles(f, u2); d.dtdxuo = read_doubles(f, u2);
  d.dlxv = read_doubles(f, v2); d.dlyv = read_doubles(f, v2); d.dpye = read_doubles(f, v2);
  d.ddpo = read_doubles(f, p2 * ke); d.weto = read_doubles(f, p2 * ke);
  d.dduo = read_doubles(f, u2 * ke); d.amsuo = read_doubles(f, u2 * ke);
  d.ddue = read_doubles(f, v2 * ke); d.amsue = read_doubles(f, v2 * ke);
  d.device = 0;

  orctm_handle* h = NULL;
  int st = orctm_create(&d, &h);
  if (st != ORCTM_OK) {
    fprintf(stderr, "create status %d: %s\n", st, orctm_last_error(NULL));
    return 2;
  }
  for (int fld = 0; fld < ORCTM_F_THO + ntr; ++fld) {
    size_t n = 0;
    if (orctm_field_size(h, fld, &n) != ORCTM_OK) return 2;
    double* a = read_doubles(f, n);
    st = orctm_upload(h, fld, a, n);
    free(a);
    if (st != ORCTM_OK) {
      fprintf(stderr, "upload %d: %s\n", fld, orctm_last_error(h));
      return 2;
    }
  }
  fclose(f);
  if (orctm_set_solver(h, solver, dv[5], 20000) != ORCTM_OK) return 2;
  for (int s = 0; s < nsteps; ++s) {
    orctm_solve_stats ss;
    st = orctm_step_hotpath(h, &ss);
    if (st != ORCTM_OK && st != ORCTM_E_NOT_CONVERGED) {
      fprintf(stderr, "step %d: %s\n", s, orctm_last_error(h));
      return 2;
    }
    printf("step %d: %d iterations, relres %.3e\n", s, ss.iterations, ss.relres);
  }
  FILE* o = fopen(argv[2], "wb");
  if (!o) return 2;
  const int outs[4] = {ORCTM_F_UOO, ORCTM_F_VOE, ORCTM_F_WNO, ORCTM_F_PNH};
  for (int k = 0; k < 4 + ntr; ++k) {
    const int fld = k < 4 ? outs[k] : ORCTM_F_THO + (k - 4);
    size_t n = 0;
    orctm_field_size(h, fld, &n);
    double* a = (double*)malloc(sizeof(double) * n);
    if (!a || orctm_download(h, fld, a, n) != ORCTM_OK) return 2;
    fwrite(a, sizeof(double), n, o);
    free(a);
  }
  fclose(o);
  orctm_destroy(h);
  return 0;
}
