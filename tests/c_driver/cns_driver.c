/*
 * A plain C caller of libcodens_b200.so (no Python, no torch): what a Fortran
 * driver does through ISO_C_BINDING, written in C.
 *
 *   cns_driver CASE OUT
 *
 * CASE is a binary case description (little-endian; written by
 * tests/test_gpu_c_driver.py): int64 nblk, ld, nbnd, nlist; int32 dims[3 nblk];
 * double phys[9]; double scheme[18] (the numeric fields of cns_scheme_t in
 * declaration order); the boundary tables type, blk, face (int32 x nbnd), mpb
 * (int64 x nbnd), mmb, partner (int32 x nbnd), cosr, sinr (double x nbnd),
 * ncbd, ncin (int64 x nlist), bceqt (double x 5 nlist); x, y, z (double x ld);
 * v (double x 5 ld).
 *
 * The driver
 *   1. creates the context and computes the metric (device arrays: the set-up
 *      of the fast path);
 *   2. runs zpres, rbord and sch_roe_euler of block 1 on plain malloc'd HOST
 *      arrays -- the copy-in/out mode of the per-routine entry points, sn
 *      passed as the block's slice with lgsnlt = nnn(1) as the reference does;
 *   3. binds device state arrays and runs three fused iterations through
 *      cns_atsch_num_step_host from a host copy of the initial state.
 * OUT receives: u after step 2 (5 ld doubles), v after step 3 (5 ld doubles),
 * the last norms (15 doubles).  Exit status 0 on success, else the failing
 * call's CNS_E* code (or 90 for a file error).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "cns_abi.h"

static FILE* in_f;

static void* rd(size_t bytes) {
  void* p = calloc(bytes > 0 ? bytes : 1, 1);
  if (!p || (bytes && fread(p, 1, bytes, in_f) != bytes)) {
    fprintf(stderr, "cns_driver: short case file\n");
    exit(90);
  }
  return p;
}

#define CALL(x)                                                                     \
  do {                                                                              \
    int rc__ = (x);                                                                 \
    if (rc__) {                                                                     \
      fprintf(stderr, "cns_driver: %s -> %d (%s)\n", #x, rc__, cns_last_error(ctx)); \
      return rc__;                                                                  \
    }                                                                               \
  } while (0)

static double* dev_zeros(size_t n) {
  void* p = NULL;
  if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return NULL;
  cudaMemset(p, 0, n * sizeof(double));
  return (double*)p;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: cns_driver CASE OUT\n");
    return 90;
  }
  in_f = fopen(argv[1], "rb");
  if (!in_f) return 90;
  int64_t* hdr = (int64_t*)rd(4 * sizeof(int64_t));
  const int nblk = (int)hdr[0], nbnd = (int)hdr[2];
  const int64_t ld = hdr[1], nlist = hdr[3];
  int32_t* dims = (int32_t*)rd(3 * nblk * sizeof(int32_t));
  double* ph = (double*)rd(9 * sizeof(double));
  double* sc = (double*)rd(18 * sizeof(double));
  int32_t* btype = (int32_t*)rd(nbnd * sizeof(int32_t));
  int32_t* bblk = (int32_t*)rd(nbnd * sizeof(int32_t));
  int32_t* bface = (int32_t*)rd(nbnd * sizeof(int32_t));
  int64_t* mpb = (int64_t*)rd(nbnd * sizeof(int64_t));
  int32_t* mmb = (int32_t*)rd(nbnd * sizeof(int32_t));
  int32_t* part = (int32_t*)rd(nbnd * sizeof(int32_t));
  double* cosr = (double*)rd(nbnd * sizeof(double));
  double* sinr = (double*)rd(nbnd * sizeof(double));
  int64_t* ncbd = (int64_t*)rd(nlist * sizeof(int64_t));
  int64_t* ncin = (int64_t*)rd(nlist * sizeof(int64_t));
  double* bceqt = (double*)rd(5 * nlist * sizeof(double));
  double* x = (double*)rd(ld * sizeof(double));
  double* y = (double*)rd(ld * sizeof(double));
  double* z = (double*)rd(ld * sizeof(double));
  double* v0 = (double*)rd(5 * ld * sizeof(double));
  fclose(in_f);

  cns_layout_t lay = {nblk, dims, ld};
  cns_phys_t phys = {ph[0], ph[1], ph[2], ph[3], ph[4], ph[5], ph[6], ph[7], ph[8]};
  cns_scheme_t sch;
  memset(&sch, 0, sizeof(sch));
  sch.ns = (int32_t)sc[0];
  sch.muscl = (int32_t)sc[1];
  sch.xk = sc[2];
  sch.ilim = (int32_t)sc[3];
  sch.eta = sc[4];
  sch.kdtl = (int32_t)sc[5];
  sch.dt1min = sc[6];
  sch.lmax = (int32_t)sc[7];
  sch.qfix_dfez = (int32_t)sc[8];
  sch.precision = (int32_t)sc[9];
  sch.kdefect = (int32_t)sc[10];
  sch.ischema = (int32_t)sc[11];
  sch.ki2 = sc[12];
  sch.ki4 = sc[13];
  sch.ncychro = (int32_t)sc[14];
  sch.icychr0 = (int32_t)sc[15];
  sch.kfmg = (int32_t)sc[16];
  sch.kdualns = (int32_t)sc[17];
  cns_bnd_t bnd = {nbnd, btype, bblk, bface, mpb, mmb, part, cosr, sinr,
                   nlist, ncbd, ncin, bceqt};
  cns_ctx* ctx = NULL;
  CALL(cns_create(&lay, &phys, &sch, &bnd, &ctx));

  /* 1. metric on device arrays, then host copies of sn and vol */
  double *dx = dev_zeros(ld), *dy = dev_zeros(ld), *dz = dev_zeros(ld);
  double *dsn = dev_zeros(9 * ld), *dvol = dev_zeros(ld);
  if (!dx || !dy || !dz || !dsn || !dvol) return CNS_ECUDA;
  cudaMemcpy(dx, x, ld * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dy, y, ld * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dz, z, ld * sizeof(double), cudaMemcpyHostToDevice);
  CALL(cns_metric(ctx, dx, dy, dz, dsn, dvol));
  double* sn = (double*)calloc(9 * ld, sizeof(double));
  double* vol = (double*)calloc(ld, sizeof(double));
  cudaMemcpy(sn, dsn, 9 * ld * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(vol, dvol, ld * sizeof(double), cudaMemcpyDeviceToHost);

  /* 2. per-routine entry points on host arrays */
  double* v = (double*)malloc(5 * ld * sizeof(double));
  memcpy(v, v0, 5 * ld * sizeof(double));
  double* ps = (double*)calloc(ld, sizeof(double));
  double* temp = (double*)calloc(ld, sizeof(double));
  double* cson = (double*)calloc(ld, sizeof(double));
  double* u = (double*)calloc(5 * ld, sizeof(double));
  const int64_t nnn1 = (int64_t)(dims[0] + 2) * (dims[1] + 2) * (dims[2] + 2);
  static const char equat[7] = {'e', 'u', '3', 'd', ' ', ' ', ' '};
  CALL(cns_zpres(ctx, 0, v, ps, temp, cson));
  CALL(cns_rbord(ctx, v, ps, temp, cson));
  /* block 1 starts at npc(1) = 0, so its sn slice starts at sn itself */
  CALL(cns_sch_roe_euler(ctx, 1, 0, u, v, NULL, equat, sn, nnn1, NULL, NULL, NULL, NULL,
                         NULL, NULL, NULL, NULL, NULL, NULL, ps));

  /* 3. the fast path: device state bound once, steps from a host copy */
  cns_state_t st;
  memset(&st, 0, sizeof(st));
  st.v = dev_zeros(5 * ld);
  st.u = dev_zeros(5 * ld);
  st.d = dev_zeros(5 * ld);
  st.dt = dev_zeros(ld);
  st.sn = dsn;
  st.vol = dvol;
  st.pression = dev_zeros(ld);
  st.ztemp = dev_zeros(ld);
  st.cson = dev_zeros(ld);
  st.mu = dev_zeros(ld);
  st.mut = dev_zeros(ld);
  st.tau = dev_zeros(9 * ld);
  if (!st.v || !st.u || !st.d || !st.dt || !st.pression || !st.ztemp || !st.cson || !st.mu ||
      !st.mut || !st.tau)
    return CNS_ECUDA;
  CALL(cns_bind_state(ctx, &st));
  double* vs = (double*)malloc(5 * ld * sizeof(double));
  memcpy(vs, v0, 5 * ld * sizeof(double));
  double norms[15];
  CALL(cns_atsch_num_step_host(ctx, vs, 3, norms));

  FILE* out = fopen(argv[2], "wb");
  if (!out) return 90;
  fwrite(u, sizeof(double), 5 * ld, out);
  fwrite(vs, sizeof(double), 5 * ld, out);
  fwrite(norms, sizeof(double), 15, out);
  fclose(out);
  CALL(cns_destroy(ctx));
  printf("cns_driver ok: %lld cells, L2(rho) = %.17g\n", (long long)ld, norms[5]);
  return 0;
}
