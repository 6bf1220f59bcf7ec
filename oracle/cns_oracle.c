/*
 * cns_oracle.c -- CPU oracle for the CodeNS hot path (test infrastructure).
 *
 * This file is the checker that tests/ and bench.py's CPU-baseline leg run
 * against the CUDA product; the product never loads it.  Each routine names
 * the reference file and lines it restates.  Parity is UNPINNED (no
 * reference outputs exist; see cns_oracle.h).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math -shared -fPIC (oracle/Makefile).
 */
#include "cns_oracle.h"
/* the real power and exponential of the injection condition and the
   Spalart-Allmaras source go through one portable implementation shared with
   the kernels (the reference's libm differs from a GPU's by an ulp here and
   there); it agrees with glibc's pow and exp within a few ulp */
#include "../codens_b200/csrc/cns_pmath.h"
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXB 1024

typedef struct {
  int ni, nj, nk;        /* ii2, jj2, kk2: real node counts (ii1=jj1=kk1=1) */
  int64_t npc;           /* 0-based offset of the block (crdms.f90:150-157) */
  int nid, njd, nkd;     /* id2-id1+1 ... with nfi=1 */
  int64_t nijd, nnn;
} blk_t;

static struct {
  int nblk;
  blk_t b[MAXB];
  int64_t ld, ncells;
  /* proprieteflu / definition */
  double gam, gam1, pinfl, pr, prt, cp, reynz, suth_a, pa1, aa1, omg;
  /* schemanum */
  int ns, muscl, ilim, kdtl, lmax, qfix_dfez;
  double xk, eta, dt1min;
  int ischema;           /* 1: Jameson (central + scalar dissipation), 7: Roe */
  double ki2, ki4;       /* Jameson dissipation coefficients ki2(lm), ki4(lm) */
  /* eta(lm), ki2(lm), ki4(lm) per block (NULL: the scalars for all) */
  double *eta_l, *ki2_l, *ki4_l;
  /* dual time stepping (kfmg = 3): dt1min is the physical time step */
  int kfmg, kdualns, icycle;
  int weno_fix; /* non-reference: WENO5 sums its three candidates everywhere */
  double *ptdual;
  /* boundary */
  int nbnd;
  int32_t *btype, *bblk, *bface, *bmmb, *bpart;
  int64_t *bmpb;
  double *bcos, *bsin;
  int64_t nlist;
  int64_t *ncbd, *ncin;
  double *nxn, *nyn, *nzn, *bceqt, *bym, *bzm;
} G;

static inline double sq(double a) { return a * a; }

/* cell (or node) (i,j,k), Fortran index values, ghost layer starting at 0 */
static inline int64_t IC(const blk_t *b, int i, int j, int k) {
  return b->npc + (int64_t)i + (int64_t)j * b->nid + (int64_t)k * b->nijd;
}
static inline int64_t ML(const blk_t *b, int i, int j, int k) {
  return (int64_t)i + (int64_t)j * b->nid + (int64_t)k * b->nijd;
}
/* sn(m,kdir,c) of the block slice starting at 9*npc (atsch_num.f90:470) */
static inline double SN(const double *sn, const blk_t *b, int64_t m, int kdir,
                        int c) {
  return sn[9 * b->npc + (int64_t)c * 3 * b->nnn + (int64_t)kdir * b->nnn + m];
}
static inline double *SNW(double *sn, const blk_t *b, int64_t m, int kdir,
                          int c) {
  return &sn[9 * b->npc + (int64_t)c * 3 * b->nnn + (int64_t)kdir * b->nnn + m];
}
static inline int64_t NINC(const blk_t *b, int dir) {
  return dir == 0 ? 1 : (dir == 1 ? (int64_t)b->nid : b->nijd);
}
static inline int NDIR(const blk_t *b, int dir) {
  return dir == 0 ? b->ni : (dir == 1 ? b->nj : b->nk);
}

int orc_setup(int nblk, const int32_t *dims, int64_t ld) {
  if (nblk < 1 || nblk > MAXB) return 1;
  G.nblk = nblk;
  int64_t off = 0;
  for (int l = 0; l < nblk; ++l) {
    blk_t *b = &G.b[l];
    b->ni = dims[3 * l];
    b->nj = dims[3 * l + 1];
    b->nk = dims[3 * l + 2];
    if (b->ni < 2 || b->nj < 2 || b->nk < 2) return 2;
    b->nid = b->ni + 2;
    b->njd = b->nj + 2;
    b->nkd = b->nk + 2;
    b->nijd = (int64_t)b->nid * b->njd;
    b->nnn = b->nijd * b->nkd;
    b->npc = off;
    off += b->nnn;
  }
  G.ncells = off;
  G.ld = ld > 0 ? ld : off;
  if (G.ld < off) return 3;
  return 0;
}
int64_t orc_npc(int l) { return G.b[l - 1].npc; }
int64_t orc_ncells(void) { return G.ncells; }

/* dfph.f90:31-35, dfnzst.f90:67 (cp=1/(gam-1)), c_nzst.f90 */
void orc_set_phys(double gam, double pinfl, double pr, double prt,
                  double reynz, double suth_a, double pa1, double aa1,
                  double omg) {
  G.gam = gam;
  G.gam1 = gam - 1.;
  G.pinfl = pinfl;
  G.pr = pr;
  G.prt = prt;
  G.cp = 1. / (gam - 1.);
  G.reynz = reynz;
  G.suth_a = suth_a;
  G.pa1 = pa1;
  G.aa1 = aa1;
  G.omg = omg;
}

void orc_set_scheme(int ns, int muscl, double xk, int ilim, double eta,
                    int kdtl, double dt1min, int lmax, int qfix_dfez) {
  G.qfix_dfez = qfix_dfez;
  G.ns = ns;
  G.muscl = muscl;
  G.xk = xk;
  G.ilim = ilim;
  G.eta = eta;
  G.kdtl = kdtl;
  G.dt1min = dt1min;
  G.lmax = lmax;
}

/* threads of the per-block loops of an iteration (OpenMP) */
void orc_set_threads(int n) {
#ifdef _OPENMP
  extern void omp_set_num_threads(int);
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

static void set_block_array(double **dst, const double *src) {
  free(*dst);
  *dst = NULL;
  if (!src) return;
  *dst = (double *)malloc(sizeof(double) * (size_t)G.nblk);
  memcpy(*dst, src, sizeof(double) * (size_t)G.nblk);
}

/* eta(lm), ki2(lm), ki4(lm) of each block (tcmd_dfpmdtd.f90,
 * tcmd_dfpmdsd.f90); NULL keeps the scalar of orc_set_scheme /
 * orc_set_dissipation for every block */
void orc_set_block_scheme(const double *eta_l, const double *ki2_l, const double *ki4_l) {
  set_block_array(&G.eta_l, eta_l);
  set_block_array(&G.ki2_l, ki2_l);
  set_block_array(&G.ki4_l, ki4_l);
}

void orc_set_dissipation(int ischema, double ki2, double ki4) {
  G.ischema = ischema;
  G.ki2 = ki2;
  G.ki4 = ki4;
}

#define DUP(dst, src, n, T)                                   \
  do {                                                        \
    free(dst);                                                \
    dst = (T *)malloc(sizeof(T) * ((n) > 0 ? (n) : 1));       \
    if ((n) > 0 && (src)) memcpy(dst, src, sizeof(T) * (n));  \
  } while (0)

int orc_set_boundaries(int nbnd, const int32_t *type, const int32_t *blk,
                       const int32_t *face, const int64_t *mpb,
                       const int32_t *mmb, const int32_t *partner,
                       const double *cosr, const double *sinr, int64_t nlist,
                       const int64_t *ncbd, const int64_t *ncin,
                       const double *bceqt) {
  G.nbnd = nbnd;
  DUP(G.btype, type, nbnd, int32_t);
  DUP(G.bblk, blk, nbnd, int32_t);
  DUP(G.bface, face, nbnd, int32_t);
  DUP(G.bmpb, mpb, nbnd, int64_t);
  DUP(G.bmmb, mmb, nbnd, int32_t);
  DUP(G.bpart, partner, nbnd, int32_t);
  DUP(G.bcos, cosr, nbnd, double);
  DUP(G.bsin, sinr, nbnd, double);
  G.nlist = nlist;
  DUP(G.ncbd, ncbd, nlist, int64_t);
  DUP(G.ncin, ncin, nlist, int64_t);
  DUP(G.bceqt, bceqt, 5 * nlist, double);
  double **geo[5] = {&G.nxn, &G.nyn, &G.nzn, &G.bym, &G.bzm};
  for (int a = 0; a < 5; ++a) {
    free(*geo[a]);
    *geo[a] = calloc((size_t)(nlist > 0 ? nlist : 1), sizeof(double));
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* geometry                                                                  */
/* ------------------------------------------------------------------------ */

/* extmhg.f90:51-100 with ex1=exs1=1, ex2=exs2=0 (solve.f90:384-385) */
static void extmhg(const blk_t *b, double *x, double *y, double *z) {
  const double ex1 = 1., ex2 = 0.;
  const int64_t nci = 1, ncj = b->nid, nck = b->nijd;
  const int i1 = 1, i2 = b->ni, j1 = 1, j2 = b->nj, k1 = 1, k2 = b->nk;
  int ks = -1;
  for (int k = k1 - 1; k <= k2 + 1; k += (k2 + 1) - (k1 - 1)) {
    ks = -ks;
    for (int j = j1; j <= j2; ++j)
      for (int i = i1; i <= i2; ++i) {
        int64_t n = IC(b, i, j, k);
        x[n] = ex1 * x[n + ks * nck] + ex2 * x[n + ks * 2 * nck];
        y[n] = ex1 * y[n + ks * nck] + ex2 * y[n + ks * 2 * nck];
        z[n] = ex1 * z[n + ks * nck] + ex2 * z[n + ks * 2 * nck];
      }
  }
  for (int k = k1 - 1; k <= k2 + 1; ++k)
    for (int j = j1; j <= j2; ++j) {
      int is = -1;
      for (int i = i1 - 1; i <= i2 + 1; i += (i2 + 1) - (i1 - 1)) {
        is = -is;
        int64_t n = IC(b, i, j, k);
        x[n] = ex1 * x[n + is * nci] + ex2 * x[n + is * 2 * nci];
        y[n] = ex1 * y[n + is * nci] + ex2 * y[n + is * 2 * nci];
        z[n] = ex1 * z[n + is * nci] + ex2 * z[n + is * 2 * nci];
      }
    }
  for (int k = k1 - 1; k <= k2 + 1; ++k) {
    int js = -1;
    for (int j = j1 - 1; j <= j2 + 1; j += (j2 + 1) - (j1 - 1)) {
      js = -js;
      for (int i = i1 - 1; i <= i2 + 1; ++i) {
        int64_t n = IC(b, i, j, k);
        x[n] = ex1 * x[n + js * ncj] + ex2 * x[n + js * 2 * ncj];
        y[n] = ex1 * y[n + js * ncj] + ex2 * y[n + js * 2 * ncj];
        z[n] = ex1 * z[n + js * ncj] + ex2 * z[n + js * 2 * ncj];
      }
    }
  }
}

/* norm.f90:57-271 called from snorm.f90 with imin=i1-1 ... imax=i2+1 */
static void snorm(const blk_t *b, const double *x, const double *y,
                  const double *z, double *sn) {
  const int64_t n0 = b->npc;
#define INC(a, bb, c) ((int64_t)(a) + (int64_t)(bb) * b->nid + (int64_t)(c) * b->nijd)
  const int imin = 0, imax = b->ni + 1, jmin = 0, jmax = b->nj + 1, kmin = 0,
            kmax = b->nk + 1;
  const int64_t nor = IC(b, 2, 2, 2);
  double dx1, dy1, dz1, dx2, dy2, dz2, vx, vy, vz, tx, ty, tz;
  /* k faces */
  dx1 = x[nor + INC(1, 1, 0)] - x[nor];
  dy1 = y[nor + INC(1, 1, 0)] - y[nor];
  dz1 = z[nor + INC(1, 1, 0)] - z[nor];
  dx2 = x[nor + INC(0, 1, 0)] - x[nor + INC(1, 0, 0)];
  dy2 = y[nor + INC(0, 1, 0)] - y[nor + INC(1, 0, 0)];
  dz2 = z[nor + INC(0, 1, 0)] - z[nor + INC(1, 0, 0)];
  tx = dy1 * dz2 - dz1 * dy2;
  ty = dz1 * dx2 - dx1 * dz2;
  tz = dx1 * dy2 - dy1 * dx2;
  vx = x[nor + INC(0, 0, 1)] - x[nor] + x[nor + INC(1, 0, 1)] - x[nor + INC(1, 0, 0)] +
       x[nor + INC(0, 1, 1)] - x[nor + INC(0, 1, 0)] + x[nor + INC(1, 1, 1)] - x[nor + INC(1, 1, 0)];
  vy = y[nor + INC(0, 0, 1)] - y[nor] + y[nor + INC(1, 0, 1)] - y[nor + INC(1, 0, 0)] +
       y[nor + INC(0, 1, 1)] - y[nor + INC(0, 1, 0)] + y[nor + INC(1, 1, 1)] - y[nor + INC(1, 1, 0)];
  vz = z[nor + INC(0, 0, 1)] - z[nor] + z[nor + INC(1, 0, 1)] - z[nor + INC(1, 0, 0)] +
       z[nor + INC(0, 1, 1)] - z[nor + INC(0, 1, 0)] + z[nor + INC(1, 1, 1)] - z[nor + INC(1, 1, 0)];
  const double psk = tx * vx + ty * vy + tz * vz;
  for (int k = kmin; k <= kmax; ++k)
    for (int j = jmin; j <= jmax - 1; ++j)
      for (int i = imin; i <= imax - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        dx1 = x[n + INC(1, 1, 0)] - x[n];
        dy1 = y[n + INC(1, 1, 0)] - y[n];
        dz1 = z[n + INC(1, 1, 0)] - z[n];
        dx2 = x[n + INC(0, 1, 0)] - x[n + INC(1, 0, 0)];
        dy2 = y[n + INC(0, 1, 0)] - y[n + INC(1, 0, 0)];
        dz2 = z[n + INC(0, 1, 0)] - z[n + INC(1, 0, 0)];
        *SNW(sn, b, m, 2, 0) = copysign(.5, psk) * (dy1 * dz2 - dz1 * dy2);
        *SNW(sn, b, m, 2, 1) = copysign(.5, psk) * (dz1 * dx2 - dx1 * dz2);
        *SNW(sn, b, m, 2, 2) = copysign(.5, psk) * (dx1 * dy2 - dy1 * dx2);
      }
  /* j faces */
  dx1 = x[nor + INC(1, 0, 1)] - x[nor];
  dy1 = y[nor + INC(1, 0, 1)] - y[nor];
  dz1 = z[nor + INC(1, 0, 1)] - z[nor];
  dx2 = x[nor + INC(0, 0, 1)] - x[nor + INC(1, 0, 0)];
  dy2 = y[nor + INC(0, 0, 1)] - y[nor + INC(1, 0, 0)];
  dz2 = z[nor + INC(0, 0, 1)] - z[nor + INC(1, 0, 0)];
  tx = dy1 * dz2 - dz1 * dy2;
  ty = dz1 * dx2 - dx1 * dz2;
  tz = dx1 * dy2 - dy1 * dx2;
  vx = x[nor + INC(0, 1, 0)] - x[nor] + x[nor + INC(1, 1, 0)] - x[nor + INC(1, 0, 0)] +
       x[nor + INC(0, 1, 1)] - x[nor + INC(0, 0, 1)] + x[nor + INC(1, 1, 1)] - x[nor + INC(1, 0, 1)];
  vy = y[nor + INC(0, 1, 0)] - y[nor] + y[nor + INC(1, 1, 0)] - y[nor + INC(1, 0, 0)] +
       y[nor + INC(0, 1, 1)] - y[nor + INC(0, 0, 1)] + y[nor + INC(1, 1, 1)] - y[nor + INC(1, 0, 1)];
  vz = z[nor + INC(0, 1, 0)] - z[nor] + z[nor + INC(1, 1, 0)] - z[nor + INC(1, 0, 0)] +
       z[nor + INC(0, 1, 1)] - z[nor + INC(0, 0, 1)] + z[nor + INC(1, 1, 1)] - z[nor + INC(1, 0, 1)];
  const double psj = tx * vx + ty * vy + tz * vz;
  for (int j = jmin; j <= jmax; ++j)
    for (int k = kmin; k <= kmax - 1; ++k)
      for (int i = imin; i <= imax - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        dx1 = x[n + INC(1, 0, 1)] - x[n];
        dy1 = y[n + INC(1, 0, 1)] - y[n];
        dz1 = z[n + INC(1, 0, 1)] - z[n];
        dx2 = x[n + INC(0, 0, 1)] - x[n + INC(1, 0, 0)];
        dy2 = y[n + INC(0, 0, 1)] - y[n + INC(1, 0, 0)];
        dz2 = z[n + INC(0, 0, 1)] - z[n + INC(1, 0, 0)];
        *SNW(sn, b, m, 1, 0) = copysign(.5, psj) * (dy1 * dz2 - dz1 * dy2);
        *SNW(sn, b, m, 1, 1) = copysign(.5, psj) * (dz1 * dx2 - dx1 * dz2);
        *SNW(sn, b, m, 1, 2) = copysign(.5, psj) * (dx1 * dy2 - dy1 * dx2);
      }
  /* i faces */
  dx1 = x[nor + INC(0, 1, 1)] - x[nor];
  dy1 = y[nor + INC(0, 1, 1)] - y[nor];
  dz1 = z[nor + INC(0, 1, 1)] - z[nor];
  dx2 = x[nor + INC(0, 0, 1)] - x[nor + INC(0, 1, 0)];
  dy2 = y[nor + INC(0, 0, 1)] - y[nor + INC(0, 1, 0)];
  dz2 = z[nor + INC(0, 0, 1)] - z[nor + INC(0, 1, 0)];
  tx = dy1 * dz2 - dz1 * dy2;
  ty = dz1 * dx2 - dx1 * dz2;
  tz = dx1 * dy2 - dy1 * dx2;
  vx = x[nor + INC(1, 0, 0)] - x[nor] + x[nor + INC(1, 1, 0)] - x[nor + INC(0, 1, 0)] +
       x[nor + INC(1, 0, 1)] - x[nor + INC(0, 0, 1)] + x[nor + INC(1, 1, 1)] - x[nor + INC(0, 1, 1)];
  vy = y[nor + INC(1, 0, 0)] - y[nor] + y[nor + INC(1, 1, 0)] - y[nor + INC(0, 1, 0)] +
       y[nor + INC(1, 0, 1)] - y[nor + INC(0, 0, 1)] + y[nor + INC(1, 1, 1)] - y[nor + INC(0, 1, 1)];
  vz = z[nor + INC(1, 0, 0)] - z[nor] + z[nor + INC(1, 1, 0)] - z[nor + INC(0, 1, 0)] +
       z[nor + INC(1, 0, 1)] - z[nor + INC(0, 0, 1)] + z[nor + INC(1, 1, 1)] - z[nor + INC(0, 1, 1)];
  const double psi = tx * vx + ty * vy + tz * vz;
  for (int i = imin; i <= imax; ++i)
    for (int k = kmin; k <= kmax - 1; ++k)
      for (int j = jmin; j <= jmax - 1; ++j) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        dx1 = x[n + INC(0, 1, 1)] - x[n];
        dy1 = y[n + INC(0, 1, 1)] - y[n];
        dz1 = z[n + INC(0, 1, 1)] - z[n];
        dx2 = x[n + INC(0, 0, 1)] - x[n + INC(0, 1, 0)];
        dy2 = y[n + INC(0, 0, 1)] - y[n + INC(0, 1, 0)];
        dz2 = z[n + INC(0, 0, 1)] - z[n + INC(0, 1, 0)];
        *SNW(sn, b, m, 0, 0) = copysign(.5, psi) * (dy1 * dz2 - dz1 * dy2);
        *SNW(sn, b, m, 0, 1) = copysign(.5, psi) * (dz1 * dx2 - dx1 * dz2);
        *SNW(sn, b, m, 0, 2) = copysign(.5, psi) * (dx1 * dy2 - dy1 * dx2);
      }
#undef INC
}

/* svol.f90:62-150 */
static void svol(const blk_t *b, const double *x, const double *y,
                 const double *z, const double *sn, double *vol) {
  const int64_t n0 = b->npc, nci = 1, ncj = b->nid, nck = b->nijd;
  double *siv = calloc(b->nnn, sizeof(double));
  double *sjv = calloc(b->nnn, sizeof(double));
  double *skv = calloc(b->nnn, sizeof(double));
  const int i1m1 = 0, i2 = b->ni, i2p1 = b->ni + 1, j1m1 = 0, j2 = b->nj,
            j2p1 = b->nj + 1, k1m1 = 0, k2 = b->nk, k2p1 = b->nk + 1;
  for (int k = k1m1; k <= k2p1; ++k)
    for (int j = j1m1; j <= j2; ++j)
      for (int i = i1m1; i <= i2; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        skv[m] = (x[n] + x[n + nci] + x[n + ncj] + x[n + nci + ncj]) * SN(sn, b, m, 2, 0) +
                 (y[n] + y[n + nci] + y[n + ncj] + y[n + nci + ncj]) * SN(sn, b, m, 2, 1) +
                 (z[n] + z[n + nci] + z[n + ncj] + z[n + nci + ncj]) * SN(sn, b, m, 2, 2);
      }
  for (int j = j1m1; j <= j2p1; ++j)
    for (int k = k1m1; k <= k2; ++k)
      for (int i = i1m1; i <= i2; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        sjv[m] = (x[n] + x[n + nci] + x[n + nck] + x[n + nci + nck]) * SN(sn, b, m, 1, 0) +
                 (y[n] + y[n + nci] + y[n + nck] + y[n + nci + nck]) * SN(sn, b, m, 1, 1) +
                 (z[n] + z[n + nci] + z[n + nck] + z[n + nci + nck]) * SN(sn, b, m, 1, 2);
      }
  for (int i = i1m1; i <= i2p1; ++i)
    for (int k = k1m1; k <= k2; ++k)
      for (int j = j1m1; j <= j2; ++j) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        siv[m] = (x[n] + x[n + ncj] + x[n + nck] + x[n + ncj + nck]) * SN(sn, b, m, 0, 0) +
                 (y[n] + y[n + ncj] + y[n + nck] + y[n + ncj + nck]) * SN(sn, b, m, 0, 1) +
                 (z[n] + z[n + ncj] + z[n + nck] + z[n + ncj + nck]) * SN(sn, b, m, 0, 2);
      }
  for (int k = k1m1; k <= k2; ++k)
    for (int j = j1m1; j <= j2; ++j)
      for (int i = i1m1; i <= i2; ++i) {
        int64_t n = IC(b, i, j, k), m1 = n - n0;
        vol[n] = 0.25 * (siv[m1 + nci] - siv[m1] + sjv[m1 + ncj] - sjv[m1] +
                         skv[m1 + nck] - skv[m1]) / 3.;
      }
  free(siv);
  free(sjv);
  free(skv);
}

/* rfsc.f90:26-57: ghost volume of a coincident boundary = partner interior */
static void rfsc(double *t) {
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    int p = G.bpart[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m)
      t[G.ncbd[G.bmpb[bb] + m]] = t[G.ncin[G.bmpb[p] + m]];
  }
}

/* per boundary entry: inward unit normal of the boundary face (initns.f90:
 * 63-150: +/- the face area vector of norm.f90, then normalised) and the
 * centre of the ghost cell (clidd.f90:64-71) */
static void boundary_geom(const double *x, const double *y, const double *z,
                          const double *sn) {
  const double eps = 1.e-10;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    const blk_t *b = &G.b[G.bblk[bb] - 1];
    const int f = G.bface[bb], dir = f / 2, upper = f % 2;
    const double is = upper ? -1. : 1.;
    const int64_t nci = 1, ncj = b->nid, nck = b->nijd;
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m;
      int64_t face_cell = upper ? G.ncbd[mb] : G.ncin[mb];
      int64_t mm = face_cell - b->npc;
      double nx = is * SN(sn, b, mm, dir, 0);
      double ny = is * SN(sn, b, mm, dir, 1);
      double nz = is * SN(sn, b, mm, dir, 2);
      double nn = sqrt(nx * nx + ny * ny + nz * nz);
      nn = nn + (copysign(1., -fabs(nn)) + 1.) * eps;
      G.nxn[mb] = nx / nn;
      G.nyn[mb] = ny / nn;
      G.nzn[mb] = nz / nn;
      int64_t n = G.ncbd[mb];
      G.bym[mb] = 0.125 * (y[n] + y[n + nci] + y[n + ncj] + y[n + nci + ncj] + y[n + nck] +
                           y[n + nci + nck] + y[n + ncj + nck] + y[n + nci + ncj + nck]);
      G.bzm[mb] = 0.125 * (z[n] + z[n + nci] + z[n + ncj] + z[n + nci + ncj] + z[n + nck] +
                           z[n + nci + nck] + z[n + ncj + nck] + z[n + nci + ncj + nck]);
    }
  }
}

/* metric.f90:24-51 -> metrics.f90:52-66 */
void orc_metric(double *x, double *y, double *z, double *sn, double *vol) {
  for (int l = 0; l < G.nblk; ++l) {
    const blk_t *b = &G.b[l];
    extmhg(b, x, y, z);
    snorm(b, x, y, z, sn);
    svol(b, x, y, z, sn, vol);
  }
  rfsc(vol);
  boundary_geom(x, y, z, sn);
}

void orc_boundary_geom(double *nxn, double *nyn, double *nzn, double *ym,
                       double *zm) {
  size_t n = sizeof(double) * (size_t)G.nlist;
  memcpy(nxn, G.nxn, n);
  memcpy(nyn, G.nyn, n);
  memcpy(nzn, G.nzn, n);
  memcpy(ym, G.bym, n);
  memcpy(zm, G.bzm, n);
}

/* ------------------------------------------------------------------------ */
/* thermodynamics and time step                                             */
/* ------------------------------------------------------------------------ */

/* zpres.f90:66-79 */
void orc_zpres(int l, const double *v, double *ps, double *temp, double *cson) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        double rhoe = v[4 * L + n] -
                      0.5 * (sq(v[L + n]) + sq(v[2 * L + n]) + sq(v[3 * L + n])) / v[n];
        ps[n] = G.gam1 * (rhoe - G.pinfl);
        temp[n] = G.gam * ps[n] / v[n];
        cson[n] = sqrt(temp[n]);
      }
}

/* zvismo.f90:77-104 (iflu=1, Sutherland; a = 110.4/tnz is passed in) */
void orc_zvismo(int l, double *mu, const double *temp) {
  const blk_t *b = &G.b[l - 1];
  const double usrey = 1. / G.reynz, a = G.suth_a;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        if (temp[n] <= 0.)
          mu[n] = 0.;
        else
          mu[n] = usrey * temp[n] * sqrt(temp[n]) * (1. + a) / (temp[n] + a);
      }
}

/* chronos.f90:110-194 (kprec=0) */
void orc_chronos(int l, const double *mu, const double *mut, const double *t,
                 double *dt, const double *sn, const double *vol,
                 const double *cson) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nci = 1, ncj = b->nid, nck = b->nijd;
  const int i1 = 1, i2 = b->ni, j1 = 1, j2 = b->nj, k1 = 1, k2 = b->nk;
  double *sfsi = calloc(b->nnn, sizeof(double));
  double *sfsj = calloc(b->nnn, sizeof(double));
  double *sfsk = calloc(b->nnn, sizeof(double));
  double *dism = calloc(b->nnn, sizeof(double));
  for (int64_t n = IC(b, i1, j1, k1); n <= IC(b, i2, j2, k2); ++n) dt[n] = 0.;
  for (int k = k1; k <= k2 - 1; ++k) {
    for (int j = j1; j <= j2 - 1; ++j)
      for (int i = i1; i <= i2; ++i) {
        int64_t m = ML(b, i, j, k);
        sfsi[m] = SN(sn, b, m, 0, 0) * SN(sn, b, m, 0, 0) +
                  SN(sn, b, m, 0, 1) * SN(sn, b, m, 0, 1) +
                  SN(sn, b, m, 0, 2) * SN(sn, b, m, 0, 2);
      }
    for (int j = j1; j <= j2; ++j)
      for (int i = i1; i <= i2 - 1; ++i) {
        int64_t m = ML(b, i, j, k);
        sfsj[m] = SN(sn, b, m, 1, 0) * SN(sn, b, m, 1, 0) +
                  SN(sn, b, m, 1, 1) * SN(sn, b, m, 1, 1) +
                  SN(sn, b, m, 1, 2) * SN(sn, b, m, 1, 2);
      }
  }
  for (int k = k1; k <= k2; ++k)
    for (int j = j1; j <= j2 - 1; ++j)
      for (int i = i1; i <= i2 - 1; ++i) {
        int64_t m = ML(b, i, j, k);
        sfsk[m] = SN(sn, b, m, 2, 0) * SN(sn, b, m, 2, 0) +
                  SN(sn, b, m, 2, 1) * SN(sn, b, m, 2, 1) +
                  SN(sn, b, m, 2, 2) * SN(sn, b, m, 2, 2);
      }
  for (int k = k1; k <= k2 - 1; ++k)
    for (int j = j1; j <= j2 - 1; ++j)
      for (int i = i1; i <= i2 - 1; ++i) {
        int64_t mn = ML(b, i, j, k), nc = n0 + mn;
        double simax = fmax(sfsi[mn + nci], sfsi[mn]);
        double sjmax = fmax(sfsj[mn + ncj], sfsj[mn]);
        double skmax = fmax(sfsk[mn + nck], sfsk[mn]);
        double smoy = sqrt(simax + sjmax + skmax);
        dism[mn] = vol[nc] / smoy;
      }
  const double etal = G.eta_l ? G.eta_l[l - 1] : G.eta;
  for (int k = k1; k <= k2 - 1; ++k)
    for (int j = j1; j <= j2 - 1; ++j)
      for (int i = i1; i <= i2 - 1; ++i) {
        int64_t nc = IC(b, i, j, k), mc = nc - n0;
        double ro = t[nc];
        double qq = (sq(t[L + nc]) + sq(t[2 * L + nc]) + sq(t[3 * L + nc])) / sq(ro);
        double q = sqrt(qq);
        double dte = dism[mc] / (q + cson[nc]);
        dt[nc] = etal * dte;
      }
  if (G.ns) {
    for (int k = k1; k <= k2 - 1; ++k)
      for (int j = j1; j <= j2 - 1; ++j)
        for (int i = i1; i <= i2 - 1; ++i) {
          int64_t nc = IC(b, i, j, k), mc = nc - n0;
          double rv1 = G.gam * (mu[nc] / G.pr + mut[nc] / G.prt) / t[nc];
          double rv = fmax(rv1, 4. / 3. * (mu[nc] + mut[nc]) / t[nc]);
          double dtv = etal * 0.25 * sq(dism[mc]) / rv;
          dt[nc] = fmin(dt[nc], dtv);
        }
  }
  free(sfsi);
  free(sfsj);
  free(sfsk);
  free(dism);
}

/* chrono.f90:113-151 (kdtl=0): dt = min(dt1min, min over real cells); a
 * value below dt1min stops the reference, here dt is left untouched and the
 * caller sees the minimum through the return of orc_step */
void orc_chrono_global(double *dt) {
  double dtmin = DBL_MAX;
  for (int l = 0; l < G.nblk; ++l) {
    const blk_t *b = &G.b[l];
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) dtmin = fmin(dtmin, dt[IC(b, i, j, k)]);
  }
  dtmin = fmin(G.dt1min, dtmin);
  for (int l = 0; l < G.nblk; ++l) {
    const blk_t *b = &G.b[l];
    for (int64_t n = b->npc; n < b->npc + b->nnn; ++n) dt[n] = dtmin;
  }
}

/* ------------------------------------------------------------------------ */
/* boundary conditions                                                       */
/* ------------------------------------------------------------------------ */

/* rbvc.f90:34-92: ghost = 0.5*(own interior + partner interior rotated by the
 * partner's periodic angle) for every coincident boundary */
static void rbvc(double *t, double *ps, double *temp, double *cson) {
  const int64_t L = G.ld;
  int64_t tot = 0;
  for (int bb = 0; bb < G.nbnd; ++bb)
    if (G.btype[bb] == ORC_BC_RC) tot += G.bmmb[bb];
  if (tot == 0) return;
  /* pack (buff(:,:,:,1)) */
  double *buff = malloc(sizeof(double) * 8 * (size_t)G.nlist);
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    const double c = G.bcos[bb], s = G.bsin[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nc = G.ncin[mb];
      double *bf = &buff[8 * mb];
      bf[0] = t[nc];
      bf[1] = t[L + nc];
      bf[2] = t[2 * L + nc] * c + t[3 * L + nc] * s;
      bf[3] = t[3 * L + nc] * c - t[2 * L + nc] * s;
      bf[4] = t[4 * L + nc];
      bf[5] = ps[nc];
      bf[6] = temp[nc];
      bf[7] = cson[nc];
    }
  }
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    const int p = G.bpart[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ndm = G.ncin[mb];
      const double *bf = &buff[8 * (G.bmpb[p] + m)];
      t[nd] = 0.5 * (t[ndm] + bf[0]);
      t[L + nd] = 0.5 * (t[L + ndm] + bf[1]);
      t[2 * L + nd] = 0.5 * (t[2 * L + ndm] + bf[2]);
      t[3 * L + nd] = 0.5 * (t[3 * L + ndm] + bf[3]);
      t[4 * L + nd] = 0.5 * (t[4 * L + ndm] + bf[4]);
      ps[nd] = 0.5 * (ps[ndm] + bf[5]);
      temp[nd] = 0.5 * (temp[ndm] + bf[6]);
      cson[nd] = 0.5 * (cson[ndm] + bf[7]);
    }
  }
  free(buff);
}

/* rbve.f90:21-33 */
static void rbve(int bb, double *t) {
  const int64_t L = G.ld;
  for (int m = 0; m < G.bmmb[bb]; ++m) {
    int64_t ml = G.bmpb[bb] + m, n = G.ncbd[ml], ni = G.ncin[ml];
    for (int c = 0; c < 5; ++c) t[c * L + n] = t[c * L + ni];
  }
}

/* clextr.f90:23-37 */
static void clextr(int bb, double *v, double *ps, double *temp, double *cson) {
  const int64_t L = G.ld;
  for (int m = 0; m < G.bmmb[bb]; ++m) {
    int64_t mb = G.bmpb[bb] + m, nl = G.ncbd[mb], ni = G.ncin[mb];
    for (int c = 0; c < 5; ++c) v[c * L + nl] = v[c * L + ni];
    ps[nl] = ps[ni];
    temp[nl] = temp[ni];
    cson[nl] = cson[ni];
  }
}

/* clpara.f90:24-40: adiabatic wall, ghost at rest with the interior rho e */
static void clpara(int bb, double *v, double *ps, double *temp, double *cson) {
  const int64_t L = G.ld;
  for (int m = 0; m < G.bmmb[bb]; ++m) {
    int64_t mb = G.bmpb[bb] + m, nc = G.ncbd[mb], ni = G.ncin[mb];
    double rhoe1 = v[4 * L + ni] -
                   0.5 * (sq(v[L + ni]) + sq(v[2 * L + ni]) + sq(v[3 * L + ni])) / v[ni];
    v[nc] = v[ni];
    v[L + nc] = 0.;
    v[2 * L + nc] = 0.;
    v[3 * L + nc] = 0.;
    v[4 * L + nc] = rhoe1;
    ps[nc] = ps[ni];
    temp[nc] = temp[ni];
    cson[nc] = cson[ni];
  }
}

/* utidd.f90 + clidd.f90:50-170: subsonic injection at imposed total pressure,
 * total temperature and flow direction (Newton on the normal velocity, at
 * most 20 sweeps, the stop test is the maximum over the whole boundary) */
static void clidd(int bb, double *v, double *ps_, double *temp, double *cson) {
  const int64_t L = G.ld;
  const int mt = G.bmmb[bb];
  const int64_t m0 = G.bmpb[bb];
  const double eps = 0.0000001;
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl, omg = G.omg;
  const double gam6 = gam / gam1;
  const double gamt = gam / sq(G.aa1);
  const double gam2t = 0.5 * gam1 / sq(G.aa1);
  double *usdn = malloc(sizeof(double) * mt), *usdn2 = malloc(sizeof(double) * mt);
  double *un = malloc(sizeof(double) * mt), *qn = malloc(sizeof(double) * mt);
  double *roc0 = malloc(sizeof(double) * mt), *am0 = malloc(sizeof(double) * mt);
  for (int m = 0; m < mt; ++m) {
    int64_t mb = m0 + m, nc = G.ncbd[mb];
    const double *bc = &G.bceqt[mb];
    double d0x = bc[G.nlist * 2], d0y = bc[G.nlist * 3], d0z = bc[G.nlist * 4];
    double nx = G.nxn[mb], ny = G.nyn[mb], nz = G.nzn[mb];
    double ym = G.bym[mb], zm = G.bzm[mb];
    usdn[m] = 1. / (d0x * nx + d0y * ny + d0z * nz);
    usdn2[m] = sq(usdn[m]);
    un[m] = omg * (ym * nz - zm * ny);
    double qxs = v[L + nc] / v[nc], qys = v[2 * L + nc] / v[nc], qzs = v[3 * L + nc] / v[nc];
    qn[m] = qxs * nx + qys * ny + qzs * nz;
    double ps = gam1 * (v[4 * L + nc] -
                        0.5 * (qxs * v[L + nc] + qys * v[2 * L + nc] + qzs * v[3 * L + nc]) - pinfl);
    roc0[m] = -sqrt(gam * ps * v[nc]);
    am0[m] = ps + roc0[m] * qn[m];
  }
  int nitn = 0;
  double residu = 1.;
  while (residu > eps && nitn < 20) {
    residu = 0.;
    for (int m = 0; m < mt; ++m) {
      int64_t mb = m0 + m;
      double rpi = G.bceqt[mb], rti = G.bceqt[G.nlist + mb];
      double b = 1. / (1. + gam2t / rti * usdn2[m] * sq(qn[m] + un[m]));
      double p = G.pa1 * rpi * cns_pow(b, gam6);
      double ro = gamt * p / (b * rti);
      double f = p + roc0[m] * qn[m] - am0[m];
      double df = roc0[m] - ro * (qn[m] + un[m]) * usdn2[m];
      double dqn = -f / df;
      double resi = fabs(dqn) / qn[m];
      qn[m] = qn[m] + dqn;
      residu = fmax(residu, resi);
    }
    nitn = nitn + 1;
  }
  for (int m = 0; m < mt; ++m) {
    int64_t mb = m0 + m, nc = G.ncbd[mb];
    double rpi = G.bceqt[mb], rti = G.bceqt[G.nlist + mb];
    double d0x = G.bceqt[G.nlist * 2 + mb], d0y = G.bceqt[G.nlist * 3 + mb],
           d0z = G.bceqt[G.nlist * 4 + mb];
    double ym = G.bym[mb], zm = G.bzm[mb];
    double b = 1. / (1. + gam2t / rti * usdn2[m] * sq(qn[m] + un[m]));
    double p = G.pa1 * rpi * cns_pow(b, gam6);
    double ro = gamt * p / (b * rti);
    double wn = qn[m] + un[m];
    double w = wn * usdn[m];
    v[nc] = ro;
    v[L + nc] = ro * (w * d0x);
    v[2 * L + nc] = ro * (w * d0y + zm * omg);
    v[3 * L + nc] = ro * (w * d0z - ym * omg);
    v[4 * L + nc] = p / gam1 + pinfl +
                    0.5 * (sq(v[L + nc]) + sq(v[2 * L + nc]) + sq(v[3 * L + nc])) / ro;
    ps_[nc] = p;
    temp[nc] = gam * p / ro;
    cson[nc] = sqrt(temp[nc]);
  }
  free(usdn);
  free(usdn2);
  free(un);
  free(qn);
  free(roc0);
  free(am0);
}

/* utprd.f90 + clprd.f90:31-59: imposed static pressure, compatibility
 * relation along the inward normal */
static void clprd(int bb, double *v, double *ps_, double *temp, double *cson) {
  const int64_t L = G.ld;
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  for (int m = 0; m < G.bmmb[bb]; ++m) {
    int64_t mb = G.bmpb[bb] + m, nl = G.ncbd[mb];
    double pres = G.bceqt[mb];
    double rho = v[nl];
    double qxs = v[L + nl] / v[nl], qys = v[2 * L + nl] / v[nl], qzs = v[3 * L + nl] / v[nl];
    double ps = gam1 * (v[4 * L + nl] - 0.5 * rho * (sq(qxs) + sq(qys) + sq(qzs)) - pinfl);
    double cs2 = gam * ps / rho;
    double roc0 = sqrt(gam * ps * rho);
    double dqn = (pres - ps) / roc0;
    double qx = qxs + dqn * G.nxn[mb];
    double qy = qys + dqn * G.nyn[mb];
    double qz = qzs + dqn * G.nzn[mb];
    double drho = (pres - ps) / cs2;
    v[nl] = v[nl] + drho;
    v[L + nl] = v[nl] * qx;
    v[2 * L + nl] = v[nl] * qy;
    v[3 * L + nl] = v[nl] * qz;
    v[4 * L + nl] = pres / gam1 + pinfl + 0.5 * v[nl] * (sq(qx) + sq(qy) + sq(qz));
    ps_[nl] = pres;
    temp[nl] = gam * ps_[nl] / v[nl];
    cson[nl] = sqrt(temp[nl]);
  }
}

/* rbord.f90:137-429: coincident halo, physical conditions, coincident halo */
void orc_rbord(double *v, double *ps, double *temp, double *cson) {
  rbvc(v, ps, temp, cson);
  for (int bb = 0; bb < G.nbnd; ++bb) {
    switch (G.btype[bb]) {
      case ORC_BC_EXTR: clextr(bb, v, ps, temp, cson); break;
      case ORC_BC_PARA:
      case ORC_BC_LP2: /* rbord.f90:374-388: 'lp2' walls take clpara */
        clpara(bb, v, ps, temp, cson);
        break;
      case ORC_BC_IDD:
        rbve(bb, v);
        clidd(bb, v, ps, temp, cson);
        break;
      case ORC_BC_PRD:
        rbve(bb, v);
        clprd(bb, v, ps, temp, cson);
        break;
      default: break;
    }
  }
  rbvc(v, ps, temp, cson);
}

static void zero_u(const blk_t *b, double *u);

/* rfve.f90:14-31: every non-coincident boundary, ghost = interior cell */
void orc_rfve(double *v, double *ps, double *temp, double *cson) {
  const int64_t L = G.ld;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] == ORC_BC_RC) continue;
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ni = G.ncin[mb];
      for (int a = 0; a < 5; ++a) v[a * L + nd] = v[a * L + ni];
      ps[nd] = ps[ni];
      temp[nd] = temp[ni];
      cson[nd] = cson[ni];
    }
  }
}

/* rfvc.f90 (same-process branch): every coincident ghost = the coincident
 * interior cell of the partner, velocity rotated by the receiver's angle */
void orc_rfvc(double *v, double *ps, double *temp, double *cson) {
  const int64_t L = G.ld;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    const int p = G.bpart[bb];
    const double c = G.bcos[bb], s = G.bsin[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], nc = G.ncin[G.bmpb[p] + m];
      v[nd] = v[nc];
      v[L + nd] = v[L + nc];
      v[2 * L + nd] = v[2 * L + nc] * c + v[3 * L + nc] * s;
      v[3 * L + nd] = v[3 * L + nc] * c - v[2 * L + nc] * s;
      v[4 * L + nd] = v[4 * L + nc];
      ps[nd] = ps[nc];
      temp[nd] = temp[nc];
      cson[nd] = cson[nc];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Jameson scheme                                                            */
/* ------------------------------------------------------------------------ */

/* one direction of dissip_jameson.f90:94-316 (i, j) and :318-431 (k) */
static void jameson_dissip_dir(const blk_t *b, int dir, double *d, const double *v,
                               const double *sn, const double *ps,
                               const double *cson, double *snu) {
  const int64_t L = G.ld, n0 = b->npc, ninc = NINC(b, dir);
  const int lb = (int)(b - G.b);
  const double ck2 = G.ki2_l ? G.ki2_l[lb] : G.ki2, ck4 = G.ki4_l ? G.ki4_l[lb] : G.ki4;
  const int kdir = dir;  /* sn(m, kdir, c): 0-based here */
  /* sensor on the real cells (:99-110) */
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        snu[m] = fabs(ps[n + ninc] - 2. * ps[n] + ps[n - ninc]) /
                 (ps[n + ninc] + 2. * ps[n] + ps[n - ninc]);
      }
  /* face quantities shared by the three loops */
#define JAM_FACE()                                                              \
  double cnds = SN(sn, b, m, kdir, 0) * SN(sn, b, m, kdir, 0) +                  \
                SN(sn, b, m, kdir, 1) * SN(sn, b, m, kdir, 1) +                  \
                SN(sn, b, m, kdir, 2) * SN(sn, b, m, kdir, 2);                   \
  double uu = 0.5 * (v[L + n] / v[n] + v[L + n - ninc] / v[n - ninc]);           \
  double vv = 0.5 * (v[2 * L + n] / v[n] + v[2 * L + n - ninc] / v[n - ninc]);   \
  double ww = 0.5 * (v[3 * L + n] / v[n] + v[3 * L + n - ninc] / v[n - ninc]);   \
  double cc = 0.5 * (cson[n] + cson[n - ninc]);                                  \
  double rl = fabs(uu * SN(sn, b, m, kdir, 0) + vv * SN(sn, b, m, kdir, 1) +     \
                   ww * SN(sn, b, m, kdir, 2)) + sqrt(cnds) * cc;
  const int nd = NDIR(b, dir);
  int lo[3], hi[3];
  /* interior faces (:112-150): face index 2..nd-1 along dir */
  lo[0] = 1; hi[0] = b->ni - 1; lo[1] = 1; hi[1] = b->nj - 1; lo[2] = 1; hi[2] = b->nk - 1;
  lo[dir] = 2; hi[dir] = nd - 1;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        double eps2 = ck2 * fmax(snu[m - ninc], snu[m]);
        double eps4 = fmax(0., ck4 - eps2);
        JAM_FACE()
        for (int a = 0; a < 5; ++a) {
          const double *w = v + a * L;
          double ds = eps2 * rl * (w[n] - w[n - ninc]) -
                      eps4 * rl * (w[n + ninc] + 3. * (w[n - ninc] - w[n]) - w[n - 2 * ninc]);
          d[a * L + n] = d[a * L + n] - ds;
          d[a * L + n - ninc] = d[a * L + n - ninc] + ds;
        }
      }
  /* lower boundary faces (:152-177), then upper ones (:179-204) */
  for (int side = 0; side < 2; ++side) {
    lo[0] = 1; hi[0] = b->ni - 1; lo[1] = 1; hi[1] = b->nj - 1; lo[2] = 1; hi[2] = b->nk - 1;
    lo[dir] = hi[dir] = side == 0 ? 1 : nd;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          double eps2 = side == 0 ? ck2 * snu[m] : ck2 * snu[m - ninc];
          JAM_FACE()
          for (int a = 0; a < 5; ++a) {
            const double *w = v + a * L;
            double ds = eps2 * rl * (w[n] - w[n - ninc]);
            if (side == 0)
              d[a * L + n] = d[a * L + n] - ds;
            else
              d[a * L + n - ninc] = d[a * L + n - ninc] + ds;
          }
        }
  }
#undef JAM_FACE
}

/* dissip_jameson.f90:4-431 (3-D): d zeroed over the block, then the i, j, k
 * dissipation fluxes */
void orc_dissip_jameson(int l, const double *v, double *d, const double *sn,
                        const double *ps, const double *cson) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, d);
  double *snu = calloc((size_t)b->nnn, sizeof(double));
  for (int dir = 0; dir < 3; ++dir) jameson_dissip_dir(b, dir, d, v, sn, ps, cson, snu);
  free(snu);
}

/* sch_jameson.f90:85-124: centred cell fluxes (with the cell stresses for
 * Navier-Stokes) over the whole block, ghosts included */
static void jameson_cell_flux(const blk_t *b, int ns, const double *v, const double *tau,
                              const double *ps, double *f) {
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  const double pinfl = G.pinfl;
  for (int64_t m = 0; m < nnn; ++m) {
    int64_t n = n0 + m;
    const double v1 = v[n], v2 = v[L + n], v3 = v[2 * L + n], v4 = v[3 * L + n],
                 v5 = v[4 * L + n], p = ps[n];
    double *F = f + 9 * m;
    if (ns) {
      const double txx = tau[n], txy = tau[L + n], txz = tau[2 * L + n],
                   tyy = tau[3 * L + n], tyz = tau[4 * L + n], tzz = tau[5 * L + n],
                   qx = tau[6 * L + n], qy = tau[7 * L + n], qz = tau[8 * L + n];
      F[0] = v2 * (v2 / v1) + p - pinfl - txx;
      F[1] = v3 * (v2 / v1) - txy;
      F[2] = v4 * (v2 / v1) - txz;
      F[3] = v3 * (v3 / v1) + p - pinfl - tyy;
      F[4] = v4 * (v3 / v1) - tyz;
      F[5] = v4 * (v4 / v1) + p - pinfl - tzz;
      F[6] = ((v5 + p - pinfl - txx) * v2 - txy * v3 - txz * v4) / v1 - qx;
      F[7] = ((v5 + p - pinfl - tyy) * v3 - txy * v2 - tyz * v4) / v1 - qy;
      F[8] = ((v5 + p - pinfl - tzz) * v4 - txz * v2 - tyz * v3) / v1 - qz;
    } else {
      F[0] = v2 * (v2 / v1) + p - pinfl;
      F[1] = v3 * (v2 / v1);
      F[2] = v4 * (v2 / v1);
      F[3] = v3 * (v3 / v1) + p - pinfl;
      F[4] = v4 * (v3 / v1);
      F[5] = v4 * (v4 / v1) + p - pinfl;
      F[6] = (v5 + p - pinfl) * v2 / v1;
      F[7] = (v5 + p - pinfl) * v3 / v1;
      F[8] = (v5 + p - pinfl) * v4 / v1;
    }
  }
}

/* the five projections of one face from the (summed or doubled) cell
 * momenta and fluxes (sch_jameson.f90:141-155); F order: xx xy xz yy yz zz
 * ex ey ez */
static void jameson_proj(const double m3[3], const double F[9], double s1, double s2,
                         double s3, double si[5]) {
  si[0] = m3[0] * s1 + m3[1] * s2 + m3[2] * s3;
  si[1] = F[0] * s1 + F[1] * s2 + F[2] * s3;
  si[2] = F[1] * s1 + F[3] * s2 + F[4] * s3;
  si[3] = F[2] * s1 + F[4] * s2 + F[5] * s3;
  si[4] = F[6] * s1 + F[7] * s2 + F[8] * s3;
}

/* sch_jameson.f90:4-437 (ityprk = 0, 3-D) */
void orc_sch_jameson(int l, double *u, const double *v, const double *d,
                     const double *tau, const double *sn, const double *ps) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  zero_u(b, u);
  double *f = malloc(sizeof(double) * 9 * (size_t)b->nnn);
  jameson_cell_flux(b, G.ns, v, tau, ps, f);
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    const int kdir = dir, nd = NDIR(b, dir);
    int lo[3], hi[3];
    /* interior faces (:135-168), lower (:170-196), upper (:198-224) */
    for (int pass = 0; pass < 3; ++pass) {
      lo[0] = 1; hi[0] = b->ni - 1; lo[1] = 1; hi[1] = b->nj - 1; lo[2] = 1; hi[2] = b->nk - 1;
      if (pass == 0) { lo[dir] = 2; hi[dir] = nd - 1; }
      else lo[dir] = hi[dir] = pass == 1 ? 1 : nd;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            int64_t n = IC(b, i, j, k), m = n - n0;
            const double s1 = SN(sn, b, m, kdir, 0), s2 = SN(sn, b, m, kdir, 1),
                         s3 = SN(sn, b, m, kdir, 2);
            double m3[3], F[9], si[5];
            if (pass == 0) {
              for (int a = 0; a < 3; ++a) m3[a] = v[(a + 1) * L + n] + v[(a + 1) * L + n - ninc];
              for (int q = 0; q < 9; ++q) F[q] = f[9 * m + q] + f[9 * (m - ninc) + q];
            } else {
              const int64_t c = pass == 1 ? n - ninc : n;  /* the ghost cell */
              for (int a = 0; a < 3; ++a) m3[a] = 2 * v[(a + 1) * L + c];
              for (int q = 0; q < 9; ++q) F[q] = 2 * f[9 * (c - n0) + q];
            }
            jameson_proj(m3, F, s1, s2, s3, si);
            for (int a = 0; a < 5; ++a) {
              if (pass != 2) u[a * L + n] = u[a * L + n] - si[a];
              if (pass != 1) u[a * L + n - ninc] = u[a * L + n - ninc] + si[a];
            }
          }
    }
  }
  free(f);
  /* normalisation and artificial dissipation (:421-437) */
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        for (int a = 0; a < 5; ++a) u[a * L + n] = 0.5 * u[a * L + n] - d[a * L + n];
      }
}

/* ------------------------------------------------------------------------ */
/* Roe flux                                                                  */
/* ------------------------------------------------------------------------ */

/* Roe dissipation |A|dW and the convective part of the face flux
 * (sch_roe_euler.f90:284-422, sch_roe.f90:326-461).  W = rho,u,v,w,p. */
static void roe_core(const double *WL, const double *WR, double sx, double sy,
                     double sz, int absam, double di[5], double *el_,
                     double *er_) {
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  double cnds = sqrt(sx * sx + sy * sy + sz * sz);
  double nx = sx / cnds, ny = sy / cnds, nz = sz / cnds;
  double al = sqrt(gam * pl / rhol);
  double ar = sqrt(gam * prr / rhor);
  double q2l = sq(ul) + sq(vl) + sq(wl);
  double q2r = sq(ur) + sq(vr) + sq(wr);
  double hl = al * al / gam1 + 0.5 * q2l;
  double hr = ar * ar / gam1 + 0.5 * q2r;
  double el = pl / (gam1 * rhol) + 0.5 * q2l + pinfl / rhol;
  double er = prr / (gam1 * rhor) + 0.5 * q2r + pinfl / rhor;
  double gd = sqrt(rhor / rhol);
  double gd1 = 1. / (1. + gd);
  double gd2 = gd * gd1;
  double rhom = sqrt(rhol * rhor);
  double rhomi = 1. / rhom;
  double um = gd1 * ul + gd2 * ur;
  double vm = gd1 * vl + gd2 * vr;
  double wm = gd1 * wl + gd2 * wr;
  double hm = gd1 * hl + gd2 * hr;
  double vitm2 = 0.5 * (sq(um) + sq(vm) + sq(wm));
  double am = absam ? sqrt(fabs(gam1 * (hm - vitm2))) : sqrt(gam1 * (hm - vitm2));
  double am2i = 1. / (am * am);
  double vn = um * nx + vm * ny + wm * nz;
  double rhoiam = rhom / am;
  double rhoami = am2i / rhoiam;
  double lam[5];
  lam[0] = fabs(vn * cnds);
  lam[1] = lam[0];
  lam[2] = lam[0];
  lam[3] = fabs(vn * cnds + am * cnds);
  lam[4] = fabs(vn * cnds - am * cnds);
  double q[5][5], p[5][5];
  q[0][0] = (1. - gam1 * vitm2 * am2i) * nx - (vm * nz - wm * ny) * rhomi;
  q[0][1] = gam1 * um * nx * am2i;
  q[0][2] = gam1 * vm * nx * am2i + nz * rhomi;
  q[0][3] = gam1 * wm * nx * am2i - ny * rhomi;
  q[0][4] = -gam1 * nx * am2i;
  q[1][0] = (1. - gam1 * vitm2 * am2i) * ny - (wm * nx - um * nz) * rhomi;
  q[1][1] = gam1 * um * ny * am2i - nz * rhomi;
  q[1][2] = gam1 * vm * ny * am2i;
  q[1][3] = gam1 * wm * ny * am2i + nx * rhomi;
  q[1][4] = -gam1 * ny * am2i;
  q[2][0] = (1. - gam1 * vitm2 * am2i) * nz - (um * ny - vm * nx) * rhomi;
  q[2][1] = gam1 * um * nz * am2i + ny * rhomi;
  q[2][2] = gam1 * vm * nz * am2i - nx * rhomi;
  q[2][3] = gam1 * wm * nz * am2i;
  q[2][4] = -gam1 * nz * am2i;
  q[3][0] = gam1 * vitm2 * rhoami - vn * rhomi;
  q[3][1] = nx * rhomi - gam1 * um * rhoami;
  q[3][2] = ny * rhomi - gam1 * vm * rhoami;
  q[3][3] = nz * rhomi - gam1 * wm * rhoami;
  q[3][4] = gam1 * rhoami;
  q[4][0] = gam1 * vitm2 * rhoami + vn * rhomi;
  q[4][1] = -nx * rhomi - gam1 * um * rhoami;
  q[4][2] = -ny * rhomi - gam1 * vm * rhoami;
  q[4][3] = -nz * rhomi - gam1 * wm * rhoami;
  q[4][4] = gam1 * rhoami;
  p[0][0] = nx;
  p[0][1] = ny;
  p[0][2] = nz;
  p[0][3] = 0.5 * rhoiam;
  p[0][4] = 0.5 * rhoiam;
  p[1][0] = um * nx;
  p[1][1] = um * ny - rhom * nz;
  p[1][2] = um * nz + rhom * ny;
  p[1][3] = 0.5 * rhoiam * (um + nx * am);
  p[1][4] = 0.5 * rhoiam * (um - nx * am);
  p[2][0] = vm * nx + rhom * nz;
  p[2][1] = vm * ny;
  p[2][2] = vm * nz - rhom * nx;
  p[2][3] = 0.5 * rhoiam * (vm + ny * am);
  p[2][4] = 0.5 * rhoiam * (vm - ny * am);
  p[3][0] = wm * nx - rhom * ny;
  p[3][1] = wm * ny + rhom * nx;
  p[3][2] = wm * nz;
  p[3][3] = 0.5 * rhoiam * (wm + nz * am);
  p[3][4] = 0.5 * rhoiam * (wm - nz * am);
  p[4][0] = vitm2 * nx + rhom * (vm * nz - wm * ny);
  p[4][1] = vitm2 * ny + rhom * (wm * nx - um * nz);
  p[4][2] = vitm2 * nz + rhom * (um * ny - vm * nx);
  p[4][3] = 0.5 * rhoiam * (hm + am * vn);
  p[4][4] = 0.5 * rhoiam * (hm - am * vn);
  double dw[5];
  dw[0] = rhor - rhol;
  dw[1] = rhor * ur - rhol * ul;
  dw[2] = rhor * vr - rhol * vl;
  dw[3] = rhor * wr - rhol * wl;
  dw[4] = rhor * er - rhol * el;
  for (int r = 0; r < 5; ++r) {
    double acc = 0.;
    for (int c = 0; c < 5; ++c) {
      double a = p[r][0] * lam[0] * q[0][c];
      for (int kk = 1; kk < 5; ++kk) a = a + p[r][kk] * lam[kk] * q[kk][c];
      acc = (c == 0) ? a * dw[0] : acc + a * dw[c];
    }
    di[r] = acc;
  }
  *el_ = el;
  *er_ = er;
}

/* primitive extrapolation with the kappa-MUSCL formula, no limiter
 * (sch_roe_euler.f90:245-273).  vv: rho,rhou,rhov,rhow,rhoE columns at cells
 * n-2,n-1,n,n+1 (index 0..3), pp: pressure at the same cells */
static void muscl_plain(const double vv[4][5], const double pp[4], double WL[5],
                        double WR[5]) {
  const double c = 0.25 * G.muscl, xk = G.xk;
  double uu[4][3];
  for (int s = 0; s < 4; ++s)
    for (int a = 0; a < 3; ++a) uu[s][a] = vv[s][a + 1] / vv[s][0];
  WL[0] = vv[1][0] + c * ((1. - xk) * (vv[1][0] - vv[0][0]) + (1. + xk) * (vv[2][0] - vv[1][0]));
  for (int a = 0; a < 3; ++a)
    WL[1 + a] = uu[1][a] + c * ((1. - xk) * (uu[1][a] - uu[0][a]) + (1. + xk) * (uu[2][a] - uu[1][a]));
  WL[4] = pp[1] + c * ((1. - xk) * (pp[1] - pp[0]) + (1. + xk) * (pp[2] - pp[1]));
  WR[0] = vv[2][0] - c * ((1. + xk) * (vv[2][0] - vv[1][0]) + (1. - xk) * (vv[3][0] - vv[2][0]));
  for (int a = 0; a < 3; ++a)
    WR[1 + a] = uu[2][a] - c * ((1. + xk) * (uu[2][a] - uu[1][a]) + (1. - xk) * (uu[3][a] - uu[2][a]));
  WR[4] = pp[2] - c * ((1. + xk) * (pp[2] - pp[1]) + (1. - xk) * (pp[3] - pp[2]));
}

/* minmod limiter of sch_roe.f90:1500-1504 */
static inline double phi(double a) {
  double m = (a < 1.) ? a : 1.;
  return (m > 0.) ? m : 0.;
}

/* limited extrapolation of sch_roe.f90:196-227 given the slope ratios at the
 * face (rm) and at the next face (rp) for the five primitive variables */
static void muscl_limited(const double vv[4][5], const double pp[4],
                          const double rm[5], const double rp[5], double WL[5],
                          double WR[5]) {
  const double c = 0.25 * G.muscl, xk = G.xk;
  double uu[4][3];
  for (int s = 0; s < 4; ++s)
    for (int a = 0; a < 3; ++a) uu[s][a] = vv[s][a + 1] / vv[s][0];
  WL[0] = vv[1][0] + c * phi(rm[0]) * (1. - xk) * (vv[1][0] - vv[0][0]) +
          c * phi(1. / rm[0]) * (1. + xk) * (vv[2][0] - vv[1][0]);
  for (int a = 0; a < 3; ++a)
    WL[1 + a] = uu[1][a] + c * phi(rm[1 + a]) * (1. - xk) * (uu[1][a] - uu[0][a]) +
                (1. + xk) * (uu[2][a] - uu[1][a]) * 0.25 * G.muscl * phi(1. / rm[1 + a]);
  WL[4] = pp[1] + c * phi(rm[4]) * (1. - xk) * (pp[1] - pp[0]) +
          c * phi(1. / rm[4]) * (1. + xk) * (pp[2] - pp[1]);
  WR[0] = vv[2][0] - c * phi(rp[0]) * (1. + xk) * (vv[2][0] - vv[1][0]) -
          c * phi(1. / rp[0]) * (1. - xk) * (vv[3][0] - vv[2][0]);
  for (int a = 0; a < 3; ++a)
    WR[1 + a] = uu[2][a] - c * phi(rp[1 + a]) * (1. + xk) * (uu[2][a] - uu[1][a]) -
                (1. - xk) * (uu[3][a] - uu[2][a]) * 0.25 * G.muscl * phi(1. / rp[1 + a]);
  WR[4] = pp[2] - c * phi(rp[4]) * (1. + xk) * (pp[2] - pp[1]) -
          c * phi(1. / rp[4]) * (1. - xk) * (pp[3] - pp[2]);
}

/* interior face flux f1..f5 (before the 0.5) of sch_roe_euler.f90:403-422 and
 * sch_roe.f90:437-461 (tau = NULL for the Euler form) */
static void face_flux(const double WL[5], const double WR[5], double sx,
                      double sy, double sz, int absam, const double *tau,
                      int64_t L, int64_t nR, int64_t nL, double f[5]) {
  const double pinfl = G.pinfl;
  double di[5], el, er;
  roe_core(WL, WR, sx, sy, sz, absam, di, &el, &er);
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  double dfxx, dfxy, dfxz, dfyy, dfyz, dfzz, dfex, dfey, dfez;
  if (!tau) {
    dfxx = rhor * sq(ur) + prr - pinfl + rhol * sq(ul) + pl - pinfl;
    dfxy = rhor * ur * vr + rhol * ul * vl;
    dfxz = rhor * ur * wr + rhol * ul * wl;
    dfyy = rhor * sq(vr) + prr - pinfl + rhol * sq(vl) + pl - pinfl;
    dfyz = rhor * vr * wr + rhol * vl * wl;
    dfzz = rhor * sq(wr) + prr - pinfl + rhol * sq(wl) + pl - pinfl;
    dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul;
    dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl;
    dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl;
  } else {
    const double *txx = tau, *txy = tau + L, *txz = tau + 2 * L, *tyy = tau + 3 * L,
                 *tyz = tau + 4 * L, *tzz = tau + 5 * L, *qx = tau + 6 * L,
                 *qy = tau + 7 * L, *qz = tau + 8 * L;
    dfxx = rhor * sq(ur) + prr - pinfl - txx[nR] + rhol * sq(ul) + pl - pinfl - txx[nL];
    dfxy = rhor * ur * vr - txy[nR] + rhol * ul * vl - txy[nL];
    dfxz = rhor * ur * wr - txz[nR] + rhol * ul * wl - txz[nL];
    dfyy = rhor * sq(vr) + prr - pinfl - tyy[nR] + rhol * sq(vl) + pl - pinfl - tyy[nL];
    dfyz = rhor * vr * wr - tyz[nR] + rhol * vl * wl - tyz[nL];
    dfzz = rhor * sq(wr) + prr - pinfl - tzz[nR] + rhol * sq(wl) + pl - pinfl - tzz[nL];
    dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul -
           (txx[nR] * ur + txy[nR] * vr + txz[nR] * wr) -
           (txx[nL] * ul + txy[nL] * vl + txz[nL] * wl) - qx[nR] - qx[nL];
    dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl -
           (txy[nR] * ur + tyy[nR] * vr + tyz[nR] * wr) -
           (txy[nL] * ul + tyy[nL] * vl + tyz[nL] * wl) - qy[nR] - qy[nL];
    dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl -
           (txz[nR] * ur + tyz[nR] * vr + tzz[nR] * wr) -
           (txz[nL] * ul + tyz[nL] * vl + tzz[nL] * wl) - qz[nR] - qz[nL];
  }
  f[0] = (rhor * ur + rhol * ul) * sx + (rhor * vr + rhol * vl) * sy +
         (rhor * wr + rhol * wl) * sz - di[0];
  f[1] = dfxx * sx + dfxy * sy + dfxz * sz - di[1];
  f[2] = dfxy * sx + dfyy * sy + dfyz * sz - di[2];
  f[3] = dfxz * sx + dfyz * sy + dfzz * sz - di[3];
  f[4] = dfex * sx + dfey * sy + dfez * sz - di[4];
}

/* physical flux of a ghost cell through a boundary face (sch_roe_euler.f90:
 * 438-513, sch_roe.f90:497-580).  ng: ghost cell; nrho: the cell whose
 * density divides the energy flux (the ghost, except the j/k lower faces of
 * sch_roe_euler, which use the interior cell: sch_roe_euler.f90:630-632). */
static void bnd_flux(const double *v, const double *ps, const double *tau,
                     int64_t L, int64_t ng, int64_t nrho, double sx, double sy,
                     double sz, double s[5]) {
  const double pinfl = G.pinfl;
  const double v1 = v[ng], v2 = v[L + ng], v3 = v[2 * L + ng], v4 = v[3 * L + ng],
               v5 = v[4 * L + ng], p = ps[ng];
  double fxx, fxy, fxz, fyy, fyz, fzz, fex, fey, fez;
  if (!tau) {
    fxx = v2 * (v2 / v1) + p - pinfl;
    fxy = v3 * (v2 / v1);
    fxz = v4 * (v2 / v1);
    fyy = v3 * (v3 / v1) + p - pinfl;
    fyz = v4 * (v3 / v1);
    fzz = v4 * (v4 / v1) + p - pinfl;
    fex = (v5 + p - pinfl) * v2 / v[nrho];
    fey = (v5 + p - pinfl) * v3 / v[nrho];
    fez = (v5 + p - pinfl) * v4 / v[nrho];
  } else {
    const double txx = tau[ng], txy = tau[L + ng], txz = tau[2 * L + ng],
                 tyy = tau[3 * L + ng], tyz = tau[4 * L + ng], tzz = tau[5 * L + ng],
                 qx = tau[6 * L + ng], qy = tau[7 * L + ng], qz = tau[8 * L + ng];
    fxx = v2 * (v2 / v1) + p - pinfl - txx;
    fxy = v3 * (v2 / v1) - txy;
    fxz = v4 * (v2 / v1) - txz;
    fyy = v3 * (v3 / v1) + p - pinfl - tyy;
    fyz = v4 * (v3 / v1) - tyz;
    fzz = v4 * (v4 / v1) + p - pinfl - tzz;
    fex = ((v5 + p - pinfl - txx) * v2 - txy * v3 - txz * v4) / v1 - qx;
    fey = ((v5 + p - pinfl - tyy) * v3 - txy * v2 - tyz * v4) / v1 - qy;
    fez = ((v5 + p - pinfl - tzz) * v4 - txz * v2 - tyz * v3) / v1 - qz;
  }
  s[0] = v2 * sx + v3 * sy + v4 * sz;
  s[1] = fxx * sx + fxy * sy + fxz * sz;
  s[2] = fxy * sx + fyy * sy + fyz * sz;
  s[3] = fxz * sx + fyz * sy + fzz * sz;
  s[4] = fex * sx + fey * sy + fez * sz;
}

static void gather_cells(const double *v, const double *ps, int64_t L,
                         int64_t n, int64_t ninc, double vv[4][5], double pp[4]) {
  for (int s = 0; s < 4; ++s) {
    int64_t c = n + (s - 2) * ninc;
    for (int a = 0; a < 5; ++a) vv[s][a] = v[a * L + c];
    pp[s] = ps[c];
  }
}

/* ranges of the (k,j,i) loop nest of one direction: real cells on the
 * tangential axes, [flo, fhi] on the face axis */
static void dir_ranges(const blk_t *b, int dir, int flo, int fhi, int lo[3],
                       int hi[3]) {
  lo[0] = 1; hi[0] = b->ni - 1;
  lo[1] = 1; hi[1] = b->nj - 1;
  lo[2] = 1; hi[2] = b->nk - 1;
  lo[dir] = flo;
  hi[dir] = fhi;
}

/* one direction of sch_roe_euler / sch_roe: interior faces (optionally with
 * the in-place limiter recurrence), then lower and upper boundary faces */
static void roe_direction(const blk_t *b, int dir, int ns, double *u,
                          const double *v, const double *tau, const double *sn,
                          const double *ps) {
  const int64_t L = G.ld, n0 = b->npc, ninc = NINC(b, dir);
  const int nd = NDIR(b, dir); /* node count along dir: faces 1..nd */
  const int absam = (!ns) && dir > 0;
  int lo[3], hi[3], idx[3];
  double *r = NULL;
  const int limited = ns && G.ilim == 1;
  if (limited) {
    r = calloc((size_t)5 * b->nnn, sizeof(double));
    /* slope differences at faces 1..nd (sch_roe.f90:146-159) */
    dir_ranges(b, dir, 1, nd, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          r[m] = v[n] - v[n - ninc];
          r[b->nnn + m] = v[L + n] / v[n] - v[L + n - ninc] / v[n - ninc];
          r[2 * b->nnn + m] = v[2 * L + n] / v[n] - v[2 * L + n - ninc] / v[n - ninc];
          r[3 * b->nnn + m] = v[3 * L + n] / v[n] - v[3 * L + n - ninc] / v[n - ninc];
          r[4 * b->nnn + m] = ps[n] - ps[n - ninc];
        }
    /* in-place ratio recurrence along each line (sch_roe.f90:161-194) */
    dir_ranges(b, dir, 2, nd - 1, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t m = ML(b, idx[0], idx[1], idx[2]);
          for (int a = 0; a < 5; ++a) {
            double *ra = r + (int64_t)a * b->nnn;
            if (fabs(ra[m - ninc] * ra[m] * ra[m + ninc]) <= DBL_MIN)
              ra[m] = 1.;
            else
              ra[m] = ra[m] / ra[m - ninc];
          }
        }
  }
  /* interior faces 2..nd-1 */
  dir_ranges(b, dir, 2, nd - 1, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double vv[4][5], pp[4], WL[5], WR[5], f[5];
        gather_cells(v, ps, L, n, ninc, vv, pp);
        if (limited && idx[dir] <= nd - 2) {
          double rm[5], rp[5];
          for (int a = 0; a < 5; ++a) {
            rm[a] = r[(int64_t)a * b->nnn + m];
            rp[a] = r[(int64_t)a * b->nnn + m + ninc];
          }
          muscl_limited(vv, pp, rm, rp, WL, WR);
        } else {
          muscl_plain(vv, pp, WL, WR);
        }
        face_flux(WL, WR, SN(sn, b, m, dir, 0), SN(sn, b, m, dir, 1),
                  SN(sn, b, m, dir, 2), absam, ns ? tau : NULL, L, n, n - ninc, f);
        for (int a = 0; a < 5; ++a) {
          u[a * L + n] = u[a * L + n] - 0.5 * f[a];
          u[a * L + n - ninc] = u[a * L + n - ninc] + 0.5 * f[a];
        }
      }
  /* lower boundary face 1 */
  dir_ranges(b, dir, 1, 1, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double s[5];
        int64_t nrho = (!ns && dir > 0) ? n : n - ninc;
        bnd_flux(v, ps, ns ? tau : NULL, L, n - ninc, nrho, SN(sn, b, m, dir, 0),
                 SN(sn, b, m, dir, 1), SN(sn, b, m, dir, 2), s);
        for (int a = 0; a < 5; ++a) u[a * L + n] = u[a * L + n] - s[a];
      }
  /* upper boundary face nd */
  dir_ranges(b, dir, nd, nd, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double s[5];
        bnd_flux(v, ps, ns ? tau : NULL, L, n, n, SN(sn, b, m, dir, 0),
                 SN(sn, b, m, dir, 1), SN(sn, b, m, dir, 2), s);
        for (int a = 0; a < 5; ++a) u[a * L + n - ninc] = u[a * L + n - ninc] + s[a];
      }
  free(r);
}

/* ---- other flux families: HLLC (ischema 14), Rusanov (ischema 9) ------ */

/* the HLLC flux through a face (sch_hllc_euler.f90:135-221,
 * sch_hllc.f90:270-357): the left or right physical flux, or the star
 * state's; absam: the sound speed from |gam1*(hm - vitm2)| (sch_hllc.f90 in
 * the i and j directions) */
static void hllc_core(const double WL[5], const double WR[5], double s1, double s2,
                      double s3, int absam, double fc[5]) {
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const double nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const double al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  const double q2l = sq(ul) + sq(vl) + sq(wl), q2r = sq(ur) + sq(vr) + sq(wr);
  const double hl = al * al / gam1 + 0.5 * q2l, hr = ar * ar / gam1 + 0.5 * q2r;
  const double el = pl / (gam1 * rhol) + 0.5 * q2l + pinfl / rhol;
  const double er = prr / (gam1 * rhor) + 0.5 * q2r + pinfl / rhor;
  const double vnl = ul * nx + vl * ny + wl * nz, vnr = ur * nx + vr * ny + wr * nz;
  const double gd = sqrt(rhor / rhol), gd1 = 1. / (1. + gd), gd2 = gd * gd1;
  const double um = gd1 * ul + gd2 * ur, vm = gd1 * vl + gd2 * vr, wm = gd1 * wl + gd2 * wr;
  const double hm = gd1 * hl + gd2 * hr;
  const double vitm2 = 0.5 * (sq(um) + sq(vm) + sq(wm));
  const double am = absam ? sqrt(fabs(gam1 * (hm - vitm2))) : sqrt(gam1 * (hm - vitm2));
  const double vnm = um * nx + vm * ny + wm * nz;
  const double sl = vnm - am, sr = vnm + am;
  const double sst = (rhor * vnr * (sr - vnr) - rhol * vnl * (sl - vnl) + pl - prr) /
                     (rhor * (sr - vnr) - rhol * (sl - vnl));
  const double pst = rhol * (vnl - sl) * (vnl - sst) + pl;
  if (sl > 0. || sr < 0.) {
    const int left = sl > 0.;
    const double rho = left ? rhol : rhor, u = left ? ul : ur, v = left ? vl : vr,
                 w = left ? wl : wr, p = left ? pl : prr, e = left ? el : er;
    const double fxx = rho * sq(u) + p - pinfl, fxy = rho * u * v, fxz = rho * u * w;
    const double fyy = rho * sq(v) + p - pinfl, fyz = rho * v * w;
    const double fzz = rho * sq(w) + p - pinfl;
    const double fex = (rho * e + p - pinfl) * u, fey = (rho * e + p - pinfl) * v,
                 fez = (rho * e + p - pinfl) * w;
    fc[0] = rho * u * s1 + rho * v * s2 + rho * w * s3;
    fc[1] = fxx * s1 + fxy * s2 + fxz * s3;
    fc[2] = fxy * s1 + fyy * s2 + fyz * s3;
    fc[3] = fxz * s1 + fyz * s2 + fzz * s3;
    fc[4] = fex * s1 + fey * s2 + fez * s3;
  } else if (sst >= 0. || sst < 0.) {
    const int left = sst >= 0.;
    const double rho = left ? rhol : rhor, u = left ? ul : ur, v = left ? vl : vr,
                 w = left ? wl : wr, p = left ? pl : prr, e = left ? el : er,
                 vn = left ? vnl : vnr, sk = left ? sl : sr;
    const double ids = 1. / (sk - sst);
    const double rhost = rho * (sk - vn);
    const double rhoust = (rhost * u + (pst - p) * nx) * ids;
    const double rhovst = (rhost * v + (pst - p) * ny) * ids;
    const double rhowst = (rhost * w + (pst - p) * nz) * ids;
    const double rhoest = (rho * e * (sk - vn) + (pst - pinfl) * sst - (p - pinfl) * vn) * ids;
    fc[0] = rhost * ids * sst * cnds;
    fc[1] = (rhoust * sst + (pst - pinfl) * nx) * cnds;
    fc[2] = (rhovst * sst + (pst - pinfl) * ny) * cnds;
    fc[3] = (rhowst * sst + (pst - pinfl) * nz) * cnds;
    fc[4] = (rhoest + pst - pinfl) * sst * cnds;
  } else {
    for (int a = 0; a < 5; ++a) fc[a] = NAN;
  }
}

/* the viscous part of sch_hllc.f90:358-375 (fv2..fv5) */
static void hllc_viscous(const double WL[5], const double WR[5], double s1, double s2,
                         double s3, const double *tau, int64_t L, int64_t nR, int64_t nL,
                         double fv[5]) {
  const double *txx = tau, *txy = tau + L, *txz = tau + 2 * L, *tyy = tau + 3 * L,
               *tyz = tau + 4 * L, *tzz = tau + 5 * L, *qx = tau + 6 * L, *qy = tau + 7 * L,
               *qz = tau + 8 * L;
  const double ul = WL[1], vl = WL[2], wl = WL[3], ur = WR[1], vr = WR[2], wr = WR[3];
  fv[0] = 0.;
  fv[1] = (txx[nR] + txx[nL]) * s1 + (txy[nR] + txy[nL]) * s2 + (txz[nR] + txz[nL]) * s3;
  fv[2] = (txy[nR] + txy[nL]) * s1 + (tyy[nR] + tyy[nL]) * s2 + (tyz[nR] + tyz[nL]) * s3;
  fv[3] = (txz[nR] + txz[nL]) * s1 + (tyz[nR] + tyz[nL]) * s2 + (tzz[nR] + tzz[nL]) * s3;
  fv[4] = (txx[nR] * ur + txy[nR] * vr + txz[nR] * wr + txx[nL] * ul + txy[nL] * vl +
           txz[nL] * wl + qx[nR] + qx[nL]) * s1 +
          (txy[nR] * ur + tyy[nR] * vr + tyz[nR] * wr + txy[nL] * ul + tyy[nL] * vl +
           tyz[nL] * wl + qy[nR] + qy[nL]) * s2 +
          (txz[nR] * ur + tyz[nR] * vr + tzz[nR] * wr + txz[nL] * ul + tyz[nL] * vl +
           tzz[nL] * wl + qz[nR] + qz[nL]) * s3;
}

/* the Rusanov flux of sch_rusanov.f90:129-185: the centred flux (viscous
 * stresses included) minus rm*(W_R - W_L), rm = |S| max(|vnl+al|, |vnr+ar|) */
static void rusanov_flux(const double WL[5], const double WR[5], double s1, double s2,
                         double s3, const double *tau, int64_t L, int64_t nR, int64_t nL,
                         double f[5]) {
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const double nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const double al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  const double q2l = sq(ul) + sq(vl) + sq(wl), q2r = sq(ur) + sq(vr) + sq(wr);
  const double el = pl / (gam1 * rhol) + 0.5 * q2l + pinfl / rhol;
  const double er = prr / (gam1 * rhor) + 0.5 * q2r + pinfl / rhor;
  const double vnl = ul * nx + vl * ny + wl * nz, vnr = ur * nx + vr * ny + wr * nz;
  const double al1 = fabs(vnl + al), ar1 = fabs(vnr + ar);
  const double rm = cnds * (al1 >= ar1 ? al1 : ar1);
  double di[5];
  di[0] = rm * (rhor - rhol);
  di[1] = rm * (rhor * ur - rhol * ul);
  di[2] = rm * (rhor * vr - rhol * vl);
  di[3] = rm * (rhor * wr - rhol * wl);
  di[4] = rm * (rhor * er - rhol * el);
  const double *txx = tau, *txy = tau + L, *txz = tau + 2 * L, *tyy = tau + 3 * L,
               *tyz = tau + 4 * L, *tzz = tau + 5 * L, *qx = tau + 6 * L, *qy = tau + 7 * L,
               *qz = tau + 8 * L;
  const double dfxx = rhor * sq(ur) + prr - pinfl - txx[nR] + rhol * sq(ul) + pl - pinfl - txx[nL];
  const double dfxy = rhor * ur * vr - txy[nR] + rhol * ul * vl - txy[nL];
  const double dfxz = rhor * ur * wr - txz[nR] + rhol * ul * wl - txz[nL];
  const double dfyy = rhor * sq(vr) + prr - pinfl - tyy[nR] + rhol * sq(vl) + pl - pinfl - tyy[nL];
  const double dfyz = rhor * vr * wr - tyz[nR] + rhol * vl * wl - tyz[nL];
  const double dfzz = rhor * sq(wr) + prr - pinfl - tzz[nR] + rhol * sq(wl) + pl - pinfl - tzz[nL];
  const double dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul -
                      (txx[nR] * ur + txy[nR] * vr + txz[nR] * wr) -
                      (txx[nL] * ul + txy[nL] * vl + txz[nL] * wl) - qx[nR] - qx[nL];
  const double dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl -
                      (txy[nR] * ur + tyy[nR] * vr + tyz[nR] * wr) -
                      (txy[nL] * ul + tyy[nL] * vl + tyz[nL] * wl) - qy[nR] - qy[nL];
  const double dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl -
                      (txz[nR] * ur + tyz[nR] * vr + tzz[nR] * wr) -
                      (txz[nL] * ul + tyz[nL] * vl + tzz[nL] * wl) - qz[nR] - qz[nL];
  f[0] = (rhor * ur + rhol * ul) * s1 + (rhor * vr + rhol * vl) * s2 +
         (rhor * wr + rhol * wl) * s3 - di[0];
  f[1] = dfxx * s1 + dfxy * s2 + dfxz * s3 - di[1];
  f[2] = dfxy * s1 + dfyy * s2 + dfyz * s3 - di[2];
  f[3] = dfxz * s1 + dfyz * s2 + dfzz * s3 - di[3];
  f[4] = dfex * s1 + dfey * s2 + dfez * s3 - di[4];
}

/* the AUSM+ splittings of sch_ausmp.f90:1010-1033 (sign(1,x) = +-1 by the
 * sign bit of x) */
static double sgn1(double x) { return copysign(1., x); }
static double ausm_fmp(double aa) {
  return 0.25 * (1. + sgn1(fabs(aa) - 1.)) * (aa + fabs(aa)) +
         0.125 * (1. - sgn1(fabs(aa) - 1.)) * sq(aa + 1.);
}
static double ausm_fmm(double xa) {
  return 0.25 * (1. + sgn1(fabs(xa) - 1.)) * (xa - fabs(xa)) -
         0.125 * (1. - sgn1(fabs(xa) - 1.)) * sq(xa - 1.);
}
static double ausm_fpp(double ta) {
  return 0.25 * (1. + sgn1(fabs(ta) - 1.)) * (1. + sgn1(fabs(ta))) +
         0.125 * (1. - sgn1(fabs(ta) - 1.)) * sq(ta + 1.) * (2. - ta + 0.75 * ta * sq(ta - 1.));
}
static double ausm_fpm(double ra) {
  return 0.25 * (1. + sgn1(fabs(ra) - 1.)) * (1. - sgn1(fabs(ra))) +
         0.125 * (1. - sgn1(fabs(ra) - 1.)) * sq(ra - 1.) * (2. + ra - 0.75 * ra * sq(ra + 1.));
}

/* the work and heat-flux terms sch_ausmp.f90:81-83 stores in d(n,1:3) */
static void ausm_dterm(const double *v, const double *tau, int64_t L, int64_t n, double dd[3]) {
  const double v1 = v[n], v2 = v[L + n], v3 = v[2 * L + n], v4 = v[3 * L + n];
  const double txx = tau[n], txy = tau[L + n], txz = tau[2 * L + n], tyy = tau[3 * L + n],
               tyz = tau[4 * L + n], tzz = tau[5 * L + n];
  dd[0] = (txx * v2 + txy * v3 + txz * v4) / v1 + tau[6 * L + n];
  dd[1] = (tyy * v3 + txy * v2 + tyz * v4) / v1 + tau[7 * L + n];
  dd[2] = (tzz * v4 + txz * v2 + tyz * v3) / v1 + tau[8 * L + n];
}

/* the AUSM+ flux of sch_ausmp.f90:255-298 (hi1..hi5) */
static void ausm_flux(const double WL[5], const double WR[5], double s1, double s2, double s3,
                      const double *v, const double *tau, int64_t L, int64_t nR, int64_t nL,
                      double hi[5]) {
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const double al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  const double hl = al * al / gam1 + 0.5 * (sq(ul) + sq(vl) + sq(wl));
  const double hr = ar * ar / gam1 + 0.5 * (sq(ur) + sq(vr) + sq(wr));
  const double ai = sqrt(al * ar);
  const double cml = (ul * s1 + vl * s2 + wl * s3) / (al * cnds);
  const double cmr = (ur * s1 + vr * s2 + wr * s3) / (ar * cnds);
  const double psi = 2. * (pl * ausm_fpp(cml) + prr * ausm_fpm(cmr)) - 2. * pinfl;
  const double cmi = ausm_fmp(cml) + ausm_fmm(cmr);
  const double dm = 0.5 * ai * (cmi * (rhol + rhor) - fabs(cmi) * (rhor - rhol)) * cnds;
  const double *txx = tau, *txy = tau + L, *txz = tau + 2 * L, *tyy = tau + 3 * L,
               *tyz = tau + 4 * L, *tzz = tau + 5 * L;
  double dR[3], dL[3];
  ausm_dterm(v, tau, L, nR, dR);
  ausm_dterm(v, tau, L, nL, dL);
  hi[0] = dm;
  hi[1] = dm * (ul + ur) - fabs(dm) * (ur - ul) + psi * s1 - (txx[nR] + txx[nL]) * s1 -
          (txy[nR] + txy[nL]) * s2 - (txz[nR] + txz[nL]) * s3;
  hi[2] = dm * (vl + vr) - fabs(dm) * (vr - vl) + psi * s2 - (txy[nR] + txy[nL]) * s1 -
          (tyy[nR] + tyy[nL]) * s2 - (tyz[nR] + tyz[nL]) * s3;
  hi[3] = dm * (wl + wr) - fabs(dm) * (wr - wl) + psi * s3 - (txz[nR] + txz[nL]) * s1 -
          (tyz[nR] + tyz[nL]) * s2 - (tzz[nR] + tzz[nL]) * s3;
  hi[4] = dm * (hl + hr) - fabs(dm) * (hr - hl) - (dR[0] + dL[0]) * s1 -
          (dR[1] + dL[1]) * s2 - (dR[2] + dL[2]) * s3;
}

enum { ORC_FL_HLLC = 1, ORC_FL_RUSANOV = 2, ORC_FL_AUSM = 3 };

/* one direction of sch_hllc_euler (fl HLLC, ns 0), sch_hllc (fl HLLC, ns 1)
 * or sch_rusanov (fl RUSANOV, always with the stresses): the same loop
 * nests as roe_direction (interior faces, then lower and upper boundary
 * faces); the minmod limiter only in sch_hllc */
static void flux_direction(const blk_t *b, int dir, int fl, int ns, double *u,
                           const double *v, const double *tau, const double *sn,
                           const double *ps) {
  const int64_t L = G.ld, n0 = b->npc, ninc = NINC(b, dir);
  const int nd = NDIR(b, dir);
  const int absam = fl == ORC_FL_HLLC && ns && dir < 2;
  const int visc = ns || fl == ORC_FL_RUSANOV;
  int lo[3], hi[3], idx[3];
  double *r = NULL;
  const int limited = (fl == ORC_FL_HLLC || fl == ORC_FL_AUSM) && ns && G.ilim == 1;
  if (limited) {
    r = calloc((size_t)5 * b->nnn, sizeof(double));
    dir_ranges(b, dir, 1, nd, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          r[m] = v[n] - v[n - ninc];
          r[b->nnn + m] = v[L + n] / v[n] - v[L + n - ninc] / v[n - ninc];
          r[2 * b->nnn + m] = v[2 * L + n] / v[n] - v[2 * L + n - ninc] / v[n - ninc];
          r[3 * b->nnn + m] = v[3 * L + n] / v[n] - v[3 * L + n - ninc] / v[n - ninc];
          r[4 * b->nnn + m] = ps[n] - ps[n - ninc];
        }
    dir_ranges(b, dir, 2, nd - 1, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t m = ML(b, idx[0], idx[1], idx[2]);
          for (int a = 0; a < 5; ++a) {
            double *ra = r + (int64_t)a * b->nnn;
            if (fabs(ra[m - ninc] * ra[m] * ra[m + ninc]) <= DBL_MIN)
              ra[m] = 1.;
            else
              ra[m] = ra[m] / ra[m - ninc];
          }
        }
  }
  dir_ranges(b, dir, 2, nd - 1, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double vv[4][5], pp[4], WL[5], WR[5], f[5];
        gather_cells(v, ps, L, n, ninc, vv, pp);
        if (limited && idx[dir] <= nd - 2) {
          double rm[5], rp[5];
          for (int a = 0; a < 5; ++a) {
            rm[a] = r[(int64_t)a * b->nnn + m];
            rp[a] = r[(int64_t)a * b->nnn + m + ninc];
          }
          muscl_limited(vv, pp, rm, rp, WL, WR);
        } else {
          muscl_plain(vv, pp, WL, WR);
        }
        const double s1 = SN(sn, b, m, dir, 0), s2 = SN(sn, b, m, dir, 1),
                     s3 = SN(sn, b, m, dir, 2);
        if (fl == ORC_FL_AUSM) {
          ausm_flux(WL, WR, s1, s2, s3, v, tau, L, n, n - ninc, f);
          u[n] = u[n] - f[0];
          for (int a = 1; a < 5; ++a) u[a * L + n] = u[a * L + n] - 0.5 * f[a];
          u[n - ninc] = u[n - ninc] + f[0];
          for (int a = 1; a < 5; ++a) u[a * L + n - ninc] = u[a * L + n - ninc] + 0.5 * f[a];
        } else if (fl == ORC_FL_RUSANOV) {
          rusanov_flux(WL, WR, s1, s2, s3, tau, L, n, n - ninc, f);
          for (int a = 0; a < 5; ++a) {
            u[a * L + n] = u[a * L + n] - 0.5 * f[a];
            u[a * L + n - ninc] = u[a * L + n - ninc] + 0.5 * f[a];
          }
        } else if (!ns) {
          hllc_core(WL, WR, s1, s2, s3, absam, f);
          for (int a = 0; a < 5; ++a) {
            u[a * L + n] = u[a * L + n] - f[a];
            u[a * L + n - ninc] = u[a * L + n - ninc] + f[a];
          }
        } else {
          double fv[5];
          hllc_core(WL, WR, s1, s2, s3, absam, f);
          hllc_viscous(WL, WR, s1, s2, s3, tau, L, n, n - ninc, fv);
          u[n] = u[n] - f[0];
          for (int a = 1; a < 5; ++a) u[a * L + n] = u[a * L + n] - f[a] + 0.5 * fv[a];
          u[n - ninc] = u[n - ninc] + f[0];
          for (int a = 1; a < 5; ++a)
            u[a * L + n - ninc] = u[a * L + n - ninc] + f[a] - 0.5 * fv[a];
        }
      }
  dir_ranges(b, dir, 1, 1, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double sb[5];
        int64_t nrho = (!visc && dir > 0) ? n : n - ninc;
        bnd_flux(v, ps, visc ? tau : NULL, L, n - ninc, nrho, SN(sn, b, m, dir, 0),
                 SN(sn, b, m, dir, 1), SN(sn, b, m, dir, 2), sb);
        for (int a = 0; a < 5; ++a) u[a * L + n] = u[a * L + n] - sb[a];
      }
  dir_ranges(b, dir, nd, nd, lo, hi);
  for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
    for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
      for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
        int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
        double sb[5];
        bnd_flux(v, ps, visc ? tau : NULL, L, n, n, SN(sn, b, m, dir, 0),
                 SN(sn, b, m, dir, 1), SN(sn, b, m, dir, 2), sb);
        for (int a = 0; a < 5; ++a) u[a * L + n - ninc] = u[a * L + n - ninc] + sb[a];
      }
  free(r);
}

static void zero_u(const blk_t *b, double *u) {
  for (int a = 0; a < 5; ++a)
    for (int64_t n = b->npc; n < b->npc + b->nnn; ++n) u[a * G.ld + n] = 0.;
}

/* sch_roe_euler.f90:205-1000 (ityprk=0, 3-D) */
void orc_sch_roe_euler(int l, double *u, const double *v, const double *sn,
                       const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) roe_direction(b, dir, 0, u, v, NULL, sn, ps);
}

/* sch_roe.f90:102-1462 (ityprk=0, 3-D) */
void orc_sch_roe(int l, double *u, const double *v, const double *tau,
                 const double *sn, const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) roe_direction(b, dir, 1, u, v, tau, sn, ps);
}

/* sch_hllc_euler.f90:4-891 (ityprk=0, 3-D) */
void orc_sch_hllc_euler(int l, double *u, const double *v, const double *sn,
                        const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) flux_direction(b, dir, ORC_FL_HLLC, 0, u, v, NULL, sn, ps);
}

/* sch_hllc.f90:4-1403 (ityprk=0, 3-D) */
void orc_sch_hllc(int l, double *u, const double *v, const double *tau, const double *sn,
                  const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) flux_direction(b, dir, ORC_FL_HLLC, 1, u, v, tau, sn, ps);
}

/* sch_ausmp.f90:4-1157 (ityprk=0, 3-D; Navier-Stokes only, as the
 * reference calls it) */
void orc_sch_ausmp(int l, double *u, const double *v, const double *tau, const double *sn,
                   const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) flux_direction(b, dir, ORC_FL_AUSM, 1, u, v, tau, sn, ps);
}

/* sch_rusanov.f90:4-791 (ityprk=0, 3-D; the stresses enter whatever the
 * equations, zero for Euler) */
void orc_sch_rusanov(int l, double *u, const double *v, const double *tau, const double *sn,
                     const double *ps) {
  const blk_t *b = &G.b[l - 1];
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir)
    flux_direction(b, dir, ORC_FL_RUSANOV, G.ns, u, v, tau, sn, ps);
}

/* ------------------------------------------------------------------------ */
/* WENO5 (sch_weno5_3d.f90, ischema 12): Jiang & Shu's fifth-order scheme,   */
/* characteristic-wise on Roe-averaged eigenvectors, each field upwinded by  */
/* the sign of its eigenvalue, with Henrick's mapped weights                 */
/* ------------------------------------------------------------------------ */

/* sch_weno5_3d.f90:148-166: the cell's flux tensor as the five values the
 * projection reads per component c (0 x, 1 y, 2 z): rho u_c and the c-th
 * column of the momentum and energy fluxes */
static void weno_cell_flux(const double *v, const double *ps, int64_t n, double f[3][5]) {
  const int64_t L = G.ld;
  const double v1 = v[n], v2 = v[L + n], v3 = v[2 * L + n], v4 = v[3 * L + n],
               v5 = v[4 * L + n], p = ps[n], pinfl = G.pinfl;
  const double fxx = v2 * (v2 / v1) + p - pinfl, fxy = v3 * (v2 / v1), fxz = v4 * (v2 / v1);
  const double fyy = v3 * (v3 / v1) + p - pinfl, fyz = v4 * (v3 / v1);
  const double fzz = v4 * (v4 / v1) + p - pinfl;
  const double fex = (v5 + p - pinfl) * v2 / v1, fey = (v5 + p - pinfl) * v3 / v1,
               fez = (v5 + p - pinfl) * v4 / v1;
  const double t[3][5] = {{v2, fxx, fxy, fxz, fex}, {v3, fxy, fyy, fyz, fey},
                          {v4, fxz, fyz, fzz, fez}};
  memcpy(f, t, sizeof(t));
}

/* Henrick's map g(w) = w (ga + ga^2 - 3 ga w + w^2) / (ga^2 + w (1 - 2 ga)):
 * the numerator's and denominator's factors as sch_weno5_3d.f90:530-535
 * writes them */
static inline double weno_map_num(double ga, double w) {
  return ga + ga * ga - 3. * ga * w + w * w;
}
static inline double weno_map_den(double ga, double w) { return ga * ga + w * (1. - 2. * ga); }

/* one characteristic field (sch_weno5_3d.f90:333-620 for field 1): q holds
 * its projected flux at the six points i-2..i+3; the three third-order
 * candidates on the stencils upwind of the eigenvalue lam, their smoothness
 * indicators (squared), the normalised weights mapped by Henrick's g and
 * normalised again; the weighted sum of the first nterm candidates (the
 * reference keeps three in the x and y fluxes of the i direction, two
 * everywhere else) */
static double weno_field(const double q[6], double lam, int nterm) {
  const double c20 = 1. / 3., c21 = -7. / 6., c22 = 11. / 6., c10 = -1. / 6., c11 = 5. / 6.;
  const double ga1 = 0.1, ga2 = 0.6, ga3 = 0.3, c1 = 13. / 12., c2 = 0.25, eps = 1.e-6;
  const double sg = copysign(1., lam);
  const double up = 0.5 * (1. + sg), dn = 0.5 * (1. - sg);
  const double f1 = up * (q[0] * c20 + q[1] * c21 + q[2] * c22) +
                    dn * (q[1] * c10 + q[2] * c11 + q[3] * c20);
  const double f2 = up * (q[1] * c10 + q[2] * c11 + q[3] * c20) +
                    dn * (q[2] * c20 + q[3] * c11 + q[4] * c10);
  const double f3 = up * (q[2] * c20 + q[3] * c11 + q[4] * c10) +
                    dn * (q[3] * c22 + q[4] * c21 + q[5] * c20);
  const double s1 = sq(q[5] - 2. * q[4] + q[3]), s2 = sq(q[4] - 2. * q[3] + q[2]),
               s3 = sq(q[3] - 2. * q[2] + q[1]), s4 = sq(q[2] - 2. * q[1] + q[0]);
  const double t1 = sq(q[5] - 4. * q[4] + 3. * q[3]), t2 = sq(q[4] - 4. * q[3] + 3. * q[2]),
               t3 = sq(q[4] - q[2]), t4 = sq(q[3] - q[1]),
               t5 = sq(3. * q[3] - 4. * q[2] + q[1]), t6 = sq(3. * q[2] - 4. * q[1] + q[0]);
  /* (...)**iexp with iexp = 2 */
  const double b1 = sq(up * (c1 * s4 + c2 * t6) + dn * (c1 * s3 + c2 * t5) + eps);
  const double b2 = sq(up * (c1 * s3 + c2 * t4) + dn * (c1 * s2 + c2 * t3) + eps);
  const double b3 = sq(up * (c1 * s2 + c2 * t2) + dn * (c1 * s1 + c2 * t1) + eps);
  const double ww1 = up * (ga1 / b1) + dn * (ga3 / b1);
  const double ww2 = ga2 / b2;
  const double ww3 = up * (ga3 / b3) + dn * (ga1 / b3);
  const double sw = ww1 + ww2 + ww3;
  const double w1 = ww1 / sw, w2 = ww2 / sw, w3 = ww3 / sw;
  const double m1 = w1 * 0.5 * (1. + sg) * weno_map_num(ga1, w1) / weno_map_den(ga1, w1) +
                    w1 * 0.5 * (1. - sg) * weno_map_num(ga3, w1) / weno_map_den(ga3, w1);
  const double m2 = w2 * weno_map_num(ga2, w2) / weno_map_den(ga2, w2);
  const double m3 = w3 * 0.5 * (1. + sg) * weno_map_num(ga3, w3) / weno_map_den(ga3, w3) +
                    w3 * 0.5 * (1. - sg) * weno_map_num(ga1, w3) / weno_map_den(ga1, w3);
  const double swm = m1 + m2 + m3;
  const double x1 = m1 / swm, x2 = m2 / swm, x3 = m3 / swm;
  return nterm == 3 ? x1 * f1 + x2 * f2 + x3 * f3 : x1 * f1 + x2 * f2;
}

/* the stencil point s (-2..3) of face n | n + ninc along dir: the flat index
 * n + s ninc, as the reference forms it.  Near a block face it lands in the
 * block's spare slots (i = ni + 1 of the row before or of the same row,
 * j = nj + 1 of the plane before or of the same plane, k = nk + 1), which
 * no cell routine writes; at the first interior k face (k = 1) the point
 * k = -1 lies before the block, where the reference's flux work arrays are
 * read out of bounds (undefined), and this restatement takes the ghost plane
 * k = 0 there */
static int64_t weno_point(const blk_t *b, int dir, int64_t n, int k, int s) {
  if (dir == 2 && k + s < 0) return n - (int64_t)k * b->nijd;
  return n + s * NINC(b, dir);
}

/* the interior face n | n1 = n + ninc (sch_weno5_3d.f90:240-1252): Roe
 * average, left (Q) and right (P) eigenvectors, the x, y and z fluxes of the
 * six stencil points reconstructed field by field, back to the conserved
 * variables and projected on the face; fv the central viscous flux (times 2) */
static void weno5_face(const blk_t *b, int dir, int64_t n, int k, const double *v,
                       const double *ps, const double *tau, const double *sn, double df[5],
                       double fv[5]) {
  const int64_t L = G.ld, ninc = NINC(b, dir), n1 = n + ninc, m1 = n1 - b->npc;
  const double gam = G.gam, gam1 = G.gam1;
  const double s1 = SN(sn, b, m1, dir, 0), s2 = SN(sn, b, m1, dir, 1), s3 = SN(sn, b, m1, dir, 2);
  const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const double nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const double ul = v[L + n] / v[n], vl = v[2 * L + n] / v[n], wl = v[3 * L + n] / v[n];
  const double ur = v[L + n1] / v[n1], vr = v[2 * L + n1] / v[n1], wr = v[3 * L + n1] / v[n1];
  const double al = sqrt(gam * ps[n] / v[n]), ar = sqrt(gam * ps[n1] / v[n1]);
  const double hl = al * al / gam1 + 0.5 * (ul * ul + vl * vl + wl * wl);
  const double hr = ar * ar / gam1 + 0.5 * (ur * ur + vr * vr + wr * wr);
  const double gd = sqrt(v[n1] / v[n]), gd1 = 1. / (1. + gd), gd2 = gd * gd1;
  const double rhom = sqrt(v[n] * v[n1]), rhomi = 1. / rhom;
  const double um = gd1 * ul + gd2 * ur, vm = gd1 * vl + gd2 * vr, wm = gd1 * wl + gd2 * wr;
  const double hm = gd1 * hl + gd2 * hr;
  const double vitm2 = 0.5 * (um * um + vm * vm + wm * wm);
  const double am = sqrt(fabs(gam1 * (hm - vitm2)));
  const double am2i = 1. / (am * am);
  const double vn = um * nx + vm * ny + wm * nz;
  const double rhoiam = rhom / am, rhoami = am2i / rhoiam;
  const double lam[5] = {vn, vn, vn, vn + am, vn - am};
  const double Q[5][5] = {
      {(1. - gam1 * vitm2 * am2i) * nx - (vm * nz - wm * ny) * rhomi, gam1 * um * nx * am2i,
       gam1 * vm * nx * am2i + nz * rhomi, gam1 * wm * nx * am2i - ny * rhomi,
       -gam1 * nx * am2i},
      {(1. - gam1 * vitm2 * am2i) * ny - (wm * nx - um * nz) * rhomi,
       gam1 * um * ny * am2i - nz * rhomi, gam1 * vm * ny * am2i,
       gam1 * wm * ny * am2i + nx * rhomi, -gam1 * ny * am2i},
      {(1. - gam1 * vitm2 * am2i) * nz - (um * ny - vm * nx) * rhomi,
       gam1 * um * nz * am2i + ny * rhomi, gam1 * vm * nz * am2i - nx * rhomi,
       gam1 * wm * nz * am2i, -gam1 * nz * am2i},
      {gam1 * vitm2 * rhoami - vn * rhomi, nx * rhomi - gam1 * um * rhoami,
       ny * rhomi - gam1 * vm * rhoami, nz * rhomi - gam1 * wm * rhoami, gam1 * rhoami},
      {gam1 * vitm2 * rhoami + vn * rhomi, -nx * rhomi - gam1 * um * rhoami,
       -ny * rhomi - gam1 * vm * rhoami, -nz * rhomi - gam1 * wm * rhoami, gam1 * rhoami}};
  const double P[5][5] = {
      {nx, ny, nz, 0.5 * rhoiam, 0.5 * rhoiam},
      {um * nx, um * ny - rhom * nz, um * nz + rhom * ny, 0.5 * rhoiam * (um + nx * am),
       0.5 * rhoiam * (um - nx * am)},
      {vm * nx + rhom * nz, vm * ny, vm * nz - rhom * nx, 0.5 * rhoiam * (vm + ny * am),
       0.5 * rhoiam * (vm - ny * am)},
      {wm * nx - rhom * ny, wm * ny + rhom * nx, wm * nz, 0.5 * rhoiam * (wm + nz * am),
       0.5 * rhoiam * (wm - nz * am)},
      {vitm2 * nx + rhom * (vm * nz - wm * ny), vitm2 * ny + rhom * (wm * nx - um * nz),
       vitm2 * nz + rhom * (um * ny - vm * nx), 0.5 * rhoiam * (hm + am * vn),
       0.5 * rhoiam * (hm - am * vn)}};
  double fl[6][3][5];
  for (int p = 0; p < 6; ++p) weno_cell_flux(v, ps, weno_point(b, dir, n, k, p - 2), fl[p]);
  double out[3][5];
  for (int c = 0; c < 3; ++c) {
    /* three candidates in the x and y fluxes of the i direction, two
       elsewhere (sch_weno5_3d.f90:616, 911, 1206, 1639, 1934, 2229, 2662,
       2957, 3252); the flagged fix sums three everywhere */
    const int nterm = (G.weno_fix || (dir == 0 && c < 2)) ? 3 : 2;
    double fc[5];
    for (int kf = 0; kf < 5; ++kf) {
      double q[6];
      for (int p = 0; p < 6; ++p)
        q[p] = Q[kf][0] * fl[p][c][0] + Q[kf][1] * fl[p][c][1] + Q[kf][2] * fl[p][c][2] +
               Q[kf][3] * fl[p][c][3] + Q[kf][4] * fl[p][c][4];
      fc[kf] = weno_field(q, lam[kf], nterm);
    }
    for (int r = 0; r < 5; ++r)
      out[c][r] = fc[0] * P[r][0] + fc[1] * P[r][1] + fc[2] * P[r][2] + fc[3] * P[r][3] +
                  fc[4] * P[r][4];
  }
  for (int r = 0; r < 5; ++r) df[r] = out[0][r] * s1 + out[1][r] * s2 + out[2][r] * s3;
  const double *txx = tau, *txy = tau + L, *txz = tau + 2 * L, *tyy = tau + 3 * L,
               *tyz = tau + 4 * L, *tzz = tau + 5 * L, *qx = tau + 6 * L, *qy = tau + 7 * L,
               *qz = tau + 8 * L;
  fv[0] = 0.;
  fv[1] = (txx[n] + txx[n1]) * s1 + (txy[n] + txy[n1]) * s2 + (txz[n] + txz[n1]) * s3;
  fv[2] = (txy[n] + txy[n1]) * s1 + (tyy[n] + tyy[n1]) * s2 + (tyz[n] + tyz[n1]) * s3;
  fv[3] = (txz[n] + txz[n1]) * s1 + (tyz[n] + tyz[n1]) * s2 + (tzz[n] + tzz[n1]) * s3;
  fv[4] = (txx[n] * ul + txy[n] * vl + txz[n] * wl + qx[n] + txx[n1] * ur + txy[n1] * vr +
           txz[n1] * wr + qx[n1]) * s1 +
          (txy[n] * ul + tyy[n] * vl + tyz[n] * wl + qy[n] + txy[n1] * ur + tyy[n1] * vr +
           tyz[n1] * wr + qy[n1]) * s2 +
          (txz[n] * ul + tyz[n] * vl + tzz[n] * wl + qz[n] + txz[n1] * ur + tyz[n1] * vr +
           tzz[n1] * wr + qz[n1]) * s3;
}

/* sch_weno5_3d.f90:3302-3500: the flux through a boundary face from the
 * ghost cell g alone (convective minus viscous), face vector s */
static void weno5_boundary(int64_t g, const double *v, const double *ps, const double *tau,
                           double s1, double s2, double s3, double f[5]) {
  const int64_t L = G.ld;
  double fl[3][5];
  weno_cell_flux(v, ps, g, fl);
  const double fxx = fl[0][1], fxy = fl[0][2], fxz = fl[0][3], fex = fl[0][4];
  const double fyy = fl[1][2], fyz = fl[1][3], fey = fl[1][4], fzz = fl[2][3], fez = fl[2][4];
  const double txx = tau[g], txy = tau[L + g], txz = tau[2 * L + g], tyy = tau[3 * L + g],
               tyz = tau[4 * L + g], tzz = tau[5 * L + g], qx = tau[6 * L + g],
               qy = tau[7 * L + g], qz = tau[8 * L + g];
  const double v1 = v[g], v2 = v[L + g], v3 = v[2 * L + g], v4 = v[3 * L + g];
  f[0] = v2 * s1 + v3 * s2 + v4 * s3;
  f[1] = (fxx - txx) * s1 + (fxy - txy) * s2 + (fxz - txz) * s3;
  f[2] = (fxy - txy) * s1 + (fyy - tyy) * s2 + (fyz - tyz) * s3;
  f[3] = (fxz - txz) * s1 + (fyz - tyz) * s2 + (fzz - tzz) * s3;
  f[4] = (fex - (txx * v2 + txy * v3 + txz * v4) / v1 - qx) * s1 +
         (fey - (txy * v2 + tyy * v3 + tyz * v4) / v1 - qy) * s2 +
         (fez - (txz * v2 + tyz * v3 + tzz * v4) / v1 - qz) * s3;
}

/* sch_weno5_3d.f90:146-3500 (ityprk = 0): u zeroed over the block; the
 * interior faces of i (i = 1..ni-2), j, k in the reference's loop order, each
 * adding to its upper cell first (u - df + fv/2) then its lower one
 * (u + df - fv/2); then the boundary faces i1, i2, j1, j2, k1, k2 from their
 * ghost cells.  tau: the nine stress and heat-flux arrays (zero for Euler) */
void orc_set_weno_fix(int on) { G.weno_fix = on ? 1 : 0; }

void orc_sch_weno5_3d(int l, double *u, const double *v, const double *tau, const double *sn,
                      const double *ps) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  zero_u(b, u);
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    int hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
    hi[dir] -= 1;
    for (int k = 1; k <= hi[2]; ++k)
      for (int j = 1; j <= hi[1]; ++j)
        for (int i = 1; i <= hi[0]; ++i) {
          const int64_t n = IC(b, i, j, k), n1 = n + ninc;
          double df[5], fv[5];
          weno5_face(b, dir, n, k, v, ps, tau, sn, df, fv);
          u[n1] = u[n1] - df[0];
          for (int a = 1; a < 5; ++a) u[a * L + n1] = u[a * L + n1] - df[a] + 0.5 * fv[a];
          u[n] = u[n] + df[0];
          for (int a = 1; a < 5; ++a) u[a * L + n] = u[a * L + n] + df[a] - 0.5 * fv[a];
        }
  }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    const int nd = NDIR(b, dir);
    for (int side = 0; side < 2; ++side) {
      int lo[3] = {1, 1, 1}, hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
      lo[dir] = hi[dir] = side ? nd - 1 : 1;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            const int64_t n = IC(b, i, j, k), g = side ? n + ninc : n - ninc;
            const int64_t mf = (side ? n + ninc : n) - n0;
            double f[5];
            weno5_boundary(g, v, ps, tau, SN(sn, b, mf, dir, 0), SN(sn, b, mf, dir, 1),
                           SN(sn, b, mf, dir, 2), f);
            for (int a = 0; a < 5; ++a)
              u[a * L + n] = side ? u[a * L + n] + f[a] : u[a * L + n] - f[a];
          }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* viscous stresses                                                          */
/* ------------------------------------------------------------------------ */

/* zgrad2.f90:62-497 with unit weights (inivec.f90:110; metric3 only runs for
 * the weighted schemes, cpfw.f90:235) then zfluto.f90:38-57 */
static void zgrad2_zfluto(const blk_t *b, const double *s, const double *mu,
                          const double *mut, double *tau, const double *sn,
                          const double *vol, const double *temp) {
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  double *vx = calloc(nnn, sizeof(double)), *vy = calloc(nnn, sizeof(double)),
         *vz = calloc(nnn, sizeof(double));
  double *g = calloc((size_t)12 * nnn, sizeof(double)); /* dvxx..dvzz, dtx..dtz */
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 0; j <= b->nj; ++j)
      for (int i = 0; i <= b->ni; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        vx[m] = s[L + n] / s[n];
        vy[m] = s[2 * L + n] / s[n];
        vz[m] = s[3 * L + n] / s[n];
      }
  /* component order in g: xx,xy,xz,yx,yy,yz,zx,zy,zz,tx,ty,tz */
  const int order[3] = {2, 1, 0}; /* k faces, then j, then i */
  for (int oi = 0; oi < 3; ++oi) {
    const int dir = order[oi];
    const int64_t ninc = NINC(b, dir);
    const int nd = NDIR(b, dir);
    int lo[3], hi[3], idx[3];
    dir_ranges(b, dir, 2, nd - 1, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          double sv[3] = {SN(sn, b, m, dir, 0), SN(sn, b, m, dir, 1), SN(sn, b, m, dir, 2)};
          double fv[4] = {vx[m] + vx[m - ninc], vy[m] + vy[m - ninc],
                          vz[m] + vz[m - ninc], temp[n] + temp[n - ninc]};
          for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c) {
              double sk = fv[a] * sv[c];
              g[(3 * a + c) * nnn + m] = g[(3 * a + c) * nnn + m] - sk;
              g[(3 * a + c) * nnn + m - ninc] = g[(3 * a + c) * nnn + m - ninc] + sk;
            }
        }
    dir_ranges(b, dir, 1, 1, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          double fv[4] = {vx[m - ninc], vy[m - ninc], vz[m - ninc], temp[n - ninc]};
          for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c)
              g[(3 * a + c) * nnn + m] =
                  g[(3 * a + c) * nnn + m] - SN(sn, b, m, dir, c) * 2 * fv[a];
        }
    dir_ranges(b, dir, nd, nd, lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          double fv[4] = {vx[m], vy[m], vz[m], temp[n]};
          for (int a = 0; a < 4; ++a)
            for (int c = 0; c < 3; ++c)
              g[(3 * a + c) * nnn + m - ninc] =
                  g[(3 * a + c) * nnn + m - ninc] + SN(sn, b, m, dir, c) * 2 * fv[a];
        }
  }
  const double eps = 0.00001, ds3 = 2. / 3.;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        double ts = copysign(0.5, -vol[n]);
        double vols = (0.5 + ts) * eps + (0.5 - ts) * vol[n];
        double c0 = .5 / (vols + DBL_MIN);
        double gg[12];
        for (int a = 0; a < 12; ++a) gg[a] = g[a * nnn + m] * c0;
        const double dvxx = gg[0], dvxy = gg[1], dvxz = gg[2], dvyx = gg[3],
                     dvyy = gg[4], dvyz = gg[5], dvzx = gg[6], dvzy = gg[7],
                     dvzz = gg[8], dtx = gg[9], dty = gg[10], dtz = gg[11];
        double mm = mu[n] + mut[n];
        tau[n] = ds3 * (mu[n] + mut[n]) * (2 * dvxx - dvyy - dvzz);
        tau[3 * L + n] = ds3 * (mu[n] + mut[n]) * (2 * dvyy - dvxx - dvzz);
        tau[5 * L + n] = ds3 * (mu[n] + mut[n]) * (2 * dvzz - dvxx - dvyy);
        tau[L + n] = mm * (dvxy + dvyx);
        tau[2 * L + n] = mm * (dvxz + dvzx);
        tau[4 * L + n] = mm * (dvyz + dvzy);
        double kq = G.cp * (mu[n] / G.pr + mut[n] / G.prt);
        tau[6 * L + n] = kq * dtx;
        tau[7 * L + n] = kq * dty;
        tau[8 * L + n] = kq * dtz;
      }
  free(vx);
  free(vy);
  free(vz);
  free(g);
}

/* zvisqc.f90:134-205: gradients + stresses per block, then ghost values:
 * rbte.f90 (copy of the interior cell) on every non-coincident boundary and
 * rbtc.f90:30-100 (average with the rotated partner) on coincident ones */
void orc_zvisqc(const double *v, const double *mu, const double *mut,
                double *tau, const double *sn, const double *vol,
                const double *temp) {
  const int64_t L = G.ld;
  for (int l = 0; l < G.nblk; ++l)
    zgrad2_zfluto(&G.b[l], v, mu, mut, tau, sn, vol, temp);
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] == ORC_BC_RC) continue;
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ndm = G.ncin[mb];
      for (int a = 0; a < 9; ++a) tau[a * L + nd] = tau[a * L + ndm];
    }
  }
  double *buff = malloc(sizeof(double) * 9 * (size_t)(G.nlist > 0 ? G.nlist : 1));
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    const double sr = -G.bsin[bb], cr = G.bcos[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nc = G.ncin[mb];
      double *bf = &buff[9 * mb];
      const double txx = tau[nc], txy = tau[L + nc], txz = tau[2 * L + nc],
                   tyy = tau[3 * L + nc], tyz = tau[4 * L + nc], tzz = tau[5 * L + nc];
      bf[0] = txx;
      bf[1] = cr * txy - sr * txz;
      bf[2] = cr * txz + sr * txy;
      bf[3] = cr * cr * tyy - 2. * cr * sr * tyz + sr * sr * tzz;
      bf[4] = -cr * sr * (tzz - tyy) + (2. * cr * cr - 1.) * tyz;
      bf[5] = sr * sr * tyy + 2. * cr * sr * tyz + cr * cr * tzz;
      bf[6] = tau[6 * L + nc];
      bf[7] = cr * tau[7 * L + nc] - sr * tau[8 * L + nc];
      bf[8] = cr * tau[8 * L + nc] + sr * tau[7 * L + nc];
    }
  }
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_RC) continue;
    const int p = G.bpart[bb];
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ndm = G.ncin[mb];
      const double *bf = &buff[9 * (G.bmpb[p] + m)];
      for (int a = 0; a < 9; ++a) tau[a * L + nd] = 0.5 * (tau[a * L + ndm] + bf[a]);
    }
  }
  free(buff);
}

/* ------------------------------------------------------------------------ */
/* implicit phase                                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  double *coefe[3], *coefdiag, *d2w[5], *df[9], *rv;
} impl_work;

static void impl_alloc(const blk_t *b, impl_work *w) {
  for (int a = 0; a < 3; ++a) w->coefe[a] = calloc(b->nnn, sizeof(double));
  w->coefdiag = calloc(b->nnn, sizeof(double));
  for (int a = 0; a < 5; ++a) w->d2w[a] = calloc(b->nnn, sizeof(double));
  for (int a = 0; a < 9; ++a) w->df[a] = calloc(b->nnn, sizeof(double));
  w->rv = calloc(b->nnn, sizeof(double));
}
static void impl_free(impl_work *w) {
  for (int a = 0; a < 3; ++a) free(w->coefe[a]);
  free(w->coefdiag);
  for (int a = 0; a < 5; ++a) free(w->d2w[a]);
  for (int a = 0; a < 9; ++a) free(w->df[a]);
  free(w->rv);
}

/* df index: 0 xx, 1 xy, 2 xz, 3 ex, 4 yy, 5 yz, 6 ey, 7 zz, 8 ez */
enum { DXX = 0, DXY, DXZ, DEX, DYY, DYZ, DEY, DZZ, DEZ };

/* face loop of one Jacobi sub-iteration (implimf_eu.f90:269-313,
 * implimf_3d.f90:236-420); eu selects the implimf_eu form of tn */
static void jacobi_faces(const blk_t *b, int eu, const double *d,
                         const double *sn, impl_work *w) {
  const int64_t L = G.ld, n0 = b->npc;
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    int lo[3], hi[3], idx[3];
    dir_ranges(b, dir, 1, NDIR(b, dir), lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          const double sx = SN(sn, b, m, dir, 0), sy = SN(sn, b, m, dir, 1),
                       sz = SN(sn, b, m, dir, 2);
          double tn[5];
          double **df = w->df;
#define AV(arr, mm) ((arr)[mm] + (arr)[(mm) - ninc])
          if (eu) {
            tn[0] = 0.5 * ((d[L + n] + d[L + n - ninc]) * sx +
                           (d[2 * L + n] + d[2 * L + n - ninc]) * sy +
                           (d[3 * L + n] + d[3 * L + n - ninc]) * sz);
            tn[1] = 0.5 * (AV(df[DXX], m) * sx + AV(df[DXY], m) * sy + AV(df[DXZ], m) * sz);
            tn[2] = 0.5 * (AV(df[DXY], m) * sx + AV(df[DYY], m) * sy + AV(df[DYZ], m) * sz);
            tn[3] = 0.5 * (AV(df[DXZ], m) * sx + AV(df[DYZ], m) * sy + AV(df[DZZ], m) * sz);
            tn[4] = 0.5 * (AV(df[DEX], m) * sx + AV(df[DEY], m) * sy + AV(df[DEZ], m) * sz);
          } else {
            tn[0] = 0.5 * (d[L + n] + d[L + n - ninc]) * sx +
                    0.5 * (d[2 * L + n] + d[2 * L + n - ninc]) * sy +
                    0.5 * (d[3 * L + n] + d[3 * L + n - ninc]) * sz;
            tn[1] = 0.5 * AV(df[DXX], m) * sx + 0.5 * AV(df[DXY], m) * sy + 0.5 * AV(df[DXZ], m) * sz;
            tn[2] = 0.5 * AV(df[DXY], m) * sx + 0.5 * AV(df[DYY], m) * sy + 0.5 * AV(df[DYZ], m) * sz;
            tn[3] = 0.5 * AV(df[DXZ], m) * sx + 0.5 * AV(df[DYZ], m) * sy + 0.5 * AV(df[DZZ], m) * sz;
            tn[4] = 0.5 * AV(df[DEX], m) * sx + 0.5 * AV(df[DEY], m) * sy + 0.5 * AV(df[DEZ], m) * sz;
          }
#undef AV
          const double ce = w->coefe[dir][m], cep = w->coefe[dir][m + ninc];
          for (int a = 0; a < 5; ++a) {
            w->d2w[a][m] = w->d2w[a][m] + tn[a] + ce * d[a * L + n - ninc] +
                           cep * d[a * L + n + ninc];
            w->d2w[a][m - ninc] = w->d2w[a][m - ninc] - tn[a];
          }
        }
  }
}

/* implimf_eu.f90:79-330 (ityprk=0; kfmg=3 adds the physical time term) */
void orc_implimf_eu(int l, const double *u, const double *dt, double *v,
                    double *d, const double *sn, const double *vol,
                    const double *ps, const double *cson, int lmx) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  /* implimf_eu.f90:82-85: fact = 1.5/dt1min with dual time stepping */
  const double gam1 = G.gam1, pinfl = G.pinfl, fact = G.kfmg == 3 ? 1.5 / G.dt1min : 0.;
  impl_work w;
  impl_alloc(b, &w);
  for (int a = 0; a < 5; ++a)
    for (int64_t n = n0; n < n0 + b->nnn; ++n) d[a * L + n] = 0.;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        w.coefdiag[m] = vol[n] * (fact + 1. / dt[n]);
      }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    int lo[3], hi[3], idx[3];
    dir_ranges(b, dir, 1, NDIR(b, dir), lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          const double sx = SN(sn, b, m, dir, 0), sy = SN(sn, b, m, dir, 1),
                       sz = SN(sn, b, m, dir, 2);
          double cnds = sx * sx + sy * sy + sz * sz;
          double norm = 1. / v[n], norm1 = 1. / v[n - ninc];
          double uu = 0.5 * (v[L + n] * norm + v[L + n - ninc] * norm1);
          double vv = 0.5 * (v[2 * L + n] * norm + v[2 * L + n - ninc] * norm1);
          double ww = 0.5 * (v[3 * L + n] * norm + v[3 * L + n - ninc] * norm1);
          double cc = 0.5 * (cson[n] + cson[n - ninc]);
          w.coefe[dir][m] = 0.5 * (fabs(uu * sx + vv * sy + ww * sz)) + sqrt(cnds) * cc;
        }
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t m = ML(b, idx[0], idx[1], idx[2]);
          w.coefdiag[m] = w.coefdiag[m] + w.coefe[dir][m] + w.coefe[dir][m + ninc];
        }
  }
  for (int ls = 1; ls <= lmx; ++ls) {
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          for (int a = 0; a < 5; ++a) w.d2w[a][m] = -u[a * L + n];
        }
    jacobi_faces(b, 1, d, sn, &w);
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          for (int a = 0; a < 5; ++a) d[a * L + n] = w.d2w[a][m] / w.coefdiag[m];
          double wi1 = 1. / (v[n] + d[n]);
          double ui = v[L + n] + d[L + n];
          double vi = v[2 * L + n] + d[2 * L + n];
          double wi = v[3 * L + n] + d[3 * L + n];
          double wi5 = v[4 * L + n] + d[4 * L + n];
          double pres = gam1 * (wi5 - .5 * wi1 * (sq(ui) + sq(vi) + sq(wi)) - pinfl);
          double norm = 1. / v[n];
          const double v2 = v[L + n], v3 = v[2 * L + n], v4 = v[3 * L + n],
                       v5 = v[4 * L + n], p = ps[n];
          double fxx = v2 * (v2 * norm) + p;
          double fxy = v3 * (v2 * norm);
          double fxz = v4 * (v2 * norm);
          double fyy = v3 * (v3 * norm) + p;
          double fyz = v4 * (v3 * norm);
          double fzz = v4 * (v4 * norm) + p;
          double fex = (v5 + p - pinfl) * v2 * norm;
          double fey = (v5 + p - pinfl) * v3 * norm;
          double fez = (v5 + p - pinfl) * v4 * norm;
          w.df[DXX][m] = wi1 * sq(ui) + pres - fxx;
          w.df[DXY][m] = wi1 * ui * vi - fxy;
          w.df[DXZ][m] = wi1 * ui * wi - fxz;
          w.df[DEX][m] = wi1 * ui * (wi5 + pres - pinfl) - fex;
          w.df[DYY][m] = wi1 * sq(vi) + pres - fyy;
          w.df[DYZ][m] = wi1 * vi * wi - fyz;
          w.df[DEY][m] = wi1 * vi * (wi5 + pres - pinfl) - fey;
          w.df[DZZ][m] = wi1 * sq(wi) + pres - fzz;
          /* implimf_eu.f90:312: the *wi factor of the z energy flux is
           * missing in the reference and is reproduced here unless the
           * flagged non-reference option asks for it */
          w.df[DEZ][m] = G.qfix_dfez ? wi1 * wi * (wi5 + pres - pinfl) - fez
                                     : wi1 * (wi5 + pres - pinfl) - fez;
        }
  }
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        for (int a = 0; a < 5; ++a) v[a * L + n] = v[a * L + n] + d[a * L + n];
      }
  impl_free(&w);
}

/* implimf_3d.f90:64-490 (ityprk=0; kfmg=3 adds the physical time term) */
void orc_implimf_3d(int l, const double *u, const double *dt, double *v,
                    double *d, const double *mu, const double *mut,
                    const double *sn, const double *vol, const double *ps,
                    const double *cson, int lmx) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  const double gam = G.gam, gam1 = G.gam1, pinfl = G.pinfl;
  impl_work w;
  impl_alloc(b, &w);
  for (int a = 0; a < 5; ++a)
    for (int64_t n = n0; n < n0 + b->nnn; ++n) d[a * L + n] = 0.;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k), m = n - n0;
        w.rv[m] = gam * (mu[n] / G.pr + mut[n] / G.prt) / v[n];
        w.coefdiag[m] = vol[n] / dt[n];
      }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    int lo[3], hi[3], idx[3];
    dir_ranges(b, dir, 1, NDIR(b, dir), lo, hi);
    for (idx[2] = lo[2]; idx[2] <= hi[2]; ++idx[2])
      for (idx[1] = lo[1]; idx[1] <= hi[1]; ++idx[1])
        for (idx[0] = lo[0]; idx[0] <= hi[0]; ++idx[0]) {
          int64_t n = IC(b, idx[0], idx[1], idx[2]), m = n - n0;
          const double sx = SN(sn, b, m, dir, 0), sy = SN(sn, b, m, dir, 1),
                       sz = SN(sn, b, m, dir, 2);
          double cnds = sx * sx + sy * sy + sz * sz;
          double uu = 0.5 * (v[L + n] / v[n] + v[L + n - ninc] / v[n - ninc]);
          double vv = 0.5 * (v[2 * L + n] / v[n] + v[2 * L + n - ninc] / v[n - ninc]);
          double ww = 0.5 * (v[3 * L + n] / v[n] + v[3 * L + n - ninc] / v[n - ninc]);
          double vn = uu * sx + vv * sy + ww * sz;
          double cc = 0.5 * (cson[n] + cson[n - ninc]);
          w.coefe[dir][m] = 0.5 * (fabs(vn) + sqrt(cnds) * cc) +
                            (w.rv[m] + w.rv[m - ninc]) * cnds / (vol[n] + vol[n - ninc]);
        }
  }
  const int64_t nci = 1, ncj = b->nid, nck = b->nijd;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t m = ML(b, i, j, k);
        w.coefdiag[m] = w.coefdiag[m] + w.coefe[0][m] + w.coefe[0][m + nci] +
                        w.coefe[1][m] + w.coefe[1][m + ncj] + w.coefe[2][m] +
                        w.coefe[2][m + nck];
      }
  /* implimf_3d.f90:213-224: the physical time term of dual time stepping
   * (fact = 1.5, dtpas = dt1min) */
  if (G.kfmg == 3)
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          w.coefdiag[m] = w.coefdiag[m] + 1.5 * vol[n] / G.dt1min;
        }
  for (int ls = 1; ls <= lmx; ++ls) {
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          for (int a = 0; a < 5; ++a) w.d2w[a][m] = -u[a * L + n];
        }
    jacobi_faces(b, 0, d, sn, &w);
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k), m = n - n0;
          for (int a = 0; a < 5; ++a) d[a * L + n] = w.d2w[a][m] / w.coefdiag[m];
          double wi1 = v[n] + d[n];
          double wi2 = v[L + n] + d[L + n];
          double wi3 = v[2 * L + n] + d[2 * L + n];
          double wi4 = v[3 * L + n] + d[3 * L + n];
          double wi5 = v[4 * L + n] + d[4 * L + n];
          double ui = wi2 / wi1, vi = wi3 / wi1, wi = wi4 / wi1;
          double pres = gam1 * (wi5 - .5 * wi1 * (sq(ui) + sq(vi) + sq(wi)) - pinfl);
          const double v1 = v[n], v2 = v[L + n], v3 = v[2 * L + n], v4 = v[3 * L + n],
                       v5 = v[4 * L + n], p = ps[n];
          double fxx = v2 * (v2 / v1) + p;
          double fxy = v3 * (v2 / v1);
          double fxz = v4 * (v2 / v1);
          double fyy = v3 * (v3 / v1) + p;
          double fyz = v4 * (v3 / v1);
          double fzz = v4 * (v4 / v1) + p;
          double fex = (v5 + p - pinfl) * v2 / v1;
          double fey = (v5 + p - pinfl) * v3 / v1;
          double fez = (v5 + p - pinfl) * v4 / v1;
          w.df[DXX][m] = wi1 * sq(ui) + pres - fxx;
          w.df[DXY][m] = wi1 * ui * vi - fxy;
          w.df[DXZ][m] = wi1 * ui * wi - fxz;
          w.df[DEX][m] = ui * (wi5 + pres - pinfl) - fex;
          w.df[DYY][m] = wi1 * sq(vi) + pres - fyy;
          w.df[DYZ][m] = wi1 * vi * wi - fyz;
          w.df[DEY][m] = vi * (wi5 + pres - pinfl) - fey;
          w.df[DZZ][m] = wi1 * sq(wi) + pres - fzz;
          w.df[DEZ][m] = wi * (wi5 + pres - pinfl) - fez;
        }
  }
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        for (int a = 0; a < 5; ++a) v[a * L + n] = v[a * L + n] + d[a * L + n];
      }
  impl_free(&w);
}

/* ------------------------------------------------------------------------ */
/* residual norms                                                            */
/* ------------------------------------------------------------------------ */

/* residu.f90:89-241 per block, combined as in rscpsv.f90:79-150 */
void orc_rscpsv(const double *u0, const double *v, const double *dt,
                double *out) {
  const int64_t L = G.ld;
  double g1[5] = {0}, g2[5] = {0}, gmax[5] = {0};
  int64_t npts = 0;
  for (int l = 0; l < G.nblk; ++l) {
    const blk_t *b = &G.b[l];
    double d1[5] = {0}, d2[5] = {0}, dmax[5] = {0};
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          int64_t n = IC(b, i, j, k);
          for (int a = 0; a < 5; ++a) {
            double res = (v[a * L + n] - u0[a * L + n]) / dt[n];
            d1[a] = d1[a] + fabs(res);
            d2[a] = d2[a] + res * res;
            dmax[a] = fmax(dmax[a], fabs(res));
          }
        }
    const int64_t nmax = (int64_t)(b->ni - 1) * (b->nj - 1) * (b->nk - 1);
    const double coef = 1. / (double)nmax;
    for (int a = 0; a < 5; ++a) {
      d1[a] = coef * d1[a];
      d2[a] = sqrt(coef * d2[a]);
      g1[a] = g1[a] + (double)nmax * d1[a];
      g2[a] = g2[a] + (double)nmax * sq(d2[a]);
      gmax[a] = fmax(gmax[a], fabs(dmax[a]));
    }
    npts += nmax;
  }
  for (int a = 0; a < 5; ++a) {
    out[a] = g1[a] / (double)npts;
    out[5 + a] = sqrt(g2[a] / (double)npts);
    out[10 + a] = gmax[a];
  }
}

/* ------------------------------------------------------------------------ */
/* one iteration                                                             */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* turbulence transport terms on the mean-flow path                          */
/* ------------------------------------------------------------------------ */

/* the flat range indc(i1,j1,k1)..indc(i2m1,j2m1,k2m1) the fludc routines
 * sweep (ghost cells inside the range included) */
static void flat_real_range(const blk_t *b, int64_t *n0, int64_t *n1) {
  *n0 = IC(b, 1, 1, 1);
  *n1 = IC(b, b->ni - 1, b->nj - 1, b->nk - 1);
}

/* met_fludc.f90:72-85 (alfak, alfae: modeleturb) */
void orc_met_fludc(int l, const double *mu, const double *mut, double *fd5x, double *fd5y,
                   double *fd5z, double *fd6x, double *fd6y, double *fd6z, double alfak,
                   double alfae) {
  const blk_t *b = &G.b[l - 1];
  int64_t n0, n1;
  flat_real_range(b, &n0, &n1);
  for (int64_t n = n0; n <= n1; ++n) {
    fd5x[n] = (mu[n] + mut[n] / alfak) * fd5x[n];
    fd5y[n] = (mu[n] + mut[n] / alfak) * fd5y[n];
    fd5z[n] = (mu[n] + mut[n] / alfak) * fd5z[n];
  }
  for (int64_t n = n0; n <= n1; ++n) {
    fd6x[n] = (mu[n] + mut[n] / alfae) * fd6x[n];
    fd6y[n] = (mu[n] + mut[n] / alfae) * fd6y[n];
    fd6z[n] = (mu[n] + mut[n] / alfae) * fd6z[n];
  }
}

/* met_fludcsa.f90:92-104 (sigma: modeleturb); s is (ld, 7) */
void orc_met_fludcsa(int l, const double *s, const double *mu, double *fd5x, double *fd5y,
                     double *fd5z, double *fd6x, double *fd6y, double *fd6z, double sigma) {
  const blk_t *b = &G.b[l - 1];
  int64_t n0, n1;
  flat_real_range(b, &n0, &n1);
  const double sigma1 = 1. / sigma;
  for (int64_t n = n0; n <= n1; ++n) {
    const double smutot = sigma1 * (mu[n] + s[5 * G.ld + n]);
    fd5x[n] = smutot * fd5x[n];
    fd5y[n] = smutot * fd5y[n];
    fd5z[n] = smutot * fd5z[n];
    fd6x[n] = 0.;
    fd6y[n] = 0.;
    fd6z[n] = 0.;
  }
}

/* met_roe2o.f90:288-296: minmod-type limiter */
static double amimd(double a, double b) {
  const double s = copysign(1.0, a);
  return s * fmax(0., fmin(fabs(a), b * s));
}
static double fi1(double x, double y, double z) { return amimd(x, amimd(y, z)); }
/* met_roe2oh.f90:318-323: Harten's entropy-fixed |a| */
static double psi_h(double aa, double eps) {
  return 0.5 * (1. + copysign(1.0, fabs(aa) - eps)) * fabs(aa) +
         0.25 * (1. - copysign(1.0, fabs(aa) - eps)) * (aa * aa + eps * eps) / eps;
}

/* met_roe2o.f90:26-286 / met_roe2oh.f90 (harten): TVD Roe dissipation of the
 * two transport variables t(:,6:7) into d(:,6:7); directions k, j, i; every
 * face of a direction (boundary faces included) in one ascending loop, the
 * slope differences extended by one face past each end */
void orc_met_roe2o(int l, const double *t, double *d, const double *sn, int harten,
                   double epsroe) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  /* zero d(:,6:7) over i 0..ni, j 0..nj, k 0..nk (:53-62) */
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 0; j <= b->nj; ++j)
      for (int i = 0; i <= b->ni; ++i) {
        const int64_t n = IC(b, i, j, k);
        d[5 * L + n] = 0.;
        d[6 * L + n] = 0.;
      }
  double *del6 = calloc((size_t)b->nnn, sizeof(double));
  double *del7 = calloc((size_t)b->nnn, sizeof(double));
  static const int order[3] = {2, 1, 0};
  for (int o = 0; o < 3; ++o) {
    const int dir = order[o];
    const int64_t ninc = NINC(b, dir);
    const int nd = NDIR(b, dir);
    /* slope differences on the faces 1..nd (the i direction also fills the
     * j = nj row, unused), then the extension at faces 0 and nd+1 */
    int lo[3] = {1, 1, 1}, hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
    lo[dir] = 1;
    hi[dir] = nd;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int64_t n = IC(b, i, j, k), m = n - n0;
          del6[m] = t[5 * L + n] - t[5 * L + n - ninc];
          del7[m] = t[6 * L + n] - t[6 * L + n - ninc];
        }
    for (int side = 0; side < 2; ++side) {
      int lo2[3] = {1, 1, 1}, hi2[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
      lo2[dir] = hi2[dir] = side == 0 ? 0 : nd + 1;
      const int64_t is = side == 0 ? 1 : -1;
      for (int k = lo2[2]; k <= hi2[2]; ++k)
        for (int j = lo2[1]; j <= hi2[1]; ++j)
          for (int i = lo2[0]; i <= hi2[0]; ++i) {
            const int64_t m = IC(b, i, j, k) - n0;
            del6[m] = del6[m + is * ninc];
            del7[m] = del7[m + is * ninc];
          }
    }
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int64_t n = IC(b, i, j, k), m = n - n0, m1 = m - ninc, m2 = m + ninc,
                        n1 = n - ninc;
          const double rro = 2 * t[n], rro1 = 2 * t[n1];
          const double u = t[L + n] / rro + t[L + n1] / rro1;
          const double v = t[2 * L + n] / rro + t[2 * L + n1] / rro1;
          const double w = t[3 * L + n] / rro + t[3 * L + n1] / rro1;
          const double s1 = SN(sn, b, m, dir, 0), s2 = SN(sn, b, m, dir, 1),
                       s3 = SN(sn, b, m, dir, 2);
          double coef;
          if (harten) {
            const double etot = t[4 * L + n] / rro + t[4 * L + n1] / rro1;
            const double q2 = 0.5 * (u * u + v * v + w * w);
            const double c = sqrt(G.gam * G.gam1 * (etot - q2));
            const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
            const double rlam = (u * s1 + v * s2 + w * s3) / cnds;
            coef = 0.5 * psi_h(rlam, epsroe * c) * cnds;
          } else {
            const double rlam = u * s1 + v * s2 + w * s3;
            coef = 0.5 * fabs(rlam);
          }
          double dd = coef * (del6[m] - fi1(del6[m1], del6[m], del6[m2]));
          d[5 * L + n] = d[5 * L + n] - dd;
          d[5 * L + n1] = d[5 * L + n1] + dd;
          dd = coef * (del7[m] - fi1(del7[m1], del7[m], del7[m2]));
          d[6 * L + n] = d[6 * L + n] - dd;
          d[6 * L + n1] = d[6 * L + n1] + dd;
        }
  }
  free(del6);
  free(del7);
}

/* ------------------------------------------------------------------------ */
/* Spalart-Allmaras                                                          */
/* ------------------------------------------------------------------------ */

/* the model constants of atlecdon.f90:193-204 */
#define SA_CB1 0.1355
#define SA_SIGMA (2. / 3.)
#define SA_CB2 0.622
#define SA_KAPPA 0.41
#define SA_CV1 7.1
/* the modified vorticity of Allmaras, Johnson & Spalart (ICCFD7-1902, 2012,
 * eq. 12): the flagged non-reference source fix (orc_set_sa_fix) */
#define SA_CV2 0.7
#define SA_CV3 0.9
static int SA_FIX = 0;
void orc_set_sa_fix(int on) { SA_FIX = on ? 1 : 0; }

/* met_samut.f90:35-46: mut = v6 fv1 on the real cells (x**3 as x*x*x) */
void orc_met_samut(int l, const double *v, const double *mu, double *mut) {
  const blk_t *b = &G.b[l - 1];
  const double cv13 = SA_CV1 * SA_CV1 * SA_CV1;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        const double xkhi = v[5 * G.ld + n] / mu[n];
        const double xkhi3 = xkhi * xkhi * xkhi;
        const double fv1 = xkhi3 / (xkhi3 + cv13);
        mut[n] = v[5 * G.ld + n] * fv1;
      }
}

/* sch_turb.f90:4-290 (3-D, no wall law): centred fluxes of the transport
 * variables, v(:,6:7) (q - (fd5, fd6)), summed per cell like sch_jameson,
 * then u6 = 0.5 u6 - vol ts6 - d6 (and 7) */
void orc_sch_turb(int l, double *u, const double *v, const double *d, const double *fd5x,
                  const double *fd5y, const double *fd5z, const double *fd6x,
                  const double *fd6y, const double *fd6z, const double *ts6,
                  const double *ts7, const double *sn, const double *vol) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc;
  for (int64_t n = n0; n < n0 + b->nnn; ++n) {
    u[5 * L + n] = 0.;
    u[6 * L + n] = 0.;
  }
  double *f = malloc(sizeof(double) * 6 * (size_t)b->nnn);
  for (int64_t m = 0; m < b->nnn; ++m) {
    const int64_t n = n0 + m;
    if (v[n] == 0.) { /* cells never set (outside the flat range) */
      for (int q = 0; q < 6; ++q) f[6 * m + q] = 0.;
      continue;
    }
    f[6 * m + 0] = v[5 * L + n] * (v[L + n] / v[n]) - fd5x[n];
    f[6 * m + 1] = v[5 * L + n] * (v[2 * L + n] / v[n]) - fd5y[n];
    f[6 * m + 2] = v[5 * L + n] * (v[3 * L + n] / v[n]) - fd5z[n];
    f[6 * m + 3] = v[6 * L + n] * (v[L + n] / v[n]) - fd6x[n];
    f[6 * m + 4] = v[6 * L + n] * (v[2 * L + n] / v[n]) - fd6y[n];
    f[6 * m + 5] = v[6 * L + n] * (v[3 * L + n] / v[n]) - fd6z[n];
  }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    const int nd = NDIR(b, dir);
    int lo[3], hi[3];
    for (int pass = 0; pass < 3; ++pass) {
      lo[0] = 1; hi[0] = b->ni - 1; lo[1] = 1; hi[1] = b->nj - 1; lo[2] = 1; hi[2] = b->nk - 1;
      if (pass == 0) { lo[dir] = 2; hi[dir] = nd - 1; }
      else lo[dir] = hi[dir] = pass == 1 ? 1 : nd;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            const int64_t n = IC(b, i, j, k), m = n - n0;
            const double s1 = SN(sn, b, m, dir, 0), s2 = SN(sn, b, m, dir, 1),
                         s3 = SN(sn, b, m, dir, 2);
            double F[6];
            if (pass == 0) {
              for (int q = 0; q < 6; ++q) F[q] = f[6 * m + q] + f[6 * (m - ninc) + q];
            } else {
              const int64_t cg = (pass == 1 ? m - ninc : m);
              for (int q = 0; q < 6; ++q) F[q] = 2 * f[6 * cg + q];
            }
            const double si6 = F[0] * s1 + F[1] * s2 + F[2] * s3;
            const double si7 = F[3] * s1 + F[4] * s2 + F[5] * s3;
            if (pass != 2) {
              u[5 * L + n] = u[5 * L + n] - si6;
              u[6 * L + n] = u[6 * L + n] - si7;
            }
            if (pass != 1) {
              u[5 * L + n - ninc] = u[5 * L + n - ninc] + si6;
              u[6 * L + n - ninc] = u[6 * L + n - ninc] + si7;
            }
          }
    }
  }
  free(f);
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        u[5 * L + n] = 0.5 * u[5 * L + n] - vol[n] * ts6[n] - d[5 * L + n];
        u[6 * L + n] = 0.5 * u[6 * L + n] - vol[n] * ts7[n] - d[6 * L + n];
      }
}

/* x**6 as gcc expands an integer power: x3 = (x*x)*x, x6 = x3*x3 */
static inline double pow6(double x) {
  const double x3 = x * x * x;
  return x3 * x3;
}

/* teq_grads.f90:4-374 (unit weights, the two branches coincide): Green-Gauss
 * gradient of the cell field s (block-local index m) over the directions k,
 * j, i -- interior faces (the lower one subtracted in a first sweep of each
 * row, the upper one added in a second), then the lower and the upper
 * boundary faces with twice the ghost value -- times 0.5 / vol on the flat
 * range of the real cells */
static void teq_grads(const blk_t *b, const double *sn, const double *vol, const double *s,
                      double *dsdx, double *dsdy, double *dsdz) {
  const int64_t n0 = b->npc;
  for (int64_t m = 0; m < b->nnn; ++m) dsdx[m] = dsdy[m] = dsdz[m] = 0.;
  static const int order[3] = {2, 1, 0};
  double *g[3] = {dsdx, dsdy, dsdz};
  for (int o = 0; o < 3; ++o) {
    const int dir = order[o];
    const int64_t ninc = NINC(b, dir);
    const int nd = NDIR(b, dir);
    int lo[3] = {1, 1, 1}, hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
    lo[dir] = 2;
    hi[dir] = nd - 1;
    /* the subtracting and the adding sweeps touch different cells of a
     * face, so running them face by face gives every cell the same order */
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int64_t m = IC(b, i, j, k) - n0;
          for (int c = 0; c < 3; ++c) g[c][m] = g[c][m] - SN(sn, b, m, dir, c) * (s[m] + s[m - ninc]);
        }
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int64_t m = IC(b, i, j, k) - n0;
          for (int c = 0; c < 3; ++c)
            g[c][m - ninc] = g[c][m - ninc] + SN(sn, b, m, dir, c) * (s[m] + s[m - ninc]);
        }
    for (int side = 0; side < 2; ++side) {
      int lo2[3] = {1, 1, 1}, hi2[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
      lo2[dir] = hi2[dir] = side == 0 ? 1 : nd;
      for (int k = lo2[2]; k <= hi2[2]; ++k)
        for (int j = lo2[1]; j <= hi2[1]; ++j)
          for (int i = lo2[0]; i <= hi2[0]; ++i) {
            const int64_t m = IC(b, i, j, k) - n0;
            for (int c = 0; c < 3; ++c) {
              if (side == 0)
                g[c][m] = g[c][m] - SN(sn, b, m, dir, c) * 2 * s[m - ninc];
              else
                g[c][m - ninc] = g[c][m - ninc] + SN(sn, b, m, dir, c) * 2 * s[m];
            }
          }
    }
  }
  const int64_t n1 = IC(b, 1, 1, 1), n2 = IC(b, b->ni - 1, b->nj - 1, b->nk - 1);
  for (int64_t n = n1; n <= n2; ++n) {
    const int64_t m = n - n0;
    const double ts = copysign(0.5, -vol[n]);
    const double vols = (0.5 + ts) * 0.000001 + (0.5 - ts) * vol[n];
    const double c0 = 0.5 / (vols + DBL_MIN);
    dsdx[m] = dsdx[m] * c0;
    dsdy[m] = dsdy[m] * c0;
    dsdz[m] = dsdz[m] * c0;
  }
}

/* teq_gradv.f90:4-170: gradients of u, v, w (v is (ld, 7); the density
 * floor of 1e-20 is applied to the values read, not written back).  dv:
 * [9][nnn] block-local, order xx xy xz yx yy yz zx zy zz */
void orc_teq_gradv(int l, const double *sn, const double *vol, const double *v, double *dv) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  double *s = calloc((size_t)nnn, sizeof(double));
  for (int c = 0; c < 3; ++c) {
    for (int k = 0; k <= b->nk; ++k)
      for (int j = 0; j <= b->nj; ++j)
        for (int i = 0; i <= b->ni; ++i) {
          const int64_t n = IC(b, i, j, k);
          s[n - n0] = v[(c + 1) * L + n] / fmax(v[n], 1.e-20);
        }
    teq_grads(b, sn, vol, s, dv + (3 * c) * nnn, dv + (3 * c + 1) * nnn, dv + (3 * c + 2) * nnn);
  }
  free(s);
}

/* met_smsa.f90:4-186 with met_difsa.f90:4-104: the Spalart-Allmaras source
 * ts6 (qcxts5), ts7 = 0 (qcyts6) and the source-derivative bound cfke on the
 * real cells.  v is (ld, 7); dv from orc_teq_gradv (block-local); fd5x..z the
 * diffusion densities (txxf5x..); dist the wall distance */
void orc_met_smsa(int l, const double *sn, const double *vol, const double *v,
                  const double *mu, const double *dist, const double *dv,
                  const double *fd5x, const double *fd5y, const double *fd5z, double *ts6,
                  double *ts7, double *cfke) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  const double cb1 = SA_CB1, sigma = SA_SIGMA, cb2 = SA_CB2, kappa = SA_KAPPA, cv1 = SA_CV1;
  const double cw1 = cb1 / (kappa * kappa) + (1 + cb2) / sigma;
  const double cw2 = 0.3, cw3 = 2., ct3 = 1.1, ct4 = 2.;
  double *t = calloc((size_t)nnn, sizeof(double));
  double *dx = calloc((size_t)nnn, sizeof(double)), *dy = calloc((size_t)nnn, sizeof(double)),
         *dz = calloc((size_t)nnn, sizeof(double)), *sdif = calloc((size_t)nnn, sizeof(double));
  /* met_difsa: gradient of rho nu~, sdif = grad . fd5 * cb2 / sigma */
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 0; j <= b->nj; ++j)
      for (int i = 0; i <= b->ni; ++i) {
        const int64_t n = IC(b, i, j, k);
        t[n - n0] = v[5 * L + n];
      }
  teq_grads(b, sn, vol, t, dx, dy, dz);
  const int64_t n1 = IC(b, 1, 1, 1), n2 = IC(b, b->ni - 1, b->nj - 1, b->nk - 1);
  for (int64_t n = n1; n <= n2; ++n) {
    const int64_t m = n - n0;
    sdif[m] = dx[m] * fd5x[n] + dy[m] * fd5y[n] + dz[m] * fd5z[n];
    sdif[m] = sdif[m] * cb2 / sigma;
  }
  /* gradient of the density */
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 0; j <= b->nj; ++j)
      for (int i = 0; i <= b->ni; ++i) {
        const int64_t n = IC(b, i, j, k);
        t[n - n0] = v[n];
      }
  teq_grads(b, sn, vol, t, dx, dy, dz);
  const double kappa2 = kappa * kappa, uns6 = 1. / 6., cv13 = cv1 * cv1 * cv1;
  const double cw36 = pow6(cw3), cv133 = 3. * cv13, ct42 = 2. * ct4, cb2sig = cb2 / sigma;
  const double *dvxx = dv, *dvxy = dv + nnn, *dvxz = dv + 2 * nnn, *dvyx = dv + 3 * nnn,
               *dvyy = dv + 4 * nnn, *dvyz = dv + 5 * nnn, *dvzx = dv + 6 * nnn,
               *dvzy = dv + 7 * nnn, *dvzz = dv + 8 * nnn;
  (void)dvxx;
  (void)dvyy;
  (void)dvzz;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        const double v6 = v[5 * L + n], v1 = v[n];
        const double vort = sqrt(sq(dvzy[m] - dvyz[m]) + sq(dvxz[m] - dvzx[m]) +
                                 sq(dvyx[m] - dvxy[m]));
        const double xkhi = v6 / mu[n];
        const double xkhi2 = xkhi * xkhi;
        const double xkhi3 = xkhi2 * xkhi;
        const double dist2 = dist[n] * dist[n];
        const double nutilde = v6 / v1;
        const double kapd2 = kappa2 * dist2;
        const double fv1 = xkhi3 / (xkhi3 + cv13);
        const double fv2 = 1. - (xkhi / (1 + xkhi * fv1));
        const double sbar = nutilde * fv2 / kapd2;
        double stilde, rtilde;
        if (!SA_FIX || sbar >= -SA_CV2 * vort)
          stilde = vort + sbar;
        else
          stilde = vort + vort * (SA_CV2 * SA_CV2 * vort + SA_CV3 * sbar) /
                              ((SA_CV3 - 2. * SA_CV2) * vort - sbar);
        if (SA_FIX && !(stilde > 0.)) {
          rtilde = 1.;
        } else {
          rtilde = nutilde / (stilde * kapd2);
          rtilde = fmin(rtilde, 1.);
        }
        const double rtil6 = pow6(rtilde);
        const double ft2 = ct3 * cns_exp(-ct4 * xkhi2);
        const double sm1 = cb1 * (1. - ft2) * stilde * v6;
        const double xg = rtilde + cw2 * (rtil6 - rtilde);
        const double xg6 = pow6(xg);
        const double fw = xg * cns_pow((1. + cw36) / (xg6 + cw36), uns6);
        const double sm2 = -(cw1 * fw - cb1 * ft2 / kappa2) * v6 * nutilde / dist2;
        ts6[n] = sm1 + sm2 + sdif[m];
        ts7[n] = 0.;
        const double xkhi4 = xkhi3 * xkhi;
        const double dfv1 =
            (SA_FIX && !(xkhi4 > 0.)) ? 0. : cv133 * sq(fv1) / (mu[n] * xkhi4);
        const double dfv2 = (xkhi2 * dfv1 - 1. / mu[n]) / sq(1. + xkhi * fv1);
        const double dst = (fv2 / v1 + nutilde * dfv2) / kapd2;
        double dpr, dxg, dfw;
        if (!SA_FIX) {
          dpr = (1. / v1 - nutilde * dst / stilde) / (stilde * kapd2);
          dxg = dpr * (1. + cw2 * (6. * rtil6 / rtilde - 1.));
          dfw = (1. - xg6 / (xg6 + cw36)) * fw * dxg / xg;
        } else {
          /* r constant where clipped; r^5 without r^6 / r; no division by
           * xg = 0 */
          dpr = (rtilde < 1. && stilde > 0.)
                    ? (1. / v1 - nutilde * dst / stilde) / (stilde * kapd2) : 0.;
          const double r2 = rtilde * rtilde;
          dxg = dpr * (1. + cw2 * (6. * (r2 * r2 * rtilde) - 1.));
          dfw = xg != 0. ? (1. - xg6 / (xg6 + cw36)) * fw * dxg / xg : 0.;
        }
        const double dft2 = -ct42 * xkhi * ft2;
        const double dsm1 = cb1 * ((1. - ft2) * (stilde + dst * v6) - stilde * v6 * dft2);
        const double dsm2 = 2. * sm2 / v6 - (cw1 * dfw - cb1 * dft2 / kappa2) * nutilde * v6 / dist2;
        /* met_smsa.f90:177 reads txxf5x.. at the block-local index m (the
         * global cell for block 1 only); reproduced */
        const double dsdif = -cb2sig * (fd5x[m] * dx[m] + fd5y[m] * dy[m] + fd5z[m] * dz[m]) / sq(v1);
        cfke[n] = fabs(dsm1 + dsm2 + dsdif);
      }
  free(t);
  free(dx);
  free(dy);
  free(dz);
  free(sdif);
}

/* impli2_eqt_3d.f90:4-330 (no wall law): implicit phase of the two
 * transport equations -- coefficients, then for the directions i, j, k two
 * alternating-line sweeps each (a tridiagonal solve along every line of the
 * direction, the other directions' neighbours taken from the previous
 * iterate), then v(:,6:7) += dw on the real cells.  cmt: the model's
 * diffusion constant (1 for 1SA) */
void orc_impli2_eqt_3d(int l, const double *u, const double *dt, double *v, const double *mu,
                       const double *mut, const double *cfke, const double *sn,
                       const double *vol, double cmt) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  const int64_t nci = 1, ncj = b->nid, nck = b->nijd;
  double *dw6 = calloc(nnn, sizeof(double)), *dw7 = calloc(nnn, sizeof(double));
  double *ce = calloc(3 * nnn, sizeof(double)), *rv = calloc(nnn, sizeof(double));
  double *uf = calloc(3 * nnn, sizeof(double)), *cd = calloc(nnn, sizeof(double));
  double *al = calloc(nnn, sizeof(double)), *b6 = calloc(nnn, sizeof(double)),
         *b7 = calloc(nnn, sizeof(double));
  double *o6 = calloc(nnn, sizeof(double)), *o7 = calloc(nnn, sizeof(double));
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        rv[m] = (mu[n] + mut[n] / cmt) / v[n];
        cd[m] = vol[n] / dt[n] + cfke[n] * vol[n];
      }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    int lo[3] = {1, 1, 1}, hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
    hi[dir] = NDIR(b, dir);
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int64_t n = IC(b, i, j, k), m = n - n0;
          const double s1 = SN(sn, b, m, dir, 0), s2 = SN(sn, b, m, dir, 1),
                       s3 = SN(sn, b, m, dir, 2);
          const double cnds = s1 * s1 + s2 * s2 + s3 * s3;
          const double uu = 0.5 * (v[L + n] / v[n] + v[L + n - ninc] / v[n - ninc]);
          const double vv = 0.5 * (v[2 * L + n] / v[n] + v[2 * L + n - ninc] / v[n - ninc]);
          const double ww = 0.5 * (v[3 * L + n] / v[n] + v[3 * L + n - ninc] / v[n - ninc]);
          uf[dir * nnn + m] = 0.5 * (uu * s1 + vv * s2 + ww * s3);
          ce[dir * nnn + m] = fabs(uf[dir * nnn + m]) +
                              (rv[m] + rv[m - ninc]) * cnds / (vol[n] + vol[n - ninc]);
        }
  }
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t m = IC(b, i, j, k) - n0;
        cd[m] = cd[m] + ce[m] + ce[m + nci] + ce[nnn + m] + ce[nnn + m + ncj] + ce[2 * nnn + m] +
                ce[2 * nnn + m + nck];
      }
  for (int dir = 0; dir < 3; ++dir) {
    const int64_t ninc = NINC(b, dir);
    const int d1 = (dir + 1) % 3, d2 = (dir + 2) % 3;
    /* the two other directions in the reference's order (i: j, k; j: i, k;
     * k: i, j) */
    const int oa = d1 < d2 ? d1 : d2, ob = d1 < d2 ? d2 : d1;
    const int64_t inca = NINC(b, oa), incb = NINC(b, ob);
    const double *ua = uf + oa * nnn, *ub = uf + ob * nnn, *ud = uf + dir * nnn;
    const double *ca = ce + oa * nnn, *cb = ce + ob * nnn, *cdir = ce + dir * nnn;
    for (int64_t m = 0; m < nnn; ++m) al[m] = b6[m] = b7[m] = 0.;
    for (int sw = 0; sw < 2; ++sw) {
      /* backward recurrence on every line, from the previous iterate */
      int lo[3] = {1, 1, 1}, hi[3] = {b->ni - 1, b->nj - 1, b->nk - 1};
      const int nd = NDIR(b, dir);
      for (int p = nd - 1; p >= 1; --p) {
        lo[dir] = hi[dir] = p;
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
              const int64_t n = IC(b, i, j, k), m = n - n0;
              const double td = -ua[m + inca] + ua[m] - ub[m + incb] + ub[m];
              const double tpa = ca[m + inca] - ua[m + inca], tma = ca[m] + ua[m];
              const double tpb = cb[m + incb] - ub[m + incb], tmb = cb[m] + ub[m];
              const double di6 = -u[5 * L + n] + td * dw6[m] + tma * dw6[m - inca] +
                                 tpa * dw6[m + inca] + tmb * dw6[m - incb] + tpb * dw6[m + incb];
              const double di7 = -u[6 * L + n] + td * dw7[m] + tma * dw7[m - inca] +
                                 tpa * dw7[m + inca] + tmb * dw7[m - incb] + tpb * dw7[m + incb];
              const double ai = cdir[m] + ud[m];
              const double bi = cd[m] + ud[m + ninc] - ud[m];
              const double cci = -cdir[m + ninc] + ud[m + ninc];
              al[m] = ai / (bi + cci * al[m + ninc]);
              b6[m] = (di6 - cci * b6[m + ninc]) / (bi + cci * al[m + ninc]);
              b7[m] = (di7 - cci * b7[m + ninc]) / (bi + cci * al[m + ninc]);
            }
      }
      /* forward substitution */
      memcpy(o6, dw6, nnn * sizeof(double));
      memcpy(o7, dw7, nnn * sizeof(double));
      for (int p = 1; p <= nd - 1; ++p) {
        lo[dir] = hi[dir] = p;
        for (int k = lo[2]; k <= hi[2]; ++k)
          for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
              const int64_t m = IC(b, i, j, k) - n0;
              dw6[m] = al[m] * dw6[m - ninc] + b6[m];
              dw7[m] = al[m] * dw7[m - ninc] + b7[m];
            }
      }
    }
  }
  /* impli2_eqt_3d.f90:384-405 (lparoi 1): no increment in the first cell
   * of the block's wall-law walls */
  for (int bb = 0; bb < G.nbnd; ++bb)
    if (G.btype[bb] == ORC_BC_LP2 && G.bblk[bb] == l)
      for (int m = 0; m < G.bmmb[bb]; ++m) {
        const int64_t ni = G.ncin[G.bmpb[bb] + m] - n0;
        dw6[ni] = 0.;
        dw7[ni] = 0.;
      }
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        v[5 * L + n] = v[5 * L + n] + dw6[m];
        v[6 * L + n] = v[6 * L + n] + dw7[m];
      }
  free(dw6); free(dw7); free(ce); free(rv); free(uf); free(cd); free(al); free(b6); free(b7);
  free(o6); free(o7);
}

/* ------------------------------------------------------------------------ */
/* Spalart-Allmaras transport step (met_num.f90 for equat '1SA ': kcutke 2,  */
/* kfludis 2, ksecmb 2, kcmut 2, kditur 2, klroe 2, kparoi 0)                */
/* ------------------------------------------------------------------------ */

/* the wall boundaries: cl 'pa..' (adiabatic wall) and 'lp..' (wall-law
 * wall) -- atcaldis3.f90:171 */
static int is_wall(int bb) { return G.btype[bb] == ORC_BC_PARA || G.btype[bb] == ORC_BC_LP2; }

/* atindnor.f90 + atccfp.f90:56-72: node increments of a wall facet (dm1,
 * dm2 span the face, ndm3 moves from the interior cell's lower node to the
 * face for the upper faces i2, j2, k2) */
static void facet_incs(const blk_t *b, int face, int64_t *dm1, int64_t *dm2, int64_t *ndm3) {
  const int dir = face / 2, upper = face % 2;
  if (dir == 0) { *dm1 = b->nid; *dm2 = b->nijd; }
  else if (dir == 1) { *dm1 = 1; *dm2 = b->nijd; }
  else { *dm1 = 1; *dm2 = b->nid; }
  *ndm3 = upper ? NINC(b, dir) : 0;
}

/* atcaldis3.f90 with the default attachment of every block to every wall
 * (at_lecopt: idefaut = 1, igr = jgr = kgr = 1 -> atdist_3.f90:34-58): the
 * distance from each real cell centre (atccc.f90:36-60) to the nearest wall
 * facet centre (atccfp.f90:60-72), brute force over the facets in boundary
 * list order; dist = sqrt(min d^2) on the real cells */
int orc_atcaldis3(const double *x, const double *y, const double *z, double *dist) {
  int64_t nw = 0;
  for (int bb = 0; bb < G.nbnd; ++bb)
    if (is_wall(bb)) nw += G.bmmb[bb];
  if (nw == 0) return 1;
  double *xp = malloc(sizeof(double) * nw), *yp = malloc(sizeof(double) * nw),
         *zp = malloc(sizeof(double) * nw);
  int64_t q = 0;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (!is_wall(bb)) continue;
    const blk_t *b = &G.b[G.bblk[bb] - 1];
    int64_t dm1, dm2, ndm3;
    facet_incs(b, G.bface[bb], &dm1, &dm2, &ndm3);
    for (int m = 0; m < G.bmmb[bb]; ++m, ++q) {
      const int64_t nci = G.ncin[G.bmpb[bb] + m] + ndm3;
      xp[q] = (x[nci] + x[nci + dm1] + x[nci + dm2] + x[nci + dm1 + dm2]) * .25;
      yp[q] = (y[nci] + y[nci + dm1] + y[nci + dm2] + y[nci + dm1 + dm2]) * .25;
      zp[q] = (z[nci] + z[nci + dm1] + z[nci + dm2] + z[nci + dm1 + dm2]) * .25;
    }
  }
  for (int l = 1; l <= G.nblk; ++l) {
    const blk_t *b = &G.b[l - 1];
    const int64_t a = 1, bj = b->nid, ck = b->nijd;
#pragma omp parallel for schedule(static)
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          const int64_t n = IC(b, i, j, k), n1 = n + ck;
          const double xcc = ((x[n] + x[n + a] + x[n + bj] + x[n + a + bj]) +
                              (x[n1] + x[n1 + a] + x[n1 + bj] + x[n1 + a + bj])) * 0.125;
          const double ycc = ((y[n] + y[n + a] + y[n + bj] + y[n + a + bj]) +
                              (y[n1] + y[n1 + a] + y[n1 + bj] + y[n1 + a + bj])) * 0.125;
          const double zcc = ((z[n] + z[n + a] + z[n + bj] + z[n + a + bj]) +
                              (z[n1] + z[n1 + a] + z[n1 + bj] + z[n1 + a + bj])) * 0.125;
          double dmini = 1.e+20;
          for (int64_t f = 0; f < nw; ++f) {
            const double d2 = (xcc - xp[f]) * (xcc - xp[f]) + (ycc - yp[f]) * (ycc - yp[f]) +
                              (zcc - zp[f]) * (zcc - zp[f]);
            if (d2 < dmini) dmini = d2;
          }
          dist[n] = sqrt(dmini);
        }
  }
  free(xp); free(yp); free(zp);
  return 0;
}

/* met_bord.f90:24-258 with kparoi = 0 (met_rbvc before and after: every
 * ghost depends on interior cells only, so one pass gives the same values):
 * coincident ghosts = average with the partner's interior cell
 * (met_rbvc.f90:53-62), idd = (rokinf, roeinf), para = 0, extr / prd =
 * the interior cell (met_rbve) */
void orc_met_bord(double *v, double rokinf, double roeinf) {
  const int64_t L = G.ld;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      const int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ni = G.ncin[mb];
      switch (G.btype[bb]) {
        case ORC_BC_RC: {
          const int64_t nc = G.ncin[G.bmpb[G.bpart[bb]] + m];
          v[5 * L + nd] = 0.5 * (v[5 * L + ni] + v[5 * L + nc]);
          v[6 * L + nd] = 0.5 * (v[6 * L + ni] + v[6 * L + nc]);
          break;
        }
        case ORC_BC_IDD:
          v[5 * L + nd] = rokinf;
          v[6 * L + nd] = roeinf;
          break;
        case ORC_BC_PARA:
        case ORC_BC_LP2: /* met_bord.f90:296-305, kparoi = 0 */
          v[5 * L + nd] = 0.;
          v[6 * L + nd] = 0.;
          break;
        default:
          v[5 * L + nd] = v[5 * L + ni];
          v[6 * L + nd] = v[6 * L + ni];
          break;
      }
    }
  }
}

/* met_gradtr.f90:48-130: fd5 = grad(s6 / s1), fd6 = grad(s7 / s1) by
 * teq_grads over the flat range of the real cells (ghost cells inside the
 * range receive the zero teq_grads leaves there) */
void orc_met_gradtr(int l, const double *sn, const double *vol, const double *s, double *fd5x,
                    double *fd5y, double *fd5z, double *fd6x, double *fd6y, double *fd6z) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  double *tt = calloc((size_t)nnn, sizeof(double));
  double *g = calloc((size_t)(3 * nnn), sizeof(double));
  double *out[2][3] = {{fd5x, fd5y, fd5z}, {fd6x, fd6y, fd6z}};
  int64_t n1, n2;
  flat_real_range(b, &n1, &n2);
  for (int q = 0; q < 2; ++q) {
    for (int k = 0; k <= b->nk; ++k)
      for (int j = 0; j <= b->nj; ++j)
        for (int i = 0; i <= b->ni; ++i) {
          const int64_t n = IC(b, i, j, k);
          tt[n - n0] = s[(5 + q) * L + n] / s[n];
        }
    teq_grads(b, sn, vol, tt, g, g + nnn, g + 2 * nnn);
    for (int64_t n = n1; n <= n2; ++n)
      for (int c = 0; c < 3; ++c) out[q][c][n] = g[c * nnn + n - n0];
  }
  free(tt); free(g);
}

/* met_rbse.f90:19-31 (every non-coincident boundary: ghost = interior) and
 * met_rbsc.f90:38-70 (coincident: average with the partner's interior
 * cell) on the six diffusion densities */
void orc_met_rbse(double *fd5x, double *fd5y, double *fd5z, double *fd6x, double *fd6y,
                  double *fd6z) {
  double *f[6] = {fd5x, fd5y, fd5z, fd6x, fd6y, fd6z};
  for (int bb = 0; bb < G.nbnd; ++bb)
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      const int64_t mb = G.bmpb[bb] + m, nd = G.ncbd[mb], ndm = G.ncin[mb];
      if (G.btype[bb] == ORC_BC_RC) {
        const int64_t nc = G.ncin[G.bmpb[G.bpart[bb]] + m];
        for (int q = 0; q < 6; ++q) f[q][nd] = 0.5 * (f[q][ndm] + f[q][nc]);
      } else {
        for (int q = 0; q < 6; ++q) f[q][nd] = f[q][ndm];
      }
    }
}

/* met_cutsa.f90:35-48: s6 < 0 -> epsk, s7 = 0 on the real cells */
void orc_met_cutsa(int l, double *s, double epsk) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        if (s[5 * L + n] < 0.) s[5 * L + n] = epsk;
        s[6 * L + n] = 0.;
      }
}

static struct {
  int on, harten;
  const double *dist;
  double rokinf, roeinf, epsk, epsroe, sigma;
  double *fd, *ts, *cfke;  /* 6 ld, 2 ld, ld */
} SA;

void orc_set_sa(int on, const double *dist, double rokinf, double roeinf, double epsk,
                int harten, double epsroe, double sigma, double *fd, double *ts,
                double *cfke) {
  SA.on = on;
  SA.dist = dist;
  SA.rokinf = rokinf;
  SA.roeinf = roeinf;
  SA.epsk = epsk;
  SA.harten = harten;
  SA.epsroe = epsroe;
  SA.sigma = sigma;
  SA.fd = fd;
  SA.ts = ts;
  SA.cfke = cfke;
}

/* ------------------------------------------------------------------------ */
/* wall laws of the adiabatic wall-law walls 'lp2' (lparoi = 1; air,          */
/* iflu = 1; no transition, ktransi = 0)                                    */
/* ------------------------------------------------------------------------ */

/* rbord.f90:377-379 */
#define WL_VKAR 0.41
#define WL_CLLOG 5.25
#define WL_YP0 11.13

static int has_lp2(void) {
  for (int bb = 0; bb < G.nbnd; ++bb)
    if (G.btype[bb] == ORC_BC_LP2) return 1;
  return 0;
}

typedef struct {
  double t1, t2, t3, n1, n2, n3, top, dudy, rop, mup;
} wall_fr;

/* the friction law of lpsa1.f90:111-160 and lparoi1.f90:111-160 for list
 * entry mb: unit tangent of the first cell's velocity, Crocco wall
 * temperature, Sutherland wall viscosity, wall density, Van Driest's
 * velocity v1t = co asin(v1t / co), then the wall stress of the linear law
 * or ten fixed-point passes of the log law */
static wall_fr wall_friction(int64_t mb, const double *v, const double *mu, const double *mut,
                             const double *dist, const double *temp) {
  const int64_t L = G.ld, ni = G.ncin[mb];
  wall_fr f;
  const double v1x = v[L + ni] / v[ni], v1y = v[2 * L + ni] / v[ni], v1z = v[3 * L + ni] / v[ni];
  f.n1 = G.nxn[mb];
  f.n2 = G.nyn[mb];
  f.n3 = G.nzn[mb];
  const double tn = v1x * f.n1 + v1y * f.n2 + v1z * f.n3;
  double t1 = v1x - tn * f.n1, t2 = v1y - tn * f.n2, t3 = v1z - tn * f.n3;
  const double tt = sqrt(sq(t1) + sq(t2) + sq(t3));
  f.t1 = t1 = t1 / tt;
  f.t2 = t2 = t2 / tt;
  f.t3 = t3 = t3 / tt;
  double v1t = v1x * t1 + v1y * t2 + v1z * t3;
  const double temp1 = temp[ni];
  const double pka = G.cp * (mu[ni] / G.pr + mut[ni] / G.prt);
  const double pkb = mu[ni] + mut[ni];
  const double tparoi = temp1 + 0.5 * pkb * sq(v1t) / pka;
  const double sv = G.suth_a; /* 110.4 / tnz */
  f.mup = mu[ni] * sqrt(tparoi / temp1) * (1. + sv / temp1) / (1. + sv / tparoi);
  f.rop = v[ni] * temp1 / tparoi;
  const double co = sqrt(2. * pka * tparoi / pkb);
  v1t = co * cns_asin(v1t / co);
  const double d = dist[ni];
  const double upyp1 = f.rop * v1t * d / f.mup;
  double top = f.mup * v1t / d;
  if (upyp1 <= WL_YP0 * WL_YP0) {
    f.dudy = top / f.mup;
  } else {
    for (int it = 1; it <= 10; ++it)
      top = f.rop * sq(v1t) / sq(cns_log(d * sqrt(f.rop * top) / f.mup) / WL_VKAR + WL_CLLOG);
    f.dudy = sqrt(top / f.rop) / (WL_VKAR * d);
  }
  f.top = top;
  return f;
}

/* lpsa.f90:70-100 -> lpsa1.f90:111-236 on the 'lp2' walls of block l in
 * boundary order: mut of the first cell from the mixing length with van
 * Driest's damping, rho nu~ there from the closed-form root of
 * mut = rho nu~ fv1 (floored at epsk), rho nu~ = 0 in the ghost */
void orc_lpsa(int l, double *v, const double *mu, double *mut, const double *dist,
              const double *temp, double epsk) {
  const int64_t L = G.ld;
  const double c13 = 1. / 3., c18 = 1. / 18., cv1 = SA_CV1;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_LP2 || G.bblk[bb] != l) continue;
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      const int64_t mb = G.bmpb[bb] + m, ni = G.ncin[mb], nc = G.ncbd[mb];
      const wall_fr f = wall_friction(mb, v, mu, mut, dist, temp);
      const double d = dist[ni];
      const double yplus1 = d * sqrt(f.top * f.rop) / f.mup;
      mut[ni] = v[ni] * sq(WL_VKAR) * sq(d) * f.dudy * sq(1. - cns_exp(-yplus1 / 26.));
      const double ca = mut[ni];
      const double cb = mu[ni] * mu[ni] * mu[ni] * mut[ni] * (cv1 * cv1 * cv1);
      const double c1 = cb * sqrt(3.) * sqrt(256. * cb + 27. * (sq(ca) * sq(ca)));
      const double c2 = 0.5 * cb * sq(ca) + c18 * c1;
      const double c3 = -(0.5 * cb * sq(ca)) + c18 * c1;
      const double c4 = 4. * fabs(cns_pow(c3, c13) - cns_pow(c2, c13));
      const double rc4 = sqrt(sq(ca) + c4);
      const double rnutilde =
          0.25 * (ca + rc4) + 0.25 * sqrt(2.) *
                                  sqrt(sq(ca) * rc4 - 2. * cns_pow(c3, c13) * rc4 +
                                       2. * cns_pow(c2, c13) * rc4 + sq(ca) * ca) /
                                  cns_pow(rc4, 0.5);
      v[5 * L + ni] = fmax(rnutilde, epsk);
      v[5 * L + nc] = 0.;
    }
  }
}

/* cllparoi1.f90:89-124 -> lparoi1.f90:111-229 on every 'lp2' wall in
 * boundary order: the wall stress tensor top (t n + n t) in the ghost and
 * the first cell, the first cell's heat flux -n top (u . t), none in the
 * ghost; tau (ld, 9): txx txy txz tyy tyz tzz qcx qcy qcz */
void orc_cllparoi1(const double *v, const double *dist, const double *mu, const double *mut,
                   double *tau, const double *temp) {
  const int64_t L = G.ld;
  for (int bb = 0; bb < G.nbnd; ++bb) {
    if (G.btype[bb] != ORC_BC_LP2) continue;
    for (int m = 0; m < G.bmmb[bb]; ++m) {
      const int64_t mb = G.bmpb[bb] + m, ni = G.ncin[mb], nc = G.ncbd[mb];
      const wall_fr f = wall_friction(mb, v, mu, mut, dist, temp);
      const double top = f.top;
      tau[nc] = 2. * f.t1 * f.n1 * top;
      tau[3 * L + nc] = 2. * f.t2 * f.n2 * top;
      tau[5 * L + nc] = 2. * f.t3 * f.n3 * top;
      tau[L + nc] = (f.t2 * f.n1 + f.t1 * f.n2) * top;
      tau[2 * L + nc] = (f.t1 * f.n3 + f.t3 * f.n1) * top;
      tau[4 * L + nc] = (f.t2 * f.n3 + f.t3 * f.n2) * top;
      for (int a = 0; a < 6; ++a) tau[a * L + ni] = tau[a * L + nc];
      const double qc1 = top * ((v[L + ni] * f.t1 + v[2 * L + ni] * f.t2 + v[3 * L + ni] * f.t3) /
                                v[ni]);
      tau[6 * L + ni] = -f.n1 * qc1;
      tau[7 * L + ni] = -f.n2 * qc1;
      tau[8 * L + ni] = -f.n3 * qc1;
      tau[6 * L + nc] = 0.;
      tau[7 * L + nc] = 0.;
      tau[8 * L + nc] = 0.;
    }
  }
}

double orc_asin(double x) { return cns_asin(x); }

/* ------------------------------------------------------------------------ */
/* k-epsilon of Jones & Launder (equat '2JL', atlecdon.f90:113-128: kcutke  */
/* 1, kfludis 1, ksecmb 1, kcmut 1, kparoi 0, kesst 0; cke1 1.55, cke2 2,    */
/* cmu 0.09; no wall law)                                                    */
/* ------------------------------------------------------------------------ */

#define KE_CKE1 1.55
#define KE_CKE2 2.
#define KE_CMU 0.09

/* met_prod.f90:41-66: the production of k, -rho u'u' : grad u with the
 * Boussinesq stresses; dv and tprod [nnn] block-local */
void orc_met_prod(int l, const double *mut, const double *s, const double *dv, double *tprod) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  const double *dxx = dv, *dxy = dv + nnn, *dxz = dv + 2 * nnn, *dyx = dv + 3 * nnn,
               *dyy = dv + 4 * nnn, *dyz = dv + 5 * nnn, *dzx = dv + 6 * nnn,
               *dzy = dv + 7 * nnn, *dzz = dv + 8 * nnn;
  const double ds3 = 2. / 3.;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        const double torxx = ds3 * (-s[5 * L + n] - mut[n] * (-2 * dxx[m] + dyy[m] + dzz[m]));
        const double toryy = ds3 * (-s[5 * L + n] - mut[n] * (-2 * dyy[m] + dxx[m] + dzz[m]));
        const double torzz = ds3 * (-s[5 * L + n] - mut[n] * (-2 * dzz[m] + dyy[m] + dxx[m]));
        const double torxy = mut[n] * (dxy[m] + dyx[m]);
        const double torxz = mut[n] * (dxz[m] + dzx[m]);
        const double toryz = mut[n] * (dzy[m] + dyz[m]);
        tprod[m] = dxx[m] * torxx + dyy[m] * toryy + dzz[m] * torzz +
                   torxy * (dxy[m] + dyx[m]) + torxz * (dxz[m] + dzx[m]) +
                   toryz * (dzy[m] + dyz[m]);
      }
}

/* met_exgr.f90:60-100 with ex1 = 1, ex2 = 0: a gradient's ghost values
 * from the neighbouring cell -- the k ghosts of the real (i, j), then the
 * i ghosts of every k plane, then the j ghosts of every (i, k) */
static void met_exgr(const blk_t *b, double *ds) {
  const int64_t nci = 1, ncj = b->nid, nck = b->nijd, n0 = b->npc;
  const double ex1 = 1., ex2 = 0.;
  for (int side = 0; side < 2; ++side) {
    const int k = side ? b->nk : 0;
    const int64_t ks = side ? -1 : 1;
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t m = IC(b, i, j, k) - n0;
        ds[m] = ex1 * ds[m + ks * nck] + ex2 * ds[m + 2 * ks * nck];
      }
  }
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int side = 0; side < 2; ++side) {
        const int i = side ? b->ni : 0;
        const int64_t is = side ? -1 : 1;
        const int64_t m = IC(b, i, j, k) - n0;
        ds[m] = ex1 * ds[m + is * nci] + ex2 * ds[m + 2 * is * nci];
      }
  for (int k = 0; k <= b->nk; ++k)
    for (int side = 0; side < 2; ++side) {
      const int j = side ? b->nj : 0;
      const int64_t js = side ? -1 : 1;
      for (int i = 0; i <= b->ni; ++i) {
        const int64_t m = IC(b, i, j, k) - n0;
        ds[m] = ex1 * ds[m + js * ncj] + ex2 * ds[m + 2 * js * ncj];
      }
    }
}

/* met_smke.f90:93-118 for equat '2JL ' (met_exgr on the nine velocity
 * gradients, met_bark, met_bare, met_smkes): ts6, ts7 (qcxts5, qcyts6)
 * the k and epsilon sources and cfke the bound of their derivative, on the
 * real cells (global index); dv [9][nnn] block-local, its ghosts
 * extrapolated in place */
void orc_met_smke(int l, const double *sn, const double *vol, const double *v,
                  const double *mu, const double *mut, const double *tprod, double *dv,
                  double *ts6, double *ts7, double *cfke) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  for (int c = 0; c < 9; ++c) met_exgr(b, dv + c * nnn);
  double *t = calloc((size_t)nnn, sizeof(double)), *bark = calloc((size_t)nnn, sizeof(double)),
         *bare = calloc((size_t)nnn, sizeof(double));
  double *dx = calloc((size_t)nnn, sizeof(double)), *dy = calloc((size_t)nnn, sizeof(double)),
         *dz = calloc((size_t)nnn, sizeof(double));
  /* met_bark.f90:91-126: bark = -2 mu |grad sqrt(k)|^2 (k per unit mass) */
  for (int k = 0; k <= b->nk; ++k)
    for (int j = 0; j <= b->nj; ++j)
      for (int i = 0; i <= b->ni; ++i) {
        const int64_t n = IC(b, i, j, k);
        t[n - n0] = sqrt(v[5 * L + n] / v[n]);
      }
  teq_grads(b, sn, vol, t, dx, dy, dz);
  int64_t r0, r1;
  flat_real_range(b, &r0, &r1);
  for (int64_t n = r0; n <= r1; ++n) {
    const int64_t m = n - n0;
    bark[m] = dx[m] * dx[m] + dy[m] * dy[m] + dz[m] * dz[m];
    bark[m] = -2. * mu[n] * bark[m];
  }
  /* met_bare.f90:64-318: bare = 2 mut mu / rho * sum of the squared
   * gradients of the nine velocity gradients, in the order xx .. zz */
  for (int c = 0; c < 9; ++c) {
    teq_grads(b, sn, vol, dv + c * nnn, dx, dy, dz);
    for (int k = 1; k <= b->nk - 1; ++k)
      for (int j = 1; j <= b->nj - 1; ++j)
        for (int i = 1; i <= b->ni - 1; ++i) {
          const int64_t m = IC(b, i, j, k) - n0;
          bare[m] = bare[m] + dx[m] * dx[m] + dy[m] * dy[m] + dz[m] * dz[m];
        }
  }
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        bare[m] = 2. * mut[n] * mu[n] * bare[m] / v[n];
      }
  /* met_smkes.f90:45-73 (f1 = 1; lparoi = 0) */
  const double f1 = 1.;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        const double s6 = v[5 * L + n], s7 = v[6 * L + n];
        const double retur = sq(s6) / (s7 * mu[n]);
        const double arg = -sq(retur);
        const double f2 = 1. - 0.3 * cns_exp(arg);
        const double esk = s7 / s6;
        const double roe2sk = (s7 * s7) / s6;
        ts6[n] = tprod[m] - s7 + bark[m];
        ts7[n] = KE_CKE1 * f1 * tprod[m] * esk - KE_CKE2 * f2 * roe2sk + bare[m];
        const double c1f1 = KE_CKE1 * f1, c2f2 = KE_CKE2 * f2;
        const double d = -bark[m];
        const double x = c1f1 * tprod[m] - c2f2 * s7;
        const double g = fmax(0., d * (d - 2. * (x - c2f2 * s7)));
        const double rdelta = sqrt(sq(x - c2f2 * s7) + 4 * x * s7 + g);
        const double bb = x - c2f2 * s7 - d;
        const double xl1 = 0.5 * (bb + rdelta) / s6, xl2 = 0.5 * (bb - rdelta) / s6;
        cfke[n] = fmax(fabs(xl1), fabs(xl2));
      }
  free(t); free(bark); free(bare); free(dx); free(dy); free(dz);
}

/* met_kemut.f90:52-65 ('2JL', kesst = 0, lparoi = 0): mut = f_mu cmu
 * rho k^2 / eps, f_mu = exp(-2.5 / (1 + Re_t / 50)), Re_t = rho k^2 / (mu eps) */
void orc_met_kemut(int l, const double *v, const double *mu, double *mut) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        const double retur = sq(v[5 * L + n]) / (v[6 * L + n] * mu[n]);
        const double mut0 = KE_CMU * retur * mu[n];
        const double fmu = cns_exp(-2.5 / (1. + retur / 50.));
        mut[n] = fmu * mut0;
      }
}

/* met_cutke.f90:43-60: k below epsk or epsilon below epse resets both, on
 * i = 1..ni (the upper i ghost included), the real j and k */
void orc_met_cutke(int l, double *s, double epsk, double epse) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni; ++i) {
        const int64_t n = IC(b, i, j, k);
        if (s[5 * L + n] < epsk) {
          s[5 * L + n] = epsk;
          s[6 * L + n] = epse;
        }
        if (s[6 * L + n] < epse) {
          s[5 * L + n] = epsk;
          s[6 * L + n] = epse;
        }
      }
}

/* the first cycle's turbulence initialisation (atsch_num.f90:256-345) on
 * the real cells: met_inisa.f90:36-44 (v6 = mut), met_inmut.f90 (mut =
 * mu / 10), met_ini.f90 = teq_gradv + met_brad.f90:37-51 (v6 = mut |omega| /
 * sqrt(cmu), v7 = mut |omega|^2; dv [9][nnn] block-local) */
void orc_met_inisa(int l, double *v, const double *mut) {
  const blk_t *b = &G.b[l - 1];
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        v[5 * G.ld + n] = mut[n];
      }
}

void orc_met_inmut(int l, const double *mu, double *mut) {
  const blk_t *b = &G.b[l - 1];
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k);
        mut[n] = mu[n] * 1.e-1;
      }
}

void orc_met_ini(int l, double *v, const double *mut, const double *sn, const double *vol,
                 double *dv) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld, n0 = b->npc, nnn = b->nnn;
  orc_teq_gradv(l, sn, vol, v, dv);
  const double cmu1 = 1. / sqrt(KE_CMU);
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        const int64_t n = IC(b, i, j, k), m = n - n0;
        const double omeg = sqrt(sq(dv[7 * nnn + m] - dv[5 * nnn + m]) +
                                 sq(dv[2 * nnn + m] - dv[6 * nnn + m]) +
                                 sq(dv[3 * nnn + m] - dv[nnn + m]));
        v[5 * L + n] = cmu1 * mut[n] * omeg;
        v[6 * L + n] = mut[n] * omeg * omeg;
      }
}

static struct {
  int on;
  double rokinf, roeinf, epsk, epse, alfak, alfae;
  int harten;
  double epsroe;
  double *fd, *ts, *cfke; /* 6 ld, 2 ld, ld */
} KE;

void orc_set_ke(int on, double rokinf, double roeinf, double epsk, double epse, double alfak,
                double alfae, int harten, double epsroe, double *fd, double *ts, double *cfke) {
  KE.on = on;
  KE.rokinf = rokinf;
  KE.roeinf = roeinf;
  KE.epsk = epsk;
  KE.epse = epse;
  KE.alfak = alfak;
  KE.alfae = alfae;
  KE.harten = harten;
  KE.epsroe = epsroe;
  KE.fd = fd;
  KE.ts = ts;
  KE.cfke = cfke;
}

/* met_num.f90:145-790 for '2JL ': turbulence ghosts; per block velocity
 * gradients, production, grad(k/rho) and grad(eps/rho), the sources and
 * the diffusion densities; their ghosts; per block Roe dissipation,
 * explicit balance, implicit line Jacobi (cmt = 1, impli2_eqt_3d.f90:85)
 * and the clip; mut of the model.  v, u, d are (ld, 7). */
void orc_met_num_ke(double *v, double *u, double *d, const double *dt, const double *mu,
                    double *mut, const double *sn, const double *vol) {
  const int64_t L = G.ld;
  double *fd = KE.fd, *ts6 = KE.ts, *ts7 = KE.ts + L;
  double *f5x = fd, *f5y = fd + L, *f5z = fd + 2 * L, *f6x = fd + 3 * L, *f6y = fd + 4 * L,
         *f6z = fd + 5 * L;
  orc_met_bord(v, KE.rokinf, KE.roeinf);
  for (int l = 1; l <= G.nblk; ++l) {
    const blk_t *b = &G.b[l - 1];
    double *dv = calloc((size_t)(9 * b->nnn), sizeof(double));
    double *tprod = calloc((size_t)b->nnn, sizeof(double));
    orc_teq_gradv(l, sn, vol, v, dv);
    orc_met_prod(l, mut, v, dv, tprod);
    orc_met_gradtr(l, sn, vol, v, f5x, f5y, f5z, f6x, f6y, f6z);
    orc_met_smke(l, sn, vol, v, mu, mut, tprod, dv, ts6, ts7, KE.cfke);
    orc_met_fludc(l, mu, mut, f5x, f5y, f5z, f6x, f6y, f6z, KE.alfak, KE.alfae);
    free(dv);
    free(tprod);
  }
  orc_met_rbse(f5x, f5y, f5z, f6x, f6y, f6z);
  for (int l = 1; l <= G.nblk; ++l) {
    orc_met_roe2o(l, v, d, sn, KE.harten, KE.epsroe);
    orc_sch_turb(l, u, v, d, f5x, f5y, f5z, f6x, f6y, f6z, ts6, ts7, sn, vol);
    orc_impli2_eqt_3d(l, u, dt, v, mu, mut, KE.cfke, sn, vol, 1.0);
    orc_met_cutke(l, v, KE.epsk, KE.epse);
  }
  for (int l = 1; l <= G.nblk; ++l) orc_met_kemut(l, v, mu, mut);
}

/* met_num.f90:145-790 for 1SA, after rbord: turbulence ghosts; per block
 * (in block order, which met_smsa.f90:177's block-local read of txxf5x
 * depends on) velocity gradients, grad(nu~), source, diffusion densities;
 * their ghosts; per block Roe dissipation, explicit balance, implicit line
 * Jacobi and the clip; mut = v6 fv1.  v, u, d are (ld, 7). */
void orc_met_num(double *v, double *u, double *d, const double *dt, const double *mu,
                 double *mut, const double *sn, const double *vol, const double *temp) {
  const int64_t L = G.ld;
  double *fd = SA.fd, *ts6 = SA.ts, *ts7 = SA.ts + L;
  double *f5x = fd, *f5y = fd + L, *f5z = fd + 2 * L, *f6x = fd + 3 * L, *f6y = fd + 4 * L,
         *f6z = fd + 5 * L;
  orc_met_bord(v, SA.rokinf, SA.roeinf);
  for (int l = 1; l <= G.nblk; ++l) {
    const blk_t *b = &G.b[l - 1];
    double *dv = calloc((size_t)(9 * b->nnn), sizeof(double));
    orc_teq_gradv(l, sn, vol, v, dv);
    /* met_num.f90:193-279: the wall law after teq_gradv and met_prod */
    orc_lpsa(l, v, mu, mut, SA.dist, temp, SA.epsk);
    orc_met_gradtr(l, sn, vol, v, f5x, f5y, f5z, f6x, f6y, f6z);
    orc_met_smsa(l, sn, vol, v, mu, SA.dist, dv, f5x, f5y, f5z, ts6, ts7, SA.cfke);
    orc_met_fludcsa(l, v, mu, f5x, f5y, f5z, f6x, f6y, f6z, SA.sigma);
    free(dv);
  }
  orc_met_rbse(f5x, f5y, f5z, f6x, f6y, f6z);
  for (int l = 1; l <= G.nblk; ++l) {
    orc_met_roe2o(l, v, d, sn, SA.harten, SA.epsroe);
    orc_sch_turb(l, u, v, d, f5x, f5y, f5z, f6x, f6y, f6z, ts6, ts7, sn, vol);
    orc_impli2_eqt_3d(l, u, dt, v, mu, mut, SA.cfke, sn, vol, 1.0);
    orc_met_cutsa(l, v, SA.epsk);
  }
  for (int l = 1; l <= G.nblk; ++l) orc_met_samut(l, v, mu, mut);
}

/* atsch_num.f90:245-1134 for ischema<=4 (Jameson, kprec=0), kmf=1, steady:
 * zpres/zvismo, chrono, rfve (first cycle only) and rfvc, dissip_jameson
 * (before rbord: the physical ghosts are the previous iteration's), rbord,
 * zvisqc, sch_jameson, the implicit phase.  dis holds the dissipation (the
 * reference reuses d for it; implimf then overwrites d with the increment). */
int orc_step_jameson(double *v, double *u, double *d, double *dis, double *dt,
                     const double *sn, const double *vol, double *ps, double *temp,
                     double *cson, double *mu, double *mut, double *tau, int first_cycle) {
  for (int l = 1; l <= G.nblk; ++l) orc_zpres(l, v, ps, temp, cson);
  if (G.ns)
    for (int l = 1; l <= G.nblk; ++l) orc_zvismo(l, mu, temp);
  for (int l = 1; l <= G.nblk; ++l) orc_chronos(l, mu, mut, v, dt, sn, vol, cson);
  if (G.kdtl == 0) orc_chrono_global(dt);
  if (first_cycle) orc_rfve(v, ps, temp, cson);
  orc_rfvc(v, ps, temp, cson);
  for (int l = 1; l <= G.nblk; ++l) orc_dissip_jameson(l, v, dis, sn, ps, cson);
  orc_rbord(v, ps, temp, cson);
  if (SA.on) orc_met_num(v, u, d, dt, mu, mut, sn, vol, temp);
  if (KE.on) orc_met_num_ke(v, u, d, dt, mu, mut, sn, vol);
  if (G.ns) {
    orc_zvisqc(v, mu, mut, tau, sn, vol, temp);
    /* atsch_num.f90:579-604: the wall law of the 'lp2' walls */
    if (has_lp2()) orc_cllparoi1(v, SA.dist, mu, mut, tau, temp);
  }
  for (int l = 1; l <= G.nblk; ++l) orc_sch_jameson(l, u, v, dis, tau, sn, ps);
  if (G.kfmg == 3)
    for (int l = 1; l <= G.nblk; ++l) orc_sch_dual(l, u, v, G.icycle, vol, G.ptdual);
  for (int l = 1; l <= G.nblk; ++l) {
    if (G.ns)
      orc_implimf_3d(l, u, dt, v, d, mu, mut, sn, vol, ps, cson, G.lmax);
    else
      orc_implimf_eu(l, u, dt, v, d, sn, vol, ps, cson, G.lmax);
  }
  return 0;
}

/* atsch_num.f90:245-1134 for ischema=7 (Roe), kmf=1 (implicit), steady */
int orc_step(double *v, double *u, double *d, double *dt, const double *sn,
             const double *vol, double *ps, double *temp, double *cson,
             double *mu, double *mut, double *tau, int compute_dt) {
#pragma omp parallel for schedule(dynamic, 1)
  for (int l = 1; l <= G.nblk; ++l) {
    orc_zpres(l, v, ps, temp, cson);
    if (G.ns) orc_zvismo(l, mu, temp);
    if (compute_dt) orc_chronos(l, mu, mut, v, dt, sn, vol, cson);
  }
  if (compute_dt && G.kdtl == 0) orc_chrono_global(dt);
  orc_rbord(v, ps, temp, cson);
  if (SA.on) orc_met_num(v, u, d, dt, mu, mut, sn, vol, temp);
  if (KE.on) orc_met_num_ke(v, u, d, dt, mu, mut, sn, vol);
  if (G.ns) {
    orc_zvisqc(v, mu, mut, tau, sn, vol, temp);
    /* atsch_num.f90:579-604: the wall law of the 'lp2' walls */
    if (has_lp2()) orc_cllparoi1(v, SA.dist, mu, mut, tau, temp);
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int l = 1; l <= G.nblk; ++l) {
    /* atsch_num.f90:628-983: the flux family by ischema */
    if (G.ischema == 9)
      orc_sch_rusanov(l, u, v, tau, sn, ps);
    else if (G.ischema == 12)
      orc_sch_weno5_3d(l, u, v, tau, sn, ps);
    else if (G.ischema == 5)
      orc_sch_ausmp(l, u, v, tau, sn, ps);
    else if (G.ischema == 14 && G.ns)
      orc_sch_hllc(l, u, v, tau, sn, ps);
    else if (G.ischema == 14)
      orc_sch_hllc_euler(l, u, v, sn, ps);
    else if (G.ns)
      orc_sch_roe(l, u, v, tau, sn, ps);
    else
      orc_sch_roe_euler(l, u, v, sn, ps);
    if (G.kfmg == 3) orc_sch_dual(l, u, v, G.icycle, vol, G.ptdual);
    if (G.ns)
      orc_implimf_3d(l, u, dt, v, d, mu, mut, sn, vol, ps, cson, G.lmax);
    else
      orc_implimf_eu(l, u, dt, v, d, sn, vol, ps, cson, G.lmax);
  }
  return 0;
}

/* ---- reference grid and flow files ------------------------------------- */
/* Fortran unformatted sequential files as gfortran writes them: a logical
 * record is subrecords of at most maxsub data bytes, each framed by 4-byte
 * byte counts; the leading count is negated when another subrecord follows,
 * the trailing one when a subrecord precedes.  Return codes: 0, 8 (open,
 * read or write failure), 9 (records do not match the layout). */
enum { ORC_EIO = 8, ORC_EFORMAT = 9 };

static int orc_put_record(FILE *f, const double *buf, int64_t n, int64_t maxsub) {
  const unsigned char *p = (const unsigned char *)buf;
  int64_t left = 8 * n;
  int sub = 0;
  do {
    int64_t len = left > maxsub ? maxsub : left;
    int32_t lead = (int32_t)(left > len ? -len : len);
    int32_t trail = (int32_t)(sub > 0 ? -len : len);
    if (fwrite(&lead, 4, 1, f) != 1) return ORC_EIO;
    if (len > 0 && fwrite(p, 1, (size_t)len, f) != (size_t)len) return ORC_EIO;
    if (fwrite(&trail, 4, 1, f) != 1) return ORC_EIO;
    p += len;
    left -= len;
    ++sub;
  } while (left > 0);
  return 0;
}

/* the first n doubles of the next logical record (a Fortran READ of n items) */
static int orc_get_record(FILE *f, double *buf, int64_t n) {
  unsigned char *p = (unsigned char *)buf;
  int64_t need = 8 * n;
  int sub = 0;
  for (;;) {
    int32_t lead, trail;
    if (fread(&lead, 4, 1, f) != 1) return ORC_EFORMAT;
    int64_t len = lead < 0 ? -(int64_t)lead : lead;
    for (int64_t b = 0; b < len; ++b) {
      int ch = fgetc(f);
      if (ch == EOF) return ORC_EFORMAT;
      if (need > 0) {
        *p++ = (unsigned char)ch;
        --need;
      }
    }
    if (fread(&trail, 4, 1, f) != 1) return ORC_EFORMAT;
    if ((trail < 0 ? -(int64_t)trail : trail) != len) return ORC_EFORMAT;
    if ((sub > 0) != (trail < 0)) return ORC_EFORMAT;
    ++sub;
    if (lead >= 0) break;
  }
  return need > 0 ? ORC_EFORMAT : 0;
}

/* (i, j, k) box of a record over block b: 0 real nodes, 1 real cells,
 * 2 cells with the ghost layer (chdgcv.f90, chdacc.f90) */
static void orc_box(const blk_t *b, int what, int lo[3], int hi[3]) {
  int n[3] = {b->ni, b->nj, b->nk};
  for (int a = 0; a < 3; ++a) {
    lo[a] = what == 2 ? 0 : 1;
    hi[a] = what == 1 ? n[a] - 1 : n[a];
  }
}

static int64_t orc_box_count(const int lo[3], const int hi[3]) {
  return (int64_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

/* writdg.f90:46-48 / writda.f90:78-97: the array over the box, i fastest;
 * centre: cvccg.f90's .125*(sum of the 8 nodes of the cell) */
static int orc_put_array(FILE *f, const blk_t *b, const double *x, int centre,
                         const int lo[3], const int hi[3], int64_t maxsub, double *buf) {
  int64_t m = 0;
  int64_t inc1 = 1, inc2 = b->nid, inc3 = b->nijd;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        int64_t n = b->npc + i + (int64_t)j * b->nid + (int64_t)k * b->nijd;
        if (!centre) {
          buf[m++] = x[n];
        } else {
          buf[m++] = .125 * (x[n] + x[n + inc3] + x[n + inc1] + x[n + inc1 + inc3] +
                             x[n + inc2] + x[n + inc2 + inc3] + x[n + inc1 + inc2] +
                             x[n + inc1 + inc2 + inc3]);
        }
      }
  return orc_put_record(f, buf, m, maxsub);
}

/* readdg.f90:71-80 / readda.f90:88-118: one record into the array's box */
static int orc_get_array(FILE *f, const blk_t *b, double *x, const int lo[3], const int hi[3],
                         double *buf) {
  int rc = orc_get_record(f, buf, orc_box_count(lo, hi));
  if (rc) return rc;
  int64_t m = 0;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i)
        x[b->npc + i + (int64_t)j * b->nid + (int64_t)k * b->nijd] = buf[m++];
  return 0;
}


static void orc_equat(const char *equat, int *ns, int *ke) {
  char q[8] = "       ";
  for (int a = 0; a < 7 && equat[a]; ++a) q[a] = equat[a];
  *ns = q[0] == 'n' && q[1] == 's';
  *ke = q[5] == 'k' && q[6] == 'e';
}

static double *orc_block_buffer(void) {
  int64_t mx = 1;
  for (int l = 0; l < G.nblk; ++l)
    if (G.b[l].nnn > mx) mx = G.b[l].nnn;
  return (double *)malloc(sizeof(double) * (size_t)mx);
}

/* svgr.f90 for l = 1..nblk: disc cvcv (nodes, cvcvg), cvcc / cvcf (cell
 * centres of the real cells / with the ghost layer, cvccg) */
int orc_writdg(const char *path, const char *disc, const double *x, const double *y,
               const double *z, int64_t maxsub) {
  int what = !strncmp(disc, "cvcv", 4) ? 0 : !strncmp(disc, "cvcc", 4) ? 1
             : !strncmp(disc, "cvcf", 4) ? 2 : -1;
  if (what < 0) return 1;
  FILE *f = fopen(path, "wb");
  if (!f) return ORC_EIO;
  double *buf = orc_block_buffer();
  int rc = 0;
  for (int l = 0; l < G.nblk && !rc; ++l) {
    int lo[3], hi[3];
    orc_box(&G.b[l], what, lo, hi);
    const double *c[3] = {x, y, z};
    for (int a = 0; a < 3 && !rc; ++a)
      rc = orc_put_array(f, &G.b[l], c[a], what != 0, lo, hi, maxsub, buf);
  }
  free(buf);
  if (fclose(f) && !rc) rc = ORC_EIO;
  return rc;
}

/* ingr.f90:49 -> readdg.f90:71-80 for l = 1..nblk */
int orc_readdg(const char *path, double *x, double *y, double *z) {
  FILE *f = fopen(path, "rb");
  if (!f) return ORC_EIO;
  double *buf = orc_block_buffer();
  int rc = 0;
  for (int l = 0; l < G.nblk && !rc; ++l) {
    int lo[3], hi[3];
    orc_box(&G.b[l], 0, lo, hi);
    double *c[3] = {x, y, z};
    for (int a = 0; a < 3 && !rc; ++a) rc = orc_get_array(f, &G.b[l], c[a], lo, hi, buf);
  }
  free(buf);
  fclose(f);
  return rc;
}

/* svfw.f90 for l = 1..nblk: chdacc.f90 (disc cccc = real cells, cccf = with
 * the ghost layer) -> writda.f90:78-97: v1..v5, mut ('ns'), v6, v7 ('ke') */
int orc_writda(const char *path, const char *disc, const char *equat, const double *v,
               const double *mut, int64_t maxsub) {
  int what = !strncmp(disc, "cccc", 4) ? 1 : !strncmp(disc, "cccf", 4) ? 2 : -1;
  if (what < 0) return 1;
  int ns, ke;
  orc_equat(equat, &ns, &ke);
  FILE *f = fopen(path, "wb");
  if (!f) return ORC_EIO;
  double *buf = orc_block_buffer();
  int rc = 0;
  for (int l = 0; l < G.nblk && !rc; ++l) {
    const blk_t *b = &G.b[l];
    int lo[3], hi[3];
    orc_box(b, what, lo, hi);
    for (int a = 0; a < 5 && !rc; ++a) rc = orc_put_array(f, b, v + a * G.ld, 0, lo, hi, maxsub, buf);
    if (ns && !rc) rc = orc_put_array(f, b, mut, 0, lo, hi, maxsub, buf);
    for (int a = 5; a < 7 && ke && !rc; ++a)
      rc = orc_put_array(f, b, v + a * G.ld, 0, lo, hi, maxsub, buf);
  }
  free(buf);
  if (fclose(f) && !rc) rc = ORC_EIO;
  return rc;
}

/* infw.f90:64 -> readda.f90:88-131 for l = 1..nblk */
int orc_readda(const char *path, const char *equat, int keinit, double *v, double *mut) {
  int ns, ke;
  orc_equat(equat, &ns, &ke);
  FILE *f = fopen(path, "rb");
  if (!f) return ORC_EIO;
  double *buf = orc_block_buffer();
  int rc = 0;
  for (int l = 0; l < G.nblk && !rc; ++l) {
    const blk_t *b = &G.b[l];
    int lo[3], hi[3];
    orc_box(b, 1, lo, hi);
    for (int a = 0; a < 5 && !rc; ++a) rc = orc_get_array(f, b, v + a * G.ld, lo, hi, buf);
    if (ns && !rc) rc = orc_get_array(f, b, mut, lo, hi, buf);
    if (ke && keinit == 0) {
      for (int a = 5; a < 7 && !rc; ++a) rc = orc_get_array(f, b, v + a * G.ld, lo, hi, buf);
    } else if (ke) {
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i) {
            int64_t n = b->npc + i + (int64_t)j * b->nid + (int64_t)k * b->nijd;
            v[5 * G.ld + n] = 0.;
            v[6 * G.ld + n] = 0.;
          }
    }
  }
  free(buf);
  fclose(f);
  return rc;
}

/* ---- dual time stepping (kfmg = 3) -------------------------------------- */
void orc_set_dual(int kfmg, int kdualns, int icycle, double *ptdual) {
  G.kfmg = kfmg;
  G.kdualns = kdualns;
  G.icycle = icycle;
  G.ptdual = ptdual;
}

/* sch_dual.f90:18-52 (kdualns 0, 1) and sch_dual2.f90:18-52 (kdualns 2):
 * u += vol/dt1min * (fact*v + ptdual) on the real cells */
void orc_sch_dual(int l, double *u, const double *v, int icycle, const double *vol,
                  const double *ptdual) {
  const blk_t *b = &G.b[l - 1];
  const int64_t L = G.ld;
  double fact = G.kdualns == 2 ? 11. / 6. : 1.5;
  if (icycle <= 1) fact = 1.;
  const double dti = 1. / G.dt1min;
  for (int k = 1; k <= b->nk - 1; ++k)
    for (int j = 1; j <= b->nj - 1; ++j)
      for (int i = 1; i <= b->ni - 1; ++i) {
        int64_t n = IC(b, i, j, k);
        double c0 = vol[n] * dti;
        for (int a = 0; a < 5; ++a) u[a * L + n] = u[a * L + n] + c0 * (fact * v[a * L + n] + ptdual[a * L + n]);
      }
}

/* the real cells of every block, in block, k, j, i order */
#define FOR_REAL_CELLS(n)                                 \
  for (int l_ = 0; l_ < G.nblk; ++l_)                     \
    for (int k_ = 1; k_ <= G.b[l_].nk - 1; ++k_)          \
      for (int j_ = 1; j_ <= G.b[l_].nj - 1; ++j_)        \
        for (int i_ = 1; i_ <= G.b[l_].ni - 1; ++i_)      \
          for (int64_t n = IC(&G.b[l_], i_, j_, k_), once_ = 1; once_; once_ = 0)

/* utinia.f90:140-160 / readda.f90:150-176 (vdual = vdual1 = vdual2 = v)
 * then sch_duin.f90 (ptdual = -vdual) */
void orc_sch_duin(const double *v, double *ptdual, double *vdual, double *vdual1,
                  double *vdual2) {
  const int64_t L = G.ld;
  FOR_REAL_CELLS(n) {
    for (int a = 0; a < 5; ++a) {
      vdual[a * L + n] = v[a * L + n];
      vdual1[a * L + n] = v[a * L + n];
      vdual2[a * L + n] = v[a * L + n];
      ptdual[a * L + n] = -vdual[a * L + n];
    }
  }
}

/* sch_duup.f90 (kdualns 0, 1): vdual1 = vdual, vdual = v,
 * ptdual = -2 vdual + 0.5 vdual1; sch_duup2.f90 (kdualns 2): vdual2 =
 * vdual1, vdual1 = vdual, vdual = v, ptdual = -3 vdual + 1.5 vdual1 - vdual2/3 */
void orc_sch_duup(const double *v, double *ptdual, double *vdual, double *vdual1,
                  double *vdual2) {
  const int64_t L = G.ld;
  const double c13 = 1. / 3.;
  FOR_REAL_CELLS(n) {
    for (int a = 0; a < 5; ++a) {
      const int64_t q = a * L + n;
      if (G.kdualns == 2) {
        vdual2[q] = vdual1[q];
        vdual1[q] = vdual[q];
        vdual[q] = v[q];
        ptdual[q] = -3. * vdual[q] + 1.5 * vdual1[q] - c13 * vdual2[q];
      } else {
        vdual1[q] = vdual[q];
        vdual[q] = v[q];
        ptdual[q] = -2. * vdual[q] + 0.5 * vdual1[q];
      }
    }
  }
}
#undef FOR_REAL_CELLS

/* the portable exponential and real power (cns_pmath.h) as the checker sees
   them, for the tests that compare them with the host libm */
double orc_pow(double x, double y) { return cns_pow(x, y); }
double orc_exp(double t) { return cns_exp(t); }
