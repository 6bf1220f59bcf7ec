// cns_ke.cu -- the k-epsilon model of Jones & Launder in the reference's
// transport step (equat '2JL': met_prod, met_smke with met_exgr, met_bark,
// met_bare and met_smkes, met_kemut, met_cutke; kesst 0, no wall law).
//
// Per real cell, one thread each: the production of k from the velocity
// gradients; the sources of k and epsilon with their low-Reynolds terms
// (|grad sqrt(k)|^2 and the squared second derivatives of the velocity,
// through the Green-Gauss gradients of cns_sa.cu) and the bound of their
// derivative; the eddy viscosity; the clip.  The ghost values of the nine
// velocity gradients are copied from the neighbouring cell in three
// ordered passes (k ghosts, then i, then j) as met_exgr runs them.
// FP64, --fmad=false, the reference's expression order; exp through
// cns_pmath.h: bit-identical to the CPU restatement.
#include "cns_kernels.cuh"
#include "cns_pmath.h"

namespace cns {

namespace {

constexpr double kCke1 = 1.55, kCke2 = 2., kCmu = 0.09;  // atlecdon.f90:124-128

// met_prod.f90:41-66 on the real cells; dv (global index, 9 rows xx xy xz
// yx yy yz zx zy zz)
__global__ void __launch_bounds__(kTile) k_met_prod(const Blk* __restrict__ blks, Space sp,
                                                    long long ld,
                                                    const double* __restrict__ mut,
                                                    const double* __restrict__ s,
                                                    const double* __restrict__ dv,
                                                    double* __restrict__ tprod) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double dxx = dv[n], dxy = dv[ld + n], dxz = dv[2 * ld + n], dyx = dv[3 * ld + n],
               dyy = dv[4 * ld + n], dyz = dv[5 * ld + n], dzx = dv[6 * ld + n],
               dzy = dv[7 * ld + n], dzz = dv[8 * ld + n];
  const double ds3 = 2. / 3.;
  const double s6 = s[5 * ld + n], mt = mut[n];
  const double torxx = ds3 * (-s6 - mt * (-2 * dxx + dyy + dzz));
  const double toryy = ds3 * (-s6 - mt * (-2 * dyy + dxx + dzz));
  const double torzz = ds3 * (-s6 - mt * (-2 * dzz + dyy + dxx));
  const double torxy = mt * (dxy + dyx);
  const double torxz = mt * (dxz + dzx);
  const double toryz = mt * (dzy + dyz);
  tprod[n] = dxx * torxx + dyy * toryy + dzz * torzz + torxy * (dxy + dyx) +
             torxz * (dxz + dzx) + toryz * (dzy + dyz);
}

// met_exgr.f90:60-100 (ex1 = 1, ex2 = 0) on the nine gradients of block B,
// pass p, one side per launch (lower, then upper: the order of the
// reference's loops, which matters where a block is one cell thick and the
// two sides read each other): 0 the k ghosts of the real (i, j); 1 the i
// ghosts of every k plane and real j; 2 the j ghosts of every k plane and
// i = 0..ni
__global__ void __launch_bounds__(256) k_exgr(Blk B, int p, int side, long long ld,
                                             double* __restrict__ dv) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k;
  long long inc;
  if (p == 0) {
    const long long ni = B.ni - 1;
    if (t >= ni * (B.nj - 1)) return;
    i = 1 + (int)(t % ni);
    j = 1 + (int)(t / ni);
    k = side ? B.nk : 0;
    inc = B.nijd;
  } else if (p == 1) {
    const long long nj = B.nj - 1;
    if (t >= nj * (B.nk + 1)) return;
    j = 1 + (int)(t % nj);
    k = (int)(t / nj);
    i = side ? B.ni : 0;
    inc = 1;
  } else {
    const long long ni = B.ni + 1;
    if (t >= ni * (B.nk + 1)) return;
    i = (int)(t % ni);
    k = (int)(t / ni);
    j = side ? B.nj : 0;
    inc = B.nid;
  }
  const long long s = side ? -inc : inc;
  const long long m = cell_index(B, i, j, k);
  const double ex1 = 1., ex2 = 0.;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    double* d = dv + c * ld;
    d[m] = ex1 * d[m + s] + ex2 * d[m + 2 * s];
  }
}

// met_bare.f90:64-300: bare += |grad a|^2 for the three gradients a whose
// Green-Gauss gradients g holds (9 rows: a0 x y z, a1 x y z, a2 x y z), in
// that order; first: bare starts from 0
__global__ void __launch_bounds__(kTile) k_bare_acc(const Blk* __restrict__ blks, Space sp,
                                                    long long ld, const double* __restrict__ g,
                                                    double* __restrict__ bare, int first) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  double acc = first ? 0. : bare[n];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double gx = g[(3 * q) * ld + n], gy = g[(3 * q + 1) * ld + n],
                 gz = g[(3 * q + 2) * ld + n];
    acc = acc + gx * gx + gy * gy + gz * gz;
  }
  bare[n] = acc;
}

// met_bark.f90:122-126, met_bare.f90:308-316 and met_smkes.f90:45-73 (f1 = 1,
// lparoi = 0) on the real cells: gt the gradient of sqrt(k / rho) [3][ld],
// bare the sum of met_bare; ts6, ts7 the sources of k and epsilon, cfke the
// bound of their derivative
__global__ void __launch_bounds__(kTile) k_smkes(const Blk* __restrict__ blks, Space sp,
                                                 long long ld, const double* __restrict__ s,
                                                 const double* __restrict__ mu,
                                                 const double* __restrict__ mut,
                                                 const double* __restrict__ tprod,
                                                 const double* __restrict__ gt,
                                                 const double* __restrict__ bare_sum,
                                                 double* __restrict__ ts6,
                                                 double* __restrict__ ts7,
                                                 double* __restrict__ cfke) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double gx = gt[n], gy = gt[ld + n], gz = gt[2 * ld + n];
  double bark = gx * gx + gy * gy + gz * gz;
  bark = -2. * mu[n] * bark;
  const double bare = 2. * mut[n] * mu[n] * bare_sum[n] / s[n];
  const double f1 = 1.;
  const double s6 = s[5 * ld + n], s7 = s[6 * ld + n], tp = tprod[n];
  const double retur = (s6 * s6) / (s7 * mu[n]);
  const double arg = -(retur * retur);
  const double f2 = 1. - 0.3 * cns_exp(arg);
  const double esk = s7 / s6;
  const double roe2sk = (s7 * s7) / s6;
  ts6[n] = tp - s7 + bark;
  ts7[n] = kCke1 * f1 * tp * esk - kCke2 * f2 * roe2sk + bare;
  const double c1f1 = kCke1 * f1, c2f2 = kCke2 * f2;
  const double d = -bark;
  const double x = c1f1 * tp - c2f2 * s7;
  const double g = fmax(0., d * (d - 2. * (x - c2f2 * s7)));
  const double xm = x - c2f2 * s7;
  const double rdelta = sqrt(xm * xm + 4 * x * s7 + g);
  const double bb = x - c2f2 * s7 - d;
  const double xl1 = 0.5 * (bb + rdelta) / s6, xl2 = 0.5 * (bb - rdelta) / s6;
  cfke[n] = fmax(fabs(xl1), fabs(xl2));
}

// met_kemut.f90:52-65 ('2JL', kesst 0, lparoi 0) on the real cells
__global__ void __launch_bounds__(kTile) k_kemut(const Blk* __restrict__ blks, Space sp,
                                                 long long ld, const double* __restrict__ v,
                                                 const double* __restrict__ mu,
                                                 double* __restrict__ mut) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double v6 = v[5 * ld + n];
  const double retur = (v6 * v6) / (v[6 * ld + n] * mu[n]);
  const double mut0 = kCmu * retur * mu[n];
  const double fmu = cns_exp(-2.5 / (1. + retur / 50.));
  mut[n] = fmu * mut0;
}

// met_cutke.f90:43-60 on i = 1..ni (the thread of i = ni - 1 also takes the
// upper i ghost, which the reference's loop reaches), the real j and k
__device__ __forceinline__ void cutke_cell(double* v, long long ld, long long n, double epsk,
                                           double epse) {
  if (v[5 * ld + n] < epsk) {
    v[5 * ld + n] = epsk;
    v[6 * ld + n] = epse;
  }
  if (v[6 * ld + n] < epse) {
    v[5 * ld + n] = epsk;
    v[6 * ld + n] = epse;
  }
}

__global__ void __launch_bounds__(kTile) k_cutke(const Blk* __restrict__ blks, Space sp,
                                                 long long ld, double* __restrict__ v,
                                                 double epsk, double epse) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  cutke_cell(v, ld, n, epsk, epse);
  if (i == B.ni - 1) cutke_cell(v, ld, n + 1, epsk, epse);
}

// the turbulence initialisation of the first cycle (atsch_num.f90:256-345)
// on the real cells: mode 0 met_inisa.f90:36-44 (rho nu~ = mut), mode 1
// met_inmut.f90 (mut = mu / 10), mode 2 met_brad.f90:37-51 (Bradshaw:
// rho k = mut |omega| / sqrt(cmu), rho eps = mut |omega|^2; dv the velocity
// gradients, global index)
__global__ void __launch_bounds__(kTile) k_turb_init(const Blk* __restrict__ blks, Space sp,
                                                     int mode, long long ld, double* v,
                                                     double* mut, const double* __restrict__ mu,
                                                     const double* __restrict__ dv) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  if (mode == 0) {
    v[5 * ld + n] = mut[n];
  } else if (mode == 1) {
    mut[n] = mu[n] * 1.e-1;
  } else {
    const double cmu1 = 1. / sqrt(kCmu);
    const double a1 = dv[7 * ld + n] - dv[5 * ld + n];  // dvzy - dvyz
    const double a2 = dv[2 * ld + n] - dv[6 * ld + n];  // dvxz - dvzx
    const double a3 = dv[3 * ld + n] - dv[ld + n];      // dvyx - dvxy
    const double omeg = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
    v[5 * ld + n] = cmu1 * mut[n] * omeg;
    v[6 * ld + n] = mut[n] * omeg * omeg;
  }
}

inline int grid_of(const Space& s) { return s.ntiles; }

}  // namespace

cudaError_t launch_turb_init(const Blk* blks, Space cells, int mode, long long ld, double* v,
                             double* mut, const double* mu, const double* dv, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_turb_init<<<grid_of(cells), kTile, 0, st>>>(blks, cells, mode, ld, v, mut, mu, dv);
  return cudaGetLastError();
}

cudaError_t launch_met_prod(const Blk* blks, Space cells, long long ld, const double* mut,
                            const double* s, const double* dv, double* tprod, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_met_prod<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, mut, s, dv, tprod);
  return cudaGetLastError();
}

cudaError_t launch_exgr(const Blk& B, long long ld, double* dv, cudaStream_t st) {
  const long long cnt[3] = {(long long)(B.ni - 1) * (B.nj - 1),
                            (long long)(B.nj - 1) * (B.nk + 1),
                            (long long)(B.ni + 1) * (B.nk + 1)};
  for (int p = 0; p < 3; ++p)
    for (int side = 0; side < 2 && cnt[p] > 0; ++side)
      k_exgr<<<(unsigned)((cnt[p] + 255) / 256), 256, 0, st>>>(B, p, side, ld, dv);
  return cudaGetLastError();
}

cudaError_t launch_smke(const Blk* blks, Space cells, long long ld, const double* s,
                        const double* mu, const double* mut, const double* sn,
                        const double* vol, const double* tprod, const double* dv, double* w,
                        double* ts6, double* ts7, double* cfke, long long n0, long long n1,
                        cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  // w: gt [3][ld], g [9][ld], bare [ld], scalars [1][ld]
  double *gt = w, *g = w + 3 * ld, *bare = w + 12 * ld, *sc = w + 13 * ld;
  // met_bark: the gradient of sqrt(s6 / s1) over the block's cells
  cudaError_t e = launch_teq_grads(blks, cells, 3, 1, s, nullptr, ld, sn, vol, gt, sc, n0, n1,
                                   st);
  // met_bare: the gradients of the nine velocity gradients, three at a time
  for (int q = 0; q < 3 && e == cudaSuccess; ++q) {
    e = launch_teq_grads(blks, cells, 1, 3, s, dv + 3 * q * ld, ld, sn, vol, g, nullptr, 0, 0,
                         st);
    if (e == cudaSuccess)
      k_bare_acc<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, g, bare, q == 0);
  }
  if (e == cudaSuccess)
    k_smkes<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, s, mu, mut, tprod, gt, bare, ts6,
                                              ts7, cfke);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t launch_kemut(const Blk* blks, Space cells, long long ld, const double* v,
                         const double* mu, double* mut, cudaStream_t st) {
  if (cells.ntiles > 0) k_kemut<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, v, mu, mut);
  return cudaGetLastError();
}

cudaError_t launch_cutke(const Blk* blks, Space cells, long long ld, double* v, double epsk,
                         double epse, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_cutke<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, v, epsk, epse);
  return cudaGetLastError();
}

}  // namespace cns
