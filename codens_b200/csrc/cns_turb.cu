// cns_turb.cu -- the turbulence-transport terms of the reference: the
// diffusion coefficients of the transport equations (met_fludc.f90 for
// k-epsilon, met_fludcsa.f90 for Spalart-Allmaras), the TVD Roe dissipation
// of the two transport variables (met_roe2o.f90, with Harten's entropy fix
// met_roe2oh.f90), the Spalart-Allmaras eddy viscosity (met_samut.f90) and
// the transport equations' explicit balance (sch_turb.f90).
//
// The transport state t and the dissipation d are the reference's (ld, 7)
// arrays (columns 6 and 7: the transport variables).  FP64, --fmad=false,
// reference expression order: bit-identical.
#include "cns_kernels.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

// met_fludc.f90:72-85 over the flat range [n0, n1]
__global__ void __launch_bounds__(256) k_fludc(long long n0, long long n1,
                                              const double* __restrict__ mu,
                                              const double* __restrict__ mut, double* fd5x,
                                              double* fd5y, double* fd5z, double* fd6x,
                                              double* fd6y, double* fd6z, double alfak,
                                              double alfae) {
  const long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n > n1) return;
  const double m = mu[n], mt = mut[n];
  fd5x[n] = (m + mt / alfak) * fd5x[n];
  fd5y[n] = (m + mt / alfak) * fd5y[n];
  fd5z[n] = (m + mt / alfak) * fd5z[n];
  fd6x[n] = (m + mt / alfae) * fd6x[n];
  fd6y[n] = (m + mt / alfae) * fd6y[n];
  fd6z[n] = (m + mt / alfae) * fd6z[n];
}

// met_fludcsa.f90:92-104 over the flat range [n0, n1]; s6 = s(:,6)
__global__ void __launch_bounds__(256) k_fludcsa(long long n0, long long n1,
                                                const double* __restrict__ s6,
                                                const double* __restrict__ mu, double* fd5x,
                                                double* fd5y, double* fd5z, double* fd6x,
                                                double* fd6y, double* fd6z, double sigma1) {
  const long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n > n1) return;
  const double smutot = sigma1 * (mu[n] + s6[n]);
  fd5x[n] = smutot * fd5x[n];
  fd5y[n] = smutot * fd5y[n];
  fd5z[n] = smutot * fd5z[n];
  fd6x[n] = 0.;
  fd6y[n] = 0.;
  fd6z[n] = 0.;
}

// met_roe2o.f90:288-296
__device__ __forceinline__ double amimd(double a, double b) {
  const double s = copysign(1.0, a);
  return s * fmax(0., fmin(fabs(a), b * s));
}
__device__ __forceinline__ double fi1(double x, double y, double z) {
  return amimd(x, amimd(y, z));
}
// met_roe2oh.f90:318-323
__device__ __forceinline__ double psi_h(double aa, double eps) {
  return 0.5 * (1. + copysign(1.0, fabs(aa) - eps)) * fabs(aa) +
         0.25 * (1. - copysign(1.0, fabs(aa) - eps)) * (aa * aa + eps * eps) / eps;
}

// slope difference of variable col on face q (1..nd) along dir, extended past
// the ends as met_roe2o.f90:75-88 does (face 0 = face 1, face nd+1 = face nd)
__device__ __forceinline__ double face_del(const double* __restrict__ t, long long n,
                                           long long inc, int p, int q, int nd) {
  const int qq = q < 1 ? 1 : (q > nd ? nd : q);
  const long long c = n + (long long)(qq - p) * inc;
  return t[c] - t[c - inc];
}

// TVD Roe dissipation of t(:,6:7) on one face (met_roe2o.f90:89-114 and the
// j, i twins; met_roe2oh.f90 with harten), into G[dir][0..1][n]
__global__ void __launch_bounds__(kTile) k_roe2o_face(const Blk* __restrict__ blks, Space sp,
                                                      int dir, int harten, double epsroe,
                                                      double gam, double gam1,
                                                      const double* __restrict__ t,
                                                      long long ld,
                                                      const double* __restrict__ sn,
                                                      double* __restrict__ G) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const long long n1 = n - inc;
  const double rro = 2 * t[n], rro1 = 2 * t[n1];
  const double u = t[ld + n] / rro + t[ld + n1] / rro1;
  const double v = t[2 * ld + n] / rro + t[2 * ld + n1] / rro1;
  const double w = t[3 * ld + n] / rro + t[3 * ld + n1] / rro1;
  const double s1 = sn_ptr(sn, B, dir, 0)[n], s2 = sn_ptr(sn, B, dir, 1)[n],
               s3 = sn_ptr(sn, B, dir, 2)[n];
  double coef;
  if (harten) {
    const double etot = t[4 * ld + n] / rro + t[4 * ld + n1] / rro1;
    const double q2 = 0.5 * (u * u + v * v + w * w);
    const double c = sqrt(gam * gam1 * (etot - q2));
    const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
    const double rlam = (u * s1 + v * s2 + w * s3) / cnds;
    coef = 0.5 * psi_h(rlam, epsroe * c) * cnds;
  } else {
    const double rlam = u * s1 + v * s2 + w * s3;
    coef = 0.5 * fabs(rlam);
  }
  double* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
  for (int a = 0; a < 2; ++a) {
    const double* tc = t + (5 + a) * ld;
    const double dm = face_del(tc, n, inc, p, p, nd);
    const double dm1 = face_del(tc, n, inc, p, p - 1, nd);
    const double dm2 = face_del(tc, n, inc, p, p + 1, nd);
    Gd[a * ld + n] = coef * (dm - fi1(dm1, dm, dm2));
  }
}

// d(:,6:7) of every cell of i 0..ni, j 0..nj, k 0..nk: per direction (k, j,
// i) the lower face subtracts, the upper face adds, where the face exists
// (the other two indices real); the ghost rows receive their one face
__global__ void __launch_bounds__(kTile) k_roe2o_acc(const Blk* __restrict__ blks, Space sp,
                                                     const double* __restrict__ G,
                                                     long long ld, double* __restrict__ d) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  --i;
  --j;
  --k;
  const long long n = cell_index(B, i, j, k);
  double acc[2] = {0., 0.};
  const int idx[3] = {i, j, k};
  const int lim[3] = {B.ni, B.nj, B.nk};
#pragma unroll
  for (int o = 0; o < 3; ++o) {
    const int dir = 2 - o;
    const int d1 = (dir + 1) % 3, d2 = (dir + 2) % 3;
    if (idx[d1] < 1 || idx[d1] > lim[d1] - 1 || idx[d2] < 1 || idx[d2] > lim[d2] - 1) continue;
    const int p = idx[dir], nd = lim[dir];
    const long long inc = ninc_of(B, dir);
    const double* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      if (p >= 1) acc[a] = acc[a] - Gd[a * ld + n];
      if (p + 1 <= nd) acc[a] = acc[a] + Gd[a * ld + n + inc];
    }
  }
  d[5 * ld + n] = acc[0];
  d[6 * ld + n] = acc[1];
}

// met_samut.f90:35-46 on the real cells: mut = v6 fv1 (x**3 as x*x*x)
__global__ void __launch_bounds__(kTile) k_samut(const Blk* __restrict__ blks, Space sp,
                                                 const double* __restrict__ v6,
                                                 const double* __restrict__ mu,
                                                 double* __restrict__ mut, double cv13) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double xkhi = v6[n] / mu[n];
  const double xkhi3 = xkhi * xkhi * xkhi;
  const double fv1 = xkhi3 / (xkhi3 + cv13);
  mut[n] = v6[n] * fv1;
}

// centred cell fluxes of the transport variables (sch_turb.f90:84-93)
__device__ __forceinline__ void turb_cell_flux(const double* __restrict__ v, long long ld,
                                               long long n, const double* const fd[6],
                                               double F[6]) {
  const double qx = v[ld + n] / v[n], qy = v[2 * ld + n] / v[n], qz = v[3 * ld + n] / v[n];
  const double t6 = v[5 * ld + n], t7 = v[6 * ld + n];
  F[0] = t6 * qx - fd[0][n];
  F[1] = t6 * qy - fd[1][n];
  F[2] = t6 * qz - fd[2][n];
  F[3] = t7 * qx - fd[3][n];
  F[4] = t7 * qy - fd[4][n];
  F[5] = t7 * qz - fd[5][n];
}

struct FdPtrs {
  const double* p[6];
};

// one face of sch_turb.f90:95-273 into G[dir][0..1][n]: interior faces sum
// the two cells' fluxes, boundary faces take twice the ghost cell's
__global__ void __launch_bounds__(kTile) k_turb_face(const Blk* __restrict__ blks, Space sp,
                                                     int dir, const double* __restrict__ v,
                                                     long long ld, FdPtrs fdp,
                                                     const double* __restrict__ sn,
                                                     double* __restrict__ G) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const double s1 = sn_ptr(sn, B, dir, 0)[n], s2 = sn_ptr(sn, B, dir, 1)[n],
               s3 = sn_ptr(sn, B, dir, 2)[n];
  double F[6];
  if (p >= 2 && p <= nd - 1) {
    double Fl[6];
    turb_cell_flux(v, ld, n, fdp.p, F);
    turb_cell_flux(v, ld, n - inc, fdp.p, Fl);
#pragma unroll
    for (int q = 0; q < 6; ++q) F[q] = F[q] + Fl[q];
  } else {
    turb_cell_flux(v, ld, p == 1 ? n - inc : n, fdp.p, F);
#pragma unroll
    for (int q = 0; q < 6; ++q) F[q] = 2. * F[q];
  }
  double* Gd = G + (long long)dir * 5 * ld;
  Gd[n] = F[0] * s1 + F[1] * s2 + F[2] * s3;
  Gd[ld + n] = F[3] * s1 + F[4] * s2 + F[5] * s3;
}

// per-cell sum in the reference's order, then u6 = 0.5 u6 - vol ts6 - d6
// (sch_turb.f90:276-287) and the same for 7
__global__ void __launch_bounds__(kTile) k_turb_acc(const Blk* __restrict__ blks, Space sp,
                                                    const double* __restrict__ G, long long ld,
                                                    const double* __restrict__ vol,
                                                    const double* __restrict__ ts6,
                                                    const double* __restrict__ ts7,
                                                    const double* __restrict__ d,
                                                    double* __restrict__ u) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double acc[2] = {0., 0.};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const bool upper_first = (p == 1) && nd >= 3;
    const double* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const double gl = Gd[a * ld + n], gu = Gd[a * ld + n + inc];
      if (upper_first) {
        acc[a] = acc[a] + gu;
        acc[a] = acc[a] - gl;
      } else {
        acc[a] = acc[a] - gl;
        acc[a] = acc[a] + gu;
      }
    }
  }
  u[5 * ld + n] = 0.5 * acc[0] - vol[n] * ts6[n] - d[5 * ld + n];
  u[6 * ld + n] = 0.5 * acc[1] - vol[n] * ts7[n] - d[6 * ld + n];
}

}  // namespace

cudaError_t launch_fludc(long long n0, long long n1, const double* mu, const double* mut,
                         double* const fd[6], double alfak, double alfae, cudaStream_t st) {
  if (n1 >= n0)
    k_fludc<<<(int)((n1 - n0 + 256) / 256), 256, 0, st>>>(n0, n1, mu, mut, fd[0], fd[1], fd[2],
                                                          fd[3], fd[4], fd[5], alfak, alfae);
  return cudaGetLastError();
}

cudaError_t launch_fludcsa(long long n0, long long n1, const double* s6, const double* mu,
                           double* const fd[6], double sigma, cudaStream_t st) {
  const double sigma1 = 1. / sigma;
  if (n1 >= n0)
    k_fludcsa<<<(int)((n1 - n0 + 256) / 256), 256, 0, st>>>(n0, n1, s6, mu, fd[0], fd[1],
                                                            fd[2], fd[3], fd[4], fd[5], sigma1);
  return cudaGetLastError();
}

cudaError_t launch_samut(const Blk* blks, Space cells, const double* v6, const double* mu,
                         double* mut, cudaStream_t st) {
  const double cv1 = 7.1;  // atlecdon.f90:200
  if (cells.ntiles > 0)
    k_samut<<<grid_of(cells), kTile, 0, st>>>(blks, cells, v6, mu, mut, cv1 * cv1 * cv1);
  return cudaGetLastError();
}

cudaError_t launch_sch_turb(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                            const double* v, long long ld, const double* const fd[6],
                            const double* ts6, const double* ts7, const double* d,
                            const double* sn, const double* vol, double* G, double* u,
                            cudaStream_t st) {
  FdPtrs fdp;
  for (int q = 0; q < 6; ++q) fdp.p[q] = fd[q];
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles > 0)
      k_turb_face<<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, v, ld, fdp, sn, G);
  }
  if (cells.ntiles > 0)
    k_turb_acc<<<grid_of(cells), kTile, 0, st>>>(blks, cells, G, ld, vol, ts6, ts7, d, u);
  return cudaGetLastError();
}

cudaError_t launch_roe2o(const Blk* blks, const SpaceBuf* faces, Space cells_ext, int l0,
                         int harten, double epsroe, double gam, double gam1, const double* t,
                         long long ld, const double* sn, double* G, double* d,
                         cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles > 0)
      k_roe2o_face<<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, harten, epsroe, gam, gam1, t,
                                                  ld, sn, G);
  }
  if (cells_ext.ntiles > 0)
    k_roe2o_acc<<<grid_of(cells_ext), kTile, 0, st>>>(blks, cells_ext, G, ld, d);
  return cudaGetLastError();
}

}  // namespace cns
