// cns_sa.cu -- the Spalart-Allmaras source of the reference: the Green-Gauss
// cell gradients of teq_grads.f90 (velocity gradients for teq_gradv.f90,
// the gradients of rho nu~ and rho inside met_difsa.f90 / met_smsa.f90) and
// the source term met_smsa.f90 with its derivative bound.
//
// Gradient: one thread per real cell evaluates the face values S (s_upper +
// s_lower) (interior) or (2 S) s_ghost (boundary) of its six faces and sums
// them in the reference's order -- directions k, j, i; within a direction
// the lower face subtracted then the upper added, the first cell of a line
// (lower face on the boundary) taking its upper face first -- and
// multiplies by 0.5 / vol.
// FP64, --fmad=false: bit-identical gradients.  The source uses exp and a
// real power, whose last bit may differ from the host libm's.
#include "cns_kernels.cuh"
#include "cns_pmath.h"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

// SA constants (atlecdon.f90:193-204)
constexpr double kCb1 = 0.1355, kSigma = 2. / 3., kCb2 = 0.622, kKappa = 0.41;
constexpr double kCv1 = 7.1, kCw2 = 0.3, kCw3 = 2., kCt3 = 1.1, kCt4 = 2.;
// the modified vorticity of Allmaras, Johnson & Spalart (ICCFD7-1902, 2012,
// eq. 12), used by the flagged non-reference source fix
constexpr double kCv2 = 0.7, kCv3 = 0.9;

__device__ __forceinline__ double pow6(double x) {  // gcc's x**6: x3 * x3
  const double x3 = x * x * x;
  return x3 * x3;
}

// scalar q of cell n: mode 0 = the velocity component q (teq_gradv.f90:
// t(:,q+1) / max(t(:,1), 1e-20)), mode 1 = the field f, mode 2 = the
// transport variable q per unit mass (met_gradtr.f90:78-84: s(:,6+q) / s(:,1)),
// mode 3 = sqrt(s(:,6) / s(:,1)) (met_bark.f90:91-99)
__device__ __forceinline__ double scalar_of(int mode, const double* __restrict__ v,
                                            const double* __restrict__ f, long long ld,
                                            long long n, int q) {
  if (mode == 0) return v[(q + 1) * ld + n] / fmax(v[n], 1.e-20);
  if (mode == 2) return v[(5 + q) * ld + n] / v[n];
  if (mode == 3) return sqrt(v[5 * ld + n] / v[n]);
  return f[q * ld + n];
}

// the scalars of modes 0 and 2 over the flat cell range [n0, n1) into
// sc[q][ld], once per cell (the gradient kernel reads each six more times)
template <int NSC>
__global__ void __launch_bounds__(256) k_teq_scalars(int mode, const double* __restrict__ v,
                                                    long long ld, long long n0, long long n1,
                                                    double* __restrict__ sc) {
  const long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n1) return;
#pragma unroll
  for (int q = 0; q < NSC; ++q) sc[q * ld + n] = scalar_of(mode, v, nullptr, ld, n, q);
}

// teq_grads.f90:38-346 per real cell: the Green-Gauss sum over the six faces
// in the reference's order -- directions k, j, i; within a direction the
// lower face subtracted then the upper one added, except that the first cell
// of a line (lower face on the boundary) takes its upper face first -- then
// times 0.5 / vol.  A face value is S (s_upper + s_lower) inside the block
// and (S * 2) s_ghost on a boundary face; every cell evaluates its six face
// values itself (the face's two cells compute the same operands in the same
// order, so the value is the one a stored face buffer would hold).
template <int NSC>
__global__ void __launch_bounds__(kTile) k_teq_cell(const Blk* __restrict__ blks, Space sp,
                                                    int mode, const double* __restrict__ v,
                                                    const double* __restrict__ f, long long ld,
                                                    const double* __restrict__ sn,
                                                    const double* __restrict__ vol,
                                                    double* __restrict__ out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double s0[NSC];
#pragma unroll
  for (int q = 0; q < NSC; ++q) s0[q] = scalar_of(mode, v, f, ld, n, q);
  double acc[NSC * 3];
#pragma unroll
  for (int a = 0; a < NSC * 3; ++a) acc[a] = 0.;
#pragma unroll
  for (int o = 0; o < 3; ++o) {
    const int dir = 2 - o;
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const bool upper_first = (p == 1) && nd >= 3;
    const double* s0p = sn_ptr(sn, B, dir, 0);
    const double* s1p = sn_ptr(sn, B, dir, 1);
    const double* s2p = sn_ptr(sn, B, dir, 2);
    const double Sl[3] = {s0p[n], s1p[n], s2p[n]};
    const double Su[3] = {s0p[n + inc], s1p[n + inc], s2p[n + inc]};
#pragma unroll
    for (int q = 0; q < NSC; ++q) {
      const double sl = scalar_of(mode, v, f, ld, n - inc, q);
      const double su = scalar_of(mode, v, f, ld, n + inc, q);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double gl = p >= 2 ? Sl[c] * (s0[q] + sl) : Sl[c] * 2 * sl;
        const double gu = p + 1 <= nd - 1 ? Su[c] * (su + s0[q]) : Su[c] * 2 * su;
        double& x = acc[q * 3 + c];
        if (upper_first) {
          x = x + gu;
          x = x - gl;
        } else {
          x = x - gl;
          x = x + gu;
        }
      }
    }
  }
  // teq_grads.f90:338-346
  const double ts = copysign(0.5, -vol[n]);
  const double vols = (0.5 + ts) * 0.000001 + (0.5 - ts) * vol[n];
  const double c0 = 0.5 / (vols + 2.2250738585072014e-308);
#pragma unroll
  for (int a = 0; a < NSC * 3; ++a) out[a * ld + n] = acc[a] * c0;
}

// met_smsa.f90:102-176 on the real cells; dv (global index, 9 rows: xx xy
// xz yx yy yz zx zy zz), grt / grr: the gradients of rho nu~ and of rho
__global__ void __launch_bounds__(kTile) k_smsa(
    const Blk* __restrict__ blks, Space sp, long long ld, const double* __restrict__ v,
    const double* __restrict__ mu, const double* __restrict__ dist,
    const double* __restrict__ dv, const double* __restrict__ grt,
    const double* __restrict__ grr, const double* __restrict__ fd5x,
    const double* __restrict__ fd5y, const double* __restrict__ fd5z,
    double* __restrict__ ts6, double* __restrict__ ts7, double* __restrict__ cfke, int fix) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const long long m = n - B.npc;  // met_smsa.f90:177 reads txxf5x.. at this index
  const double cw1 = kCb1 / (kKappa * kKappa) + (1 + kCb2) / kSigma;
  const double kappa2 = kKappa * kKappa, uns6 = 1. / 6., cv13 = kCv1 * kCv1 * kCv1;
  const double cw36 = pow6(kCw3), cv133 = 3. * cv13, ct42 = 2. * kCt4, cb2sig = kCb2 / kSigma;
  // met_difsa.f90:96-101
  double sdif = grt[n] * fd5x[n] + grt[ld + n] * fd5y[n] + grt[2 * ld + n] * fd5z[n];
  sdif = sdif * kCb2 / kSigma;
  const double v6 = v[5 * ld + n], v1 = v[n];
  const double a1 = dv[7 * ld + n] - dv[5 * ld + n];  // dvzy - dvyz
  const double a2 = dv[2 * ld + n] - dv[6 * ld + n];  // dvxz - dvzx
  const double a3 = dv[3 * ld + n] - dv[ld + n];      // dvyx - dvxy
  const double vort = sqrt(a1 * a1 + a2 * a2 + a3 * a3);
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
  if (!fix || sbar >= -kCv2 * vort) {
    stilde = vort + sbar;
  } else {
    stilde = vort + vort * (kCv2 * kCv2 * vort + kCv3 * sbar) / ((kCv3 - 2. * kCv2) * vort - sbar);
  }
  if (fix && !(stilde > 0.)) {
    rtilde = 1.;
  } else {
    rtilde = nutilde / (stilde * kapd2);
    rtilde = fmin(rtilde, 1.);
  }
  const double rtil6 = pow6(rtilde);
  const double ft2 = kCt3 * cns_exp(-kCt4 * xkhi2);
  const double sm1 = kCb1 * (1. - ft2) * stilde * v6;
  const double xg = rtilde + kCw2 * (rtil6 - rtilde);
  const double xg6 = pow6(xg);
  const double fw = xg * cns_pow((1. + cw36) / (xg6 + cw36), uns6);
  const double sm2 = -(cw1 * fw - kCb1 * ft2 / kappa2) * v6 * nutilde / dist2;
  ts6[n] = sm1 + sm2 + sdif;
  ts7[n] = 0.;
  const double xkhi4 = xkhi3 * xkhi;
  const double dfv1 =
      (fix && !(xkhi4 > 0.)) ? 0. : cv133 * (fv1 * fv1) / (mu[n] * xkhi4);
  const double t1 = 1. + xkhi * fv1;
  const double dfv2 = (xkhi2 * dfv1 - 1. / mu[n]) / (t1 * t1);
  const double dst = (fv2 / v1 + nutilde * dfv2) / kapd2;
  double dpr, dxg, dfw;
  if (!fix) {
    dpr = (1. / v1 - nutilde * dst / stilde) / (stilde * kapd2);
    dxg = dpr * (1. + kCw2 * (6. * rtil6 / rtilde - 1.));
    dfw = (1. - xg6 / (xg6 + cw36)) * fw * dxg / xg;
  } else {
    // r is constant where it is clipped; r^5 without r^6 / r; no division
    // by xg = 0
    dpr = (rtilde < 1. && stilde > 0.)
              ? (1. / v1 - nutilde * dst / stilde) / (stilde * kapd2) : 0.;
    const double r2 = rtilde * rtilde;
    dxg = dpr * (1. + kCw2 * (6. * (r2 * r2 * rtilde) - 1.));
    dfw = xg != 0. ? (1. - xg6 / (xg6 + cw36)) * fw * dxg / xg : 0.;
  }
  const double dft2 = -ct42 * xkhi * ft2;
  const double dsm1 = kCb1 * ((1. - ft2) * (stilde + dst * v6) - stilde * v6 * dft2);
  const double dsm2 = 2. * sm2 / v6 - (cw1 * dfw - kCb1 * dft2 / kappa2) * nutilde * v6 / dist2;
  const double dsdif =
      -cb2sig * (fd5x[m] * grr[n] + fd5y[m] * grr[ld + n] + fd5z[m] * grr[2 * ld + n]) /
      (v1 * v1);
  cfke[n] = fabs(dsm1 + dsm2 + dsdif);
}

// impli2_eqt_3d.f90:93-103: rv and the time-step part of the diagonal
__global__ void __launch_bounds__(kTile) k_i2_cell(const Blk* __restrict__ blks, Space sp,
                                                   const double* __restrict__ v,
                                                   const double* __restrict__ mu,
                                                   const double* __restrict__ mut,
                                                   const double* __restrict__ dt,
                                                   const double* __restrict__ cfke,
                                                   const double* __restrict__ vol, double cmt,
                                                   double* __restrict__ rv,
                                                   double* __restrict__ cd) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  rv[n] = (mu[n] + mut[n] / cmt) / v[n];
  cd[n] = vol[n] / dt[n] + cfke[n] * vol[n];
}

// impli2_eqt_3d.f90:104-160: face velocity flux u_dir and coefficient of one
// face (boundary faces included)
__global__ void __launch_bounds__(kTile) k_i2_face(const Blk* __restrict__ blks, Space sp,
                                                   int dir, const double* __restrict__ v,
                                                   long long ld, const double* __restrict__ sn,
                                                   const double* __restrict__ vol,
                                                   const double* __restrict__ rv,
                                                   double* __restrict__ uf,
                                                   double* __restrict__ ce) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const long long inc = ninc_of(B, dir), nl = n - inc;
  const double s1 = sn_ptr(sn, B, dir, 0)[n], s2 = sn_ptr(sn, B, dir, 1)[n],
               s3 = sn_ptr(sn, B, dir, 2)[n];
  const double cnds = s1 * s1 + s2 * s2 + s3 * s3;
  const double uu = 0.5 * (v[ld + n] / v[n] + v[ld + nl] / v[nl]);
  const double vv = 0.5 * (v[2 * ld + n] / v[n] + v[2 * ld + nl] / v[nl]);
  const double ww = 0.5 * (v[3 * ld + n] / v[n] + v[3 * ld + nl] / v[nl]);
  const double u = 0.5 * (uu * s1 + vv * s2 + ww * s3);
  uf[(long long)dir * ld + n] = u;
  ce[(long long)dir * ld + n] = fabs(u) + (rv[n] + rv[nl]) * cnds / (vol[n] + vol[nl]);
}

// impli2_eqt_3d.f90:161-171
__global__ void __launch_bounds__(kTile) k_i2_diag(const Blk* __restrict__ blks, Space sp,
                                                   long long ld, const double* __restrict__ ce,
                                                   double* __restrict__ cd) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long m = cell_index(B, i, j, k);
  cd[m] = cd[m] + ce[m] + ce[m + 1] + ce[ld + m] + ce[ld + m + B.nid] + ce[2 * ld + m] +
          ce[2 * ld + m + B.nijd];
}

// one alternating-line sweep of direction dir (impli2_eqt_3d.f90:172-291),
// in two kernels.  k_i2_rhs (a thread per real cell, fully parallel): the
// tridiagonal coefficients ai, bi, cci of the cell and the right-hand sides
// di6, di7, whose neighbours in the two other directions come from the
// previous iterate.  k_i2_line (a thread per line): the backward recurrence
// into al/b6/b7 (written over ai/bi/cci) and the forward substitution into
// the new iterate -- the only sequential part, reading five values per cell.
// The expressions and their order are the reference's, so the split is
// bit-identical to evaluating everything inside the line loop.
__global__ void __launch_bounds__(kTile) k_i2_rhs(
    const Blk* __restrict__ blks, Space sp, int dir, long long ld,
    const double* __restrict__ u, const double* __restrict__ uf,
    const double* __restrict__ ce, const double* __restrict__ cd,
    const double* __restrict__ o6, const double* __restrict__ o7, double* __restrict__ ta,
    double* __restrict__ tb, double* __restrict__ tc, double* __restrict__ d6,
    double* __restrict__ d7) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const int oa = dir == 0 ? 1 : 0, ob = dir == 2 ? 1 : 2;
  const long long inc = ninc_of(B, dir), inca = ninc_of(B, oa), incb = ninc_of(B, ob);
  const double *ua = uf + (long long)oa * ld, *ub = uf + (long long)ob * ld,
               *ud = uf + (long long)dir * ld;
  const double *ca = ce + (long long)oa * ld, *cb = ce + (long long)ob * ld,
               *cdir = ce + (long long)dir * ld;
  const long long m = cell_index(B, i, j, k);
  const double td = -ua[m + inca] + ua[m] - ub[m + incb] + ub[m];
  const double tpa = ca[m + inca] - ua[m + inca], tma = ca[m] + ua[m];
  const double tpb = cb[m + incb] - ub[m + incb], tmb = cb[m] + ub[m];
  d6[m] = -u[5 * ld + m] + td * o6[m] + tma * o6[m - inca] + tpa * o6[m + inca] +
          tmb * o6[m - incb] + tpb * o6[m + incb];
  d7[m] = -u[6 * ld + m] + td * o7[m] + tma * o7[m - inca] + tpa * o7[m + inca] +
          tmb * o7[m - incb] + tpb * o7[m + incb];
  ta[m] = cdir[m] + ud[m];
  tb[m] = cd[m] + ud[m + inc] - ud[m];
  tc[m] = -cdir[m + inc] + ud[m + inc];
}

// The recurrence reads the coefficients from arrays it does not write, so
// the loads of the next kLineUnroll cells are issued while the current ones
// are consumed (a thread walks its line alone: memory latency, not
// bandwidth, bounds this kernel; a chunk of eight dependent division steps
// covers an HBM round trip).  Few threads run it, so it may use up to 255
// registers a thread for the two chunks in flight.
constexpr int kLineUnroll = 8;
// CTAs of kLineCta threads, kTile / kLineCta per tile of lines: a direction
// has only as many threads as lines (8192 i-lines on a 256x128x64 block),
// so small CTAs spread them over every SM instead of a third of them
constexpr int kLineCta = 32;

// RCP: the reduced-precision forms' variant, one division per step (the
// reciprocal of the pivot times each numerator).  The sweep only shapes the
// pseudo-time increment, so the fixed point is unchanged; the dependent
// chain per step shrinks from three divisions to one.
template <bool RCP>
__global__ void __launch_bounds__(kLineCta, 1) k_i2_line(const Blk* __restrict__ blks, Space sp,
                                                      int dir, const double* __restrict__ ta,
                                                      const double* __restrict__ tb,
                                                      const double* __restrict__ tc,
                                                      const double* __restrict__ d6,
                                                      const double* __restrict__ d7,
                                                      double* __restrict__ al,
                                                      double* __restrict__ b6,
                                                      double* __restrict__ b7,
                                                      double* __restrict__ n6,
                                                      double* __restrict__ n7) {
  int b, i, j, k;
  constexpr int kSub = kTile / kLineCta;
  if (!space_elem_at(sp, blockIdx.x / kSub, (blockIdx.x % kSub) * kLineCta + threadIdx.x, b, i,
                     j, k))
    return;
  const Blk& B = blks[b];
  const long long inc = ninc_of(B, dir);
  const int nc = nd_of(B, dir) - 1;             // cells on the line
  const long long m1 = cell_index(B, i, j, k);  // the line's first cell (p = 1)
  constexpr int U = kLineUnroll;
  // backward recurrence over p = nc .. 1 (step q = nc - p); the values at
  // p + 1 carried, zero past the end (the reference's never-written ghost
  // entries)
  double aln = 0., b6n = 0., b7n = 0.;
  double xa[U], xb[U], xc[U], x6[U], x7[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int p = nc - u;
    if (p >= 1) {
      const long long m = m1 + (long long)(p - 1) * inc;
      xa[u] = ta[m];
      xb[u] = tb[m];
      xc[u] = tc[m];
      x6[u] = d6[m];
      x7[u] = d7[m];
    }
  }
  for (int q0 = 0; q0 < nc; q0 += U) {
    double ya[U], yb[U], yc[U], y6[U], y7[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      ya[u] = xa[u];
      yb[u] = xb[u];
      yc[u] = xc[u];
      y6[u] = x6[u];
      y7[u] = x7[u];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = nc - (q0 + U + u);
      if (p >= 1) {
        const long long m = m1 + (long long)(p - 1) * inc;
        xa[u] = ta[m];
        xb[u] = tb[m];
        xc[u] = tc[m];
        x6[u] = d6[m];
        x7[u] = d7[m];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = nc - (q0 + u);
      if (p >= 1) {
        const long long m = m1 + (long long)(p - 1) * inc;
        const double den = yb[u] + yc[u] * aln;
        if (RCP) {
          const double r = 1. / den;
          aln = ya[u] * r;
          b6n = (y6[u] - yc[u] * b6n) * r;
          b7n = (y7[u] - yc[u] * b7n) * r;
        } else {
          aln = ya[u] / den;
          b6n = (y6[u] - yc[u] * b6n) / den;
          b7n = (y7[u] - yc[u] * b7n) / den;
        }
        al[m] = aln;
        b6[m] = b6n;
        b7[m] = b7n;
      }
    }
  }
  // forward substitution over p = 1 .. nc (the cell before the line's first
  // is a ghost: 0), the next chunk's al/b6/b7 (this thread's own stores of
  // the backward pass) loaded ahead in the same way
  double w6 = 0., w7 = 0.;
  double fa[U], f6[U], f7[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const int p = 1 + u;
    if (p <= nc) {
      const long long m = m1 + (long long)(p - 1) * inc;
      fa[u] = al[m];
      f6[u] = b6[m];
      f7[u] = b7[m];
    }
  }
  for (int p0 = 1; p0 <= nc; p0 += U) {
    double ga[U], g6[U], g7[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      ga[u] = fa[u];
      g6[u] = f6[u];
      g7[u] = f7[u];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = p0 + U + u;
      if (p <= nc) {
        const long long m = m1 + (long long)(p - 1) * inc;
        fa[u] = al[m];
        f6[u] = b6[m];
        f7[u] = b7[m];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int p = p0 + u;
      if (p <= nc) {
        const long long m = m1 + (long long)(p - 1) * inc;
        w6 = ga[u] * w6 + g6[u];
        w7 = ga[u] * w7 + g7[u];
        n6[m] = w6;
        n7[m] = w7;
      }
    }
  }
}

// v(:,6:7) += dw on the real cells (impli2_eqt_3d.f90:321-329)
__global__ void __launch_bounds__(kTile) k_i2_update(const Blk* __restrict__ blks, Space sp,
                                                     long long ld,
                                                     const double* __restrict__ w6,
                                                     const double* __restrict__ w7,
                                                     double* __restrict__ v) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  v[5 * ld + n] = v[5 * ld + n] + w6[n];
  v[6 * ld + n] = v[6 * ld + n] + w7[n];
}

// ---------------------------------------------------------------------------
// wall distance (atcaldis3.f90 -> atdist_3.f90, every block attached to every
// wall): facet centres of the adiabatic-wall boundaries (atccfp.f90:60-72) in
// boundary list order, then per real cell the cell centre (atccc.f90:36-60)
// and the smallest squared distance to a facet centre.  The facet centres are
// staged through shared memory in chunks, every thread of the CTA scanning
// the same chunk; the minimum of a set is order-free, so dist is bit-exact.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_wall_facets(Bnd bd, const Blk* __restrict__ blks,
                                                    const long long* __restrict__ went,
                                                    long long nw, const double* __restrict__ x,
                                                    const double* __restrict__ y,
                                                    const double* __restrict__ z,
                                                    double* __restrict__ par) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nw) return;
  const long long e = went[q];
  const int bb = bd.ent_bnd[e];
  const Blk& B = blks[bd.blk[bb]];
  const int face = bd.face[bb], dir = face / 2;
  const long long dm1 = dir == 0 ? (long long)B.nid : 1LL;
  const long long dm2 = dir == 2 ? (long long)B.nid : B.nijd;
  const long long nci = bd.ncin[e] + ((face & 1) ? ninc_of(B, dir) : 0LL);
  par[q] = (x[nci] + x[nci + dm1] + x[nci + dm2] + x[nci + dm1 + dm2]) * .25;
  par[nw + q] = (y[nci] + y[nci + dm1] + y[nci + dm2] + y[nci + dm1 + dm2]) * .25;
  par[2 * nw + q] = (z[nci] + z[nci + dm1] + z[nci + dm2] + z[nci + dm1 + dm2]) * .25;
}

constexpr int kWallChunk = 1024;

__global__ void __launch_bounds__(kTile) k_wall_dist(const Blk* __restrict__ blks, Space sp,
                                                     const double* __restrict__ x,
                                                     const double* __restrict__ y,
                                                     const double* __restrict__ z,
                                                     const double* __restrict__ par,
                                                     long long nw, double* __restrict__ dist) {
  __shared__ double sx[kWallChunk], sy[kWallChunk], sz[kWallChunk];
  int b, i, j, k;
  const bool live = space_elem(sp, threadIdx.x, b, i, j, k);
  double xcc = 0., ycc = 0., zcc = 0.;
  long long n = 0;
  if (live) {
    const Blk& B = blks[b];
    n = cell_index(B, i, j, k);
    const long long a = 1, bj = B.nid, n1 = n + B.nijd;
    xcc = ((x[n] + x[n + a] + x[n + bj] + x[n + a + bj]) +
           (x[n1] + x[n1 + a] + x[n1 + bj] + x[n1 + a + bj])) * 0.125;
    ycc = ((y[n] + y[n + a] + y[n + bj] + y[n + a + bj]) +
           (y[n1] + y[n1 + a] + y[n1 + bj] + y[n1 + a + bj])) * 0.125;
    zcc = ((z[n] + z[n + a] + z[n + bj] + z[n + a + bj]) +
           (z[n1] + z[n1 + a] + z[n1 + bj] + z[n1 + a + bj])) * 0.125;
  }
  double dmini = 1.e+20;
  for (long long f0 = 0; f0 < nw; f0 += kWallChunk) {
    const int cnt = (int)min((long long)kWallChunk, nw - f0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      sx[q] = par[f0 + q];
      sy[q] = par[nw + f0 + q];
      sz[q] = par[2 * nw + f0 + q];
    }
    __syncthreads();
    for (int q = 0; q < cnt; ++q) {
      const double d2 = (xcc - sx[q]) * (xcc - sx[q]) + (ycc - sy[q]) * (ycc - sy[q]) +
                        (zcc - sz[q]) * (zcc - sz[q]);
      dmini = d2 < dmini ? d2 : dmini;
    }
  }
  if (live) dist[n] = sqrt(dmini);
}

// met_bord.f90:24-258 (kparoi = 0) on v(:,6:7): coincident ghosts average
// with the partner's interior cell (met_rbvc.f90:53-62), idd ghosts take
// (rokinf, roeinf), walls 0, extrapolation and outlet the interior cell
__global__ void __launch_bounds__(256) k_turb_bord(Bnd bd, double* v, long long ld,
                                                  double rokinf, double roeinf) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int bb = bd.ent_bnd[e];
  const long long nd = bd.ncbd[e], ni = bd.ncin[e];
  double* v6 = v + 5 * ld;
  double* v7 = v + 6 * ld;
  switch (bd.type[bb]) {
    case BC_RC: {
      const long long nc = bd.ncin[bd.mpb[bd.partner[bb]] + (e - bd.mpb[bb])];
      v6[nd] = 0.5 * (v6[ni] + v6[nc]);
      v7[nd] = 0.5 * (v7[ni] + v7[nc]);
      break;
    }
    case BC_IDD:
      v6[nd] = rokinf;
      v7[nd] = roeinf;
      break;
    case BC_PARA:
    case BC_LP2:  // met_bord.f90:296-305 with kparoi = 0
      v6[nd] = 0.;
      v7[nd] = 0.;
      break;
    default:
      v6[nd] = v6[ni];
      v7[nd] = v7[ni];
      break;
  }
}

// ---------------------------------------------------------------------------
// wall laws of the adiabatic wall-law walls 'lp2' (lparoi = 1; constants of
// rbord.f90:377-379; air, iflu = 1; no transition, ktransi = 0).  lpsa1.f90
// and lparoi1.f90 share the friction law: the unit tangent t of the first
// cell's velocity, the Crocco wall temperature, the wall viscosity
// (Sutherland) and density, Van Driest's compressible velocity, and the wall
// stress top of the linear law (u+ y+ <= yp0^2) or of ten fixed-point passes
// of the log law.  One launch per boundary in list order: a corner cell next
// to two such walls sees the writes of the earlier boundary first, as in the
// reference's boundary loop.
struct WallFriction {
  double t1, t2, t3, n1, n2, n3, top, dudy, rop, mup;
};

__device__ __forceinline__ WallFriction wall_friction(const Bnd& bd, long long e, Phys ph,
                                                      WallLaw wl, long long ld,
                                                      const double* v, const double* mu,
                                                      const double* mut, const double* dist,
                                                      const double* temp) {
  const long long ni = bd.ncin[e];
  WallFriction f;
  const double v1x = v[ld + ni] / v[ni], v1y = v[2 * ld + ni] / v[ni],
               v1z = v[3 * ld + ni] / v[ni];
  f.n1 = bd.nxn[e];
  f.n2 = bd.nyn[e];
  f.n3 = bd.nzn[e];
  const double tn = v1x * f.n1 + v1y * f.n2 + v1z * f.n3;
  double t1 = v1x - tn * f.n1, t2 = v1y - tn * f.n2, t3 = v1z - tn * f.n3;
  const double tt = sqrt(t1 * t1 + t2 * t2 + t3 * t3);
  t1 = t1 / tt;
  t2 = t2 / tt;
  t3 = t3 / tt;
  f.t1 = t1;
  f.t2 = t2;
  f.t3 = t3;
  double v1t = v1x * t1 + v1y * t2 + v1z * t3;
  const double temp1 = temp[ni];
  const double pka = ph.cp * (mu[ni] / ph.pr + mut[ni] / ph.prt);
  const double pkb = mu[ni] + mut[ni];
  const double tparoi = temp1 + 0.5 * pkb * (v1t * v1t) / pka;
  const double sv = ph.suth_a;
  const double mup = mu[ni] * sqrt(tparoi / temp1) * (1. + sv / temp1) / (1. + sv / tparoi);
  const double rop = v[ni] * temp1 / tparoi;
  f.rop = rop;
  f.mup = mup;
  const double co = sqrt(2. * pka * tparoi / pkb);
  v1t = co * cns_asin(v1t / co);
  const double d = dist[ni];
  const double upyp1 = rop * v1t * d / mup;
  double top = mup * v1t / d;
  if (upyp1 <= wl.yp0 * wl.yp0) {
    f.dudy = top / mup;
  } else {
    for (int it = 0; it < 10; ++it) {
      const double q = cns_log(d * sqrt(rop * top) / mup) / wl.vkar + wl.cllog;
      top = rop * (v1t * v1t) / (q * q);
    }
    f.dudy = sqrt(top / rop) / (wl.vkar * d);
  }
  f.top = top;
  return f;
}

// lpsa1.f90:70-236: mut and rho nu~ of the first cell from the wall law
// (mut = rho (kappa d)^2 du/dy (1 - exp(-y+/26))^2, then nu~ from the
// closed-form root of mut = rho nu~ fv1), the wall ghost's rho nu~ = 0
__global__ void __launch_bounds__(128) k_lpsa1(Bnd bd, long long e0, int cnt, Phys ph,
                                              WallLaw wl, long long ld, double* v,
                                              const double* __restrict__ mu, double* mut,
                                              const double* __restrict__ dist,
                                              const double* __restrict__ temp) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= cnt) return;
  const long long e = e0 + m, ni = bd.ncin[e], nc = bd.ncbd[e];
  const WallFriction f = wall_friction(bd, e, ph, wl, ld, v, mu, mut, dist, temp);
  const double d = dist[ni];
  const double yplus1 = d * sqrt(f.top * f.rop) / f.mup;
  const double ex = 1. - cns_exp(-yplus1 / 26.);
  const double mt = v[ni] * (wl.vkar * wl.vkar) * (d * d) * f.dudy * (ex * ex);
  mut[ni] = mt;
  const double c13 = 1. / 3., c18 = 1. / 18.;
  const double ca = mt;
  const double mu1 = mu[ni];
  const double cb = mu1 * mu1 * mu1 * mt * (wl.cv1 * wl.cv1 * wl.cv1);
  const double ca2 = ca * ca;
  const double c1 = cb * sqrt(3.) * sqrt(256. * cb + 27. * (ca2 * ca2));
  const double c2 = 0.5 * cb * ca2 + c18 * c1;
  const double c3 = -(0.5 * cb * ca2) + c18 * c1;
  const double p3 = cns_pow(c3, c13), p2 = cns_pow(c2, c13);
  const double c4 = 4. * fabs(p3 - p2);
  const double rc4 = sqrt(ca2 + c4);
  const double rnut = 0.25 * (ca + rc4) +
                      0.25 * sqrt(2.) *
                          sqrt(ca2 * rc4 - 2. * p3 * rc4 + 2. * p2 * rc4 + ca2 * ca) /
                          cns_pow(rc4, 0.5);
  v[5 * ld + ni] = fmax(rnut, wl.epsk);
  v[5 * ld + nc] = 0.;
}

// lparoi1.f90:77-229: the wall stress tensor top (t n + n t) in the wall
// ghost and the first cell, the first cell's heat flux -n top (u . t) and
// none in the ghost
__global__ void __launch_bounds__(128) k_lparoi1(Bnd bd, long long e0, int cnt, Phys ph,
                                                WallLaw wl, long long ld,
                                                const double* __restrict__ v,
                                                const double* __restrict__ mu,
                                                const double* __restrict__ mut,
                                                const double* __restrict__ dist,
                                                const double* __restrict__ temp, double* tau) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= cnt) return;
  const long long e = e0 + m, ni = bd.ncin[e], nc = bd.ncbd[e];
  const WallFriction f = wall_friction(bd, e, ph, wl, ld, v, mu, mut, dist, temp);
  const double top = f.top;
  const double t[6] = {2. * f.t1 * f.n1 * top,           (f.t2 * f.n1 + f.t1 * f.n2) * top,
                       (f.t1 * f.n3 + f.t3 * f.n1) * top, 2. * f.t2 * f.n2 * top,
                       (f.t2 * f.n3 + f.t3 * f.n2) * top, 2. * f.t3 * f.n3 * top};
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    tau[a * ld + nc] = t[a];
    tau[a * ld + ni] = t[a];
  }
  const double qc1 =
      top * ((v[ld + ni] * f.t1 + v[2 * ld + ni] * f.t2 + v[3 * ld + ni] * f.t3) / v[ni]);
  tau[6 * ld + ni] = -f.n1 * qc1;
  tau[7 * ld + ni] = -f.n2 * qc1;
  tau[8 * ld + ni] = -f.n3 * qc1;
  tau[6 * ld + nc] = 0.;
  tau[7 * ld + nc] = 0.;
  tau[8 * ld + nc] = 0.;
}

// impli2_eqt_3d.f90:384-405: the increments of rho nu~ and of the second
// variable vanish in the first cell of every wall-law wall
__global__ void __launch_bounds__(256) k_i2_wall_freeze(const long long* __restrict__ ni,
                                                       long long cnt, double* w6, double* w7) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cnt) return;
  w6[ni[q]] = 0.;
  w7[ni[q]] = 0.;
}

// met_rbse.f90:19-31 (non-coincident boundaries: ghost = interior) and
// met_rbsc.f90:38-70 (coincident: average with the partner's interior cell)
// on the six diffusion densities fd (6 rows of ld)
struct Fd6 {
  double* p[6];
};

__global__ void __launch_bounds__(256) k_fd_ghosts(Bnd bd, Fd6 fd) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int bb = bd.ent_bnd[e];
  const long long nd = bd.ncbd[e], ndm = bd.ncin[e];
  if (bd.type[bb] == BC_RC) {
    const long long nc = bd.ncin[bd.mpb[bd.partner[bb]] + (e - bd.mpb[bb])];
#pragma unroll
    for (int q = 0; q < 6; ++q) fd.p[q][nd] = 0.5 * (fd.p[q][ndm] + fd.p[q][nc]);
  } else {
#pragma unroll
    for (int q = 0; q < 6; ++q) fd.p[q][nd] = fd.p[q][ndm];
  }
}

// met_cutsa.f90:35-48 on the real cells
__global__ void __launch_bounds__(kTile) k_cutsa(const Blk* __restrict__ blks, Space sp,
                                                 double* v, long long ld, double epsk) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  if (v[5 * ld + n] < 0.) v[5 * ld + n] = epsk;
  v[6 * ld + n] = 0.;
}

}  // namespace

cudaError_t launch_wall_dist(const Bnd& bd, const Blk* blks, Space cells,
                             const long long* went, long long nw, const double* x,
                             const double* y, const double* z, double* par, double* dist,
                             cudaStream_t st) {
  if (nw <= 0) return cudaErrorInvalidValue;
  k_wall_facets<<<(int)((nw + 255) / 256), 256, 0, st>>>(bd, blks, went, nw, x, y, z, par);
  if (cells.ntiles > 0)
    k_wall_dist<<<grid_of(cells), kTile, 0, st>>>(blks, cells, x, y, z, par, nw, dist);
  return cudaGetLastError();
}

cudaError_t launch_turb_bord(const Bnd& bd, double* v, long long ld, double rokinf,
                             double roeinf, cudaStream_t st) {
  if (bd.nlist > 0)
    k_turb_bord<<<(int)((bd.nlist + 255) / 256), 256, 0, st>>>(bd, v, ld, rokinf, roeinf);
  return cudaGetLastError();
}

cudaError_t launch_fd_ghosts(const Bnd& bd, double* const fd[6], cudaStream_t st) {
  Fd6 f;
  for (int q = 0; q < 6; ++q) f.p[q] = fd[q];
  if (bd.nlist > 0) k_fd_ghosts<<<(int)((bd.nlist + 255) / 256), 256, 0, st>>>(bd, f);
  return cudaGetLastError();
}

cudaError_t launch_cutsa(const Blk* blks, Space cells, double* v, long long ld, double epsk,
                         cudaStream_t st) {
  if (cells.ntiles > 0) k_cutsa<<<grid_of(cells), kTile, 0, st>>>(blks, cells, v, ld, epsk);
  return cudaGetLastError();
}

cudaError_t launch_teq_grads(const Blk* blks, Space cells, int mode, int nsc,
                             const double* v, const double* f, long long ld, const double* sn,
                             const double* vol, double* out, double* sc, long long n0,
                             long long n1, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  if (mode != 1) {
    const int g = (int)((n1 - n0 + 255) / 256);
    if (nsc == 3)
      k_teq_scalars<3><<<g, 256, 0, st>>>(mode, v, ld, n0, n1, sc);
    else if (nsc == 2)
      k_teq_scalars<2><<<g, 256, 0, st>>>(mode, v, ld, n0, n1, sc);
    else
      k_teq_scalars<1><<<g, 256, 0, st>>>(mode, v, ld, n0, n1, sc);
    mode = 1;
    f = sc;
  }
  {
    if (nsc == 3)
      k_teq_cell<3><<<grid_of(cells), kTile, 0, st>>>(blks, cells, mode, v, f, ld, sn, vol, out);
    else if (nsc == 2)
      k_teq_cell<2><<<grid_of(cells), kTile, 0, st>>>(blks, cells, mode, v, f, ld, sn, vol, out);
    else
      k_teq_cell<1><<<grid_of(cells), kTile, 0, st>>>(blks, cells, mode, v, f, ld, sn, vol, out);
  }
  return cudaGetLastError();
}

cudaError_t launch_impli2(const Blk* blks, const SpaceBuf* faces, const SpaceBuf* lines,
                          Space cells, int l0, long long ld, const double* u, const double* dt,
                          double* v, const double* mu, const double* mut, const double* cfke,
                          const double* sn, const double* vol, double cmt, double* w,
                          int rcp, const long long* wall_ni, long long nwall,
                          cudaStream_t st) {
  // scratch w: rv, cd, uf[3], ce[3], al, b6, b7, two iterates x (6, 7),
  // the tridiagonal coefficients ta, tb, tc and right-hand sides d6, d7 of
  // a sweep = 20 ld.  rv and the iterates start at zero (their ghost
  // entries are the reference's zeroed rv and never-written neighbours);
  // every other entry read is written first.
  double *rv = w, *cd = w + ld, *uf = w + 2 * ld, *ce = w + 5 * ld, *al = w + 8 * ld,
         *b6 = w + 9 * ld, *b7 = w + 10 * ld;
  double* it[2][2] = {{w + 11 * ld, w + 12 * ld}, {w + 13 * ld, w + 14 * ld}};
  double *ta = w + 15 * ld, *tb = w + 16 * ld, *tc = w + 17 * ld, *d6 = w + 18 * ld,
         *d7 = w + 19 * ld;
  cudaError_t e = cudaMemsetAsync(rv, 0, sizeof(double) * ld, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(w + 11 * ld, 0, sizeof(double) * 4 * ld, st);
  if (e != cudaSuccess) return e;
  if (cells.ntiles == 0) return cudaSuccess;
  k_i2_cell<<<grid_of(cells), kTile, 0, st>>>(blks, cells, v, mu, mut, dt, cfke, vol, cmt, rv,
                                              cd);
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles > 0)
      k_i2_face<<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, v, ld, sn, vol, rv, uf, ce);
  }
  k_i2_diag<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, ce, cd);
  int cur = 0;
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = lines[dir].view(l0);
    for (int sw = 0; sw < 2; ++sw) {
      k_i2_rhs<<<grid_of(cells), kTile, 0, st>>>(blks, cells, dir, ld, u, uf, ce, cd,
                                                 it[cur][0], it[cur][1], ta, tb, tc, d6, d7);
      const int lg = grid_of(sp) * (kTile / kLineCta);
      if (sp.ntiles > 0 && rcp)
        k_i2_line<true><<<lg, kLineCta, 0, st>>>(blks, sp, dir, ta, tb, tc, d6, d7, al, b6, b7,
                                                 it[1 - cur][0], it[1 - cur][1]);
      else if (sp.ntiles > 0)
        k_i2_line<false><<<lg, kLineCta, 0, st>>>(blks, sp, dir, ta, tb, tc, d6, d7, al, b6,
                                                  b7, it[1 - cur][0], it[1 - cur][1]);
      cur = 1 - cur;
    }
  }
  if (nwall > 0)
    k_i2_wall_freeze<<<(unsigned)((nwall + 255) / 256), 256, 0, st>>>(wall_ni, nwall,
                                                                     it[cur][0], it[cur][1]);
  k_i2_update<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, it[cur][0], it[cur][1], v);
  return cudaGetLastError();
}

cudaError_t launch_lpsa1(const Bnd& bd, long long e0, int cnt, Phys ph, WallLaw wl,
                         long long ld, double* v, const double* mu, double* mut,
                         const double* dist, const double* temp, cudaStream_t st) {
  if (cnt > 0)
    k_lpsa1<<<(cnt + 127) / 128, 128, 0, st>>>(bd, e0, cnt, ph, wl, ld, v, mu, mut, dist, temp);
  return cudaGetLastError();
}

cudaError_t launch_lparoi1(const Bnd& bd, long long e0, int cnt, Phys ph, WallLaw wl,
                           long long ld, const double* v, const double* mu, const double* mut,
                           const double* dist, const double* temp, double* tau,
                           cudaStream_t st) {
  if (cnt > 0)
    k_lparoi1<<<(cnt + 127) / 128, 128, 0, st>>>(bd, e0, cnt, ph, wl, ld, v, mu, mut, dist,
                                                 temp, tau);
  return cudaGetLastError();
}

cudaError_t launch_smsa(const Blk* blks, Space cells, long long ld, const double* v,
                        const double* mu, const double* dist, const double* dv,
                        const double* grt, const double* grr, const double* const fd5[3],
                        double* ts6, double* ts7, double* cfke, int fix, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_smsa<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, v, mu, dist, dv, grt, grr,
                                             fd5[0], fd5[1], fd5[2], ts6, ts7, cfke, fix);
  return cudaGetLastError();
}

}  // namespace cns
