// cns_weno.cu -- the WENO5 residual of the reference (sch_weno5_3d.f90,
// ischema 12): Jiang & Shu's fifth-order scheme applied characteristic-wise
// on Roe-averaged eigenvectors, each characteristic field upwinded by the
// sign of its eigenvalue, with Henrick's mapped weights.
//
// Work: one launch per direction computes every interior face of that
// direction (one thread per face, indexed by its lower cell) into the face
// buffer G (convective flux on the face area) and V (half the central
// viscous flux); one launch then sums, per real cell, its interior faces
// direction by direction (lower face then upper, as the reference's loops
// reach the cell) and then its boundary faces i1, i2, j1, j2, k1, k2, whose
// flux comes from the ghost cell alone and is evaluated in place.
//
// FP64, --fmad=false, the reference's expression order: bit-identical to the
// CPU restatement.  The stencils read the block's flat arrays at
// n - 2 ninc .. n + 3 ninc as the reference does; near a block face that
// lands in the spare slots of the cell arrays (i = ni + 1, j = nj + 1,
// k = nk + 1), which no cell routine writes.  At the first interior k face
// the point k = -1 lies before the block, where the reference reads its
// flux work arrays out of bounds (undefined); the kernel takes the ghost
// plane k = 0 there.
#include "cns_kernels.cuh"

namespace cns {

namespace {

// sch_weno5_3d.f90:148-166: component c (0 x, 1 y, 2 z) of cell n's flux
// tensor, as the five values the projection reads: rho u_c and the c-th
// column of the momentum and energy fluxes
__device__ __forceinline__ void weno_cell_flux(const double* __restrict__ v,
                                               const double* __restrict__ ps, long long ld,
                                               long long n, int c, double pinfl, double f[5]) {
  const double v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n],
               v5 = v[4 * ld + n], p = ps[n];
  const double vc = c == 0 ? v2 : (c == 1 ? v3 : v4);
  f[0] = vc;
  // fxx fxy fxz / fxy fyy fyz / fxz fyz fzz: the off-diagonal entries are
  // the higher-index momentum times the lower-index velocity, the diagonal
  // adds p - pinfl
  if (c == 0) {
    f[1] = v2 * (v2 / v1) + p - pinfl;
    f[2] = v3 * (v2 / v1);
    f[3] = v4 * (v2 / v1);
  } else if (c == 1) {
    f[1] = v3 * (v2 / v1);
    f[2] = v3 * (v3 / v1) + p - pinfl;
    f[3] = v4 * (v3 / v1);
  } else {
    f[1] = v4 * (v2 / v1);
    f[2] = v4 * (v3 / v1);
    f[3] = v4 * (v4 / v1) + p - pinfl;
  }
  f[4] = (v5 + p - pinfl) * vc / v1;
}

__device__ __forceinline__ double weno_map_num(double ga, double w) {
  return ga + ga * ga - 3. * ga * w + w * w;
}
__device__ __forceinline__ double weno_map_den(double ga, double w) {
  return ga * ga + w * (1. - 2. * ga);
}

// one characteristic field (sch_weno5_3d.f90:333-620 for field 1): q at the
// points i-2..i+3; the three third-order candidates upwind of lam, their
// smoothness indicators squared, weights normalised, mapped by Henrick's g
// and normalised again; the weighted sum of the first nterm candidates
__device__ __forceinline__ double weno_field(const double q[6], double lam, int nterm) {
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

// the Roe-averaged state of a face and the derived scalars its left (Q) and
// right (P) eigenvector matrices are built from (sch_weno5_3d.f90:240-332)
struct RoeState {
  double nx, ny, nz, um, vm, wm, hm, vitm2, am, am2i, vn, rhom, rhomi, rhoiam, rhoami, gam1;
};

// row kf of Q (sch_weno5_3d.f90:282-306)
__device__ __forceinline__ void q_row(const RoeState& R, int kf, double q[5]) {
  const double nx = R.nx, ny = R.ny, nz = R.nz, um = R.um, vm = R.vm, wm = R.wm;
  const double gam1 = R.gam1, vitm2 = R.vitm2, am2i = R.am2i, rhomi = R.rhomi,
               rhoami = R.rhoami, vn = R.vn;
  switch (kf) {
    case 0:
      q[0] = (1. - gam1 * vitm2 * am2i) * nx - (vm * nz - wm * ny) * rhomi;
      q[1] = gam1 * um * nx * am2i;
      q[2] = gam1 * vm * nx * am2i + nz * rhomi;
      q[3] = gam1 * wm * nx * am2i - ny * rhomi;
      q[4] = -gam1 * nx * am2i;
      break;
    case 1:
      q[0] = (1. - gam1 * vitm2 * am2i) * ny - (wm * nx - um * nz) * rhomi;
      q[1] = gam1 * um * ny * am2i - nz * rhomi;
      q[2] = gam1 * vm * ny * am2i;
      q[3] = gam1 * wm * ny * am2i + nx * rhomi;
      q[4] = -gam1 * ny * am2i;
      break;
    case 2:
      q[0] = (1. - gam1 * vitm2 * am2i) * nz - (um * ny - vm * nx) * rhomi;
      q[1] = gam1 * um * nz * am2i + ny * rhomi;
      q[2] = gam1 * vm * nz * am2i - nx * rhomi;
      q[3] = gam1 * wm * nz * am2i;
      q[4] = -gam1 * nz * am2i;
      break;
    case 3:
      q[0] = gam1 * vitm2 * rhoami - vn * rhomi;
      q[1] = nx * rhomi - gam1 * um * rhoami;
      q[2] = ny * rhomi - gam1 * vm * rhoami;
      q[3] = nz * rhomi - gam1 * wm * rhoami;
      q[4] = gam1 * rhoami;
      break;
    default:
      q[0] = gam1 * vitm2 * rhoami + vn * rhomi;
      q[1] = -nx * rhomi - gam1 * um * rhoami;
      q[2] = -ny * rhomi - gam1 * vm * rhoami;
      q[3] = -nz * rhomi - gam1 * wm * rhoami;
      q[4] = gam1 * rhoami;
  }
}

// column kf of P (sch_weno5_3d.f90:308-332)
__device__ __forceinline__ void p_col(const RoeState& R, int kf, double p[5]) {
  const double nx = R.nx, ny = R.ny, nz = R.nz, um = R.um, vm = R.vm, wm = R.wm;
  const double rhom = R.rhom, rhoiam = R.rhoiam, am = R.am, hm = R.hm, vitm2 = R.vitm2,
               vn = R.vn;
  switch (kf) {
    case 0:
      p[0] = nx;
      p[1] = um * nx;
      p[2] = vm * nx + rhom * nz;
      p[3] = wm * nx - rhom * ny;
      p[4] = vitm2 * nx + rhom * (vm * nz - wm * ny);
      break;
    case 1:
      p[0] = ny;
      p[1] = um * ny - rhom * nz;
      p[2] = vm * ny;
      p[3] = wm * ny + rhom * nx;
      p[4] = vitm2 * ny + rhom * (wm * nx - um * nz);
      break;
    case 2:
      p[0] = nz;
      p[1] = um * nz + rhom * ny;
      p[2] = vm * nz - rhom * nx;
      p[3] = wm * nz;
      p[4] = vitm2 * nz + rhom * (um * ny - vm * nx);
      break;
    case 3:
      p[0] = 0.5 * rhoiam;
      p[1] = 0.5 * rhoiam * (um + nx * am);
      p[2] = 0.5 * rhoiam * (vm + ny * am);
      p[3] = 0.5 * rhoiam * (wm + nz * am);
      p[4] = 0.5 * rhoiam * (hm + am * vn);
      break;
    default:
      p[0] = 0.5 * rhoiam;
      p[1] = 0.5 * rhoiam * (um - nx * am);
      p[2] = 0.5 * rhoiam * (vm - ny * am);
      p[3] = 0.5 * rhoiam * (wm - nz * am);
      p[4] = 0.5 * rhoiam * (hm - am * vn);
  }
}

// interior faces of direction DIR: the thread of real cell (i, j, k) with
// index p <= nd - 2 along DIR computes the face to its upper neighbour
// (sch_weno5_3d.f90:240-1252) into G[DIR][5][ld] and half the viscous flux
// into V[DIR][4][ld], at the lower cell's index
template <int DIR>
__global__ void __launch_bounds__(kTile) k_weno_face(const Blk* __restrict__ blks, Space sp,
                                                     Phys ph, int fix,
                                                     const double* __restrict__ v, long long ld,
                                                     const double* __restrict__ ps,
                                                     const double* __restrict__ tau,
                                                     const double* __restrict__ sn,
                                                     double* __restrict__ G,
                                                     double* __restrict__ V) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const int p = DIR == 0 ? i : (DIR == 1 ? j : k);
  if (p > nd_of(B, DIR) - 2) return;
  const long long ninc = ninc_of(B, DIR);
  const long long n = cell_index(B, i, j, k), n1 = n + ninc;
  const double gam = ph.gam, gam1 = ph.gam1;
  const double s1 = sn_ptr(sn, B, DIR, 0)[n1], s2 = sn_ptr(sn, B, DIR, 1)[n1],
               s3 = sn_ptr(sn, B, DIR, 2)[n1];
  const double cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const double nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const double ul = v[ld + n] / v[n], vl = v[2 * ld + n] / v[n], wl = v[3 * ld + n] / v[n];
  const double ur = v[ld + n1] / v[n1], vr = v[2 * ld + n1] / v[n1],
               wr = v[3 * ld + n1] / v[n1];
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
  const RoeState R{nx, ny, nz, um, vm, wm, hm, vitm2, am, am2i, vn, rhom, rhomi, rhoiam, rhoami,
                   gam1};
  // the six stencil points n + s ninc (s = -2..3); k = -1 (below the
  // block) is taken at the ghost plane k = 0
  long long pt[6];
#pragma unroll
  for (int s = 0; s < 6; ++s)
    pt[s] = (DIR == 2 && k + s - 2 < 0) ? n - (long long)k * B.nijd : n + (s - 2) * ninc;
  double df[5];
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    // the reference sums three candidates in the x and y fluxes of the i
    // direction and two everywhere else (sch_weno5_3d.f90:616, 911, 1206,
    // 1639, 1934, 2229, 2662, 2957, 3252); fix: three everywhere
    const int nterm = (fix || (DIR == 0 && c < 2)) ? 3 : 2;
    double fl[6][5];
#pragma unroll
    for (int s = 0; s < 6; ++s) weno_cell_flux(v, ps, ld, pt[s], c, ph.pinfl, fl[s]);
    // field by field: its row of Q, its reconstructed flux, and its share
    // of P times the fluxes (summed over the fields in order, as the
    // reference's fc1*p11 + fc2*p12 + ... rounds)
    double oc[5];
#pragma unroll 1
    for (int kf = 0; kf < 5; ++kf) {
      double qr[5], pc[5];
      q_row(R, kf, qr);
      p_col(R, kf, pc);
      double q[6];
#pragma unroll
      for (int s = 0; s < 6; ++s)
        q[s] = qr[0] * fl[s][0] + qr[1] * fl[s][1] + qr[2] * fl[s][2] + qr[3] * fl[s][3] +
               qr[4] * fl[s][4];
      const double fck = weno_field(q, kf < 3 ? vn : (kf == 3 ? vn + am : vn - am), nterm);
#pragma unroll
      for (int r = 0; r < 5; ++r) oc[r] = kf == 0 ? fck * pc[r] : oc[r] + fck * pc[r];
    }
    const double sc = c == 0 ? s1 : (c == 1 ? s2 : s3);
#pragma unroll
    for (int r = 0; r < 5; ++r) df[r] = c == 0 ? oc[r] * sc : df[r] + oc[r] * sc;
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) G[(DIR * 5 + r) * ld + n] = df[r];
  const double *txx = tau, *txy = tau + ld, *txz = tau + 2 * ld, *tyy = tau + 3 * ld,
               *tyz = tau + 4 * ld, *tzz = tau + 5 * ld, *qx = tau + 6 * ld, *qy = tau + 7 * ld,
               *qz = tau + 8 * ld;
  const double fv2 =
      (txx[n] + txx[n1]) * s1 + (txy[n] + txy[n1]) * s2 + (txz[n] + txz[n1]) * s3;
  const double fv3 =
      (txy[n] + txy[n1]) * s1 + (tyy[n] + tyy[n1]) * s2 + (tyz[n] + tyz[n1]) * s3;
  const double fv4 =
      (txz[n] + txz[n1]) * s1 + (tyz[n] + tyz[n1]) * s2 + (tzz[n] + tzz[n1]) * s3;
  const double fv5 = (txx[n] * ul + txy[n] * vl + txz[n] * wl + qx[n] + txx[n1] * ur +
                      txy[n1] * vr + txz[n1] * wr + qx[n1]) * s1 +
                     (txy[n] * ul + tyy[n] * vl + tyz[n] * wl + qy[n] + txy[n1] * ur +
                      tyy[n1] * vr + tyz[n1] * wr + qy[n1]) * s2 +
                     (txz[n] * ul + tyz[n] * vl + tzz[n] * wl + qz[n] + txz[n1] * ur +
                      tyz[n1] * vr + tzz[n1] * wr + qz[n1]) * s3;
  V[(DIR * 4 + 0) * ld + n] = 0.5 * fv2;
  V[(DIR * 4 + 1) * ld + n] = 0.5 * fv3;
  V[(DIR * 4 + 2) * ld + n] = 0.5 * fv4;
  V[(DIR * 4 + 3) * ld + n] = 0.5 * fv5;
}

// sch_weno5_3d.f90:3302-3500: the flux through a boundary face from the
// ghost cell g alone (convective minus viscous), face vector (s1, s2, s3)
__device__ __forceinline__ void weno_boundary(const double* __restrict__ v,
                                              const double* __restrict__ ps,
                                              const double* __restrict__ tau, long long ld,
                                              long long g, double pinfl, double s1, double s2,
                                              double s3, double f[5]) {
  const double v1 = v[g], v2 = v[ld + g], v3 = v[2 * ld + g], v4 = v[3 * ld + g],
               v5 = v[4 * ld + g], p = ps[g];
  const double fxx = v2 * (v2 / v1) + p - pinfl, fxy = v3 * (v2 / v1), fxz = v4 * (v2 / v1);
  const double fyy = v3 * (v3 / v1) + p - pinfl, fyz = v4 * (v3 / v1);
  const double fzz = v4 * (v4 / v1) + p - pinfl;
  const double fex = (v5 + p - pinfl) * v2 / v1, fey = (v5 + p - pinfl) * v3 / v1,
               fez = (v5 + p - pinfl) * v4 / v1;
  const double txx = tau[g], txy = tau[ld + g], txz = tau[2 * ld + g], tyy = tau[3 * ld + g],
               tyz = tau[4 * ld + g], tzz = tau[5 * ld + g], qx = tau[6 * ld + g],
               qy = tau[7 * ld + g], qz = tau[8 * ld + g];
  f[0] = v2 * s1 + v3 * s2 + v4 * s3;
  f[1] = (fxx - txx) * s1 + (fxy - txy) * s2 + (fxz - txz) * s3;
  f[2] = (fxy - txy) * s1 + (fyy - tyy) * s2 + (fyz - tyz) * s3;
  f[3] = (fxz - txz) * s1 + (fyz - tyz) * s2 + (fzz - tzz) * s3;
  f[4] = (fex - (txx * v2 + txy * v3 + txz * v4) / v1 - qx) * s1 +
         (fey - (txy * v2 + tyy * v3 + tyz * v4) / v1 - qy) * s2 +
         (fez - (txz * v2 + tyz * v3 + tzz * v4) / v1 - qz) * s3;
}

// per real cell: the interior faces of i, j, k (lower face u - df + fv/2,
// upper face u + df - fv/2), then the boundary faces i1, i2, j1, j2, k1, k2
// (u -/+ the ghost flux), from u = 0
__global__ void __launch_bounds__(kTile) k_weno_acc(const Blk* __restrict__ blks, Space sp,
                                                    Phys ph, const double* __restrict__ v,
                                                    long long ld, const double* __restrict__ ps,
                                                    const double* __restrict__ tau,
                                                    const double* __restrict__ sn,
                                                    const double* __restrict__ G,
                                                    const double* __restrict__ V,
                                                    double* __restrict__ u,
                                                    float* __restrict__ u32) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long ninc = ninc_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const int nd = nd_of(B, dir);
    if (p >= 2) {
      const long long f = n - ninc;
      acc[0] = acc[0] - G[(dir * 5) * ld + f];
#pragma unroll
      for (int a = 1; a < 5; ++a)
        acc[a] = acc[a] - G[(dir * 5 + a) * ld + f] + V[(dir * 4 + a - 1) * ld + f];
    }
    if (p <= nd - 2) {
      acc[0] = acc[0] + G[(dir * 5) * ld + n];
#pragma unroll
      for (int a = 1; a < 5; ++a)
        acc[a] = acc[a] + G[(dir * 5 + a) * ld + n] - V[(dir * 4 + a - 1) * ld + n];
    }
  }
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long ninc = ninc_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const int nd = nd_of(B, dir);
    const double* s0p = sn_ptr(sn, B, dir, 0);
    const double* s1p = sn_ptr(sn, B, dir, 1);
    const double* s2p = sn_ptr(sn, B, dir, 2);
    double f[5];
    if (p == 1) {
      weno_boundary(v, ps, tau, ld, n - ninc, ph.pinfl, s0p[n], s1p[n], s2p[n], f);
#pragma unroll
      for (int a = 0; a < 5; ++a) acc[a] = acc[a] - f[a];
    }
    if (p == nd - 1) {
      const long long m = n + ninc;
      weno_boundary(v, ps, tau, ld, m, ph.pinfl, s0p[m], s1p[m], s2p[m], f);
#pragma unroll
      for (int a = 0; a < 5; ++a) acc[a] = acc[a] + f[a];
    }
  }
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    u[a * ld + n] = acc[a];
    if (u32) u32[a * ld + n] = (float)acc[a];
  }
}

}  // namespace

cudaError_t launch_weno5(const Blk* blks, Space cells, Phys ph, int fix, const double* v,
                         long long ld,
                         const double* ps, const double* tau, const double* sn, double* G,
                         double* V, double* u, float* u32, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  k_weno_face<0><<<cells.ntiles, kTile, 0, st>>>(blks, cells, ph, fix, v, ld, ps, tau, sn, G,
                                                  V);
  k_weno_face<1><<<cells.ntiles, kTile, 0, st>>>(blks, cells, ph, fix, v, ld, ps, tau, sn, G,
                                                  V);
  k_weno_face<2><<<cells.ntiles, kTile, 0, st>>>(blks, cells, ph, fix, v, ld, ps, tau, sn, G,
                                                  V);
  k_weno_acc<<<cells.ntiles, kTile, 0, st>>>(blks, cells, ph, v, ld, ps, tau, sn, G, V, u,
                                              u32);
  return cudaGetLastError();
}

}  // namespace cns
