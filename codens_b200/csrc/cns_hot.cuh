// cns_hot.cuh -- the hot kernels of the iteration, templated on the real type
// T of their arithmetic and storage:
//   k_ratio       limiter slope-ratio recurrence (sch_roe.f90:146-194)
//   k_face_flux   Roe-MUSCL face flux, Euler or Navier-Stokes (sch_roe*.f90)
//   k_accumulate  face-owned residual accumulation, always summed in FP64
//   k_jacobi_rc   first point-Jacobi sweep, per cell (implimf_eu.f90,
//                 implimf_3d.f90)
//   k_jacobi_25d  the following sweeps, 2.5D-blocked through shared memory
//   k_update      v += d in FP64 and the residual-norm partials
//
// The FP64 instantiations (cns_flow.cu, built with --fmad=false) evaluate the
// reference expressions in the reference's order and are bit-identical to
// the reference semantics.  The FP32 instantiations (cns_mixed.cu, built with
// FMA contraction) are the reduced-precision half of the mixed-precision
// forms, where FP64 stays for metrics, the residual accumulation, the state
// update and the norms.  Every literal is written T(...) so that the FP32
// instantiation never promotes to double.
//
// Included by exactly one translation unit per precision; all kernels live in
// an anonymous namespace.
#pragma once
#include <cfloat>
#include <type_traits>

#include "cns_kernels.cuh"

namespace cns {
namespace {

template <class T>
struct PhysT {
  T gam, gam1, pinfl;
  __device__ explicit PhysT(const Phys& p) : gam(T(p.gam)), gam1(T(p.gam1)), pinfl(T(p.pinfl)) {}
};

template <class T>
__device__ __forceinline__ T sqT(T a) { return a * a; }

template <class T>
__device__ __forceinline__ T tinyT();
template <>
__device__ __forceinline__ double tinyT<double>() { return 2.2250738585072014e-308; }
template <>
__device__ __forceinline__ float tinyT<float>() { return FLT_MIN; }

// ---------------------------------------------------------------------------
// limiter ratios
// ---------------------------------------------------------------------------

// One thread walks one grid line for one of the five variables (blockIdx.y:
// rho, u, v, w, p).  The ratio at face m divides by the ALREADY UPDATED ratio
// of face m-1 and resets to 1 when |r(m-1) r(m) r(m+1)| <= tiny: a
// sequential line recurrence, kept as such.
template <class T>
__global__ void __launch_bounds__(kTile) k_ratio(const Blk* __restrict__ blks,
                                                 Space sp, int dir,
                                                 const T* __restrict__ v,
                                                 const T* __restrict__ prim,
                                                 long long ld,
                                                 const T* __restrict__ ps,
                                                 T* __restrict__ R) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const int nd = nd_of(B, dir);
  if (nd < 3) return;
  const long long inc = ninc_of(B, dir);
  const int a = blockIdx.y;
  const T* x = a == 0 ? v : (a == 4 ? ps : prim + (long long)(a - 1) * ld);
  T* Ra = R + ((long long)dir * 5 + a) * ld;
  const long long n0 = cell_index(B, i, j, k) - inc;   // position 0 of the line
  T x0 = x[n0], x1 = x[n0 + inc], x2 = x[n0 + 2 * inc];
  T rprev = x1 - x0;   // face 1 (never updated)
  T dcur = x2 - x1;    // face 2
  for (int f = 2; f <= nd - 1; ++f) {
    const long long n = n0 + (long long)f * inc;
    const T x3 = x[n + inc];
    const T dnext = x3 - x2;
    T r;
    if (fabs(rprev * dcur * dnext) <= tinyT<T>())
      r = T(1.);
    else
      r = dcur / rprev;
    Ra[n] = r;
    rprev = r;
    dcur = dnext;
    x2 = x3;
  }
}

// ---------------------------------------------------------------------------
// Roe-MUSCL face flux
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T phi_mm(T a) {  // minmod, sch_roe.f90:1500-1504
  const T m = (a < T(1.)) ? a : T(1.);
  return (m > T(0.)) ? m : T(0.);
}

// kappa-MUSCL without limiter (sch_roe_euler.f90:245-273); cells c[0..3] are
// n-2, n-1, n, n+1 as (rho, u, v, w, p)
template <class T>
__device__ __forceinline__ void muscl_plain(const T c[4][5], T c4, T xk, T WL[5],
                                            T WR[5]) {
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    WL[a] = c[1][a] + c4 * ((T(1.) - xk) * (c[1][a] - c[0][a]) +
                            (T(1.) + xk) * (c[2][a] - c[1][a]));
    WR[a] = c[2][a] - c4 * ((T(1.) + xk) * (c[2][a] - c[1][a]) +
                            (T(1.) - xk) * (c[3][a] - c[2][a]));
  }
}

// limited MUSCL (sch_roe.f90:196-227): rho and p use one product order, the
// velocities another; rm are the ratios at this face, rp at the next
template <class T>
__device__ __forceinline__ void muscl_limited(const T c[4][5], T c4, int muscl,
                                              T xk, const T rm[5], const T rp[5],
                                              T WL[5], T WR[5]) {
  const T mu = T(muscl);
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    if (a == 0 || a == 4) {
      WL[a] = c[1][a] + c4 * phi_mm(rm[a]) * (T(1.) - xk) * (c[1][a] - c[0][a]) +
              c4 * phi_mm(T(1.) / rm[a]) * (T(1.) + xk) * (c[2][a] - c[1][a]);
      WR[a] = c[2][a] - c4 * phi_mm(rp[a]) * (T(1.) + xk) * (c[2][a] - c[1][a]) -
              c4 * phi_mm(T(1.) / rp[a]) * (T(1.) - xk) * (c[3][a] - c[2][a]);
    } else {
      WL[a] = c[1][a] + c4 * phi_mm(rm[a]) * (T(1.) - xk) * (c[1][a] - c[0][a]) +
              (T(1.) + xk) * (c[2][a] - c[1][a]) * T(0.25) * mu * phi_mm(T(1.) / rm[a]);
      WR[a] = c[2][a] - c4 * phi_mm(rp[a]) * (T(1.) + xk) * (c[2][a] - c[1][a]) -
              (T(1.) - xk) * (c[3][a] - c[2][a]) * T(0.25) * mu * phi_mm(T(1.) / rp[a]);
    }
  }
}

// row r of the right eigenvector matrix P at the Roe state
template <class T>
__device__ __forceinline__ void p_row(int r, T nx, T ny, T nz, T um, T vm, T wm,
                                      T hm, T am, T vn, T vitm2, T rhom, T rhoiam,
                                      T p[5]) {
  const T h = T(0.5);
  switch (r) {
    case 0:
      p[0] = nx; p[1] = ny; p[2] = nz;
      p[3] = h * rhoiam; p[4] = h * rhoiam;
      break;
    case 1:
      p[0] = um * nx; p[1] = um * ny - rhom * nz; p[2] = um * nz + rhom * ny;
      p[3] = h * rhoiam * (um + nx * am); p[4] = h * rhoiam * (um - nx * am);
      break;
    case 2:
      p[0] = vm * nx + rhom * nz; p[1] = vm * ny; p[2] = vm * nz - rhom * nx;
      p[3] = h * rhoiam * (vm + ny * am); p[4] = h * rhoiam * (vm - ny * am);
      break;
    case 3:
      p[0] = wm * nx - rhom * ny; p[1] = wm * ny + rhom * nx; p[2] = wm * nz;
      p[3] = h * rhoiam * (wm + nz * am); p[4] = h * rhoiam * (wm - nz * am);
      break;
    default:
      p[0] = vitm2 * nx + rhom * (vm * nz - wm * ny);
      p[1] = vitm2 * ny + rhom * (wm * nx - um * nz);
      p[2] = vitm2 * nz + rhom * (um * ny - vm * nx);
      p[3] = h * rhoiam * (hm + am * vn);
      p[4] = h * rhoiam * (hm - am * vn);
  }
}

// Roe dissipation |A|(W_R - W_L) of sch_roe_euler.f90:284-402 (di), plus the
// specific total energies el, er used by the centred part
template <class T>
__device__ __forceinline__ void roe_dissipation(const T WL[5], const T WR[5], T sx,
                                                T sy, T sz, bool absam,
                                                const PhysT<T>& ph, T di[5],
                                                T& el, T& er) {
  const T gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl;
  const T one = T(1.), h = T(0.5);
  const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const T s2 = sx * sx + sy * sy + sz * sz;
  const T q2l = sqT(ul) + sqT(vl) + sqT(wl);
  const T q2r = sqT(ur) + sqT(vr) + sqT(wr);
#ifdef CNS_RECIP_DIV
  // the mixed form's residual (not a parity path): reciprocal square roots
  // where a root and its inverse are both used (|S|, the Roe density
  // sqrt(rho_L rho_R) and sound speed), the inverse densities and the
  // density ratio from 1/sqrt(rho_L rho_R), products with reciprocals
  // instead of divisions: 2 divisions and 3 reciprocal roots per face
  // instead of 17 divisions and 6 roots; the same quantities to FP64
  // rounding
  const T icnds = rsqrt(s2), cnds = s2 * icnds;
  const T nx = sx * icnds, ny = sy * icnds, nz = sz * icnds;
  const T rlr = rhol * rhor, rhomi = rsqrt(rlr), rhom = rlr * rhomi;
  const T ilr = rhomi * rhomi;                  // 1 / (rho_L rho_R)
  const T irl = rhor * ilr, irr = rhol * ilr;   // 1 / rho_L, 1 / rho_R
  const T igam1 = one / gam1;
  const T al2 = gam * pl * irl, ar2 = gam * prr * irr;
  const T hl = al2 * igam1 + h * q2l;
  const T hr = ar2 * igam1 + h * q2r;
  el = pl * igam1 * irl + h * q2l + pinfl * irl;
  er = prr * igam1 * irr + h * q2r + pinfl * irr;
  const T gd = rhor * rhomi;                    // sqrt(rho_R / rho_L)
  const T gd1 = one / (one + gd);
  const T gd2 = gd * gd1;
  const T um = gd1 * ul + gd2 * ur;
  const T vm = gd1 * vl + gd2 * vr;
  const T wm = gd1 * wl + gd2 * wr;
  const T hm = gd1 * hl + gd2 * hr;
  const T vitm2 = h * (sqT(um) + sqT(vm) + sqT(wm));
  const T vn = um * nx + vm * ny + wm * nz;
  const T am2 = absam ? fabs(gam1 * (hm - vitm2)) : gam1 * (hm - vitm2);
  const T iam = rsqrt(am2), am = am2 * iam;
  const T am2i = iam * iam;
  const T rhoiam = rhom * iam;
  const T rhoami = iam * rhomi;
#else
  const T cnds = sqrt(s2);
  const T nx = sx / cnds, ny = sy / cnds, nz = sz / cnds;
  const T al = sqrt(gam * pl / rhol);
  const T ar = sqrt(gam * prr / rhor);
  const T hl = al * al / gam1 + h * q2l;
  const T hr = ar * ar / gam1 + h * q2r;
  el = pl / (gam1 * rhol) + h * q2l + pinfl / rhol;
  er = prr / (gam1 * rhor) + h * q2r + pinfl / rhor;
  const T gd = sqrt(rhor / rhol);
  const T gd1 = one / (one + gd);
  const T gd2 = gd * gd1;
  const T rhom = sqrt(rhol * rhor);
  const T rhomi = one / rhom;
  const T um = gd1 * ul + gd2 * ur;
  const T vm = gd1 * vl + gd2 * vr;
  const T wm = gd1 * wl + gd2 * wr;
  const T hm = gd1 * hl + gd2 * hr;
  const T vitm2 = h * (sqT(um) + sqT(vm) + sqT(wm));
  const T am = absam ? sqrt(fabs(gam1 * (hm - vitm2))) : sqrt(gam1 * (hm - vitm2));
  const T am2i = one / (am * am);
  const T vn = um * nx + vm * ny + wm * nz;
  const T rhoiam = rhom / am;
  const T rhoami = am2i / rhoiam;
#endif
  const T lam1 = fabs(vn * cnds);
  const T lam4 = fabs(vn * cnds + am * cnds);
  const T lam5 = fabs(vn * cnds - am * cnds);
  T dw[5];
  dw[0] = rhor - rhol;
  dw[1] = rhor * ur - rhol * ul;
  dw[2] = rhor * vr - rhol * vl;
  dw[3] = rhor * wr - rhol * wl;
  dw[4] = rhor * er - rhol * el;
#ifdef CNS_RECIP_DIV
  // the mixed form: (P Lambda Q) dW associated as P (Lambda (Q dW)) -- the
  // rows of Q dotted with dW in closed form, then each row of P with the
  // five weighted characteristic amplitudes: ~50 multiply-adds instead of
  // ~150 and no 5x5 Q held in registers (the same product to rounding)
  T w[5];
  {
    const T S = um * dw[1] + vm * dw[2] + wm * dw[3] - dw[4];
    const T A = (one - gam1 * vitm2 * am2i) * dw[0] + gam1 * am2i * S;
    const T B = gam1 * rhoami * (vitm2 * dw[0] - S);
    const T C = rhomi * (nx * dw[1] + ny * dw[2] + nz * dw[3] - vn * dw[0]);
    w[0] = lam1 * (nx * A + rhomi * (nz * dw[2] - ny * dw[3] - (vm * nz - wm * ny) * dw[0]));
    w[1] = lam1 * (ny * A + rhomi * (nx * dw[3] - nz * dw[1] - (wm * nx - um * nz) * dw[0]));
    w[2] = lam1 * (nz * A + rhomi * (ny * dw[1] - nx * dw[2] - (um * ny - vm * nx) * dw[0]));
    w[3] = lam4 * (B + C);
    w[4] = lam5 * (B - C);
  }
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    T p[5];
    p_row(r, nx, ny, nz, um, vm, wm, hm, am, vn, vitm2, rhom, rhoiam, p);
    di[r] = p[0] * w[0] + p[1] * w[1] + p[2] * w[2] + p[3] * w[3] + p[4] * w[4];
  }
#else
  T q[5][5];
  q[0][0] = (one - gam1 * vitm2 * am2i) * nx - (vm * nz - wm * ny) * rhomi;
  q[0][1] = gam1 * um * nx * am2i;
  q[0][2] = gam1 * vm * nx * am2i + nz * rhomi;
  q[0][3] = gam1 * wm * nx * am2i - ny * rhomi;
  q[0][4] = -gam1 * nx * am2i;
  q[1][0] = (one - gam1 * vitm2 * am2i) * ny - (wm * nx - um * nz) * rhomi;
  q[1][1] = gam1 * um * ny * am2i - nz * rhomi;
  q[1][2] = gam1 * vm * ny * am2i;
  q[1][3] = gam1 * wm * ny * am2i + nx * rhomi;
  q[1][4] = -gam1 * ny * am2i;
  q[2][0] = (one - gam1 * vitm2 * am2i) * nz - (um * ny - vm * nx) * rhomi;
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
  const T lam[5] = {lam1, lam1, lam1, lam4, lam5};
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    T p[5];
    p_row(r, nx, ny, nz, um, vm, wm, hm, am, vn, vitm2, rhom, rhoiam, p);
    T pl_[5];
#pragma unroll
    for (int kk = 0; kk < 5; ++kk) pl_[kk] = p[kk] * lam[kk];
    T acc = T(0.);
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      T a = pl_[0] * q[0][c];
#pragma unroll
      for (int kk = 1; kk < 5; ++kk) a = a + pl_[kk] * q[kk][c];
      acc = (c == 0) ? a * dw[0] : acc + a * dw[c];
    }
    di[r] = acc;
  }
#endif
}

// flux families of the face kernel (atsch_num.f90:628-983 by ischema)
enum { kFluxRoe = 0, kFluxHllc = 1, kFluxRusanov = 2, kFluxAusm = 3 };

// the AUSM+ splittings of sch_ausmp.f90:1010-1033 (sign(1, x) = +-1 by the
// sign bit of x)
template <class T>
__device__ __forceinline__ T sgn1(T x) { return copysign(T(1.), x); }
template <class T>
__device__ __forceinline__ T ausm_fmp(T aa) {
  const T s = sgn1(fabs(aa) - T(1.));
  return T(0.25) * (T(1.) + s) * (aa + fabs(aa)) + T(0.125) * (T(1.) - s) * sqT(aa + T(1.));
}
template <class T>
__device__ __forceinline__ T ausm_fmm(T xa) {
  const T s = sgn1(fabs(xa) - T(1.));
  return T(0.25) * (T(1.) + s) * (xa - fabs(xa)) - T(0.125) * (T(1.) - s) * sqT(xa - T(1.));
}
template <class T>
__device__ __forceinline__ T ausm_fpp(T ta) {
  const T s = sgn1(fabs(ta) - T(1.));
  return T(0.25) * (T(1.) + s) * (T(1.) + sgn1(fabs(ta))) +
         T(0.125) * (T(1.) - s) * sqT(ta + T(1.)) *
             (T(2.) - ta + T(0.75) * ta * sqT(ta - T(1.)));
}
template <class T>
__device__ __forceinline__ T ausm_fpm(T ra) {
  const T s = sgn1(fabs(ra) - T(1.));
  return T(0.25) * (T(1.) + s) * (T(1.) - sgn1(fabs(ra))) +
         T(0.125) * (T(1.) - s) * sqT(ra - T(1.)) *
             (T(2.) + ra - T(0.75) * ra * sqT(ra + T(1.)));
}

// the work and heat-flux terms sch_ausmp.f90:81-83 stores in d(n, 1:3)
template <class T>
__device__ __forceinline__ void ausm_dterm(const T* __restrict__ v, const T* __restrict__ tau,
                                           long long ld, long long n, T dd[3]) {
  const T v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n];
  const T txx = tau[n], txy = tau[ld + n], txz = tau[2 * ld + n], tyy = tau[3 * ld + n],
          tyz = tau[4 * ld + n], tzz = tau[5 * ld + n];
  dd[0] = (txx * v2 + txy * v3 + txz * v4) / v1 + tau[6 * ld + n];
  dd[1] = (tyy * v3 + txy * v2 + tyz * v4) / v1 + tau[7 * ld + n];
  dd[2] = (tzz * v4 + txz * v2 + tyz * v3) / v1 + tau[8 * ld + n];
}

// the AUSM+ flux hi1..hi5 of sch_ausmp.f90:255-298
template <class T>
__device__ __forceinline__ void ausm_flux(const T WL[5], const T WR[5], T s1, T s2, T s3,
                                          const T* __restrict__ v, const T* __restrict__ tau,
                                          long long ld, long long nR, long long nL,
                                          const PhysT<T>& ph, T hi[5]) {
  const T gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl, h = T(0.5), two = T(2.);
  const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const T cnds = sqrt(s1 * s1 + s2 * s2 + s3 * s3);
  const T al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  const T hl = al * al / gam1 + h * (sqT(ul) + sqT(vl) + sqT(wl));
  const T hr = ar * ar / gam1 + h * (sqT(ur) + sqT(vr) + sqT(wr));
  const T ai = sqrt(al * ar);
  const T cml = (ul * s1 + vl * s2 + wl * s3) / (al * cnds);
  const T cmr = (ur * s1 + vr * s2 + wr * s3) / (ar * cnds);
  const T psi = two * (pl * ausm_fpp(cml) + prr * ausm_fpm(cmr)) - two * pinfl;
  const T cmi = ausm_fmp(cml) + ausm_fmm(cmr);
  const T dm = h * ai * (cmi * (rhol + rhor) - fabs(cmi) * (rhor - rhol)) * cnds;
  const T txxR = tau[nR], txyR = tau[ld + nR], txzR = tau[2 * ld + nR], tyyR = tau[3 * ld + nR],
          tyzR = tau[4 * ld + nR], tzzR = tau[5 * ld + nR];
  const T txxL = tau[nL], txyL = tau[ld + nL], txzL = tau[2 * ld + nL], tyyL = tau[3 * ld + nL],
          tyzL = tau[4 * ld + nL], tzzL = tau[5 * ld + nL];
  T dR[3], dL[3];
  ausm_dterm(v, tau, ld, nR, dR);
  ausm_dterm(v, tau, ld, nL, dL);
  hi[0] = dm;
  hi[1] = dm * (ul + ur) - fabs(dm) * (ur - ul) + psi * s1 - (txxR + txxL) * s1 -
          (txyR + txyL) * s2 - (txzR + txzL) * s3;
  hi[2] = dm * (vl + vr) - fabs(dm) * (vr - vl) + psi * s2 - (txyR + txyL) * s1 -
          (tyyR + tyyL) * s2 - (tyzR + tyzL) * s3;
  hi[3] = dm * (wl + wr) - fabs(dm) * (wr - wl) + psi * s3 - (txzR + txzL) * s1 -
          (tyzR + tyzL) * s2 - (tzzR + tzzL) * s3;
  hi[4] = dm * (hl + hr) - fabs(dm) * (hr - hl) - (dR[0] + dL[0]) * s1 - (dR[1] + dL[1]) * s2 -
          (dR[2] + dL[2]) * s3;
}

// the HLLC flux (sch_hllc_euler.f90:135-221, sch_hllc.f90:270-357): the
// left or right physical flux, or the star state's; absam: the sound speed
// from |gam1 (hm - vitm2)| (sch_hllc.f90, i and j directions)
template <class T>
__device__ __forceinline__ void hllc_flux(const T WL[5], const T WR[5], T s1, T s2, T s3,
                                          bool absam, const PhysT<T>& ph, T fc[5]) {
  const T gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl;
  const T one = T(1.), h = T(0.5), zero = T(0.);
  const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const T ss = s1 * s1 + s2 * s2 + s3 * s3;
  const T q2l = sqT(ul) + sqT(vl) + sqT(wl), q2r = sqT(ur) + sqT(vr) + sqT(wr);
#ifdef CNS_RECIP_DIV
  // the mixed form's residual (not a parity path): the reciprocal-root and
  // reciprocal forms of the Roe dissipation (roe_dissipation)
  const T icnds = rsqrt(ss), cnds = ss * icnds;
  const T nx = s1 * icnds, ny = s2 * icnds, nz = s3 * icnds;
  const T rlr = rhol * rhor, irlr = rsqrt(rlr), ilr = irlr * irlr;
  const T irl = rhor * ilr, irr = rhol * ilr, igam1 = one / gam1;
  const T hl = gam * pl * irl * igam1 + h * q2l, hr = gam * prr * irr * igam1 + h * q2r;
  const T el = pl * igam1 * irl + h * q2l + pinfl * irl;
  const T er = prr * igam1 * irr + h * q2r + pinfl * irr;
  const T gd = rhor * irlr;
#else
  const T cnds = sqrt(ss);
  const T nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const T al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  const T hl = al * al / gam1 + h * q2l, hr = ar * ar / gam1 + h * q2r;
  const T el = pl / (gam1 * rhol) + h * q2l + pinfl / rhol;
  const T er = prr / (gam1 * rhor) + h * q2r + pinfl / rhor;
  const T gd = sqrt(rhor / rhol);
#endif
  const T vnl = ul * nx + vl * ny + wl * nz, vnr = ur * nx + vr * ny + wr * nz;
  const T gd1 = one / (one + gd), gd2 = gd * gd1;
  const T um = gd1 * ul + gd2 * ur, vm = gd1 * vl + gd2 * vr, wm = gd1 * wl + gd2 * wr;
  const T hm = gd1 * hl + gd2 * hr;
  const T vitm2 = h * (sqT(um) + sqT(vm) + sqT(wm));
  const T am = absam ? sqrt(fabs(gam1 * (hm - vitm2))) : sqrt(gam1 * (hm - vitm2));
  const T vnm = um * nx + vm * ny + wm * nz;
  const T sl = vnm - am, sr = vnm + am;
  const T sst = (rhor * vnr * (sr - vnr) - rhol * vnl * (sl - vnl) + pl - prr) /
                (rhor * (sr - vnr) - rhol * (sl - vnl));
  const T pst = rhol * (vnl - sl) * (vnl - sst) + pl;
  if (sl > zero || sr < zero) {
    const bool left = sl > zero;
    const T rho = left ? rhol : rhor, u = left ? ul : ur, v = left ? vl : vr,
            w = left ? wl : wr, p = left ? pl : prr, e = left ? el : er;
    const T fxx = rho * sqT(u) + p - pinfl, fxy = rho * u * v, fxz = rho * u * w;
    const T fyy = rho * sqT(v) + p - pinfl, fyz = rho * v * w, fzz = rho * sqT(w) + p - pinfl;
    const T fex = (rho * e + p - pinfl) * u, fey = (rho * e + p - pinfl) * v,
            fez = (rho * e + p - pinfl) * w;
    fc[0] = rho * u * s1 + rho * v * s2 + rho * w * s3;
    fc[1] = fxx * s1 + fxy * s2 + fxz * s3;
    fc[2] = fxy * s1 + fyy * s2 + fyz * s3;
    fc[3] = fxz * s1 + fyz * s2 + fzz * s3;
    fc[4] = fex * s1 + fey * s2 + fez * s3;
  } else if (sst >= zero || sst < zero) {
    const bool left = sst >= zero;
    const T rho = left ? rhol : rhor, u = left ? ul : ur, v = left ? vl : vr,
            w = left ? wl : wr, p = left ? pl : prr, e = left ? el : er,
            vn = left ? vnl : vnr, sk = left ? sl : sr;
    const T ids = one / (sk - sst);
    const T rhost = rho * (sk - vn);
    const T rhoust = (rhost * u + (pst - p) * nx) * ids;
    const T rhovst = (rhost * v + (pst - p) * ny) * ids;
    const T rhowst = (rhost * w + (pst - p) * nz) * ids;
    const T rhoest = (rho * e * (sk - vn) + (pst - pinfl) * sst - (p - pinfl) * vn) * ids;
    fc[0] = rhost * ids * sst * cnds;
    fc[1] = (rhoust * sst + (pst - pinfl) * nx) * cnds;
    fc[2] = (rhovst * sst + (pst - pinfl) * ny) * cnds;
    fc[3] = (rhowst * sst + (pst - pinfl) * nz) * cnds;
    fc[4] = (rhoest + pst - pinfl) * sst * cnds;
  } else {
#pragma unroll
    for (int a = 0; a < 5; ++a) fc[a] = sst;  // NaN in, NaN out
  }
}

// Rusanov dissipation rm (W_R - W_L), rm = |S| max(|vnl + al|, |vnr + ar|)
// (sch_rusanov.f90:129-156), and the specific total energies el, er
template <class T>
__device__ __forceinline__ void rusanov_dissipation(const T WL[5], const T WR[5], T s1, T s2,
                                                    T s3, const PhysT<T>& ph, T di[5], T& el,
                                                    T& er) {
  const T gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl, h = T(0.5);
  const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const T ss = s1 * s1 + s2 * s2 + s3 * s3;
  const T q2l = sqT(ul) + sqT(vl) + sqT(wl), q2r = sqT(ur) + sqT(vr) + sqT(wr);
#ifdef CNS_RECIP_DIV
  // the mixed form's residual: reciprocal forms as in roe_dissipation
  const T icnds = rsqrt(ss), cnds = ss * icnds;
  const T nx = s1 * icnds, ny = s2 * icnds, nz = s3 * icnds;
  const T irlr = rsqrt(rhol * rhor), ilr = irlr * irlr;
  const T irl = rhor * ilr, irr = rhol * ilr, igam1 = T(1.) / gam1;
  const T al = sqrt(gam * pl * irl), ar = sqrt(gam * prr * irr);
  el = pl * igam1 * irl + h * q2l + pinfl * irl;
  er = prr * igam1 * irr + h * q2r + pinfl * irr;
#else
  const T cnds = sqrt(ss);
  const T nx = s1 / cnds, ny = s2 / cnds, nz = s3 / cnds;
  const T al = sqrt(gam * pl / rhol), ar = sqrt(gam * prr / rhor);
  el = pl / (gam1 * rhol) + h * q2l + pinfl / rhol;
  er = prr / (gam1 * rhor) + h * q2r + pinfl / rhor;
#endif
  const T vnl = ul * nx + vl * ny + wl * nz, vnr = ur * nx + vr * ny + wr * nz;
  const T al1 = fabs(vnl + al), ar1 = fabs(vnr + ar);
  const T rm = cnds * (al1 >= ar1 ? al1 : ar1);
  di[0] = rm * (rhor - rhol);
  di[1] = rm * (rhor * ur - rhol * ul);
  di[2] = rm * (rhor * vr - rhol * vl);
  di[3] = rm * (rhor * wr - rhol * wl);
  di[4] = rm * (rhor * er - rhol * el);
}

// primitive (rho, u, v, w, p) of cell n
template <class T>
__device__ __forceinline__ void load_prim(const T* __restrict__ v,
                                          const T* __restrict__ prim,
                                          const T* __restrict__ ps, long long ld,
                                          long long n, T c[5]) {
  c[0] = v[n];
  c[1] = prim[n];
  c[2] = prim[ld + n];
  c[3] = prim[2 * ld + n];
  c[4] = ps[n];
}

// one face per thread, direction dir: interior faces give 0.5*f (sch_roe*
// and sch_rusanov interior loops) or the HLLC flux fc (sch_hllc*), boundary
// faces give the ghost-cell physical flux s (lower face 1, upper face nd).
// Results go to G[dir][a][n], n the cell above the face; HLLC with the
// stresses also writes the halves of its viscous flux 0.5*fv to
// V[dir][a-1][n] (a = 1..4), which sch_hllc.f90 applies as a second term.
// FL: kFluxRoe, kFluxHllc, kFluxRusanov (with NS = true always) or kFluxAusm.
// Occupancy: 4 CTAs per SM for Roe (128 registers; 2, 3, 5, 6 measured
// slower), 5 for the lighter families (HLLC residual 1.59 -> 1.42 ms,
// Rusanov 1.27 -> 1.18 ms against 4 on the 4.4M-cell channel).
// The value a face contributes to the face buffer (the expressions of the
// face kernel below, shared with the fused residual kernel): face p of
// direction dir, n the cell above it.  HLLC with the stresses also writes the
// viscous halves to V (when V is given).
template <class T, bool NS, int FL>
__device__ __forceinline__ void face_flux_eval(const Blk& B, int dir, int p, long long n,
                                               const PhysT<T>& ph, const Scheme& sc,
                                               const T* __restrict__ v,
                                               const T* __restrict__ prim, long long ld,
                                               const T* __restrict__ ps,
                                               const T* __restrict__ tau,
                                               const T* __restrict__ sn,
                                               const T* __restrict__ R, T out[5],
                                               T* __restrict__ V) {
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const T sx = sn_ptr(sn, B, dir, 0)[n], sy = sn_ptr(sn, B, dir, 1)[n],
          sz = sn_ptr(sn, B, dir, 2)[n];
  const T pinfl = ph.pinfl;
  if (p == 1 || p == nd) {
    // boundary face: physical flux of the ghost cell (sch_roe_euler.f90:
    // 438-513, sch_roe.f90:497-580); the Euler j/k lower faces divide the
    // energy flux by the interior density (sch_roe_euler.f90:630-632)
    const long long ng = (p == 1) ? n - inc : n;
    // (the Euler forms of Roe and HLLC; Rusanov always has the NS form)
    const long long nrho = (!NS && p == 1 && dir > 0) ? n : ng;
    const T v1 = v[ng], v2 = v[ld + ng], v3 = v[2 * ld + ng], v4 = v[3 * ld + ng],
            v5 = v[4 * ld + ng], pg = ps[ng];
    const T qu = prim[ng], qv = prim[ld + ng], qw = prim[2 * ld + ng];
    T fxx, fxy, fxz, fyy, fyz, fzz, fex, fey, fez;
    if (!NS) {
      const T rr = v[nrho];
      fxx = v2 * qu + pg - pinfl;
      fxy = v3 * qu;
      fxz = v4 * qu;
      fyy = v3 * qv + pg - pinfl;
      fyz = v4 * qv;
      fzz = v4 * qw + pg - pinfl;
      fex = (v5 + pg - pinfl) * v2 / rr;
      fey = (v5 + pg - pinfl) * v3 / rr;
      fez = (v5 + pg - pinfl) * v4 / rr;
    } else {
      const T txx = tau[ng], txy = tau[ld + ng], txz = tau[2 * ld + ng],
              tyy = tau[3 * ld + ng], tyz = tau[4 * ld + ng], tzz = tau[5 * ld + ng],
              qx = tau[6 * ld + ng], qy = tau[7 * ld + ng], qz = tau[8 * ld + ng];
      fxx = v2 * qu + pg - pinfl - txx;
      fxy = v3 * qu - txy;
      fxz = v4 * qu - txz;
      fyy = v3 * qv + pg - pinfl - tyy;
      fyz = v4 * qv - tyz;
      fzz = v4 * qw + pg - pinfl - tzz;
      fex = ((v5 + pg - pinfl - txx) * v2 - txy * v3 - txz * v4) / v1 - qx;
      fey = ((v5 + pg - pinfl - tyy) * v3 - txy * v2 - tyz * v4) / v1 - qy;
      fez = ((v5 + pg - pinfl - tzz) * v4 - txz * v2 - tyz * v3) / v1 - qz;
    }
    out[0] = v2 * sx + v3 * sy + v4 * sz;
    out[1] = fxx * sx + fxy * sy + fxz * sz;
    out[2] = fxy * sx + fyy * sy + fyz * sz;
    out[3] = fxz * sx + fyz * sy + fzz * sz;
    out[4] = fex * sx + fey * sy + fez * sz;
  } else {
    T c[4][5];
#pragma unroll
    for (int s = 0; s < 4; ++s) load_prim(v, prim, ps, ld, n + (long long)(s - 2) * inc, c[s]);
    T WL[5], WR[5];
    const T c4 = T(0.25) * T(sc.muscl);
    const T xk = T(sc.xk);
    if (FL != kFluxRusanov && NS && sc.ilim == 1 && p <= nd - 2) {
      const T* Rd = R + (long long)dir * 5 * ld;
      T rm[5], rp[5];
#pragma unroll
      for (int a = 0; a < 5; ++a) {
        rm[a] = Rd[a * ld + n];
        rp[a] = Rd[a * ld + n + inc];
      }
      muscl_limited(c, c4, sc.muscl, xk, rm, rp, WL, WR);
    } else {
      muscl_plain(c, c4, xk, WL, WR);
    }
    if (FL == kFluxAusm) {
      // sch_ausmp.f90:289-298: hi1 whole, the others halved
      ausm_flux(WL, WR, sx, sy, sz, v, tau, ld, n, n - inc, ph, out);
#pragma unroll
      for (int a = 1; a < 5; ++a) out[a] = T(0.5) * out[a];
      return;
    }
    if (FL == kFluxHllc) {
      hllc_flux(WL, WR, sx, sy, sz, NS && dir < 2, ph, out);
      if (NS) {
        // sch_hllc.f90:358-375
        const long long nR = n, nL = n - inc;
        const T ul = WL[1], vl = WL[2], wl = WL[3], ur = WR[1], vr = WR[2], wr = WR[3];
        const T txxR = tau[nR], txyR = tau[ld + nR], txzR = tau[2 * ld + nR],
                tyyR = tau[3 * ld + nR], tyzR = tau[4 * ld + nR], tzzR = tau[5 * ld + nR];
        const T txxL = tau[nL], txyL = tau[ld + nL], txzL = tau[2 * ld + nL],
                tyyL = tau[3 * ld + nL], tyzL = tau[4 * ld + nL], tzzL = tau[5 * ld + nL];
        T fv[4];
        fv[0] = (txxR + txxL) * sx + (txyR + txyL) * sy + (txzR + txzL) * sz;
        fv[1] = (txyR + txyL) * sx + (tyyR + tyyL) * sy + (tyzR + tyzL) * sz;
        fv[2] = (txzR + txzL) * sx + (tyzR + tyzL) * sy + (tzzR + tzzL) * sz;
        fv[3] = (txxR * ur + txyR * vr + txzR * wr + txxL * ul + txyL * vl + txzL * wl +
                 tau[6 * ld + nR] + tau[6 * ld + nL]) * sx +
                (txyR * ur + tyyR * vr + tyzR * wr + txyL * ul + tyyL * vl + tyzL * wl +
                 tau[7 * ld + nR] + tau[7 * ld + nL]) * sy +
                (txzR * ur + tyzR * vr + tzzR * wr + txzL * ul + tyzL * vl + tzzL * wl +
                 tau[8 * ld + nR] + tau[8 * ld + nL]) * sz;
        if (V) {
          T* Vd = V + (long long)dir * 4 * ld;
#pragma unroll
          for (int a = 0; a < 4; ++a) Vd[a * ld + n] = T(0.5) * fv[a];
        }
      }
      return;
    }
    T di[5], el, er;
    if (FL == kFluxRusanov)
      rusanov_dissipation(WL, WR, sx, sy, sz, ph, di, el, er);
    else
      roe_dissipation(WL, WR, sx, sy, sz, (!NS) && dir > 0, ph, di, el, er);
    const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
    const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
    T dfxx, dfxy, dfxz, dfyy, dfyz, dfzz, dfex, dfey, dfez;
    if (!NS) {
      dfxx = rhor * sqT(ur) + prr - pinfl + rhol * sqT(ul) + pl - pinfl;
      dfxy = rhor * ur * vr + rhol * ul * vl;
      dfxz = rhor * ur * wr + rhol * ul * wl;
      dfyy = rhor * sqT(vr) + prr - pinfl + rhol * sqT(vl) + pl - pinfl;
      dfyz = rhor * vr * wr + rhol * vl * wl;
      dfzz = rhor * sqT(wr) + prr - pinfl + rhol * sqT(wl) + pl - pinfl;
      dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul;
      dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl;
      dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl;
    } else {
      const long long nR = n, nL = n - inc;
      const T txxR = tau[nR], txyR = tau[ld + nR], txzR = tau[2 * ld + nR],
              tyyR = tau[3 * ld + nR], tyzR = tau[4 * ld + nR], tzzR = tau[5 * ld + nR];
      const T txxL = tau[nL], txyL = tau[ld + nL], txzL = tau[2 * ld + nL],
              tyyL = tau[3 * ld + nL], tyzL = tau[4 * ld + nL], tzzL = tau[5 * ld + nL];
      dfxx = rhor * sqT(ur) + prr - pinfl - txxR + rhol * sqT(ul) + pl - pinfl - txxL;
      dfxy = rhor * ur * vr - txyR + rhol * ul * vl - txyL;
      dfxz = rhor * ur * wr - txzR + rhol * ul * wl - txzL;
      dfyy = rhor * sqT(vr) + prr - pinfl - tyyR + rhol * sqT(vl) + pl - pinfl - tyyL;
      dfyz = rhor * vr * wr - tyzR + rhol * vl * wl - tyzL;
      dfzz = rhor * sqT(wr) + prr - pinfl - tzzR + rhol * sqT(wl) + pl - pinfl - tzzL;
      dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul -
             (txxR * ur + txyR * vr + txzR * wr) - (txxL * ul + txyL * vl + txzL * wl) -
             tau[6 * ld + nR] - tau[6 * ld + nL];
      dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl -
             (txyR * ur + tyyR * vr + tyzR * wr) - (txyL * ul + tyyL * vl + tyzL * wl) -
             tau[7 * ld + nR] - tau[7 * ld + nL];
      dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl -
             (txzR * ur + tyzR * vr + tzzR * wr) - (txzL * ul + tyzL * vl + tzzL * wl) -
             tau[8 * ld + nR] - tau[8 * ld + nL];
    }
    const T f1 = (rhor * ur + rhol * ul) * sx + (rhor * vr + rhol * vl) * sy +
                 (rhor * wr + rhol * wl) * sz - di[0];
    const T f2 = dfxx * sx + dfxy * sy + dfxz * sz - di[1];
    const T f3 = dfxy * sx + dfyy * sy + dfyz * sz - di[2];
    const T f4 = dfxz * sx + dfyz * sy + dfzz * sz - di[3];
    const T f5 = dfex * sx + dfey * sy + dfez * sz - di[4];
    out[0] = T(0.5) * f1;
    out[1] = T(0.5) * f2;
    out[2] = T(0.5) * f3;
    out[3] = T(0.5) * f4;
    out[4] = T(0.5) * f5;
  }
}

template <class T, bool NS, int FL = kFluxRoe>
__global__ void __launch_bounds__(kTile, FL == kFluxRoe ? 4 : 5) k_face_flux(
    const Blk* __restrict__ blks, Space sp, int dir, Phys ph64, Scheme sc,
    const T* __restrict__ v, const T* __restrict__ prim, long long ld,
    const T* __restrict__ ps, const T* __restrict__ tau, const T* __restrict__ sn,
    const T* __restrict__ R, T* __restrict__ G, T* __restrict__ V = nullptr) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const PhysT<T> ph(ph64);
  const Blk& B = blks[b];
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const long long n = cell_index(B, i, j, k);
  T out[5];
  face_flux_eval<T, NS, FL>(B, dir, p, n, ph, sc, v, prim, ld, ps, tau, sn, R, out, V);
  T* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
  for (int a = 0; a < 5; ++a) Gd[a * ld + n] = out[a];
}

// ---------------------------------------------------------------------------
// Fused residual: the three face directions and the accumulation in one
// launch.  A CTA owns a TI x TJ patch of cell columns of one block and
// marches along k over kc planes (the 2.5D tiles of the sweeps).  Per plane
// it evaluates, once, every face its patch's cells touch -- the i faces
// i0..i0+TI of each row, the j faces j0..j0+TJ of each column and the upper
// k face of each column; the lower k face is the previous plane's upper one,
// kept in shared memory -- with face_flux_eval (the face kernel's
// expressions), then each real cell sums its six faces from shared memory in
// the order of k_accumulate.  Same bits as the face kernels + k_accumulate,
// without the face buffer's write and re-read in HBM and without the
// accumulation launch.  Per plane a CTA evaluates (TI+1)TJ + TI(TJ+1) + TI TJ
// faces for TI TJ cells: the patch-edge faces are evaluated by both
// neighbouring CTAs (1/TI + 1/TJ of the faces).
// ---------------------------------------------------------------------------
template <int TI, int TJ>
constexpr size_t residual_smem_faces() {
  return (size_t)(TI + 1) * TJ + (size_t)TI * (TJ + 1) + 2 * (size_t)TI * TJ;
}

template <class T, bool NS, int FL, int TI, int TJ, int MINB>
__global__ void __launch_bounds__(TI * TJ, MINB) k_residual_25d(
    const Blk* __restrict__ blks, Tiles tl, Phys ph64, Scheme sc, const T* __restrict__ v,
    const T* __restrict__ prim, long long ld, const T* __restrict__ ps,
    const T* __restrict__ tau, const T* __restrict__ sn, const T* __restrict__ R,
    double* __restrict__ u, float* __restrict__ u32) {
  constexpr int NT = TI * TJ, NFI = (TI + 1) * TJ, NFJ = TI * (TJ + 1);
  constexpr int NF = NFI + NFJ + 2 * NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // face values [5][NF]: i faces (x, y) at y (TI+1) + x (face i0 + x), then
  // j faces (x, y) at NFI + y TI + x (face j0 + y), then two slots of k faces
  T* sf = reinterpret_cast<T*>(smem_raw);
  const int4 t = tl.tile[tl.tile0 + blockIdx.x];
  const Blk& B = blks[t.x];  // fields read where used (not held in registers)
  const PhysT<T> ph(ph64);
  const int i0 = t.y, j0 = t.z, kbeg = t.w, kend = min(t.w + tl.kc, B.nk);
  const int tx = threadIdx.x % TI, ty = threadIdx.x / TI;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = i <= B.ni - 1 && j <= B.nj - 1;
  // one work loop per plane over the faces it needs (a single evaluation
  // site keeps the register allocation of the face kernel): the i faces, the
  // j faces, the upper k faces of the columns, and on the first plane the
  // lower k faces too
  for (int k = kbeg; k < kend; ++k) {
    const int nitems = NFI + NFJ + NT + (k == kbeg ? NT : 0);
    for (int q = threadIdx.x; q < nitems; q += NT) {
      int dir, fi, fj, fk, slot;
      bool ok;
      if (q < NFI) {
        dir = 0;
        fi = i0 + q % (TI + 1);
        fj = j0 + q / (TI + 1);
        fk = k;
        slot = q;
        ok = fi <= B.ni && fj <= B.nj - 1;
      } else if (q < NFI + NFJ) {
        const int r = q - NFI;
        dir = 1;
        fi = i0 + r % TI;
        fj = j0 + r / TI;
        fk = k;
        slot = q;
        ok = fi <= B.ni - 1 && fj <= B.nj;
      } else {
        const int r = (q - NFI - NFJ) % NT;
        const bool upper = q < NFI + NFJ + NT;  // else the first plane's lower faces
        dir = 2;
        fi = i0 + r % TI;
        fj = j0 + r / TI;
        fk = upper ? k + 1 : k;
        slot = NFI + NFJ + (fk & 1) * NT + r;
        ok = fi <= B.ni - 1 && fj <= B.nj - 1;
      }
      if (ok) {
        const int p = dir == 0 ? fi : (dir == 1 ? fj : fk);
        T out[5];
        face_flux_eval<T, NS, FL>(B, dir, p, cell_index(B, fi, fj, fk), ph, sc, v, prim, ld, ps,
                                  tau, sn, R, out, nullptr);
#pragma unroll
        for (int a = 0; a < 5; ++a) sf[a * NF + slot] = out[a];
      }
    }
    __syncthreads();
    if (own) {
      // k_accumulate's order: directions i, j, k; lower face then upper,
      // except the upper face first for the first cell of a line (nd >= 3)
      const int slo[3] = {ty * (TI + 1) + tx, NFI + ty * TI + tx,
                          NFI + NFJ + (k & 1) * NT + threadIdx.x};
      const int sup[3] = {slo[0] + 1, slo[1] + TI, NFI + NFJ + ((k + 1) & 1) * NT + threadIdx.x};
      const int pos[3] = {i, j, k};
      double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) {
        const bool upper_first = pos[dir] == 1 && nd_of(B, dir) >= 3;
#pragma unroll
        for (int a = 0; a < 5; ++a) {
          const double gl = (double)sf[a * NF + slo[dir]], gu = (double)sf[a * NF + sup[dir]];
          if (upper_first) {
            acc[a] = acc[a] + gu;
            acc[a] = acc[a] - gl;
          } else {
            acc[a] = acc[a] - gl;
            acc[a] = acc[a] + gu;
          }
        }
      }
      const long long n = cell_index(B, i, j, k);
#pragma unroll
      for (int a = 0; a < 5; ++a) {
        if (u) u[a * ld + n] = acc[a];
        if (u32) u32[a * ld + n] = (float)acc[a];
      }
    }
    __syncthreads();
  }
}

template <class T, bool NS, int FL, int TI, int TJ, int MINB>
cudaError_t residual_fused_shape(const Blk* blks, Tiles tl, Phys ph, Scheme sc, const T* v,
                                 const T* prim, long long ld, const T* ps, const T* tau,
                                 const T* sn, const T* R, double* u, float* u32,
                                 cudaStream_t st) {
  constexpr size_t sm = sizeof(T) * 5 * residual_smem_faces<TI, TJ>();
  k_residual_25d<T, NS, FL, TI, TJ, MINB><<<tl.ntiles, TI * TJ, sm, st>>>(
      blks, tl, ph, sc, v, prim, ld, ps, tau, sn, R, u, u32);
  return cudaGetLastError();
}

// the fused residual of the flux families that keep one value per face (all
// but HLLC with the stresses, whose viscous halves go through the face
// buffer path); tl: the residual's 2.5D tiles (patch 32 x 4)
template <class T>
cudaError_t residual_fused_dispatch(const Blk* blks, Tiles tl, Phys ph, Scheme sc, const T* v,
                                    const T* prim, long long ld, const T* ps, const T* tau,
                                    const T* sn, const T* R, double* u, float* u32,
                                    cudaStream_t st) {
  if (tl.ntiles == 0) return cudaSuccess;
  if (sc.ischema == 14 && sc.ns) return cudaErrorInvalidValue;
#define CNS_RES_SHAPE(A, B_)                                                              \
  if (tl.ti == A && tl.tj == B_) {                                                        \
    if (sc.ischema == 14)                                                                 \
      return residual_fused_shape<T, false, kFluxHllc, A, B_, 4>(blks, tl, ph, sc, v, prim, \
                                                                 ld, ps, tau, sn, R, u, u32, \
                                                                 st);                      \
    if (sc.ischema == 9)                                                                  \
      return residual_fused_shape<T, true, kFluxRusanov, A, B_, 4>(                       \
          blks, tl, ph, sc, v, prim, ld, ps, tau, sn, R, u, u32, st);                     \
    if (sc.ischema == 5)                                                                  \
      return residual_fused_shape<T, true, kFluxAusm, A, B_, 4>(blks, tl, ph, sc, v, prim, \
                                                                ld, ps, tau, sn, R, u, u32, st); \
    if (sc.ns)                                                                            \
      return residual_fused_shape<T, true, kFluxRoe, A, B_, 4>(blks, tl, ph, sc, v, prim, ld, \
                                                               ps, tau, sn, R, u, u32, st); \
    return residual_fused_shape<T, false, kFluxRoe, A, B_, 4>(blks, tl, ph, sc, v, prim, ld, \
                                                              ps, tau, sn, R, u, u32, st);  \
  }
  CNS_RES_SHAPE(32, 4)
  CNS_RES_SHAPE(16, 8)
#undef CNS_RES_SHAPE
  return cudaErrorInvalidValue;
}

// the FP64 face kernels of one residual by flux family (atsch_num.f90:628-983):
// ischema 14 HLLC (sch_hllc / sch_hllc_euler), 9 Rusanov (sch_rusanov, the
// stresses always), 5 AUSM+ (sch_ausmp, Navier-Stokes), else Roe; each translation unit instantiates it with its
// own contraction flags
static inline cudaError_t face_flux_dispatch(const Blk* blks, const SpaceBuf* faces, int l0,
                                             Phys ph, Scheme sc, const double* v,
                                             const double* prim, long long ld,
                                             const double* ps, const double* tau,
                                             const double* sn, const double* R, double* G,
                                             double* V, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles == 0) continue;
    const int g = sp.ntiles;
    if (sc.ischema == 14 && sc.ns)
      k_face_flux<double, true, kFluxHllc><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                               ld, ps, tau, sn, R, G, V);
    else if (sc.ischema == 14)
      k_face_flux<double, false, kFluxHllc><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v,
                                                                prim, ld, ps, tau, sn, R, G);
    else if (sc.ischema == 9)
      k_face_flux<double, true, kFluxRusanov><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v,
                                                                  prim, ld, ps, tau, sn, R, G);
    else if (sc.ischema == 5)
      k_face_flux<double, true, kFluxAusm><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                               ld, ps, tau, sn, R, G);
    else if (sc.ns)
      k_face_flux<double, true><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim, ld, ps,
                                                     tau, sn, R, G);
    else
      k_face_flux<double, false><<<g, kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim, ld, ps,
                                                      tau, sn, R, G);
  }
  return cudaGetLastError();
}

// u(n) from the six faces of the cell, summed in FP64 in the reference's
// order; with corr (defect correction, FP64) u = that sum + corr; with u32 a
// single-precision copy of u is written too
// V (HLLC with the stresses): the halves 0.5*fv of the interior faces'
// viscous flux, applied after each face's fc as sch_hllc.f90:376-385 does
template <class T>
__global__ void __launch_bounds__(kTile) k_accumulate(const Blk* __restrict__ blks,
                                                      Space sp, const T* __restrict__ G,
                                                      long long ld,
                                                      const double* __restrict__ corr,
                                                      double* __restrict__ u,
                                                      float* __restrict__ u32,
                                                      const T* __restrict__ V = nullptr) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double acc[5] = {0., 0., 0., 0., 0.};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const bool upper_first = (p == 1) && nd >= 3;
    const bool vlo = V && p >= 2, vup = V && p <= nd - 2;  // interior faces
    const T* Gd = G + (long long)dir * 5 * ld;
    const T* Vd = V + (long long)dir * 4 * ld;
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double gl = (double)Gd[a * ld + n], gu = (double)Gd[a * ld + n + inc];
      if (upper_first) {
        acc[a] = acc[a] + gu;
        if (vup && a > 0) acc[a] = acc[a] - (double)Vd[(a - 1) * ld + n + inc];
        acc[a] = acc[a] - gl;
      } else {
        acc[a] = acc[a] - gl;
        if (vlo && a > 0) acc[a] = acc[a] + (double)Vd[(a - 1) * ld + n];
        acc[a] = acc[a] + gu;
        if (vup && a > 0) acc[a] = acc[a] - (double)Vd[(a - 1) * ld + n + inc];
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double r = corr ? acc[a] + corr[a * ld + n] : acc[a];
    if (u) u[a * ld + n] = r;
    if (u32) u32[a * ld + n] = (float)r;
  }
}

// ---------------------------------------------------------------------------
// implicit phase: matrix-free point Jacobi
// ---------------------------------------------------------------------------

// df index: 0 xx, 1 xy, 2 xz, 3 ex, 4 yy, 5 yz, 6 ey, 7 zz, 8 ez

// flux increments of v+d minus those of v (implimf_eu.f90:301-312,
// implimf_3d.f90:430-463) for one cell
template <class T, bool EU>
__device__ __forceinline__ void jacobi_df(const T dn[5], T v1, T v2, T v3, T v4, T v5,
                                          T p, T qu, T qv, T qw, T gam1, T pinfl,
                                          int qfix, T f[9]) {
  const T h = T(0.5);
  if (EU) {
    const T wi1 = T(1.) / (v1 + dn[0]);
    const T ui = v2 + dn[1], vi = v3 + dn[2], wi = v4 + dn[3], wi5 = v5 + dn[4];
    const T pres = gam1 * (wi5 - h * wi1 * (sqT(ui) + sqT(vi) + sqT(wi)) - pinfl);
    const T norm = T(1.) / v1;
    const T fxx = v2 * (v2 * norm) + p;
    const T fxy = v3 * (v2 * norm);
    const T fxz = v4 * (v2 * norm);
    const T fyy = v3 * (v3 * norm) + p;
    const T fyz = v4 * (v3 * norm);
    const T fzz = v4 * (v4 * norm) + p;
    const T fex = (v5 + p - pinfl) * v2 * norm;
    const T fey = (v5 + p - pinfl) * v3 * norm;
    const T fez = (v5 + p - pinfl) * v4 * norm;
    f[0] = wi1 * sqT(ui) + pres - fxx;
    f[1] = wi1 * ui * vi - fxy;
    f[2] = wi1 * ui * wi - fxz;
    f[3] = wi1 * ui * (wi5 + pres - pinfl) - fex;
    f[4] = wi1 * sqT(vi) + pres - fyy;
    f[5] = wi1 * vi * wi - fyz;
    f[6] = wi1 * vi * (wi5 + pres - pinfl) - fey;
    f[7] = wi1 * sqT(wi) + pres - fzz;
    f[8] = qfix ? wi1 * wi * (wi5 + pres - pinfl) - fez : wi1 * (wi5 + pres - pinfl) - fez;
  } else {
    const T wi1 = v1 + dn[0];
    const T ui = (v2 + dn[1]) / wi1, vi = (v3 + dn[2]) / wi1, wi = (v4 + dn[3]) / wi1;
    const T wi5 = v5 + dn[4];
    const T pres = gam1 * (wi5 - h * wi1 * (sqT(ui) + sqT(vi) + sqT(wi)) - pinfl);
    const T fxx = v2 * qu + p;
    const T fxy = v3 * qu;
    const T fxz = v4 * qu;
    const T fyy = v3 * qv + p;
    const T fyz = v4 * qv;
    const T fzz = v4 * qw + p;
    const T fex = (v5 + p - pinfl) * v2 / v1;
    const T fey = (v5 + p - pinfl) * v3 / v1;
    const T fez = (v5 + p - pinfl) * v4 / v1;
    f[0] = wi1 * sqT(ui) + pres - fxx;
    f[1] = wi1 * ui * vi - fxy;
    f[2] = wi1 * ui * wi - fxz;
    f[3] = ui * (wi5 + pres - pinfl) - fex;
    f[4] = wi1 * sqT(vi) + pres - fyy;
    f[5] = wi1 * vi * wi - fyz;
    f[6] = vi * (wi5 + pres - pinfl) - fey;
    f[7] = wi1 * sqT(wi) + pres - fzz;
    f[8] = wi * (wi5 + pres - pinfl) - fez;
  }
}

// Reduced-precision sweep that stores no flux increments: each neighbour's
// increment f(v+d) - f(v) is recomputed from its state and iterate (ghost
// neighbours contribute zero, as their stored increments do in the reference
// sweep).  A sweep then moves the iterate and the per-iteration constants
// only.  Used by the mixed forms, where the sweeps only precondition the
// pseudo-time step.
//
// The increment is evaluated in difference form: with q the velocity, rho'
// = rho + d_rho, dq = (d_m - q d_rho) / rho' and dp = p' - p,
//   rho' u'u' - rho u u = d_rho u u + rho' (2 u du + du du) (+ dp on the
//   diagonal), u' (E' + p' - pinfl) - u (E + p - pinfl) = du H' + u (dE + dp),
// the same quantities as implimf_3d.f90:430-463 / implimf_eu.f90:301-312 in
// exact arithmetic, but exactly zero for d = 0.  The reference form cancels
// O(1) fluxes, and in FP32 that leaves a rounding residue of ~1e-7 at d = 0
// which would hold the iteration off the FP64 steady state.
template <class T>
__device__ __forceinline__ T rcpT(T a) {
  return T(1.) / a;
}
template <>
__device__ __forceinline__ float rcpT<float>(float a) {
  return __fdividef(1.f, a);
}

// FP32 form of df_diff with every operation spelled out as a rounding
// intrinsic (never contracted or reordered by the compiler).  A sweep
// evaluates the same cell's increment at different places of the kernel --
// a tile's first plane from global memory, a ring or patch cell staged in
// shared memory -- and which place a cell takes depends on the tiling; with
// explicit roundings every place gives the same bits, so the FP32 sweeps are
// independent of the tiling the autotuner picks.
template <bool EU>
__device__ __forceinline__ void df_diff_f32(const float dd[5], float rho, float E, float p,
                                            float qu, float qv, float qw, float gam1,
                                            float pinfl, int qfix, float f[9]) {
  const float r1 = __fadd_rn(rho, dd[0]);
  const float ir1 = __fdividef(1.f, r1);
  const float du = __fmul_rn(__fmaf_rn(-qu, dd[0], dd[1]), ir1);
  const float dv = __fmul_rn(__fmaf_rn(-qv, dd[0], dd[2]), ir1);
  const float dw = __fmul_rn(__fmaf_rn(-qw, dd[0], dd[3]), ir1);
  const float q2 = __fmaf_rn(qu, qu, __fmaf_rn(qv, qv, __fmul_rn(qw, qw)));
  const float qd = __fmaf_rn(qu, du, __fmaf_rn(qv, dv, __fmul_rn(qw, dw)));
  const float d2 = __fmaf_rn(du, du, __fmaf_rn(dv, dv, __fmul_rn(dw, dw)));
  const float dk = __fmaf_rn(dd[0], q2, __fmul_rn(r1, __fmaf_rn(2.f, qd, d2)));
  const float dp = __fmul_rn(gam1, __fmaf_rn(-0.5f, dk, dd[4]));
  const float h0 = __fsub_rn(__fadd_rn(E, p), pinfl);
  const float de = __fadd_rn(dd[4], dp);
  const float h1 = __fadd_rn(h0, de);
  const float d0u = __fmul_rn(dd[0], qu), d0v = __fmul_rn(dd[0], qv),
              d0w = __fmul_rn(dd[0], qw);
  f[0] = __fmaf_rn(d0u, qu, __fmaf_rn(r1, __fmaf_rn(__fmul_rn(2.f, qu), du, __fmul_rn(du, du)),
                                      dp));
  f[1] = __fmaf_rn(d0u, qv, __fmul_rn(r1, __fmaf_rn(qu, dv, __fmaf_rn(qv, du, __fmul_rn(du, dv)))));
  f[2] = __fmaf_rn(d0u, qw, __fmul_rn(r1, __fmaf_rn(qu, dw, __fmaf_rn(qw, du, __fmul_rn(du, dw)))));
  f[3] = __fmaf_rn(du, h1, __fmul_rn(qu, de));
  f[4] = __fmaf_rn(d0v, qv, __fmaf_rn(r1, __fmaf_rn(__fmul_rn(2.f, qv), dv, __fmul_rn(dv, dv)),
                                      dp));
  f[5] = __fmaf_rn(d0v, qw, __fmul_rn(r1, __fmaf_rn(qv, dw, __fmaf_rn(qw, dv, __fmul_rn(dv, dw)))));
  f[6] = __fmaf_rn(dv, h1, __fmul_rn(qv, de));
  f[7] = __fmaf_rn(d0w, qw, __fmaf_rn(r1, __fmaf_rn(__fmul_rn(2.f, qw), dw, __fmul_rn(dw, dw)),
                                      dp));
  // implimf_eu.f90:312 lacks the *wi factor of the z energy increment; the
  // Euler form keeps it unless qfix (a flagged non-reference option) is set
  f[8] = (EU && !qfix) ? __fmaf_rn(h1, ir1, -__fmul_rn(h0, qw))
                       : __fmaf_rn(dw, h1, __fmul_rn(qw, de));
}

template <class T, bool EU>
__device__ __forceinline__ void df_diff(const T dd[5], T rho, T E, T p, T qu, T qv, T qw,
                                        T gam1, T pinfl, int qfix, T f[9]) {
  if constexpr (std::is_same<T, float>::value) {
    df_diff_f32<EU>(dd, rho, E, p, qu, qv, qw, gam1, pinfl, qfix, f);
    return;
  }
  const T r1 = rho + dd[0];
  const T ir1 = rcpT(r1);
  const T du = (dd[1] - qu * dd[0]) * ir1;
  const T dv = (dd[2] - qv * dd[0]) * ir1;
  const T dw = (dd[3] - qw * dd[0]) * ir1;
  const T dk = dd[0] * (qu * qu + qv * qv + qw * qw) +
               r1 * (T(2.) * (qu * du + qv * dv + qw * dw) + du * du + dv * dv + dw * dw);
  const T dp = gam1 * (dd[4] - T(0.5) * dk);
  const T h0 = E + p - pinfl;
  const T h1 = h0 + dd[4] + dp;
  const T de = dd[4] + dp;
  f[0] = dd[0] * qu * qu + r1 * (T(2.) * qu * du + du * du) + dp;
  f[1] = dd[0] * qu * qv + r1 * (qu * dv + qv * du + du * dv);
  f[2] = dd[0] * qu * qw + r1 * (qu * dw + qw * du + du * dw);
  f[3] = du * h1 + qu * de;
  f[4] = dd[0] * qv * qv + r1 * (T(2.) * qv * dv + dv * dv) + dp;
  f[5] = dd[0] * qv * qw + r1 * (qv * dw + qw * dv + dv * dw);
  f[6] = dv * h1 + qv * de;
  f[7] = dd[0] * qw * qw + r1 * (T(2.) * qw * dw + dw * dw) + dp;
  // implimf_eu.f90:312 lacks the *wi factor of the z energy increment; the
  // Euler form keeps it unless qfix (a flagged non-reference option) is set
  f[8] = (EU && !qfix) ? h1 * ir1 - h0 * qw : dw * h1 + qw * de;
}

template <class T, bool EU>
__device__ __forceinline__ void df_of(const T* __restrict__ v, const T* __restrict__ prim,
                                      const T* __restrict__ ps, const T* __restrict__ d,
                                      long long ld, long long n, T gam1, T pinfl, int qfix,
                                      T dd[5], T f[9]) {
#pragma unroll
  for (int a = 0; a < 5; ++a) dd[a] = d[a * ld + n];
  df_diff<T, EU>(dd, v[n], v[4 * ld + n], ps[n], prim[n], prim[ld + n], prim[2 * ld + n], gam1,
                 pinfl, qfix, f);
}

template <class T, bool EU>
__device__ __forceinline__ void face_tn(const T du[5], const T dl[5], const T fu[9],
                                        const T fl[9], T sx, T sy, T sz, T tn[5]) {
  const T h = T(0.5);
  const T a2 = du[1] + dl[1], a3 = du[2] + dl[2], a4 = du[3] + dl[3];
  T s[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) s[q] = fu[q] + fl[q];
  if (EU) {
    tn[0] = h * (a2 * sx + a3 * sy + a4 * sz);
    tn[1] = h * (s[0] * sx + s[1] * sy + s[2] * sz);
    tn[2] = h * (s[1] * sx + s[4] * sy + s[5] * sz);
    tn[3] = h * (s[2] * sx + s[5] * sy + s[7] * sz);
    tn[4] = h * (s[3] * sx + s[6] * sy + s[8] * sz);
  } else {
    tn[0] = h * a2 * sx + h * a3 * sy + h * a4 * sz;
    tn[1] = h * s[0] * sx + h * s[1] * sy + h * s[2] * sz;
    tn[2] = h * s[1] * sx + h * s[4] * sy + h * s[5] * sz;
    tn[3] = h * s[2] * sx + h * s[5] * sy + h * s[7] * sz;
    tn[4] = h * s[3] * sx + h * s[6] * sy + h * s[8] * sz;
  }
}

template <class T, bool EU, bool FIRST>
__global__ void __launch_bounds__(kTile) k_jacobi_rc(
    const Blk* __restrict__ blks, Space sp, Phys ph64, int qfix, long long ld,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ prim,
    const T* __restrict__ ps, const T* __restrict__ sn, const T* __restrict__ coefe,
    const T* __restrict__ coefdiag, const T* __restrict__ d_in, T* __restrict__ d_out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const T gam1 = T(ph64.gam1), pinfl = T(ph64.pinfl);
  T d0[5], f0[9];
  if (FIRST) {
#pragma unroll
    for (int a = 0; a < 5; ++a) d0[a] = T(0.);
#pragma unroll
    for (int q = 0; q < 9; ++q) f0[q] = T(0.);
  } else {
    df_of<T, EU>(v, prim, ps, d_in, ld, n, gam1, pinfl, qfix, d0, f0);
  }
  T d2w[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) d2w[a] = -u[a * ld + n];
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const T *s0 = sn_ptr(sn, B, dir, 0), *s1 = sn_ptr(sn, B, dir, 1),
            *s2 = sn_ptr(sn, B, dir, 2);
    const T* ce = coefe + (long long)dir * ld;
    T dl[5], fl[9], du[5], fu[9];
    if (FIRST || p == 1) {
#pragma unroll
      for (int a = 0; a < 5; ++a) dl[a] = T(0.);
#pragma unroll
      for (int q = 0; q < 9; ++q) fl[q] = T(0.);
    } else {
      df_of<T, EU>(v, prim, ps, d_in, ld, n - inc, gam1, pinfl, qfix, dl, fl);
    }
    if (FIRST || p == nd - 1) {
#pragma unroll
      for (int a = 0; a < 5; ++a) du[a] = T(0.);
#pragma unroll
      for (int q = 0; q < 9; ++q) fu[q] = T(0.);
    } else {
      df_of<T, EU>(v, prim, ps, d_in, ld, n + inc, gam1, pinfl, qfix, du, fu);
    }
    T tn[5];
    face_tn<T, EU>(d0, dl, f0, fl, s0[n], s1[n], s2[n], tn);
    const T cel = ce[n], ceu = ce[n + inc];
#pragma unroll
    for (int a = 0; a < 5; ++a) d2w[a] = d2w[a] + tn[a] + cel * dl[a] + ceu * du[a];
    const long long nu = n + inc;
    face_tn<T, EU>(du, d0, fu, f0, s0[nu], s1[nu], s2[nu], tn);
#pragma unroll
    for (int a = 0; a < 5; ++a) d2w[a] = d2w[a] - tn[a];
  }
  const T cd = coefdiag[n];
#pragma unroll
  for (int a = 0; a < 5; ++a) d_out[a * ld + n] = d2w[a] / cd;
}

// ---------------------------------------------------------------------------
// 2.5D-blocked point-Jacobi sweep (every sweep after the first).
//
// A CTA owns a TI x TJ patch of cell columns of one block and marches along k
// over kc planes.  For each plane it evaluates the iterate d and the flux
// increment f(v+d) - f(v) of every cell of the patch and of its one-cell ring
// once, into shared memory; the own column's plane k-1 stays in registers.
// A cell then reads its six neighbours' (d, f) on chip, so a sweep moves d,
// v, prim, ps, u, the coefficients and the face areas about once per cell
// from HBM and evaluates each increment ~1.3 times (ring) instead of seven.
//
// Pipeline: the inputs of the increments (d, v, prim, ps of the patch and
// ring) of plane k+2 are copied into shared memory with cp.async while plane
// k is computed, and each cell's own inputs (u, face areas, coefficients)
// are loaded before the barrier that precedes its evaluation, so neither
// waits on HBM latency in the critical path.
//
// FORM 0 evaluates the increment with the reference expressions
// (jacobi_df: implimf_3d.f90:430-463, implimf_eu.f90:301-312), so the FP64
// instantiation reproduces the stored-increment sweep bit for bit (the same
// inputs through the same operations); FORM 1 uses the difference form of
// df_diff (reduced precision).  Neighbours outside the block's real cells
// contribute zero, as the reference's never-written ghost increments do.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(valid ? 8 : 0)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(valid ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// the increment of one cell read straight from global memory
template <class T, bool EU, int FORM>
__device__ __forceinline__ void cell_df(const T* __restrict__ v, const T* __restrict__ prim,
                                        const T* __restrict__ ps, const T* __restrict__ d,
                                        long long ld, long long m, T gam1, T pinfl, int qfix,
                                        T dd[5], T f[9]) {
  if (FORM == 1) {
    df_of<T, EU>(v, prim, ps, d, ld, m, gam1, pinfl, qfix, dd, f);
  } else {
#pragma unroll
    for (int a = 0; a < 5; ++a) dd[a] = d[a * ld + m];
    jacobi_df<T, EU>(dd, v[m], v[ld + m], v[2 * ld + m], v[3 * ld + m], v[4 * ld + m], ps[m],
                     EU ? T(0.) : prim[m], EU ? T(0.) : prim[ld + m],
                     EU ? T(0.) : prim[2 * ld + m], gam1, pinfl, qfix, f);
  }
}

// staged inputs of one increment: 0-4 d, then rho, rho E, p and the
// velocity (FORM 1), or v(1..5), p and the velocity (FORM 0, the reference
// expressions; the Euler form reads no velocity)
template <int FORM>
__host__ __device__ constexpr int raw_count(bool eu) {
  return FORM == 1 ? 11 : (eu ? 11 : 14);
}

// 128-thread patches fit three CTAs per SM (shared memory ~60-67 KB each):
// registers capped to match
template <class T, bool EU, int FORM, int TI, int TJ>
__global__ void __launch_bounds__(TI * TJ, TI * TJ <= 128 ? 3 : 1) k_jacobi_25d(
    const Blk* __restrict__ blks, Tiles tl, Phys ph64, int qfix, long long ld,
    const T* __restrict__ u, const T* __restrict__ v, const T* __restrict__ prim,
    const T* __restrict__ ps, const T* __restrict__ sn, const T* __restrict__ coefe,
    const T* __restrict__ coefdiag, const T* __restrict__ d_in, T* __restrict__ d_out) {
  constexpr int NX = TI + 2, NY = TJ + 2, NP = NX * NY, NT = TI * TJ;
  constexpr int NR = raw_count<FORM>(EU);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sdf = reinterpret_cast<T*>(smem_raw);  // [2 planes][14 values][NP]: d, f
  T* sraw = sdf + 2 * 14 * NP;              // [NR inputs][NP]: one staged plane
  const int4 t = tl.tile[tl.tile0 + blockIdx.x];
  const Blk B = blks[t.x];
  const int tx = threadIdx.x % TI, ty = threadIdx.x / TI;
  const int i = t.y + tx, j = t.z + ty;
  const int kbeg = t.w, kend = min(t.w + tl.kc, B.nk);
  const bool own = i <= B.ni - 1 && j <= B.nj - 1;
  const T gam1 = T(ph64.gam1), pinfl = T(ph64.pinfl);

  // the patch-and-ring points this thread stages and fills (at most two for
  // every shape: NP <= 2 NT): whether the column is inside the block's real
  // cells, and its flat index at k = 0
  constexpr int NQ = (NP + NT - 1) / NT;
  static_assert(NQ <= 2, "a thread stages at most two ring points");
  bool colin[NQ];
  long long col0[NQ];
#pragma unroll
  for (int rr = 0; rr < NQ; ++rr) {
    const int q = threadIdx.x + rr * NT;
    const int ii = t.y - 1 + q % NX, jj = t.z - 1 + q / NX;
    colin[rr] = q < NP && ii >= 1 && ii <= B.ni - 1 && jj >= 1 && jj <= B.nj - 1;
    col0[rr] = colin[rr] ? cell_index(B, ii, jj, 0) : 0;
  }
  // the increment inputs of plane kk (patch and ring) into the raw buffer;
  // cells outside the block's real cells are zero-filled
  auto stage = [&](int kk) {
    T* r = sraw;
    const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
    for (int rr = 0; rr < NQ; ++rr) {
      const int q = threadIdx.x + rr * NT;
      if (q >= NP) break;
      const bool in = colin[rr] && kin;
      const long long m = in ? col0[rr] + (long long)kk * B.nijd : 0;
#pragma unroll
      for (int a = 0; a < 5; ++a) cp_async_elem(r + a * NP + q, d_in + a * ld + m, in);
      if (FORM == 1) {
        cp_async_elem(r + 5 * NP + q, v + m, in);
        cp_async_elem(r + 6 * NP + q, v + 4 * ld + m, in);
        cp_async_elem(r + 7 * NP + q, ps + m, in);
#pragma unroll
        for (int a = 0; a < 3; ++a) cp_async_elem(r + (8 + a) * NP + q, prim + a * ld + m, in);
      } else {
#pragma unroll
        for (int a = 0; a < 5; ++a) cp_async_elem(r + (5 + a) * NP + q, v + a * ld + m, in);
        cp_async_elem(r + 10 * NP + q, ps + m, in);
        if (!EU) {
#pragma unroll
          for (int a = 0; a < 3; ++a)
            cp_async_elem(r + (11 + a) * NP + q, prim + a * ld + m, in);
        }
      }
    }
  };
  // increments of the staged plane kk into (d, f) buffer b (zero where the
  // raw inputs are zero: outside the block)
  auto fill = [&](int kk, int b) {
    const T* r = sraw;
    T* s = sdf + b * 14 * NP;
    const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
    for (int rr = 0; rr < NQ; ++rr) {
      const int q = threadIdx.x + rr * NT;
      if (q >= NP) break;
      const bool in = colin[rr] && kin;
      T dd[5], f[9];
#pragma unroll
      for (int a = 0; a < 5; ++a) dd[a] = r[a * NP + q];
      if (in) {
        if (FORM == 1)
          df_diff<T, EU>(dd, r[5 * NP + q], r[6 * NP + q], r[7 * NP + q], r[8 * NP + q],
                         r[9 * NP + q], r[10 * NP + q], gam1, pinfl, qfix, f);
        else
          jacobi_df<T, EU>(dd, r[5 * NP + q], r[6 * NP + q], r[7 * NP + q], r[8 * NP + q],
                           r[9 * NP + q], r[10 * NP + q], EU ? T(0.) : r[11 * NP + q],
                           EU ? T(0.) : r[12 * NP + q], EU ? T(0.) : r[13 * NP + q], gam1,
                           pinfl, qfix, f);
      } else {
#pragma unroll
        for (int a = 0; a < 9; ++a) f[a] = T(0.);
      }
#pragma unroll
      for (int a = 0; a < 5; ++a) s[a * NP + q] = dd[a];
#pragma unroll
      for (int a = 0; a < 9; ++a) s[(5 + a) * NP + q] = f[a];
    }
  };

  // the own column's plane kbeg-1 (registers)
  T pd[5], pf[9];
  if (own && kbeg >= 2) {
    cell_df<T, EU, FORM>(v, prim, ps, d_in, ld, cell_index(B, i, j, kbeg - 1), gam1, pinfl,
                         qfix, pd, pf);
  } else {
#pragma unroll
    for (int a = 0; a < 5; ++a) pd[a] = T(0.);
#pragma unroll
    for (int a = 0; a < 9; ++a) pf[a] = T(0.);
  }
  // one raw buffer: plane kk+1's inputs are copied in while plane kk-1 is
  // computed, after plane kk's increments have been filled from it
  stage(kbeg);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  fill(kbeg, kbeg & 1);
  __syncthreads();
  stage(kbeg + 1);
  cp_async_commit();
  const int q0 = (ty + 1) * NX + tx + 1;
  // the lower k face of plane kbeg; later planes carry it from the plane
  // below (the upper face of cell k is the lower face of cell k+1: the same
  // operands in the same order, so the carried value is bit-identical)
  T tkl[5];
  {
    const T* s = sdf + (kbeg & 1) * 14 * NP;
    T d0[5], f0[9], sk[3];
#pragma unroll
    for (int a = 0; a < 5; ++a) d0[a] = s[a * NP + q0];
#pragma unroll
    for (int a = 0; a < 9; ++a) f0[a] = s[(5 + a) * NP + q0];
    const long long n = cell_index(B, own ? i : 1, own ? j : 1, kbeg);
#pragma unroll
    for (int c = 0; c < 3; ++c) sk[c] = own ? sn_ptr(sn, B, 2, c)[n] : T(0.);
    face_tn<T, EU>(d0, pd, f0, pf, sk[0], sk[1], sk[2], tkl);
  }
  // rows of the patch are TI consecutive lanes (TI = 16 or 32)
  const bool iface = i <= B.ni && j <= B.nj - 1;  // lower i face exists (incl. i = ni)
  const bool iedge = tx == TI - 1;
  for (int k = kbeg; k < kend; ++k) {
    // this cell's own inputs, in flight across the barrier
    const long long n = cell_index(B, iface ? i : 1, iface ? j : 1, k);
    T uu[5], si[3], sj[3], sju[3], sku[3], siu[3], cel[3], ceu[3], cd;
    if (iface) {
#pragma unroll
      for (int c = 0; c < 3; ++c) si[c] = sn_ptr(sn, B, 0, c)[n];
    }
    if (own) {
#pragma unroll
      for (int a = 0; a < 5; ++a) uu[a] = u[a * ld + n];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sj[c] = sn_ptr(sn, B, 1, c)[n];
        sju[c] = sn_ptr(sn, B, 1, c)[n + B.nid];
        sku[c] = sn_ptr(sn, B, 2, c)[n + B.nijd];
        if (iedge) siu[c] = sn_ptr(sn, B, 0, c)[n + 1];
      }
#pragma unroll
      for (int dir = 0; dir < 3; ++dir) {
        cel[dir] = coefe[(long long)dir * ld + n];
        ceu[dir] = coefe[(long long)dir * ld + n + ninc_of(B, dir)];
      }
      cd = coefdiag[n];
    }
    cp_async_wait<0>();
    __syncthreads();
    fill(k + 1, (k + 1) & 1);
    __syncthreads();
    // plane k+2's inputs, in flight while plane k is computed
    stage(k + 2);
    cp_async_commit();
    const T* s = sdf + (k & 1) * 14 * NP;
    const T* su = sdf + ((k + 1) & 1) * 14 * NP;
    T d0[5], f0[9], dl[5], fl[9], du[5], fu[9], tl[5], tu[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) d0[a] = s[a * NP + q0];
#pragma unroll
    for (int a = 0; a < 9; ++a) f0[a] = s[(5 + a) * NP + q0];
    // i: the lower face by every lane, the upper one from the next lane
    // (the row's last lane evaluates its own)
#pragma unroll
    for (int a = 0; a < 5; ++a) dl[a] = s[a * NP + q0 - 1];
#pragma unroll
    for (int a = 0; a < 9; ++a) fl[a] = s[(5 + a) * NP + q0 - 1];
    face_tn<T, EU>(d0, dl, f0, fl, si[0], si[1], si[2], tl);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      du[a] = s[a * NP + q0 + 1];
      tu[a] = __shfl_down_sync(0xffffffffu, tl[a], 1, TI);
    }
    if (iedge) {
#pragma unroll
      for (int a = 0; a < 9; ++a) fu[a] = s[(5 + a) * NP + q0 + 1];
      face_tn<T, EU>(du, d0, fu, f0, siu[0], siu[1], siu[2], tu);
    }
    T d2w[5];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      d2w[a] = -uu[a];
      d2w[a] = d2w[a] + tl[a] + cel[0] * dl[a] + ceu[0] * du[a];
      d2w[a] = d2w[a] - tu[a];
    }
    // j: both faces
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      dl[a] = s[a * NP + q0 - NX];
      du[a] = s[a * NP + q0 + NX];
    }
#pragma unroll
    for (int a = 0; a < 9; ++a) {
      fl[a] = s[(5 + a) * NP + q0 - NX];
      fu[a] = s[(5 + a) * NP + q0 + NX];
    }
    face_tn<T, EU>(d0, dl, f0, fl, sj[0], sj[1], sj[2], tl);
    face_tn<T, EU>(du, d0, fu, f0, sju[0], sju[1], sju[2], tu);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      d2w[a] = d2w[a] + tl[a] + cel[1] * dl[a] + ceu[1] * du[a];
      d2w[a] = d2w[a] - tu[a];
    }
    // k: the lower face carried, the upper one evaluated and carried on
#pragma unroll
    for (int a = 0; a < 5; ++a) du[a] = su[a * NP + q0];
#pragma unroll
    for (int a = 0; a < 9; ++a) fu[a] = su[(5 + a) * NP + q0];
    face_tn<T, EU>(du, d0, fu, f0, sku[0], sku[1], sku[2], tu);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      d2w[a] = d2w[a] + tkl[a] + cel[2] * pd[a] + ceu[2] * du[a];
      d2w[a] = d2w[a] - tu[a];
      tkl[a] = tu[a];
      pd[a] = d0[a];
    }
    if (own) {
      if (FORM == 1) {
        const T rc = T(1.) / cd;
#pragma unroll
        for (int a = 0; a < 5; ++a) d_out[a * ld + n] = d2w[a] * rc;
      } else {
#pragma unroll
        for (int a = 0; a < 5; ++a) d_out[a * ld + n] = d2w[a] / cd;
      }
    }
  }
  cp_async_wait<0>();
}

template <int TI, int TJ, class T, int FORM, bool EU>
constexpr size_t jacobi_25d_smem() {
  // two planes of increments (d, f) and one staged plane of raw inputs
  return sizeof(T) * (2 * 14 + raw_count<FORM>(EU)) * (TI + 2) * (TJ + 2);
}

template <class T, int FORM, int TI, int TJ>
cudaError_t jacobi_25d_shape(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                             long long ld, const T* u, const T* v, const T* prim, const T* ps,
                             const T* sn, const T* coefe, const T* coefdiag, const T* d_in,
                             T* d_out, cudaStream_t st) {
  if (eu)
    k_jacobi_25d<T, true, FORM, TI, TJ>
        <<<tl.ntiles, TI * TJ, jacobi_25d_smem<TI, TJ, T, FORM, true>(), st>>>(
            blks, tl, ph, qfix, ld, u, v, prim, ps, sn, coefe, coefdiag, d_in, d_out);
  else
    k_jacobi_25d<T, false, FORM, TI, TJ>
        <<<tl.ntiles, TI * TJ, jacobi_25d_smem<TI, TJ, T, FORM, false>(), st>>>(
            blks, tl, ph, qfix, ld, u, v, prim, ps, sn, coefe, coefdiag, d_in, d_out);
  return cudaGetLastError();
}

template <class T, int FORM>
cudaError_t jacobi_25d_dispatch(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                                long long ld, const T* u, const T* v, const T* prim,
                                const T* ps, const T* sn, const T* coefe, const T* coefdiag,
                                const T* d_in, T* d_out, cudaStream_t st) {
  if (tl.ntiles == 0) return cudaSuccess;
#define CNS_SHAPE(A, B)                                                                   \
  if (tl.ti == A && tl.tj == B)                                                           \
    return jacobi_25d_shape<T, FORM, A, B>(blks, tl, ph, qfix, eu, ld, u, v, prim, ps, sn, \
                                           coefe, coefdiag, d_in, d_out, st);
  CNS_SHAPE(32, 4)
  CNS_SHAPE(32, 8)
  CNS_SHAPE(16, 8)
  CNS_SHAPE(16, 16)
#undef CNS_SHAPE
  return cudaErrorInvalidValue;
}

template <class T, int FORM, int TI, int TJ>
cudaError_t jacobi_25d_attr_shape() {
  cudaError_t e = cudaFuncSetAttribute(k_jacobi_25d<T, true, FORM, TI, TJ>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)jacobi_25d_smem<TI, TJ, T, FORM, true>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_jacobi_25d<T, false, FORM, TI, TJ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)jacobi_25d_smem<TI, TJ, T, FORM, false>());
  return e;
}

template <class T, int FORM>
cudaError_t jacobi_25d_attr() {
  cudaError_t e = jacobi_25d_attr_shape<T, FORM, 32, 4>();
  if (e == cudaSuccess) e = jacobi_25d_attr_shape<T, FORM, 32, 8>();
  if (e == cudaSuccess) e = jacobi_25d_attr_shape<T, FORM, 16, 8>();
  if (e == cudaSuccess) e = jacobi_25d_attr_shape<T, FORM, 16, 16>();
  return e;
}

// per-tile partial residual norms of (v_new - v_old)/dt (residu.f90:127-182)
__device__ __forceinline__ void norm_tile_reduce(const double res[5], bool valid,
                                                 double* out15) {
  __shared__ double sh[kTile / 32][15];
  double a1[5], a2[5], am[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    a1[a] = valid ? fabs(res[a]) : 0.;
    a2[a] = valid ? res[a] * res[a] : 0.;
    am[a] = a1[a];
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      a1[a] = a1[a] + __shfl_down_sync(0xffffffffu, a1[a], off);
      a2[a] = a2[a] + __shfl_down_sync(0xffffffffu, a2[a], off);
      am[a] = fmax(am[a], __shfl_down_sync(0xffffffffu, am[a], off));
    }
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      sh[w][a] = a1[a];
      sh[w][5 + a] = a2[a];
      sh[w][10 + a] = am[a];
    }
  }
  __syncthreads();
  if (threadIdx.x < 15) {
    const int q = threadIdx.x;
    double s = sh[0][q];
    for (int ww = 1; ww < kTile / 32; ++ww) s = (q >= 10) ? fmax(s, sh[ww][q]) : s + sh[ww][q];
    out15[q] = s;
  }
}

// v += d on the real cells (FP64 state update of implimf_*.f90), the residual
// norm partials and, when requested, the final increment copied to d_out.
// PAD: d in the padded layout (the FP32 iterates)
template <class T, bool PAD = false>
__global__ void __launch_bounds__(kTile) k_update(const Blk* __restrict__ blks,
                                                  Space sp, long long ld,
                                                  const T* __restrict__ d,
                                                  double* __restrict__ v,
                                                  const double* __restrict__ dt,
                                                  double* d_out, double* normpart) {
  int b, i, j, k;
  const bool valid = space_elem(sp, threadIdx.x, b, i, j, k);
  double res[5] = {0., 0., 0., 0., 0.};
  if (valid) {
    const Blk& B = blks[b];
    const long long n = cell_index(B, i, j, k);
    const long long dn = PAD ? pad_index(B, i, j, k) : n;
    const long long dld = PAD ? B.pld : ld;
    const double t = dt[n];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double vo = v[a * ld + n], dd = (double)d[a * dld + dn];
      const double vn = vo + dd;
      v[a * ld + n] = vn;
      if (d_out) d_out[a * ld + n] = dd;
      res[a] = (vn - vo) / t;
    }
  }
  if (normpart) norm_tile_reduce(res, valid, normpart + (long long)(sp.tile0 + blockIdx.x) * 15);
}

}  // namespace
}  // namespace cns
