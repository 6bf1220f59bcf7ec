// cns_adjoint.cu -- the discrete adjoint of the FP64 Euler Roe iteration
// (sch_roe_euler + implimf_eu): exact Jacobian blocks of the face fluxes,
// obtained by running the scheme's own expressions in forward-mode dual
// numbers (one seed per launch row), and the transposed products the adjoint
// iteration needs:
//
//   A^T lambda   the residual u(W) = sum of face fluxes, transposed, gathered
//                per cell over the faces whose MUSCL stencil holds it (four
//                faces per direction), with the face-normal sensitivities;
//   L^T y        the primal's implicit phase linearised at d = 0 (d = -L u
//                after lmax Jacobi sweeps: L = sum_m (D^-1 N)^m D^-1) and
//                transposed, so that the adjoint iteration
//                lambda += L^T (dJ/dW - A^T lambda) contracts at the primal's
//                asymptotic rate (the two iteration matrices are transposes
//                up to similarity); its blocks are the cells' Euler flux
//                Jacobians, evaluated on the fly.
//
// Stencil inputs per cell: the five conserved variables and the pressure
// (the residual reads the pressure array; for real cells it is zpres of the
// state, for ghost cells the boundary condition's output), so the
// derivatives with respect to W and p are kept apart and chained by the
// caller.  Built with --fmad=false like the rest of the FP64 path.
#include "cns_kernels.cuh"
#include "cns_dual.cuh"
#include "cns_hot.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

constexpr int kFaceSeeds = 27;  // 4 stencil cells x (W 5 + p) + the face normal (3)

// The Euler face flux of sch_roe_euler.f90 (the arithmetic of
// k_face_flux<T, false>) for one face from its stencil values:
// cw[s] = (rho u, ... as W1..W5, p) of the cells n-2inc, n-inc, n, n+inc.
template <class T>
__device__ void euler_face(const T cw[4][6], T sx, T sy, T sz, int p, int nd, int dir,
                           const PhysT<T>& ph, T muscl4, T xk, T out[5]) {
  const T pinfl = ph.pinfl;
  if (p == 1 || p == nd) {
    const int g = p == 1 ? 1 : 2;
    const int r = (p == 1 && dir > 0) ? 2 : g;  // sch_roe_euler.f90:630-632
    const T v1 = cw[g][0], v2 = cw[g][1], v3 = cw[g][2], v4 = cw[g][3], v5 = cw[g][4],
            pg = cw[g][5];
    const T qu = v2 / v1, qv = v3 / v1, qw = v4 / v1;
    const T rr = cw[r][0];
    const T fxx = v2 * qu + pg - pinfl;
    const T fxy = v3 * qu;
    const T fxz = v4 * qu;
    const T fyy = v3 * qv + pg - pinfl;
    const T fyz = v4 * qv;
    const T fzz = v4 * qw + pg - pinfl;
    const T fex = (v5 + pg - pinfl) * v2 / rr;
    const T fey = (v5 + pg - pinfl) * v3 / rr;
    const T fez = (v5 + pg - pinfl) * v4 / rr;
    out[0] = v2 * sx + v3 * sy + v4 * sz;
    out[1] = fxx * sx + fxy * sy + fxz * sz;
    out[2] = fxy * sx + fyy * sy + fyz * sz;
    out[3] = fxz * sx + fyz * sy + fzz * sz;
    out[4] = fex * sx + fey * sy + fez * sz;
    return;
  }
  T c[4][5];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    c[s][0] = cw[s][0];
    c[s][1] = cw[s][1] / cw[s][0];
    c[s][2] = cw[s][2] / cw[s][0];
    c[s][3] = cw[s][3] / cw[s][0];
    c[s][4] = cw[s][5];
  }
  T WL[5], WR[5];
  muscl_plain(c, muscl4, xk, WL, WR);
  T di[5], el, er;
  roe_dissipation(WL, WR, sx, sy, sz, dir > 0, ph, di, el, er);
  const T rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const T rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const T dfxx = rhor * sqT(ur) + prr - pinfl + rhol * sqT(ul) + pl - pinfl;
  const T dfxy = rhor * ur * vr + rhol * ul * vl;
  const T dfxz = rhor * ur * wr + rhol * ul * wl;
  const T dfyy = rhor * sqT(vr) + prr - pinfl + rhol * sqT(vl) + pl - pinfl;
  const T dfyz = rhor * vr * wr + rhol * vl * wl;
  const T dfzz = rhor * sqT(wr) + prr - pinfl + rhol * sqT(wl) + pl - pinfl;
  const T dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul;
  const T dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl;
  const T dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl;
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

// Jacobian of the face flux G_f (5 outputs) w.r.t. seed blockIdx.y: stored at
// J[((dir * 27 + seed) * 5 + a) * ld + n]
__global__ void __launch_bounds__(kTile) k_face_jac(const Blk* __restrict__ blks, Space sp,
                                                    int dir, Phys ph64, Scheme sc,
                                                    const double* __restrict__ v,
                                                    const double* __restrict__ ps,
                                                    long long ld,
                                                    const double* __restrict__ sn,
                                                    double* __restrict__ J) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const int seed = blockIdx.y;
  const Blk& B = blks[b];
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const long long n = cell_index(B, i, j, k);
  Dual cw[4][6];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    // stencil cells outside the block's cell range (faces 1 and nd reach
    // no further than the ghost) are never read by the boundary branch
    const int q = p + s - 2;
    const bool ok = q >= 0 && q <= nd;
    const long long m = n + (long long)(s - 2) * inc;
#pragma unroll
    for (int a = 0; a < 5; ++a) cw[s][a] = Dual(ok ? v[a * ld + m] : 1.);
    cw[s][5] = Dual(ok ? ps[m] : 1.);
  }
  Dual S[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) S[c] = Dual(sn_ptr(sn, B, dir, c)[n]);
  if (seed < 24)
    cw[seed / 6][seed % 6].d = 1.;
  else
    S[seed - 24].d = 1.;
  const PhysT<Dual> ph(ph64);
  Dual out[5];
  euler_face<Dual>(cw, S[0], S[1], S[2], p, nd, dir, ph, Dual(0.25) * Dual(sc.muscl),
                   Dual(sc.xk), out);
  double* Jd = J + ((long long)(dir * kFaceSeeds + seed) * 5) * ld;
#pragma unroll
  for (int a = 0; a < 5; ++a) Jd[a * ld + n] = out[a].d;
}

// (A^T lambda) gathered per cell (i 0..ni, j 0..nj, k 0..nk): for each face
// f of a direction whose stencil holds the cell, J_f^T (lambda(n-inc) -
// lambda(n)) (the face adds G_f to u(n-inc) and subtracts it from u(n));
// lambda is zero on ghost cells.  wbar: [6][ld] (W 1..5, p); sbar: the
// face-normal sensitivity [3 dirs][3][ld] at the face's cell index.
__device__ __forceinline__ bool real_cell(const Blk& B, int i, int j, int k) {
  return i >= 1 && i <= B.ni - 1 && j >= 1 && j <= B.nj - 1 && k >= 1 && k <= B.nk - 1;
}

__global__ void __launch_bounds__(kTile) k_adj_gather(const Blk* __restrict__ blks, Space sp,
                                                      const double* __restrict__ J,
                                                      const double* __restrict__ lam,
                                                      long long ld, double* __restrict__ wbar,
                                                      double* __restrict__ sbar) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  --i;
  --j;
  --k;
  const long long m = cell_index(B, i, j, k);
  double acc[6] = {0., 0., 0., 0., 0., 0.};
  const int idx[3] = {i, j, k};
  const int lim[3] = {B.ni, B.nj, B.nk};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const int d1 = (dir + 1) % 3, d2 = (dir + 2) % 3;
    if (idx[d1] < 1 || idx[d1] > lim[d1] - 1 || idx[d2] < 1 || idx[d2] > lim[d2] - 1) continue;
    const long long inc = ninc_of(B, dir);
    const int q = idx[dir], nd = lim[dir];
    // the face at p holds the cells p-2 .. p+1: this cell is stencil s = q - p + 2
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int p = q - s + 2;
      if (p < 1 || p > nd) continue;
      const long long n = m + (long long)(p - q) * inc;  // the face's upper cell
      int il[3] = {i, j, k}, iu[3] = {i, j, k};
      il[dir] = p - 1;
      iu[dir] = p;
      const bool lr = real_cell(B, il[0], il[1], il[2]);
      const bool ur = real_cell(B, iu[0], iu[1], iu[2]);
      double L[5];
#pragma unroll
      for (int a = 0; a < 5; ++a)
        L[a] = (lr ? lam[a * ld + n - inc] : 0.) - (ur ? lam[a * ld + n] : 0.);
      const double* Jd = J + ((long long)(dir * kFaceSeeds + s * 6) * 5) * ld;
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        double t = 0.;
#pragma unroll
        for (int a = 0; a < 5; ++a) t += Jd[((long long)c * 5 + a) * ld + n] * L[a];
        acc[c] += t;
      }
      // the face-normal sensitivity once per face (from the stencil's upper cell)
      if (s == 2 && sbar) {
        const double* Js = J + ((long long)(dir * kFaceSeeds + 24) * 5) * ld;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          double t = 0.;
#pragma unroll
          for (int a = 0; a < 5; ++a) t += Js[((long long)c * 5 + a) * ld + n] * L[a];
          sbar[((long long)dir * 3 + c) * ld + n] = t;
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 6; ++c) wbar[c * ld + m] = acc[c];
}

// 1 / cd of every real cell, once per transposed solve (the sweeps take it
// seven times a cell each)
template <class T>
__global__ void __launch_bounds__(kTile) k_inv_cd(const Blk* __restrict__ blks, Space sp,
                                                  const T* __restrict__ cd, T* __restrict__ icd) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long c = cell_index(blks[b], i, j, k);
  icd[c] = T(1.) / cd[c];
}

template <class T>
__global__ void __launch_bounds__(kTile) k_scale_cd(const Blk* __restrict__ blks, Space sp,
                                                    long long ld, const T* __restrict__ icd,
                                                    const double* __restrict__ y,
                                                    const T* __restrict__ z,
                                                    double* __restrict__ out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long c = cell_index(blks[b], i, j, k);
  const T ic = icd[c];
#pragma unroll
  for (int a = 0; a < 5; ++a)
    out[a * ld + c] = (double)((z ? z[a * ld + c] : (T)y[a * ld + c]) * ic);
}

// the linearised Jacobi update without stored blocks.  At d = 0 the
// increment f(W + d) - f(W) of a cell differentiates to the Euler flux
// Jacobians A_k(W) of that cell (jacobi_df with qfix: p = gam1 (E - |m|^2 /
// (2 rho) - pinfl), H = (E + p - pinfl) / rho), so the block of e's update
// with respect to its neighbour c across the face S is +-0.5 A(W_c) . S +
// ce I, and the own block 0.5 A(W_e) . (sum over directions of S_lower -
// S_upper).  Every block seen from c carries A(W_c): the transposed sweep
// gathers V_k = sum of +-S_k w_e over the six neighbours and its own w, and
// applies sum_k A_k(W_c)^T V_k once -- the transpose of the linearised
// sweep (its blocks, differentiated with dual numbers, agree in exact
// arithmetic).
template <class T>
__global__ void __launch_bounds__(kTile) k_sweep_ta(const Blk* __restrict__ blks, Space sp,
                                                    long long ld, const double* __restrict__ v,
                                                    const double* __restrict__ ps,
                                                    const T* __restrict__ sn,
                                                    const T* __restrict__ coefe,
                                                    const T* __restrict__ icd,
                                                    const double* __restrict__ y,
                                                    const T* __restrict__ z,
                                                    T* __restrict__ out, T gam1, T pinfl) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long c = cell_index(B, i, j, k);
  auto wof = [&](long long e, T wv[5]) {
    const T ie = icd[e];
#pragma unroll
    for (int a = 0; a < 5; ++a) wv[a] = (z ? z[a * ld + e] : (T)y[a * ld + e]) * ie;
  };
  T acc[5], V[3][5], wc[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) acc[a] = (T)y[a * ld + c];
  wof(c, wc);
  const int idx[3] = {i, j, k};
  const int lim[3] = {B.ni, B.nj, B.nk};
  T Sc[3] = {T(0.), T(0.), T(0.)};
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    T sl[3], su[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      sl[q] = sn_ptr(sn, B, dir, q)[c];
      su[q] = sn_ptr(sn, B, dir, q)[c + inc];
      Sc[q] += sl[q] - su[q];
    }
    if (dir == 0) {
#pragma unroll
      for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int a = 0; a < 5; ++a) V[q][a] = T(0.);
    }
    if (idx[dir] + 1 <= lim[dir] - 1) {  // e above: c is its lower neighbour
      T we[5];
      wof(c + inc, we);
      const T ce = coefe[(long long)dir * ld + c + inc];
#pragma unroll
      for (int a = 0; a < 5; ++a) {
        acc[a] += ce * we[a];
#pragma unroll
        for (int q = 0; q < 3; ++q) V[q][a] += su[q] * we[a];
      }
    }
    if (idx[dir] - 1 >= 1) {  // e below: c is its upper neighbour
      T we[5];
      wof(c - inc, we);
      const T ce = coefe[(long long)dir * ld + c];
#pragma unroll
      for (int a = 0; a < 5; ++a) {
        acc[a] += ce * we[a];
#pragma unroll
        for (int q = 0; q < 3; ++q) V[q][a] -= sl[q] * we[a];
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 5; ++a)
#pragma unroll
    for (int q = 0; q < 3; ++q) V[q][a] += Sc[q] * wc[a];
  // sum_k A_k^T V_k at W_c, times 0.5
  const T rho = (T)v[c], ir = T(1.) / rho;
  const T qv[3] = {(T)v[ld + c] * ir, (T)v[2 * ld + c] * ir, (T)v[3 * ld + c] * ir};
  const T hq2 = T(0.5) * (qv[0] * qv[0] + qv[1] * qv[1] + qv[2] * qv[2]);
  const T H = ((T)v[4 * ld + c] + (T)ps[c] - pinfl) * ir;
  const T g = gam1;
  T qVm[3], sumVkk = T(0.), sumqV4 = T(0.), r0 = T(0.);
#pragma unroll
  for (int kk = 0; kk < 3; ++kk) {
    qVm[kk] = qv[0] * V[kk][1] + qv[1] * V[kk][2] + qv[2] * V[kk][3];
    sumVkk += V[kk][1 + kk];
    sumqV4 += qv[kk] * V[kk][4];
    r0 += -qv[kk] * qVm[kk] + g * hq2 * V[kk][1 + kk] + (g * hq2 - H) * qv[kk] * V[kk][4];
  }
  T r[5];
  r[0] = r0;
#pragma unroll
  for (int bb = 0; bb < 3; ++bb) {
    T t = V[bb][0] + qVm[bb] + H * V[bb][4] - g * qv[bb] * sumVkk - g * qv[bb] * sumqV4;
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) t += qv[kk] * V[kk][1 + bb];
    r[1 + bb] = t;
  }
  r[4] = g * sumVkk + (g + T(1.)) * sumqV4;
#pragma unroll
  for (int a = 0; a < 5; ++a) out[a * ld + c] = acc[a] + T(0.5) * r[a];
}

}  // namespace

cudaError_t launch_face_jac(const Blk* blks, const SpaceBuf* faces, Phys ph, Scheme sc,
                            const double* v, const double* ps, long long ld, const double* sn,
                            double* J, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(-1);
    if (sp.ntiles > 0)
      k_face_jac<<<dim3(grid_of(sp), kFaceSeeds), kTile, 0, st>>>(blks, sp, dir, ph, sc, v, ps,
                                                                   ld, sn, J);
  }
  return cudaGetLastError();
}

cudaError_t launch_adj_gather(const Blk* blks, Space cells_ext, const double* J,
                              const double* lam, long long ld, double* wbar, double* sbar,
                              cudaStream_t st) {
  if (cells_ext.ntiles > 0)
    k_adj_gather<<<grid_of(cells_ext), kTile, 0, st>>>(blks, cells_ext, J, lam, ld, wbar, sbar);
  return cudaGetLastError();
}

}  // namespace cns

namespace cns {
template <class T>
cudaError_t launch_precond_ta(const Blk* blks, Space cells, long long ld, const double* v,
                              const double* ps, const T* sn, const T* coefe, const T* cd,
                              double gam1, double pinfl, int lmax, const double* y, T* z0,
                              T* z1, T* icd, double* out, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  k_inv_cd<T><<<grid_of(cells), kTile, 0, st>>>(blks, cells, cd, icd);
  const T* cur = nullptr;  // the first sweep's iterate: y
  T* bufs[2] = {z0, z1};
  for (int l = 1; l < lmax; ++l) {
    T* nxt = bufs[l & 1];
    k_sweep_ta<T><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, v, ps, sn, coefe, icd, y,
                                                    cur, nxt, (T)gam1, (T)pinfl);
    cur = nxt;
  }
  k_scale_cd<T><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, icd, y, cur, out);
  return cudaGetLastError();
}
template cudaError_t launch_precond_ta<double>(const Blk*, Space, long long, const double*,
                                               const double*, const double*, const double*,
                                               const double*, double, double, int,
                                               const double*, double*, double*, double*,
                                               double*, cudaStream_t);
template cudaError_t launch_precond_ta<float>(const Blk*, Space, long long, const double*,
                                              const double*, const float*, const float*,
                                              const float*, double, double, int, const double*,
                                              float*, float*, float*, double*, cudaStream_t);
}  // namespace cns
