// cns_mixed.cu -- the single-precision instantiations of the hot kernels and
// the helpers of the mixed-precision iteration.
//
// Mixed form (precision 1): the explicit residual, the time steps, the
// boundary conditions, the state update v += d and the norms stay FP64; the
// point-Jacobi sweeps of the implicit phase run in FP32 on single-precision
// copies of the state, velocities, pressure and face areas.  The sweeps only
// shape the pseudo-time increment, so the fixed point is the FP64 steady
// state: R64(W) = 0.
//
// Defect-correction form (precision 2): the face fluxes also run in FP32;
// every kdefect iterations the FP64 residual R64(W) and the FP32 residual
// R32(W) of the same state give corr = R64 - R32, and the iterations in
// between use R32 + corr.  Its residual stalls at the FP32 rounding level of
// the fluxes (no longer exact between refreshes), so it is a transient
// accelerator, not a steady-state solver.
//
// Built with FMA contraction (the FP32 path is not a parity path).
#include "cns_kernels.cuh"
#include "cns_hot.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

__global__ void __launch_bounds__(256) k_to_float(const double* __restrict__ a,
                                                 float* __restrict__ b, long long n) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) b[q] = (float)a[q];
}

__global__ void __launch_bounds__(kTile) k_defect(const Blk* __restrict__ blks, Space sp,
                                                  long long ld,
                                                  const double* __restrict__ u64,
                                                  const double* __restrict__ ur32,
                                                  double* __restrict__ corr) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
#pragma unroll
  for (int a = 0; a < 5; ++a) corr[a * ld + n] = u64[a * ld + n] - ur32[a * ld + n];
}

// spectral radius of the face between cells nh (upper side) and nl; rvh, rvl
// the viscous factors (zero off the real cells, as the reference's zeroed rv)
template <bool EU>
__device__ __forceinline__ float face_coef(const float* __restrict__ prim, long long ld,
                                           const double* __restrict__ vol,
                                           const double* __restrict__ cson, long long nh,
                                           long long nl, float sx, float sy, float sz,
                                           float rvh, float rvl) {
  const float cnds = sx * sx + sy * sy + sz * sz;
  const float cc = 0.5f * ((float)cson[nh] + (float)cson[nl]);
  const float uu = 0.5f * (prim[nh] + prim[nl]);
  const float vv = 0.5f * (prim[ld + nh] + prim[ld + nl]);
  const float ww = 0.5f * (prim[2 * ld + nh] + prim[2 * ld + nl]);
  const float vn = uu * sx + vv * sy + ww * sz;
  if (EU) return 0.5f * fabsf(vn) + sqrtf(cnds) * cc;
  return 0.5f * (fabsf(vn) + sqrtf(cnds) * cc) +
         (rvh + rvl) * cnds / (float)(vol[nh] + vol[nl]);
}

// the implicit coefficients of the FP32 sweeps in one pass (the FP32 form of
// implimf_3d.f90:111-203 / implimf_eu.f90:124-170): each real cell evaluates
// the spectral radii of its six faces, stores the lower faces (and the upper
// one at the end of each line) and sums the diagonal in the reference order.
// Every interior face is evaluated by both its cells (cheaper than a second
// pass over memory).
template <bool EU>
__global__ void __launch_bounds__(kTile) k_coef32(
    const Blk* __restrict__ blks, Space sp, Phys ph, long long ld,
    const double* __restrict__ dt, const double* __restrict__ v,
    const float* __restrict__ prim, const double* __restrict__ mu,
    const double* __restrict__ mut, const float* __restrict__ sn,
    const double* __restrict__ vol, const double* __restrict__ cson,
    float* __restrict__ coefe, float* __restrict__ coefdiag) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const float gp = (float)(ph.gam / ph.pr), gpt = (float)(ph.gam / ph.prt);
  auto rv_of = [&](long long m, bool real) -> float {
    if (EU || !real) return 0.f;
    return (gp * (float)mu[m] + gpt * (float)mut[m]) / (float)v[m];
  };
  const float rv0 = rv_of(n, true);
  float cd = (float)(vol[n] / dt[n]);
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const float* s0 = sn_ptr(sn, B, dir, 0);
    const float* s1 = sn_ptr(sn, B, dir, 1);
    const float* s2 = sn_ptr(sn, B, dir, 2);
    const long long nl = n - inc, nu = n + inc;
    const float cel = face_coef<EU>(prim, ld, vol, cson, n, nl, s0[n], s1[n], s2[n], rv0,
                                    rv_of(nl, p > 1));
    const float ceu = face_coef<EU>(prim, ld, vol, cson, nu, n, s0[nu], s1[nu], s2[nu],
                                    rv_of(nu, p < nd - 1), rv0);
    coefe[(long long)dir * ld + n] = cel;
    if (p == nd - 1) coefe[(long long)dir * ld + nu] = ceu;
    cd = cd + cel + ceu;
  }
  coefdiag[n] = cd;
}

}  // namespace

cudaError_t launch_coefficients32(const Blk* blks, Space cells, Phys ph, int eu, long long ld,
                                  const double* dt, const double* v, const float* prim32,
                                  const double* mu, const double* mut, const float* sn32,
                                  const double* vol, const double* cson, float* coefe32,
                                  float* coefdiag32, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  if (eu)
    k_coef32<true><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ph, ld, dt, v, prim32, mu,
                                                     mut, sn32, vol, cson, coefe32,
                                                     coefdiag32);
  else
    k_coef32<false><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ph, ld, dt, v, prim32, mu,
                                                      mut, sn32, vol, cson, coefe32,
                                                      coefdiag32);
  return cudaGetLastError();
}

cudaError_t launch_to_float(const double* a, float* b, long long n, cudaStream_t st) {
  if (n > 0) k_to_float<<<(int)((n + 255) / 256), 256, 0, st>>>(a, b, n);
  return cudaGetLastError();
}

cudaError_t launch_defect(const Blk* blks, Space cells, long long ld, const double* u64,
                          const double* ur32, double* corr, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_defect<<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, u64, ur32, corr);
  return cudaGetLastError();
}

template <>
cudaError_t launch_ratio_t<float>(const Blk* blks, const SpaceBuf* lines, int l0,
                                  const float* v, const float* prim, long long ld,
                                  const float* ps, float* R, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = lines[dir].view(l0);
    if (sp.ntiles > 0)
      k_ratio<float><<<dim3(grid_of(sp), 5), kTile, 0, st>>>(blks, sp, dir, v, prim, ld, ps, R);
  }
  return cudaGetLastError();
}

template <>
cudaError_t launch_face_flux_t<float>(const Blk* blks, const SpaceBuf* faces, int l0,
                                      Phys ph, Scheme sc, const float* v, const float* prim,
                                      long long ld, const float* ps, const float* tau,
                                      const float* sn, const float* R, float* G,
                                      cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles == 0) continue;
    if (sc.ns)
      k_face_flux<float, true><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                              ld, ps, tau, sn, R, G);
    else
      k_face_flux<float, false><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                               ld, ps, tau, sn, R, G);
  }
  return cudaGetLastError();
}

// the FP64 face fluxes of the mixed form: the parity kernel compiled in this
// translation unit, i.e. with FMA contraction (each a*b+c rounded once).  The
// result differs from the bit-exact residual by FP64 rounding only, and the
// fused multiply-adds cut the FP64 instruction count of the Roe/viscous flux.
cudaError_t launch_face_flux_fma(const Blk* blks, const SpaceBuf* faces, int l0, Phys ph,
                                 Scheme sc, const double* v, const double* prim,
                                 long long ld, const double* ps, const double* tau,
                                 const double* sn, const double* R, double* G,
                                 cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles == 0) continue;
    if (sc.ns)
      k_face_flux<double, true><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v,
                                                               prim, ld, ps, tau, sn, R, G);
    else
      k_face_flux<double, false><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v,
                                                                prim, ld, ps, tau, sn, R, G);
  }
  return cudaGetLastError();
}

template <>
cudaError_t launch_accumulate_t<float>(const Blk* blks, Space sp, const float* G,
                                       long long ld, const double* corr, double* u,
                                       float* u32, cudaStream_t st) {
  if (sp.ntiles > 0)
    k_accumulate<float><<<grid_of(sp), kTile, 0, st>>>(blks, sp, G, ld, corr, u, u32);
  return cudaGetLastError();
}

template <>
cudaError_t launch_jacobi_25d_t<float>(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                                       long long ld, const float* u, const float* v,
                                       const float* prim, const float* ps, const float* sn,
                                       const float* coefe, const float* coefdiag,
                                       const float* d_in, float* d_out, cudaStream_t st) {
  return jacobi_25d_dispatch<float, 1>(blks, tl, ph, qfix, eu, ld, u, v, prim, ps, sn, coefe,
                                       coefdiag, d_in, d_out, st);
}

cudaError_t init_jacobi_25d_float() { return jacobi_25d_attr<float, 1>(); }

// the FP32 sweeps of the mixed forms: the first per cell, the others
// 2.5D-blocked with the increments in difference form (no stored increments)
template <>
cudaError_t launch_sweeps_t<float>(const Blk* blks, Space cells, Tiles tl, Phys ph, Scheme sc,
                                   int eu, int lmx, long long ld, const float* u,
                                   const float* v, const float* prim, const float* ps,
                                   const float* sn, const float* coefe, const float* coefdiag,
                                   float* const dpp[2], int* cur_out, cudaStream_t st) {
  const int g = grid_of(cells);
  int cur = 0;
  if (lmx == 0) {
    cudaError_t e0 = cudaMemsetAsync(dpp[0], 0, sizeof(float) * 5 * ld, st);
    if (e0 != cudaSuccess) return e0;
  }
  const int q = eu ? sc.qfix_dfez : 0;
  for (int ls = 1; ls <= lmx; ++ls) {
    const int nxt = (ls == 1) ? 0 : 1 - cur;
    const float* din = dpp[cur];
    float* dout = dpp[nxt];
    if (ls == 1) {
      if (g > 0) {
        if (eu)
          k_jacobi_rc<float, true, true><<<g, kTile, 0, st>>>(blks, cells, ph, q, ld, u, v,
                                                              prim, ps, sn, coefe, coefdiag,
                                                              din, dout);
        else
          k_jacobi_rc<float, false, true><<<g, kTile, 0, st>>>(blks, cells, ph, q, ld, u, v,
                                                               prim, ps, sn, coefe, coefdiag,
                                                               din, dout);
      }
    } else {
      cudaError_t e1 = launch_jacobi_25d_t<float>(blks, tl, ph, q, eu, ld, u, v, prim, ps, sn,
                                                  coefe, coefdiag, din, dout, st);
      if (e1 != cudaSuccess) return e1;
    }
    cur = nxt;
  }
  *cur_out = cur;
  return cudaGetLastError();
}

template <>
cudaError_t launch_update_t<float>(const Blk* blks, Space cells, long long ld, const float* d,
                                   double* v, const double* dt, double* d_out,
                                   double* normpart, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_update<float><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, d, v, dt, d_out,
                                                      normpart);
  return cudaGetLastError();
}

}  // namespace cns
