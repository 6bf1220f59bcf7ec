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
    const Blk* __restrict__ blks, Space sp, Phys ph, long long ld, double dtpas,
    const double* __restrict__ dt, const double* __restrict__ v,
    const float* __restrict__ prim, const double* __restrict__ mu,
    const double* __restrict__ mut, const float* __restrict__ sn,
    const double* __restrict__ vol, const double* __restrict__ cson,
    float* __restrict__ coefe, float* __restrict__ coefdiag, float4* __restrict__ snc) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  // the coefficient lane of the sweep's face pack: float 4 (3 m + dir) + 3
  float* const sncw = reinterpret_cast<float*>(snc);
  const float gp = (float)(ph.gam / ph.pr), gpt = (float)(ph.gam / ph.prt);
  auto rv_of = [&](long long m, bool real) -> float {
    if (EU || !real) return 0.f;
    return (gp * (float)mu[m] + gpt * (float)mut[m]) / (float)v[m];
  };
  const float rv0 = rv_of(n, true);
  // dtpas > 0: dual time stepping (implimf_eu.f90:82-85, implimf_3d.f90:213-224)
  float cd = (float)(EU && dtpas > 0. ? vol[n] * (1.5 / dtpas + 1. / dt[n]) : vol[n] / dt[n]);
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
    if (snc) {
      sncw[4 * (3 * n + dir) + 3] = cel;
      if (p == nd - 1) sncw[4 * (3 * nu + dir) + 3] = ceu;
    }
    cd = cd + cel + ceu;
  }
  if (!EU && dtpas > 0.) cd = cd + (float)(1.5 * vol[n] / dtpas);
  coefdiag[n] = cd;
}

}  // namespace

cudaError_t launch_coefficients32(const Blk* blks, Space cells, Phys ph, int eu, long long ld,
                                  double dtpas,
                                  const double* dt, const double* v, const float* prim32,
                                  const double* mu, const double* mut, const float* sn32,
                                  const double* vol, const double* cson, float* coefe32,
                                  float* coefdiag32, float4* snc32, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  if (eu)
    k_coef32<true><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ph, ld, dtpas, dt, v, prim32, mu,
                                                     mut, sn32, vol, cson, coefe32,
                                                     coefdiag32, snc32);
  else
    k_coef32<false><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ph, ld, dtpas, dt, v, prim32, mu,
                                                      mut, sn32, vol, cson, coefe32,
                                                      coefdiag32, snc32);
  return cudaGetLastError();
}

namespace {
// the face lanes of the sweep's pack for every cell of every block
__global__ void __launch_bounds__(256) k_pack_faces32(const Blk* __restrict__ blks, int nblk,
                                                     long long ncells,
                                                     const float* __restrict__ sn,
                                                     float4* __restrict__ snc) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= ncells) return;
  int b = 0;
  while (b + 1 < nblk && q >= blks[b + 1].npc) ++b;
  const Blk& B = blks[b];
  if (q >= B.npc + B.nnn) return;
#pragma unroll
  for (int dir = 0; dir < 3; ++dir)
    snc[3 * q + dir] = make_float4(0.5f * sn_ptr(sn, B, dir, 0)[q], 0.5f * sn_ptr(sn, B, dir, 1)[q],
                                   0.5f * sn_ptr(sn, B, dir, 2)[q], 0.f);
}
}  // namespace

cudaError_t launch_pack_faces32(const Blk* blks, int nblk, long long ncells, const float* sn32,
                                float4* snc32, cudaStream_t st) {
  if (ncells > 0)
    k_pack_faces32<<<(int)((ncells + 255) / 256), 256, 0, st>>>(blks, nblk, ncells, sn32, snc32);
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
                                      cudaStream_t st, float* V) {
  (void)V;  // the single-precision fluxes are Roe only (defect correction)
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
                                 cudaStream_t st, double* V) {
  return face_flux_dispatch(blks, faces, l0, ph, sc, v, prim, ld, ps, tau, sn, R, G, V, st);
}

// the fused residual compiled with contraction (the mixed form's FP64
// residual: FP64 rounding from the bit-exact one, as the face kernels above)
cudaError_t launch_residual_fused_fma(const Blk* blks, Tiles tl, Phys ph, Scheme sc,
                                      const double* v, const double* prim, long long ld,
                                      const double* ps, const double* tau, const double* sn,
                                      const double* R, double* u, float* u32, cudaStream_t st) {
  return residual_fused_dispatch<double>(blks, tl, ph, sc, v, prim, ld, ps, tau, sn, R, u, u32,
                                         st);
}

template <>
cudaError_t launch_accumulate_t<float>(const Blk* blks, Space sp, const float* G,
                                       long long ld, const double* corr, double* u,
                                       float* u32, cudaStream_t st, const float* V) {
  if (sp.ntiles > 0)
    k_accumulate<float><<<grid_of(sp), kTile, 0, st>>>(blks, sp, G, ld, corr, u, u32, V);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 2.5D point-Jacobi sweep of the mixed forms (every sweep after the
// first).  The tiling, the cp.async staging of plane k+2 and the one-cell
// ring are those of k_jacobi_25d; two things differ from its FP64 form:
//
// * shared layout: the increment (d, f) of a staged cell is packed as four
//   float4 quads [d0 d1 d2 d3] [d4 f0 f1 f2] [f3 f4 f5 f6] [f7 f8 - -] in
//   quad-major arrays (quad g of point q at g * NP + q), so a cell reads a
//   neighbour with four 128-bit loads and consecutive threads touch
//   consecutive 16-byte words (no bank conflicts);
// * arithmetic: the face term tn = 0.5 (Phi(U) + Phi(L)) . S is linear in
//   the two cells' flux-increment tensors Phi (rows (d1 d2 d3), (f0 f1 f2),
//   (f1 f4 f5), (f2 f5 f7), (f3 f6 f8)), so a cell sums Phi(nb) . (+-S/2)
//   over its six neighbours plus Phi(self) . (S_lower - S_upper)/2 summed
//   over the directions: 20 fused multiply-adds per neighbour instead of the
//   two face evaluations.  The same sum in exact arithmetic (FP32 rounding
//   differs; the sweep only shapes the increment).
// ---------------------------------------------------------------------------
namespace {

struct Inc {
  float d[5], f[9];
};

__device__ __forceinline__ void quad_load(const float4* __restrict__ s, int np, int q, Inc& x) {
  const float4 a = s[q], b = s[np + q], c = s[2 * np + q], e = s[3 * np + q];
  x.d[0] = a.x; x.d[1] = a.y; x.d[2] = a.z; x.d[3] = a.w;
  x.d[4] = b.x; x.f[0] = b.y; x.f[1] = b.z; x.f[2] = b.w;
  x.f[3] = c.x; x.f[4] = c.y; x.f[5] = c.z; x.f[6] = c.w;
  x.f[7] = e.x; x.f[8] = e.y;
}

__device__ __forceinline__ void quad_store(float4* __restrict__ s, int np, int q,
                                           const float d[5], const float f[9]) {
  s[q] = make_float4(d[0], d[1], d[2], d[3]);
  s[np + q] = make_float4(d[4], f[0], f[1], f[2]);
  s[2 * np + q] = make_float4(f[3], f[4], f[5], f[6]);
  s[3 * np + q] = make_float4(f[7], f[8], 0.f, 0.f);
}

// acc += Phi(x) . w + ce * d(x)
__device__ __forceinline__ void phi_acc(const Inc& x, float w0, float w1, float w2, float ce,
                                        float acc[5]) {
  acc[0] = fmaf(x.d[1], w0, fmaf(x.d[2], w1, fmaf(x.d[3], w2, fmaf(ce, x.d[0], acc[0]))));
  acc[1] = fmaf(x.f[0], w0, fmaf(x.f[1], w1, fmaf(x.f[2], w2, fmaf(ce, x.d[1], acc[1]))));
  acc[2] = fmaf(x.f[1], w0, fmaf(x.f[4], w1, fmaf(x.f[5], w2, fmaf(ce, x.d[2], acc[2]))));
  acc[3] = fmaf(x.f[2], w0, fmaf(x.f[5], w1, fmaf(x.f[7], w2, fmaf(ce, x.d[3], acc[3]))));
  acc[4] = fmaf(x.f[3], w0, fmaf(x.f[6], w1, fmaf(x.f[8], w2, fmaf(ce, x.d[4], acc[4]))));
}

constexpr int kRawF32 = 11;  // staged inputs of one increment: d(5), rho, rho E, p, velocity

template <int TI, int TJ>
constexpr size_t sweep_f32_smem() {
  return sizeof(float4) * 2 * 4 * (TI + 2) * (TJ + 2) +
         sizeof(float) * 2 * kRawF32 * (TI + 2) * (TJ + 2);
}

// one tile (patch t of a block, kc planes) of the sweep
template <bool EU, int TI, int TJ>
__device__ __forceinline__ void sweep_f32_tile(
    const int4 t, const Blk* __restrict__ blks, const Tiles& tl, Phys ph64, int qfix,
    long long ld, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ prim, const float* __restrict__ ps, const float* __restrict__ sn,
    const float* __restrict__ coefe, const float* __restrict__ coefdiag,
    const float* __restrict__ d_in, float* __restrict__ d_out, unsigned char* smem_raw) {
  constexpr int NX = TI + 2, NY = TJ + 2, NP = NX * NY, NT = TI * TJ, NR = kRawF32;
  float4* sq = reinterpret_cast<float4*>(smem_raw);    // [2 planes][4 quads][NP]
  float* sraw = reinterpret_cast<float*>(sq + 2 * 4 * NP);  // [2 planes][NR][NP]
  const Blk B = blks[t.x];
  const int tx = threadIdx.x % TI, ty = threadIdx.x / TI;
  const int i = t.y + tx, j = t.z + ty;
  const int kbeg = t.w, kend = min(t.w + tl.kc, B.nk);
  const bool own = i <= B.ni - 1 && j <= B.nj - 1;
  const float gam1 = (float)ph64.gam1, pinfl = (float)ph64.pinfl;

  // the patch-and-ring points this thread stages and fills (at most two for
  // every shape: NP <= 2 NT): whether the column is inside the block's real
  // cells, and its flat index at k = 0
  constexpr int NQ = (NP + NT - 1) / NT;
  static_assert(NQ <= 2, "a thread stages at most two ring points");
  bool colin[NQ];
  long long col0[NQ];
#pragma unroll
  for (int r = 0; r < NQ; ++r) {
    const int q = threadIdx.x + r * NT;
    const int ii = t.y - 1 + q % NX, jj = t.z - 1 + q / NX;
    colin[r] = q < NP && ii >= 1 && ii <= B.ni - 1 && jj >= 1 && jj <= B.nj - 1;
    col0[r] = colin[r] ? cell_index(B, ii, jj, 0) : 0;
  }
  // the increment inputs of plane kk (patch and ring) into raw buffer b;
  // cells outside the block's real cells are zero-filled
  auto stage = [&](int kk, int b) {
    float* r = sraw + b * NR * NP;
    const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
    for (int rr = 0; rr < NQ; ++rr) {
      const int q = threadIdx.x + rr * NT;
      if (q >= NP) break;
      const bool in = colin[rr] && kin;
      const long long m = in ? col0[rr] + (long long)kk * B.nijd : 0;
#pragma unroll
      for (int a = 0; a < 5; ++a) cp_async_elem(r + a * NP + q, d_in + a * ld + m, in);
      cp_async_elem(r + 5 * NP + q, v + m, in);
      cp_async_elem(r + 6 * NP + q, v + 4 * ld + m, in);
      cp_async_elem(r + 7 * NP + q, ps + m, in);
#pragma unroll
      for (int a = 0; a < 3; ++a) cp_async_elem(r + (8 + a) * NP + q, prim + a * ld + m, in);
    }
  };
  // increments of the staged plane in raw buffer b into quad buffer b
  auto fill = [&](int kk, int b) {
    const float* r = sraw + b * NR * NP;
    float4* s = sq + b * 4 * NP;
    const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
    for (int rr = 0; rr < NQ; ++rr) {
      const int q = threadIdx.x + rr * NT;
      if (q >= NP) break;
      const bool in = colin[rr] && kin;
      float dd[5], f[9];
#pragma unroll
      for (int a = 0; a < 5; ++a) dd[a] = r[a * NP + q];
      if (in) {
        df_diff<float, EU>(dd, r[5 * NP + q], r[6 * NP + q], r[7 * NP + q], r[8 * NP + q],
                           r[9 * NP + q], r[10 * NP + q], gam1, pinfl, qfix, f);
      } else {
#pragma unroll
        for (int a = 0; a < 9; ++a) f[a] = 0.f;
      }
      quad_store(s, NP, q, dd, f);
    }
  };

  // the own column's plane kbeg-1 (registers), and the lower k face area
  Inc pk;
  if (own && kbeg >= 2) {
    cell_df<float, EU, 1>(v, prim, ps, d_in, ld, cell_index(B, i, j, kbeg - 1), gam1, pinfl,
                          qfix, pk.d, pk.f);
  } else {
#pragma unroll
    for (int a = 0; a < 5; ++a) pk.d[a] = 0.f;
#pragma unroll
    for (int a = 0; a < 9; ++a) pk.f[a] = 0.f;
  }
  stage(kbeg, kbeg & 1);
  cp_async_commit();
  stage(kbeg + 1, (kbeg + 1) & 1);
  cp_async_commit();
  cp_async_wait<1>();
  __syncthreads();
  fill(kbeg, kbeg & 1);
  __syncthreads();
  const int q0 = (ty + 1) * NX + tx + 1;
  for (int k = kbeg; k < kend; ++k) {
    // this cell's own inputs, in flight across the barrier
    const long long n = cell_index(B, own ? i : 1, own ? j : 1, k);
    // half face areas and face coefficients from the pack (tl.faces): the
    // cell's three lower faces and the lower faces of its i+1, j+1, k+1
    // neighbours (its upper faces); 0.5 S is exact, so the sums below equal
    // the unpacked form's bit for bit
    float uu[5], cd = 1.f;
    float4 fi, fj, fk, fiu, fju, fku;
    fi = fj = fk = fiu = fju = fku = make_float4(0.f, 0.f, 0.f, 0.f);
    if (own) {
#pragma unroll
      for (int a = 0; a < 5; ++a) uu[a] = u[a * ld + n];
      fi = tl.faces[3 * n];
      fj = tl.faces[3 * n + 1];
      fk = tl.faces[3 * n + 2];
      fiu = tl.faces[3 * (n + 1)];
      fju = tl.faces[3 * (n + B.nid) + 1];
      fku = tl.faces[3 * (n + B.nijd) + 2];
      cd = coefdiag[n];
    }
    cp_async_wait<0>();
    __syncthreads();
    // plane k+2's inputs go into the raw buffer plane k's used
    stage(k + 2, k & 1);
    cp_async_commit();
    fill(k + 1, (k + 1) & 1);
    __syncthreads();
    const float4* s = sq + (k & 1) * 4 * NP;
    const float4* su = sq + ((k + 1) & 1) * 4 * NP;
    Inc c0, x;
    quad_load(s, NP, q0, c0);
    if (own) {
      float acc[5];
#pragma unroll
      for (int a = 0; a < 5; ++a) acc[a] = -uu[a];
      // the cell itself: Phi(c) . (sum of lower minus upper areas) / 2
      phi_acc(c0, (fi.x - fiu.x) + (fj.x - fju.x) + (fk.x - fku.x),
              (fi.y - fiu.y) + (fj.y - fju.y) + (fk.y - fku.y),
              (fi.z - fiu.z) + (fj.z - fju.z) + (fk.z - fku.z), 0.f, acc);
      quad_load(s, NP, q0 - 1, x);
      phi_acc(x, fi.x, fi.y, fi.z, fi.w, acc);
      quad_load(s, NP, q0 + 1, x);
      phi_acc(x, -fiu.x, -fiu.y, -fiu.z, fiu.w, acc);
      quad_load(s, NP, q0 - NX, x);
      phi_acc(x, fj.x, fj.y, fj.z, fj.w, acc);
      quad_load(s, NP, q0 + NX, x);
      phi_acc(x, -fju.x, -fju.y, -fju.z, fju.w, acc);
      phi_acc(pk, fk.x, fk.y, fk.z, fk.w, acc);
      quad_load(su, NP, q0, x);
      phi_acc(x, -fku.x, -fku.y, -fku.z, fku.w, acc);
      const float rc = 1.f / cd;
#pragma unroll
      for (int a = 0; a < 5; ++a) d_out[a * ld + n] = acc[a] * rc;
    }
    pk = c0;
  }
  cp_async_wait<0>();
}

// The sweep over the tile list.  With tl.sched set it is a persistent
// launch: tl.grid CTAs take tiles in turn from the counter sched[0] (each
// tile's result does not depend on the CTA that runs it), and the last CTA
// to finish resets the counter pair for the next launch on the stream.
// Without it, one CTA per tile.
template <bool EU, int TI, int TJ>
__global__ void __launch_bounds__(TI * TJ) k_sweep_f32(
    const Blk* __restrict__ blks, Tiles tl, Phys ph64, int qfix, long long ld,
    const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ prim,
    const float* __restrict__ ps, const float* __restrict__ sn, const float* __restrict__ coefe,
    const float* __restrict__ coefdiag, const float* __restrict__ d_in,
    float* __restrict__ d_out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (!tl.sched) {
    sweep_f32_tile<EU, TI, TJ>(tl.tile[tl.tile0 + blockIdx.x], blks, tl, ph64, qfix, ld, u, v,
                               prim, ps, sn, coefe, coefdiag, d_in, d_out, smem_raw);
    return;
  }
  __shared__ int s_next;
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(&tl.sched[0], 1);
    __syncthreads();
    const int tt = s_next;
    __syncthreads();  // every thread has read s_next before it is taken again
    if (tt >= tl.ntiles) break;
    sweep_f32_tile<EU, TI, TJ>(tl.tile[tl.tile0 + tt], blks, tl, ph64, qfix, ld, u, v, prim,
                               ps, sn, coefe, coefdiag, d_in, d_out, smem_raw);
    __syncthreads();  // the shared buffers are free for the next tile
  }
  if (threadIdx.x == 0) {
    __threadfence();
    // every other CTA has taken its last tile before counting itself out
    if (atomicAdd(&tl.sched[1], 1) == (int)gridDim.x - 1) {
      atomicExch(&tl.sched[0], 0);
      atomicExch(&tl.sched[1], 0);
    }
  }
}

template <int TI, int TJ>
cudaError_t sweep_f32_shape(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu, long long ld,
                            const float* u, const float* v, const float* prim, const float* ps,
                            const float* sn, const float* coefe, const float* coefdiag,
                            const float* d_in, float* d_out, cudaStream_t st) {
  constexpr size_t sm = sweep_f32_smem<TI, TJ>();
  const int grid = tl.sched ? min(tl.grid, tl.ntiles) : tl.ntiles;
  if (grid <= 0 || !tl.faces) return cudaErrorInvalidValue;
  if (eu)
    k_sweep_f32<true, TI, TJ><<<grid, TI * TJ, sm, st>>>(
        blks, tl, ph, qfix, ld, u, v, prim, ps, sn, coefe, coefdiag, d_in, d_out);
  else
    k_sweep_f32<false, TI, TJ><<<grid, TI * TJ, sm, st>>>(
        blks, tl, ph, qfix, ld, u, v, prim, ps, sn, coefe, coefdiag, d_in, d_out);
  return cudaGetLastError();
}

template <int TI, int TJ>
cudaError_t sweep_f32_attr() {
  cudaError_t e = cudaFuncSetAttribute(k_sweep_f32<true, TI, TJ>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sweep_f32_smem<TI, TJ>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_f32<false, TI, TJ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sweep_f32_smem<TI, TJ>());
  return e;
}

}  // namespace

template <>
cudaError_t launch_jacobi_25d_t<float>(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                                       long long ld, const float* u, const float* v,
                                       const float* prim, const float* ps, const float* sn,
                                       const float* coefe, const float* coefdiag,
                                       const float* d_in, float* d_out, cudaStream_t st) {
  if (tl.ntiles == 0) return cudaSuccess;
#define CNS_SHAPE(A, B)                                                                   \
  if (tl.ti == A && tl.tj == B)                                                           \
    return sweep_f32_shape<A, B>(blks, tl, ph, qfix, eu, ld, u, v, prim, ps, sn, coefe,   \
                                 coefdiag, d_in, d_out, st);
  CNS_SHAPE(32, 4)
  CNS_SHAPE(32, 8)
  CNS_SHAPE(16, 8)
  CNS_SHAPE(16, 16)
#undef CNS_SHAPE
  return cudaErrorInvalidValue;
}

// resident CTAs per SM of the FP32 sweep with patch ti x tj (0: unknown shape)
int sweep_f32_blocks_per_sm(int ti, int tj, int eu) {
  int n = 0;
#define CNS_OCC(A, B)                                                                      \
  if (ti == A && tj == B) {                                                                \
    if (eu)                                                                                \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_f32<true, A, B>, A * B,   \
                                                    sweep_f32_smem<A, B>());               \
    else                                                                                   \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_f32<false, A, B>, A * B,  \
                                                    sweep_f32_smem<A, B>());               \
    return n;                                                                              \
  }
  CNS_OCC(32, 4)
  CNS_OCC(32, 8)
  CNS_OCC(16, 8)
  CNS_OCC(16, 16)
#undef CNS_OCC
  return 0;
}

cudaError_t init_jacobi_25d_float() {
  cudaError_t e = sweep_f32_attr<32, 4>();
  if (e == cudaSuccess) e = sweep_f32_attr<32, 8>();
  if (e == cudaSuccess) e = sweep_f32_attr<16, 8>();
  if (e == cudaSuccess) e = sweep_f32_attr<16, 16>();
  return e;
}

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
