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
#include <cuda.h>

#include "cns_kernels.cuh"
// the Roe dissipation of this translation unit's face fluxes with one
// reciprocal per divisor (the hot kernels are internal to each unit)
#define CNS_RECIP_DIV 1
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

// spectral radius of the face between cells h (upper side) and l, from their
// packed inputs q = (u, v, w, c) and (vol, rv); rvh, rvl the viscous factors
// (zero off the real cells, as the reference's zeroed rv)
template <bool EU>
__device__ __forceinline__ float face_coef(const float4 qh, const float4 ql, float volh,
                                           float voll, float sx, float sy, float sz,
                                           float rvh, float rvl) {
  const float cnds = sx * sx + sy * sy + sz * sz;
  const float cc = 0.5f * (qh.w + ql.w);
  const float uu = 0.5f * (qh.x + ql.x);
  const float vv = 0.5f * (qh.y + ql.y);
  const float ww = 0.5f * (qh.z + ql.z);
  const float vn = uu * sx + vv * sy + ww * sz;
  if (EU) return 0.5f * fabsf(vn) + sqrtf(cnds) * cc;
  return 0.5f * (fabsf(vn) + sqrtf(cnds) * cc) + (rvh + rvl) * cnds / (volh + voll);
}

// the implicit coefficients of the FP32 sweeps in one pass (the FP32 form of
// implimf_3d.f90:111-203 / implimf_eu.f90:124-170): each real cell evaluates
// the spectral radii of its six faces, stores the lower faces (and the upper
// one at the end of each line) and sums the diagonal in the reference order.
// Every interior face is evaluated by both its cells (cheaper than a second
// pass over memory); a neighbour's inputs are two vector loads of the packed
// cq32 = (u, v, w, c) and cv32 = (vol, rv) the primitive kernel writes.
// With d1 given, the cell's first Jacobi iterate too: with a zero previous
// iterate every face term of the first sweep is zero, so d1 = -u / cd
// (the value k_jacobi_rc<FIRST> computes, up to the sign of a zero), in
// the padded layout.
template <bool EU>
__global__ void __launch_bounds__(kTile) k_coef32(
    const Blk* __restrict__ blks, Space sp, long long ld, double dtpas,
    const double* __restrict__ dt, const double* __restrict__ vol,
    const float4* __restrict__ cq, const float2* __restrict__ cv,
    const float* __restrict__ sn, float* __restrict__ coefe, float* __restrict__ coefdiag,
    float4* __restrict__ snc, const float* __restrict__ u32, float* __restrict__ d1) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const float4 q0 = cq[n];
  const float2 c0 = cv[n];
  const float rv0 = EU ? 0.f : c0.y;
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
    const float4 ql = cq[nl], qu = cq[nu];
    const float2 cl = cv[nl], cu = cv[nu];
    const float rvl = (EU || p <= 1) ? 0.f : cl.y;
    const float rvu = (EU || p >= nd - 1) ? 0.f : cu.y;
    const float cel = face_coef<EU>(q0, ql, c0.x, cl.x, s0[n], s1[n], s2[n], rv0, rvl);
    const float ceu = face_coef<EU>(qu, q0, cu.x, c0.x, s0[nu], s1[nu], s2[nu], rvu, rv0);
    coefe[(long long)dir * ld + n] = cel;
    if (p == nd - 1) coefe[(long long)dir * ld + nu] = ceu;
    if (snc) {
      // the sweep's face pack, whole 16-byte entries (half the face's area
      // vector, as k_pack_faces32 writes it, and its coefficient): a store of
      // the coefficient lane alone would make the memory system fetch the
      // rest of each entry first
      snc[3 * n + dir] = make_float4(0.5f * s0[n], 0.5f * s1[n], 0.5f * s2[n], cel);
      if (p == nd - 1)
        snc[3 * nu + dir] = make_float4(0.5f * s0[nu], 0.5f * s1[nu], 0.5f * s2[nu], ceu);
    }
    cd = cd + cel + ceu;
  }
  if (!EU && dtpas > 0.) cd = cd + (float)(1.5 * vol[n] / dtpas);
  coefdiag[n] = cd;
  if (d1) {
    const long long pn = pad_index(B, i, j, k);
#pragma unroll
    for (int a = 0; a < 5; ++a) d1[a * B.pld + pn] = -u32[a * ld + n] / cd;
  }
}

}  // namespace

cudaError_t launch_coefficients32(const Blk* blks, Space cells, int eu, long long ld,
                                  double dtpas, const double* dt, const double* vol,
                                  const float4* cq32, const float2* cv32, const float* sn32,
                                  float* coefe32, float* coefdiag32, float4* snc32,
                                  const float* u32, float* d1, cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  if (eu)
    k_coef32<true><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, dtpas, dt, vol, cq32,
                                                     cv32, sn32, coefe32, coefdiag32, snc32,
                                                     u32, d1);
  else
    k_coef32<false><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, dtpas, dt, vol, cq32,
                                                      cv32, sn32, coefe32, coefdiag32, snc32,
                                                      u32, d1);
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

// The sweep's staged plane: the padded arrays are read as boxes of
// (TI + 4) x (TJ + 2) points per component (the patch, its one-cell ring and
// two columns of overhang that keep the box rows a multiple of 16 bytes);
// the iterate's five components and the six state values each form one box
// stack, [component][row][column] in shared memory.
template <int TI, int TJ>
struct Sw32 {
  static constexpr int NX = TI + 2, NY = TJ + 2, NP = NX * NY, NT = TI * TJ;
  static constexpr int NXP = TI + 4;          // box row (floats)
  static constexpr int PL = NY * NXP;         // one component's box (floats)
  static constexpr int RD = (5 * PL * 4 + 127) / 128 * 128;  // iterate boxes (bytes)
  static constexpr int RS = (6 * PL * 4 + 127) / 128 * 128;  // state boxes (bytes)
  static constexpr int TX = 11 * PL * 4;      // bytes one plane's boxes deliver
  static constexpr size_t QUAD = sizeof(float4) * 2 * 4 * NP;
  // 128 bytes of slack align the dynamic shared memory by hand
  static constexpr size_t SMEM = 128 + QUAD + 2 * (size_t)(RD + RS);
  static_assert(NXP * 4 % 16 == 0, "box rows must be a multiple of 16 bytes");
  static_assert(QUAD % 128 == 0, "the raw boxes start 128-byte aligned");
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// about two seconds at the B200's clocks: a box that has not landed by then
// never will, and the sweep gives up (status bit 4) instead of spinning
constexpr long long kBoxWaitCycles = 4000000000LL;

__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > kBoxWaitCycles) return false;
  return true;
}

// one 4D box (x, y, z, component) of a tensor map into shared memory,
// completing on the transaction count of bar
__device__ __forceinline__ void box_load(void* dst, const CUtensorMap* map,
                                         unsigned long long* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(0),
      "r"(smem_u32(bar))
      : "memory");
}

// the sweep's shared state of one CTA: the two quad planes, the two raw
// planes and (box staging) one transaction barrier per raw plane
struct Sw32Smem {
  float4* sq;
  unsigned char* raw;
  unsigned long long* bar;
};

// one tile (patch t of a block, kc planes) of the sweep.  Returns false
// (every thread alike) when a box wait gave up.
template <bool EU, int TI, int TJ, bool BOX>
__device__ __forceinline__ bool sweep_f32_tile(const int4 t, const Blk* __restrict__ blks,
                                               const Tiles& tl, Phys ph64, int qfix,
                                               long long ld, const Sweep32& a,
                                               const float* __restrict__ d_in,
                                               float* __restrict__ d_out,
                                               const CUtensorMap* map_d, Sw32Smem sm,
                                               unsigned& phase) {
  using S = Sw32<TI, TJ>;
  constexpr int NX = S::NX, NP = S::NP, NT = S::NT, NXP = S::NXP, PL = S::PL;
  const Blk B = blks[t.x];
  const long long pld = B.pld;
  const float* __restrict__ u = a.u;
  const float* __restrict__ st = a.st;
  const int tx = threadIdx.x % TI, ty = threadIdx.x / TI;
  const int i = t.y + tx, j = t.z + ty;
  const int kbeg = t.w, kend = min(t.w + tl.kc, B.nk);
  const bool own = i <= B.ni - 1 && j <= B.nj - 1;
  const float gam1 = (float)ph64.gam1, pinfl = (float)ph64.pinfl;
  const int x0 = t.y - 1, y0 = t.z - 1;

  // the patch-and-ring points this thread fills (at most two for every
  // shape: NP <= 2 NT): whether the column is inside the block's real cells
  // and its offset in a component's box
  constexpr int NQ = (NP + NT - 1) / NT;
  static_assert(NQ <= 2, "a thread fills at most two ring points");
  bool colin[NQ];
  int boxo[NQ];
#pragma unroll
  for (int r = 0; r < NQ; ++r) {
    const int q = threadIdx.x + r * NT;
    const int qx = q % NX, qy = q / NX;
    const int ii = x0 + qx, jj = y0 + qy;
    colin[r] = q < NP && ii >= 1 && ii <= B.ni - 1 && jj >= 1 && jj <= B.nj - 1;
    boxo[r] = qy * NXP + qx;
  }
  auto raw_d = [&](int b) { return reinterpret_cast<float*>(sm.raw + b * (S::RD + S::RS)); };
  auto raw_s = [&](int b) {
    return reinterpret_cast<float*>(sm.raw + b * (S::RD + S::RS) + S::RD);
  };
  // the increment inputs of plane kk (patch and ring) into raw plane b
  auto stage = [&](int kk, int b) {
    if (BOX) {
      if (threadIdx.x == 0) {
        // the generic-proxy reads of this raw plane (before the barrier
        // that precedes this call) are ordered before the boxes' writes
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&sm.bar[b], S::TX);
        box_load(raw_d(b), map_d + t.x, &sm.bar[b], x0, y0, kk);
        box_load(raw_s(b), static_cast<const CUtensorMap*>(a.map_st) + t.x, &sm.bar[b], x0,
                 y0, kk);
      }
    } else {
      float* rd = raw_d(b);
      float* rs = raw_s(b);
      const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
      for (int rr = 0; rr < NQ; ++rr) {
        const int q = threadIdx.x + rr * NT;
        if (q >= NP) break;
        const bool in = colin[rr] && kin;
        const long long m = in ? pad_index(B, x0 + q % NX, y0 + q / NX, kk) : B.ppc;
        const int o = boxo[rr];
#pragma unroll
        for (int c = 0; c < 5; ++c) cp_async_elem(rd + c * PL + o, d_in + c * pld + m, in);
#pragma unroll
        for (int c = 0; c < 6; ++c) cp_async_elem(rs + c * PL + o, st + c * pld + m, in);
      }
      cp_async_commit();
    }
  };
  // raw plane b of plane kk has landed (box staging: every thread waits on
  // the plane's barrier; cp.async: on its own copies).  Then a block-wide
  // vote: false when any thread's wait gave up.
  auto arrived = [&](int b, bool last_in_flight) -> bool {
    bool ok = true;
    if (BOX) {
      ok = mbar_wait_bounded(&sm.bar[b], (phase >> b) & 1u);
      phase ^= 1u << b;
    } else if (last_in_flight) {
      cp_async_wait<0>();
    } else {
      cp_async_wait<1>();
    }
    return !__syncthreads_or(!ok);
  };
  // increments of the staged plane in raw plane b into quad plane b; cells
  // outside the block's real cells are zero
  auto fill = [&](int kk, int b) {
    const float* rd = raw_d(b);
    const float* rs = raw_s(b);
    float4* s = sm.sq + b * 4 * NP;
    const bool kin = kk >= 1 && kk <= B.nk - 1;
#pragma unroll
    for (int rr = 0; rr < NQ; ++rr) {
      const int q = threadIdx.x + rr * NT;
      if (q >= NP) break;
      const bool in = colin[rr] && kin;
      const int o = boxo[rr];
      float dd[5], f[9];
#pragma unroll
      for (int c = 0; c < 5; ++c) dd[c] = in ? rd[c * PL + o] : 0.f;
      if (in) {
        df_diff<float, EU>(dd, rs[o], rs[PL + o], rs[2 * PL + o], rs[3 * PL + o],
                           rs[4 * PL + o], rs[5 * PL + o], gam1, pinfl, qfix, f);
      } else {
#pragma unroll
        for (int c = 0; c < 9; ++c) f[c] = 0.f;
      }
      quad_store(s, NP, q, dd, f);
    }
  };
  // a failed wait: the boxes still in flight are waited for (bounded) before
  // the CTA gives up, so none lands in shared memory it no longer owns
  auto drain = [&](unsigned pending) {
    if (!BOX) {
      cp_async_wait<0>();
      return;
    }
#pragma unroll
    for (int b = 0; b < 2; ++b)
      if (pending & (1u << b)) (void)mbar_wait_bounded(&sm.bar[b], (phase >> b) & 1u);
  };

  // the own column's plane kbeg-1 (registers), read from global memory
  Inc pk;
  if (own && kbeg >= 2) {
    const long long pm = pad_index(B, i, j, kbeg - 1);
#pragma unroll
    for (int c = 0; c < 5; ++c) pk.d[c] = d_in[c * pld + pm];
    df_diff<float, EU>(pk.d, st[pm], st[pld + pm], st[2 * pld + pm], st[3 * pld + pm],
                       st[4 * pld + pm], st[5 * pld + pm], gam1, pinfl, qfix, pk.f);
  } else {
#pragma unroll
    for (int c = 0; c < 5; ++c) pk.d[c] = 0.f;
#pragma unroll
    for (int c = 0; c < 9; ++c) pk.f[c] = 0.f;
  }
  stage(kbeg, kbeg & 1);
  stage(kbeg + 1, (kbeg + 1) & 1);
  if (!arrived(kbeg & 1, false)) {
    drain(1u << ((kbeg + 1) & 1));
    return false;
  }
  fill(kbeg, kbeg & 1);
  __syncthreads();
  const int q0 = (ty + 1) * NX + tx + 1;
  // the lower k face of the own cell, carried from plane to plane (the
  // upper k face of plane k is the lower one of plane k+1)
  float4 fkc = own ? tl.faces[3 * cell_index(B, i, j, kbeg) + 2]
                   : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int k = kbeg; k < kend; ++k) {
    // this cell's own inputs, in flight across the barrier
    const long long n = cell_index(B, own ? i : 1, own ? j : 1, k);
    // half face areas and face coefficients from the pack (tl.faces): the
    // cell's three lower faces and the lower faces of its i+1, j+1, k+1
    // neighbours (its upper faces); 0.5 S is exact, so the sums below equal
    // the unpacked form's bit for bit
    float uu[5], cd = 1.f;
    float4 fi, fj, fiu, fju, fku;
    const float4 fk = fkc;
    fi = fj = fiu = fju = fku = make_float4(0.f, 0.f, 0.f, 0.f);
    if (own) {
#pragma unroll
      for (int c = 0; c < 5; ++c) uu[c] = u[c * ld + n];
      fi = tl.faces[3 * n];
      fj = tl.faces[3 * n + 1];
      fiu = tl.faces[3 * (n + 1)];
      fju = tl.faces[3 * (n + B.nid) + 1];
      fku = tl.faces[3 * (n + B.nijd) + 2];
      cd = a.coefdiag[n];
    }
    fkc = fku;
    // plane k+1 has landed; plane k's raw plane is free
    if (!arrived((k + 1) & 1, true)) {
      drain(0u);
      return false;
    }
    // plane k+2's inputs go into the raw plane that plane k used
    stage(k + 2, k & 1);
    fill(k + 1, (k + 1) & 1);
    __syncthreads();
    const float4* s = sm.sq + (k & 1) * 4 * NP;
    const float4* su = sm.sq + ((k + 1) & 1) * 4 * NP;
    Inc c0, x;
    quad_load(s, NP, q0, c0);
    if (own) {
      float acc[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) acc[c] = -uu[c];
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
      const long long pn = pad_index(B, i, j, k);
#pragma unroll
      for (int c = 0; c < 5; ++c) d_out[c * pld + pn] = acc[c] * rc;
    }
    pk = c0;
  }
  // plane kend+1 (staged by the last plane) is still in flight
  if (!arrived((kend + 1) & 1, true)) return false;
  return true;
}

// The sweep over the tile list.  With tl.sched set it is a persistent
// launch: tl.grid CTAs take tiles in turn from the counter sched[0] (each
// tile's result does not depend on the CTA that runs it), and the last CTA
// to finish resets the counter pair for the next launch on the stream.
// Without it, one CTA per tile.  A CTA whose box wait gave up sets status
// bit 4 and takes no further tile.
template <bool EU, int TI, int TJ, bool BOX>
__global__ void __launch_bounds__(TI * TJ) k_sweep_f32(const Blk* __restrict__ blks, Tiles tl,
                                                      Phys ph64, int qfix, long long ld,
                                                      Sweep32 a, const float* __restrict__ d_in,
                                                      float* __restrict__ d_out,
                                                      const CUtensorMap* __restrict__ map_d) {
  extern __shared__ unsigned char smem_dyn[];
  __shared__ __align__(8) unsigned long long bar[2];
  __shared__ int s_next;
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  Sw32Smem sm{reinterpret_cast<float4*>(base), base + Sw32<TI, TJ>::QUAD, bar};
  if (BOX) {
    if (threadIdx.x == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
  }
  unsigned phase = 0;
  if (!tl.sched) {
    if (!sweep_f32_tile<EU, TI, TJ, BOX>(tl.tile[tl.tile0 + blockIdx.x], blks, tl, ph64, qfix,
                                         ld, a, d_in, d_out, map_d, sm, phase) &&
        threadIdx.x == 0)
      atomicOr(a.status, 4);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) s_next = atomicAdd(&tl.sched[0], 1);
    __syncthreads();
    const int tt = s_next;
    __syncthreads();  // every thread has read s_next before it is taken again
    if (tt >= tl.ntiles) break;
    if (!sweep_f32_tile<EU, TI, TJ, BOX>(tl.tile[tl.tile0 + tt], blks, tl, ph64, qfix, ld, a,
                                         d_in, d_out, map_d, sm, phase)) {
      if (threadIdx.x == 0) atomicOr(a.status, 4);
      break;
    }
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
int shape_index() {
  for (int sh = 0; sh < kSweepShapes; ++sh)
    if (kSweepShape[sh][0] == TI && kSweepShape[sh][1] == TJ) return sh;
  return -1;
}

template <int TI, int TJ, bool BOX>
cudaError_t sweep_f32_launch(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                             long long ld, const Sweep32& a, const float* d_in, float* d_out,
                             const CUtensorMap* map_d, cudaStream_t st) {
  constexpr size_t sm = Sw32<TI, TJ>::SMEM;
  const int grid = tl.sched ? min(tl.grid, tl.ntiles) : tl.ntiles;
  if (grid <= 0 || !tl.faces) return cudaErrorInvalidValue;
  if (eu)
    k_sweep_f32<true, TI, TJ, BOX><<<grid, TI * TJ, sm, st>>>(blks, tl, ph, qfix, ld, a, d_in,
                                                               d_out, map_d);
  else
    k_sweep_f32<false, TI, TJ, BOX><<<grid, TI * TJ, sm, st>>>(blks, tl, ph, qfix, ld, a, d_in,
                                                                d_out, map_d);
  return cudaGetLastError();
}

template <int TI, int TJ>
cudaError_t sweep_f32_shape(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu, long long ld,
                            const Sweep32& a, int din_sel, const float* d_in, float* d_out,
                            cudaStream_t st) {
  if (a.maps) {
    const CUtensorMap* m = static_cast<const CUtensorMap*>(a.maps) +
                           (long long)(shape_index<TI, TJ>() * 3 + 1 + din_sel) * a.nblk;
    Sweep32 b = a;
    b.map_st = static_cast<const CUtensorMap*>(a.maps) +
               (long long)(shape_index<TI, TJ>() * 3) * a.nblk;
    return sweep_f32_launch<TI, TJ, true>(blks, tl, ph, qfix, eu, ld, b, d_in, d_out, m, st);
  }
  return sweep_f32_launch<TI, TJ, false>(blks, tl, ph, qfix, eu, ld, a, d_in, d_out, nullptr,
                                         st);
}

template <int TI, int TJ>
cudaError_t sweep_f32_attr() {
  const int sm = (int)Sw32<TI, TJ>::SMEM;
  cudaError_t e = cudaFuncSetAttribute(k_sweep_f32<true, TI, TJ, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_f32<false, TI, TJ, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_f32<true, TI, TJ, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep_f32<false, TI, TJ, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  return e;
}

}  // namespace

cudaError_t launch_sweep32_25d(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                               long long ld, const Sweep32& a, int din_sel, const float* d_in,
                               float* d_out, cudaStream_t st) {
  if (tl.ntiles == 0) return cudaSuccess;
#define CNS_SHAPE(A, B)                                                                   \
  if (tl.ti == A && tl.tj == B)                                                           \
    return sweep_f32_shape<A, B>(blks, tl, ph, qfix, eu, ld, a, din_sel, d_in, d_out, st);
  CNS_SHAPE(32, 4)
  CNS_SHAPE(32, 8)
  CNS_SHAPE(16, 8)
  CNS_SHAPE(16, 16)
#undef CNS_SHAPE
  return cudaErrorInvalidValue;
}

// resident CTAs per SM of the FP32 sweep with patch ti x tj (0: unknown shape)
int sweep_f32_blocks_per_sm(int ti, int tj, int eu, int box) {
  int n = 0;
#define CNS_OCC1(A, B, E, X)                                                              \
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_sweep_f32<E, A, B, X>, A * B,       \
                                                Sw32<A, B>::SMEM)
#define CNS_OCC(A, B)                                                                     \
  if (ti == A && tj == B) {                                                               \
    if (eu && box) CNS_OCC1(A, B, true, true);                                            \
    else if (eu) CNS_OCC1(A, B, true, false);                                             \
    else if (box) CNS_OCC1(A, B, false, true);                                            \
    else CNS_OCC1(A, B, false, false);                                                    \
    return n;                                                                             \
  }
  CNS_OCC(32, 4)
  CNS_OCC(32, 8)
  CNS_OCC(16, 8)
  CNS_OCC(16, 16)
#undef CNS_OCC
#undef CNS_OCC1
  return 0;
}

cudaError_t init_jacobi_25d_float() {
  cudaError_t e = sweep_f32_attr<32, 4>();
  if (e == cudaSuccess) e = sweep_f32_attr<32, 8>();
  if (e == cudaSuccess) e = sweep_f32_attr<16, 8>();
  if (e == cudaSuccess) e = sweep_f32_attr<16, 16>();
  return e;
}

// The tensor maps of the box staging: for every patch shape and block, the
// state st and the two iterates as 4D tensors (column, row, plane,
// component) of the block's padded box, boxes of (ti + 4) x (tj + 2) x 1 x
// ncomp.  Reads outside the block's padded box fill with zeros (never used:
// such points lie outside the real cells).
cudaError_t encode_sweep32_maps(const std::vector<Blk>& blks, const float* st,
                                float* const dpp[2], std::vector<unsigned char>& out) {
  using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q{};
  cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
  if (e != cudaSuccess) return e;
  if (!fn || q != cudaDriverEntryPointSuccess) return cudaErrorNotSupported;
  const Encode encode = reinterpret_cast<Encode>(fn);
  const size_t nblk = blks.size();
  out.assign(sizeof(CUtensorMap) * kSweepShapes * 3 * nblk, 0);
  CUtensorMap* maps = reinterpret_cast<CUtensorMap*>(out.data());
  for (int sh = 0; sh < kSweepShapes; ++sh)
    for (int arr = 0; arr < 3; ++arr)
      for (size_t b = 0; b < nblk; ++b) {
        const Blk& B = blks[b];
        const float* base = arr == 0 ? st : dpp[arr - 1];
        const cuuint32_t ncomp = arr == 0 ? 6 : 5;
        void* addr = const_cast<float*>(base + B.ppc);
        const cuuint64_t dims[4] = {(cuuint64_t)B.pid, (cuuint64_t)B.njd, (cuuint64_t)B.nkd,
                                    ncomp};
        const cuuint64_t strides[3] = {(cuuint64_t)B.pid * 4, (cuuint64_t)B.pnijd * 4,
                                       (cuuint64_t)B.pld * 4};
        const cuuint32_t box[4] = {(cuuint32_t)kSweepShape[sh][0] + 4,
                                   (cuuint32_t)kSweepShape[sh][1] + 2, 1, ncomp};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        if ((reinterpret_cast<uintptr_t>(addr) & 15) || (strides[0] & 15) ||
            (strides[1] & 15) || (strides[2] & 15))
          return cudaErrorInvalidValue;
        const CUresult r = encode(&maps[(sh * 3 + arr) * nblk + b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                  4, addr, dims, strides, box, estr,
                                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
      }
  return cudaSuccess;
}

// the FP32 sweeps of the mixed forms after the first, whose iterate the
// coefficient kernel writes into dpp[0] (launch_coefficients32): 2.5D-blocked,
// with the increments in difference form (no stored increments)
cudaError_t launch_sweeps32(Tiles tl, const Blk* blks, Phys ph, Scheme sc, int eu, int lmx,
                            long long ld, long long ldp, const Sweep32& a,
                            float* const dpp[2], int* cur_out, cudaStream_t st) {
  int cur = 0;
  if (lmx == 0) {
    cudaError_t e0 = cudaMemsetAsync(dpp[0], 0, sizeof(float) * 5 * ldp, st);
    if (e0 != cudaSuccess) return e0;
  }
  const int q = eu ? sc.qfix_dfez : 0;
  for (int ls = 2; ls <= lmx; ++ls) {
    cudaError_t e1 = launch_sweep32_25d(blks, tl, ph, q, eu, ld, a, cur, dpp[cur], dpp[1 - cur],
                                        st);
    if (e1 != cudaSuccess) return e1;
    cur = 1 - cur;
  }
  *cur_out = cur;
  return cudaGetLastError();
}

cudaError_t launch_update32(const Blk* blks, Space cells, long long ld, const float* d,
                            double* v, const double* dt, double* normpart, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_update<float, true><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, d, v, dt, nullptr,
                                                            normpart);
  return cudaGetLastError();
}

}  // namespace cns
