// cns_jameson.cu -- the Jameson scheme of the reference (ischema <= 4,
// kprec = 0): the scalar artificial dissipation (dissip_jameson.f90), the
// centred fluxes (sch_jameson.f90) and the ghost refresh that precedes the
// dissipation in atsch_num.f90:448-508 (rfve.f90, rfvc.f90).
//
// Same decomposition as the Roe residual: one thread per face computes the
// face's dissipation or centred flux into the face buffer G[dir][5][n] (n the
// cell above the face), then one thread per cell sums its six faces in the
// reference's order (interior faces ascending, then the lower and the upper
// boundary face of each direction).  FP64, built with --fmad=false, every
// expression in the reference's order: bit-identical to the reference
// semantics.
#include "cns_kernels.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

// rfve.f90:14-31 (mode 1: every non-coincident boundary, ghost = interior)
// and the same-process branch of rfvc.f90 (mode 2: every coincident ghost =
// the partner's coincident interior cell, velocity rotated by the receiving
// boundary's angle)
__global__ void __launch_bounds__(256) k_ghost_refresh(Bnd bd, int mode, double* v,
                                                      long long ld, double* ps, double* temp,
                                                      double* cson) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int bb = bd.ent_bnd[e];
  const bool rc = bd.type[bb] == BC_RC;
  const long long nd = bd.ncbd[e];
  if (mode == 1 && !rc) {
    const long long ni = bd.ncin[e];
    for (int a = 0; a < 5; ++a) v[a * ld + nd] = v[a * ld + ni];
    ps[nd] = ps[ni];
    temp[nd] = temp[ni];
    cson[nd] = cson[ni];
  } else if (mode == 2 && rc) {
    const int p = bd.partner[bb];
    const long long nc = bd.ncin[bd.mpb[p] + (e - bd.mpb[bb])];
    const double c = bd.cosr[bb], s = bd.sinr[bb];
    const double w3 = v[2 * ld + nc], w4 = v[3 * ld + nc];
    v[nd] = v[nc];
    v[ld + nd] = v[ld + nc];
    v[2 * ld + nd] = w3 * c + w4 * s;
    v[3 * ld + nd] = w4 * c - w3 * s;
    v[4 * ld + nd] = v[4 * ld + nc];
    ps[nd] = ps[nc];
    temp[nd] = temp[nc];
    cson[nd] = cson[nc];
  }
}

// pressure sensor of cell c along one direction (dissip_jameson.f90:106-107)
__device__ __forceinline__ double sensor(const double* __restrict__ ps, long long c,
                                         long long inc) {
  return fabs(ps[c + inc] - 2. * ps[c] + ps[c - inc]) / (ps[c + inc] + 2. * ps[c] + ps[c - inc]);
}

// dissipation flux of one face (dissip_jameson.f90:112-204 and the j, k
// twins): interior faces blend 2nd and 4th differences, boundary faces use
// the 2nd difference with the sensor of their real cell
__global__ void __launch_bounds__(kTile) k_dissip_face(const Blk* __restrict__ blks, Space sp,
                                                       int dir,
                                                       const double* __restrict__ v,
                                                       long long ld,
                                                       const double* __restrict__ ps,
                                                       const double* __restrict__ cson,
                                                       const double* __restrict__ sn,
                                                       double* __restrict__ G) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const double ck2 = B.ki2, ck4 = B.ki4;  // ki2(lm), ki4(lm)
  const long long n = cell_index(B, i, j, k);
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const double s1 = sn_ptr(sn, B, dir, 0)[n], s2 = sn_ptr(sn, B, dir, 1)[n],
               s3 = sn_ptr(sn, B, dir, 2)[n];
  const double cnds = s1 * s1 + s2 * s2 + s3 * s3;
  const long long nl = n - inc;
  const double uu = 0.5 * (v[ld + n] / v[n] + v[ld + nl] / v[nl]);
  const double vv = 0.5 * (v[2 * ld + n] / v[n] + v[2 * ld + nl] / v[nl]);
  const double ww = 0.5 * (v[3 * ld + n] / v[n] + v[3 * ld + nl] / v[nl]);
  const double cc = 0.5 * (cson[n] + cson[nl]);
  const double rl = fabs(uu * s1 + vv * s2 + ww * s3) + sqrt(cnds) * cc;
  double* Gd = G + (long long)dir * 5 * ld;
  if (p >= 2 && p <= nd - 1) {
    const double eps2 = ck2 * fmax(sensor(ps, nl, inc), sensor(ps, n, inc));
    const double eps4 = fmax(0., ck4 - eps2);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double* w = v + a * ld;
      Gd[a * ld + n] = eps2 * rl * (w[n] - w[nl]) -
                       eps4 * rl * (w[n + inc] + 3. * (w[nl] - w[n]) - w[nl - inc]);
    }
  } else {
    const double eps2 = p == 1 ? ck2 * sensor(ps, n, inc) : ck2 * sensor(ps, nl, inc);
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double* w = v + a * ld;
      Gd[a * ld + n] = eps2 * rl * (w[n] - w[nl]);
    }
  }
}

// centred cell fluxes of sch_jameson.f90:85-124 (order xx xy xz yy yz zz ex
// ey ez), with the cell stresses and heat flux for Navier-Stokes
__device__ __forceinline__ void jam_cell_flux(const double* __restrict__ v,
                                              const double* __restrict__ ps,
                                              const double* __restrict__ tau, long long ld,
                                              long long n, bool ns, double pinfl,
                                              double F[9]) {
  const double v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n],
               v5 = v[4 * ld + n], p = ps[n];
  if (ns) {
    const double txx = tau[n], txy = tau[ld + n], txz = tau[2 * ld + n], tyy = tau[3 * ld + n],
                 tyz = tau[4 * ld + n], tzz = tau[5 * ld + n], qx = tau[6 * ld + n],
                 qy = tau[7 * ld + n], qz = tau[8 * ld + n];
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

// centred flux of one face (sch_jameson.f90:135-224 and the j, k twins):
// interior faces sum the two cells' fluxes, boundary faces take twice the
// ghost cell's
template <bool NS>
__global__ void __launch_bounds__(kTile) k_jam_face(const Blk* __restrict__ blks, Space sp,
                                                    int dir, double pinfl,
                                                    const double* __restrict__ v,
                                                    long long ld,
                                                    const double* __restrict__ ps,
                                                    const double* __restrict__ tau,
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
  double m3[3], F[9];
  if (p >= 2 && p <= nd - 1) {
    double Fl[9];
    jam_cell_flux(v, ps, tau, ld, n, NS, pinfl, F);
    jam_cell_flux(v, ps, tau, ld, n - inc, NS, pinfl, Fl);
#pragma unroll
    for (int a = 0; a < 3; ++a) m3[a] = v[(a + 1) * ld + n] + v[(a + 1) * ld + n - inc];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = F[q] + Fl[q];
  } else {
    const long long c = p == 1 ? n - inc : n;  // the ghost cell of the face
    jam_cell_flux(v, ps, tau, ld, c, NS, pinfl, F);
#pragma unroll
    for (int a = 0; a < 3; ++a) m3[a] = 2. * v[(a + 1) * ld + c];
#pragma unroll
    for (int q = 0; q < 9; ++q) F[q] = 2. * F[q];
  }
  double* Gd = G + (long long)dir * 5 * ld;
  Gd[n] = m3[0] * s1 + m3[1] * s2 + m3[2] * s3;
  Gd[ld + n] = F[0] * s1 + F[1] * s2 + F[2] * s3;
  Gd[2 * ld + n] = F[1] * s1 + F[3] * s2 + F[4] * s3;
  Gd[3 * ld + n] = F[2] * s1 + F[4] * s2 + F[5] * s3;
  Gd[4 * ld + n] = F[6] * s1 + F[7] * s2 + F[8] * s3;
}

// per-cell sum of the six face values in the reference's order; with dis:
// u = 0.5 * sum - dis (sch_jameson.f90:421-437), else d = sum
__global__ void __launch_bounds__(kTile) k_jam_accumulate(const Blk* __restrict__ blks,
                                                          Space sp,
                                                          const double* __restrict__ G,
                                                          long long ld,
                                                          const double* __restrict__ dis,
                                                          double* __restrict__ out,
                                                          float* __restrict__ out32) {
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
    const double* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
    for (int a = 0; a < 5; ++a) {
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
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double r = dis ? 0.5 * acc[a] - dis[a * ld + n] : acc[a];
    out[a * ld + n] = r;
    if (out32) out32[a * ld + n] = (float)r;
  }
}

}  // namespace

cudaError_t launch_ghost_refresh(const Bnd& bd, int mode, double* v, long long ld, double* ps,
                                 double* temp, double* cson, cudaStream_t st) {
  if (bd.nlist > 0)
    k_ghost_refresh<<<(int)((bd.nlist + 255) / 256), 256, 0, st>>>(bd, mode, v, ld, ps, temp,
                                                                  cson);
  return cudaGetLastError();
}

cudaError_t launch_dissip_jameson(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                                  const double* v, long long ld,
                                  const double* ps, const double* cson, const double* sn,
                                  double* G, double* d, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles > 0)
      k_dissip_face<<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, v, ld, ps, cson,
                                                   sn, G);
  }
  if (cells.ntiles > 0)
    k_jam_accumulate<<<grid_of(cells), kTile, 0, st>>>(blks, cells, G, ld, nullptr, d,
                                                       nullptr);
  return cudaGetLastError();
}

cudaError_t launch_sch_jameson(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                               int ns, double pinfl, const double* v, long long ld,
                               const double* ps, const double* tau, const double* sn,
                               const double* dis, double* G, double* u, float* u32,
                               cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles == 0) continue;
    if (ns)
      k_jam_face<true><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, pinfl, v, ld, ps, tau, sn,
                                                      G);
    else
      k_jam_face<false><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, pinfl, v, ld, ps, tau,
                                                       sn, G);
  }
  if (cells.ntiles > 0)
    k_jam_accumulate<<<grid_of(cells), kTile, 0, st>>>(blks, cells, G, ld, dis, u, u32);
  return cudaGetLastError();
}

}  // namespace cns
