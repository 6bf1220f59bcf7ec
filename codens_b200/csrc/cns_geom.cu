// cns_geom.cu -- grid metrics on the device (run once per grid).
//
// Restates metrics.f90 -> extmhg.f90 (ghost nodes), norm.f90 (face area
// vectors, oriented towards increasing index), svol.f90 (cell volumes),
// rfsc.f90 (volume of coincident ghost cells) and the boundary-entry
// geometry of initns.f90 (inward unit normals) and clidd.f90:64-71 (ghost
// cell centres).  One launch per block and phase: this runs at set-up only.
#include "cns_kernels.cuh"

namespace cns {

namespace {

// extmhg.f90:51-100 with ex1 = 1, ex2 = 0 (solve.f90:384-385)
__global__ void k_extmhg(Blk B, int phase, double* x, double* y, double* z) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double ex1 = 1., ex2 = 0.;
  int i, j, k;
  long long inc;
  int s;
  if (phase == 0) {  // k ghost planes, real i, j
    const long long ni = B.ni, nj = B.nj;
    if (t >= ni * nj * 2) return;
    i = 1 + (int)(t % ni);
    j = 1 + (int)((t / ni) % nj);
    const int side = (int)(t / (ni * nj));
    k = side == 0 ? 0 : B.nk + 1;
    s = side == 0 ? 1 : -1;
    inc = B.nijd;
  } else if (phase == 1) {  // i ghost planes, all k, real j
    const long long nj = B.nj, nkd = B.nkd;
    if (t >= nj * nkd * 2) return;
    j = 1 + (int)(t % nj);
    k = (int)((t / nj) % nkd);
    const int side = (int)(t / (nj * nkd));
    i = side == 0 ? 0 : B.ni + 1;
    s = side == 0 ? 1 : -1;
    inc = 1;
  } else {  // j ghost planes, all k and i
    const long long nid = B.nid, nkd = B.nkd;
    if (t >= nid * nkd * 2) return;
    i = (int)(t % nid);
    k = (int)((t / nid) % nkd);
    const int side = (int)(t / (nid * nkd));
    j = side == 0 ? 0 : B.nj + 1;
    s = side == 0 ? 1 : -1;
    inc = B.nid;
  }
  const long long n = cell_index(B, i, j, k);
  x[n] = ex1 * x[n + s * inc] + ex2 * x[n + s * 2 * inc];
  y[n] = ex1 * y[n + s * inc] + ex2 * y[n + s * 2 * inc];
  z[n] = ex1 * z[n + s * inc] + ex2 * z[n + s * 2 * inc];
}

// face area vector of the quadrilateral whose diagonals are (a->c) and (b->d)
__device__ __forceinline__ void diag_cross(const double* x, const double* y,
                                           const double* z, long long na,
                                           long long nc, long long nb,
                                           long long nd, double& tx, double& ty,
                                           double& tz) {
  const double dx1 = x[nc] - x[na], dy1 = y[nc] - y[na], dz1 = z[nc] - z[na];
  const double dx2 = x[nd] - x[nb], dy2 = y[nd] - y[nb], dz2 = z[nd] - z[nb];
  tx = dy1 * dz2 - dz1 * dy2;
  ty = dz1 * dx2 - dx1 * dz2;
  tz = dx1 * dy2 - dy1 * dx2;
}

// orientation sign of direction dir at the reference node (2,2,2)
// (norm.f90:57-89, 123-155, 189-221)
__device__ double orient(const Blk& B, int dir, const double* x,
                         const double* y, const double* z) {
  const long long nor = cell_index(B, 2, 2, 2);
  const long long I = 1, J = B.nid, K = B.nijd;
  double tx, ty, tz, vx, vy, vz;
  if (dir == 2) {
    diag_cross(x, y, z, nor, nor + I + J, nor + I, nor + J, tx, ty, tz);
    vx = x[nor + K] - x[nor] + x[nor + I + K] - x[nor + I] + x[nor + J + K] -
         x[nor + J] + x[nor + I + J + K] - x[nor + I + J];
    vy = y[nor + K] - y[nor] + y[nor + I + K] - y[nor + I] + y[nor + J + K] -
         y[nor + J] + y[nor + I + J + K] - y[nor + I + J];
    vz = z[nor + K] - z[nor] + z[nor + I + K] - z[nor + I] + z[nor + J + K] -
         z[nor + J] + z[nor + I + J + K] - z[nor + I + J];
  } else if (dir == 1) {
    diag_cross(x, y, z, nor, nor + I + K, nor + I, nor + K, tx, ty, tz);
    vx = x[nor + J] - x[nor] + x[nor + I + J] - x[nor + I] + x[nor + J + K] -
         x[nor + K] + x[nor + I + J + K] - x[nor + I + K];
    vy = y[nor + J] - y[nor] + y[nor + I + J] - y[nor + I] + y[nor + J + K] -
         y[nor + K] + y[nor + I + J + K] - y[nor + I + K];
    vz = z[nor + J] - z[nor] + z[nor + I + J] - z[nor + I] + z[nor + J + K] -
         z[nor + K] + z[nor + I + J + K] - z[nor + I + K];
  } else {
    diag_cross(x, y, z, nor, nor + J + K, nor + J, nor + K, tx, ty, tz);
    vx = x[nor + I] - x[nor] + x[nor + I + J] - x[nor + J] + x[nor + I + K] -
         x[nor + K] + x[nor + I + J + K] - x[nor + J + K];
    vy = y[nor + I] - y[nor] + y[nor + I + J] - y[nor + J] + y[nor + I + K] -
         y[nor + K] + y[nor + I + J + K] - y[nor + J + K];
    vz = z[nor + I] - z[nor] + z[nor + I + J] - z[nor + J] + z[nor + I + K] -
         z[nor + K] + z[nor + I + J + K] - z[nor + J + K];
  }
  return copysign(.5, tx * vx + ty * vy + tz * vz);
}

// norm.f90 loops: normals of direction dir at every node of its range
__global__ void k_snorm(Blk B, int dir, const double* x, const double* y,
                        const double* z, double* sn) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // extents: the normal direction covers 0..n+1, the other two 0..n
  const int e0 = dir == 0 ? B.ni + 2 : B.ni + 1;
  const int e1 = dir == 1 ? B.nj + 2 : B.nj + 1;
  const int e2 = dir == 2 ? B.nk + 2 : B.nk + 1;
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t % e0), j = (int)((t / e0) % e1), k = (int)(t / ((long long)e0 * e1));
  const double sgn = orient(B, dir, x, y, z);
  const long long n = cell_index(B, i, j, k), I = 1, J = B.nid, K = B.nijd;
  double tx, ty, tz;
  if (dir == 2)
    diag_cross(x, y, z, n, n + I + J, n + I, n + J, tx, ty, tz);
  else if (dir == 1)
    diag_cross(x, y, z, n, n + I + K, n + I, n + K, tx, ty, tz);
  else
    diag_cross(x, y, z, n, n + J + K, n + J, n + K, tx, ty, tz);
  sn_wptr(sn, B, dir, 0)[n] = sgn * tx;
  sn_wptr(sn, B, dir, 1)[n] = sgn * ty;
  sn_wptr(sn, B, dir, 2)[n] = sgn * tz;
}

// projection of the face-centre sum on the face area (svol.f90:62-110)
__device__ __forceinline__ double face_moment(const double* x, const double* y,
                                              const double* z, const double* s0,
                                              const double* s1, const double* s2,
                                              long long n, long long a,
                                              long long b) {
  return (x[n] + x[n + a] + x[n + b] + x[n + a + b]) * s0[n] +
         (y[n] + y[n + a] + y[n + b] + y[n + a + b]) * s1[n] +
         (z[n] + z[n + a] + z[n + b] + z[n + a + b]) * s2[n];
}

// svol.f90:130-150: cells 0..ni, 0..nj, 0..nk
__global__ void k_svol(Blk B, const double* x, const double* y, const double* z,
                       const double* sn, double* vol) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e0 = B.ni + 1, e1 = B.nj + 1, e2 = B.nk + 1;
  if (t >= (long long)e0 * e1 * e2) return;
  const int i = (int)(t % e0), j = (int)((t / e0) % e1), k = (int)(t / ((long long)e0 * e1));
  const long long n = cell_index(B, i, j, k), I = 1, J = B.nid, K = B.nijd;
  const double *i0 = sn_ptr(sn, B, 0, 0), *i1 = sn_ptr(sn, B, 0, 1), *i2 = sn_ptr(sn, B, 0, 2);
  const double *j0 = sn_ptr(sn, B, 1, 0), *j1 = sn_ptr(sn, B, 1, 1), *j2 = sn_ptr(sn, B, 1, 2);
  const double *k0 = sn_ptr(sn, B, 2, 0), *k1 = sn_ptr(sn, B, 2, 1), *k2 = sn_ptr(sn, B, 2, 2);
  const double siv1 = face_moment(x, y, z, i0, i1, i2, n, J, K);
  const double siv2 = face_moment(x, y, z, i0, i1, i2, n + I, J, K);
  const double sjv1 = face_moment(x, y, z, j0, j1, j2, n, I, K);
  const double sjv4 = face_moment(x, y, z, j0, j1, j2, n + J, I, K);
  const double skv1 = face_moment(x, y, z, k0, k1, k2, n, I, J);
  const double skv5 = face_moment(x, y, z, k0, k1, k2, n + K, I, J);
  vol[n] = 0.25 * (siv2 - siv1 + sjv4 - sjv1 + skv5 - skv1) / 3.;
}

// rfsc.f90:26-57 for one list entry of a coincident boundary
__global__ void k_rfsc(Bnd bd, double* vol) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int b = bd.ent_bnd[e];
  if (bd.type[b] != BC_RC) return;
  const long long m = e - bd.mpb[b];
  vol[bd.ncbd[e]] = vol[bd.ncin[bd.mpb[bd.partner[b]] + m]];
}

// initns.f90:63-150 (inward unit normal) and clidd.f90:64-71 (ghost centre)
__global__ void k_bnd_geom(const Blk* blks, Bnd bd, const double* y,
                           const double* z, const double* sn) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int b = bd.ent_bnd[e];
  const Blk B = blks[bd.blk[b]];
  const int f = bd.face[b], dir = f / 2, upper = f % 2;
  const double is = upper ? -1. : 1., eps = 1.e-10;
  const long long nf = upper ? bd.ncbd[e] : bd.ncin[e];
  double nx = is * sn_ptr(sn, B, dir, 0)[nf];
  double ny = is * sn_ptr(sn, B, dir, 1)[nf];
  double nz = is * sn_ptr(sn, B, dir, 2)[nf];
  double nn = sqrt(nx * nx + ny * ny + nz * nz);
  nn = nn + (copysign(1., -fabs(nn)) + 1.) * eps;
  bd.nxn[e] = nx / nn;
  bd.nyn[e] = ny / nn;
  bd.nzn[e] = nz / nn;
  const long long n = bd.ncbd[e], I = 1, J = B.nid, K = B.nijd;
  bd.ym[e] = 0.125 * (y[n] + y[n + I] + y[n + J] + y[n + I + J] + y[n + K] +
                      y[n + I + K] + y[n + J + K] + y[n + I + J + K]);
  bd.zm[e] = 0.125 * (z[n] + z[n + I] + z[n + J] + z[n + I + J] + z[n + K] +
                      z[n + I + K] + z[n + J + K] + z[n + I + J + K]);
}

inline int nblocks_for(long long n, int bs) { return (int)((n + bs - 1) / bs); }

}  // namespace

cudaError_t launch_metric(const HostLayout& lay, const Blk* dblks, const Bnd& bd,
                          double* x, double* y, double* z, double* sn,
                          double* vol, cudaStream_t st) {
  const int bs = 256;
  for (const Blk& B : lay.blks) {
    const long long n0 = (long long)B.ni * B.nj * 2;
    const long long n1 = (long long)B.nj * B.nkd * 2;
    const long long n2 = (long long)B.nid * B.nkd * 2;
    k_extmhg<<<nblocks_for(n0, bs), bs, 0, st>>>(B, 0, x, y, z);
    k_extmhg<<<nblocks_for(n1, bs), bs, 0, st>>>(B, 1, x, y, z);
    k_extmhg<<<nblocks_for(n2, bs), bs, 0, st>>>(B, 2, x, y, z);
  }
  for (const Blk& B : lay.blks) {
    for (int dir = 0; dir < 3; ++dir) {
      const long long e = (long long)(dir == 0 ? B.ni + 2 : B.ni + 1) *
                          (dir == 1 ? B.nj + 2 : B.nj + 1) *
                          (dir == 2 ? B.nk + 2 : B.nk + 1);
      k_snorm<<<nblocks_for(e, bs), bs, 0, st>>>(B, dir, x, y, z, sn);
    }
  }
  for (const Blk& B : lay.blks) {
    const long long e = (long long)(B.ni + 1) * (B.nj + 1) * (B.nk + 1);
    k_svol<<<nblocks_for(e, bs), bs, 0, st>>>(B, x, y, z, sn, vol);
  }
  if (bd.nlist > 0) {
    k_rfsc<<<nblocks_for(bd.nlist, bs), bs, 0, st>>>(bd, vol);
    k_bnd_geom<<<nblocks_for(bd.nlist, bs), bs, 0, st>>>(dblks, bd, y, z, sn);
  }
  return cudaGetLastError();
}

}  // namespace cns
