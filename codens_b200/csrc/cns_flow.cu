// cns_flow.cu -- per-iteration kernels of the CodeNS hot path on sm_100a:
// thermodynamics (zpres, zvismo), local time step (chronos), boundary
// conditions and coincident halos (rbord, rbte, rbtc), viscous gradients and
// stresses (zgrad2 + zfluto), Roe-MUSCL face fluxes (sch_roe_euler, sch_roe
// with the in-place limiter recurrence), the face-owned accumulation of the
// residual, the matrix-free point-Jacobi implicit phase (implimf_eu,
// implimf_3d) and the residual norms (residu, rscpsv).
//
// Residual accumulation is face-owned, not atomic: each face flux is computed
// once into a face buffer, then every cell sums its six faces in exactly the
// order in which the reference's loops add them (interior faces in ascending
// order, then the lower and the upper boundary face), which keeps the FP64
// result bit-identical.
#include <math_constants.h>

#include "cns_kernels.cuh"
#include "cns_pmath.h"
#include "cns_hot.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

// ---------------------------------------------------------------------------
// thermodynamics
// ---------------------------------------------------------------------------

// zpres.f90:66-79 and, for the Navier-Stokes equations, zvismo.f90:77-104,
// of cell n; returns c (and mu through *mu_n when with_mu)
__device__ __forceinline__ double zpres_cell(Phys ph, int with_mu,
                                             const double* __restrict__ v, long long ld,
                                             long long n, double* ps, double* temp,
                                             double* cson, double* mu, int* status,
                                             double* mu_n) {
  const double v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n],
               v5 = v[4 * ld + n];
  const double rhoe = v5 - 0.5 * (sq(v2) + sq(v3) + sq(v4)) / v1;
  const double p = ph.gam1 * (rhoe - ph.pinfl);
  const double t = ph.gam * p / v1;
  ps[n] = p;
  temp[n] = t;
  const double c = sqrt(t);
  cson[n] = c;
  if (with_mu) {
    // the reference aborts on T <= 0 (zvismo.f90:123-127); here the status
    // word records it and the host turns it into an error code
    double m;
    if (t <= 0.) {
      m = 0.;
      atomicOr(status, 1);
    } else {
      const double usrey = 1. / ph.reynz, a = ph.suth_a;
      m = usrey * t * sqrt(t) * (1. + a) / (t + a);
    }
    mu[n] = m;
    *mu_n = m;
  }
  return c;
}

__global__ void __launch_bounds__(kTile) k_zpres(const Blk* __restrict__ blks,
                                                 Space sp, Phys ph, int with_mu,
                                                 const double* __restrict__ v,
                                                 long long ld, double* ps,
                                                 double* temp, double* cson,
                                                 double* mu, int* status) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  double m;
  (void)zpres_cell(ph, with_mu, v, ld, n, ps, temp, cson, mu, status, &m);
}

// zvismo.f90:77-104 alone (temperature already known)
__global__ void __launch_bounds__(kTile) k_zvismo(const Blk* __restrict__ blks,
                                                  Space sp, Phys ph, double* mu,
                                                  const double* __restrict__ temp,
                                                  int* status) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double t = temp[n];
  if (t <= 0.) {
    mu[n] = 0.;
    atomicOr(status, 1);
  } else {
    const double usrey = 1. / ph.reynz, a = ph.suth_a;
    mu[n] = usrey * t * sqrt(t) * (1. + a) / (t + a);
  }
}

// primitive velocities u = rho u / rho (and v, w) of every cell of a flat
// range, once per iteration after the boundary conditions: the face fluxes,
// the limiter ratios, the gradients and the implicit phase all use these very
// quotients (the reference recomputes them at every use, with identical
// results), so sharing them changes no bit
template <bool SHADOW>
__global__ void __launch_bounds__(256) k_prim(long long n0, long long n1,
                                             const double* __restrict__ v,
                                             long long ld, double* __restrict__ prim,
                                             const double* __restrict__ ps, PrimShadow sh) {
  const long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n1) return;
  const double r = v[n];
  const double q0 = v[ld + n] / r, q1 = v[2 * ld + n] / r, q2 = v[3 * ld + n] / r;
  prim[n] = q0;
  prim[ld + n] = q1;
  prim[2 * ld + n] = q2;
  if (SHADOW) {
    // the single-precision copies (PrimShadow)
    const float r32 = (float)r, e32 = (float)v[4 * ld + n], p32 = (float)ps[n];
    const float u32 = (float)q0, w1 = (float)q1, w2 = (float)q2;
    const Blk* __restrict__ blks = sh.blks;
    const int nblk = sh.nblk;
    float* __restrict__ st32 = sh.st32;
    sh.cq32[n] = make_float4(u32, w1, w2, (float)sh.cson[n]);
    sh.cv32[n] = make_float2(
        (float)sh.vol[n],
        sh.eu ? 0.f : (sh.gp * (float)sh.mu[n] + sh.gpt * (float)sh.mut[n]) / r32);
    if (sh.v32) {
      sh.prim32[n] = u32;
      sh.prim32[ld + n] = w1;
      sh.prim32[2 * ld + n] = w2;
      sh.v32[n] = r32;
#pragma unroll
      for (int a = 1; a < 4; ++a) sh.v32[a * ld + n] = (float)v[a * ld + n];
      sh.v32[4 * ld + n] = e32;
      sh.ps32[n] = p32;
    }
    if (st32) {
      // the cell's block (blocks in increasing npc) and (i, j, k) in it
      int lo = 0, hi = nblk - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (blks[mid].npc <= n) lo = mid;
        else hi = mid - 1;
      }
      const Blk& B = blks[lo];
      const long long q = n - B.npc;
      if (q < B.nnn) {
        // (i, j, k) by 32-bit divisions (a block holds fewer than 2^31 cells)
        const unsigned q32 = (unsigned)q, nijd = (unsigned)B.nijd, nid = (unsigned)B.nid;
        const unsigned k = q32 / nijd, rem = q32 - k * nijd;
        const unsigned j = rem / nid, i = rem - j * nid;
        const long long pn = pad_index(B, i, j, k);
        st32[pn] = r32;
        st32[B.pld + pn] = e32;
        st32[2 * B.pld + pn] = p32;
        st32[3 * B.pld + pn] = u32;
        st32[4 * B.pld + pn] = w1;
        st32[5 * B.pld + pn] = w2;
      }
    }
  }
}

// chronos.f90:110-194 (kprec = 0)
// the local time step of cell nc (chronos.f90:110-194, kprec = 0) from its
// state t (rho, rho u, rho v, rho w), sound speed c and viscosities mu, mut
__device__ __forceinline__ double chronos_cell(const Blk& B, Phys ph, Scheme sc,
                                               const double* __restrict__ t, long long ld,
                                               long long nc, const double* __restrict__ sn,
                                               const double* __restrict__ vol, double c,
                                               double mu_c, double mut_c) {
  double sf[3][2];
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const double *s0 = sn_ptr(sn, B, dir, 0), *s1 = sn_ptr(sn, B, dir, 1),
                 *s2 = sn_ptr(sn, B, dir, 2);
    sf[dir][0] = s0[nc] * s0[nc] + s1[nc] * s1[nc] + s2[nc] * s2[nc];
    sf[dir][1] = s0[nc + inc] * s0[nc + inc] + s1[nc + inc] * s1[nc + inc] +
                 s2[nc + inc] * s2[nc + inc];
  }
  const double simax = fmax(sf[0][1], sf[0][0]);
  const double sjmax = fmax(sf[1][1], sf[1][0]);
  const double skmax = fmax(sf[2][1], sf[2][0]);
  const double smoy = sqrt(simax + sjmax + skmax);
  const double dism = vol[nc] / smoy;
  const double ro = t[nc];
  const double qq = (sq(t[ld + nc]) + sq(t[2 * ld + nc]) + sq(t[3 * ld + nc])) / sq(ro);
  const double q = sqrt(qq);
  const double dte = dism / (q + c);
  double d = B.eta * dte;
  if (sc.ns) {
    const double rv1 = ph.gam * (mu_c / ph.pr + mut_c / ph.prt) / t[nc];
    const double rv = fmax(rv1, 4. / 3. * (mu_c + mut_c) / t[nc]);
    const double dtv = B.eta * 0.25 * sq(dism) / rv;
    d = fmin(d, dtv);
  }
  return d;
}

__global__ void __launch_bounds__(kTile) k_chronos(
    const Blk* __restrict__ blks, Space sp, Phys ph, Scheme sc,
    const double* __restrict__ mu, const double* __restrict__ mut,
    const double* __restrict__ t, long long ld, double* dt,
    const double* __restrict__ sn, const double* __restrict__ vol,
    const double* __restrict__ cson) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long nc = cell_index(B, i, j, k);
  dt[nc] = chronos_cell(B, ph, sc, t, ld, nc, sn, vol, cson[nc], sc.ns ? mu[nc] : 0.,
                        sc.ns ? mut[nc] : 0.);
}

// zpres (+ zvismo) and chronos of each real cell in one pass: the time step
// takes the sound speed and viscosity just computed (the values the separate
// kernels store and re-read)
__global__ void __launch_bounds__(kTile) k_zpres_chronos(
    const Blk* __restrict__ blks, Space sp, Phys ph, Scheme sc, const double* __restrict__ v,
    long long ld, double* ps, double* temp, double* cson, double* mu,
    const double* __restrict__ mut, double* dt, const double* __restrict__ sn,
    const double* __restrict__ vol, int* status) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double m = 0.;
  const double c = zpres_cell(ph, sc.ns, v, ld, n, ps, temp, cson, mu, status, &m);
  dt[n] = chronos_cell(B, ph, sc, v, ld, n, sn, vol, c, m, sc.ns ? mut[n] : 0.);
}

// ---------------------------------------------------------------------------
// boundary conditions (rbord.f90:137-429)
// ---------------------------------------------------------------------------

// one list entry of a coincident, extrapolation, adiabatic-wall or
// outlet-pressure boundary; injection boundaries are handled by k_clidd.
// rbvc runs before and after the physical conditions in the reference; every
// ghost cell depends on interior cells only, so one pass gives the same values.
__global__ void __launch_bounds__(256) k_rbord(Bnd bd, Phys ph, double* v,
                                              long long ld, double* ps,
                                              double* temp, double* cson) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int bb = bd.ent_bnd[e];
  const int kind = bd.type[bb];
  const long long nd = bd.ncbd[e], ni = bd.ncin[e];
  if (kind == BC_RC) {  // rbvc.f90:40-92
    const int p = bd.partner[bb];
    const long long nc = bd.ncin[bd.mpb[p] + (e - bd.mpb[bb])];
    const double c = bd.cosr[p], s = bd.sinr[p];
    const double b0 = v[nc], b1 = v[ld + nc];
    const double b2 = v[2 * ld + nc] * c + v[3 * ld + nc] * s;
    const double b3 = v[3 * ld + nc] * c - v[2 * ld + nc] * s;
    const double b4 = v[4 * ld + nc];
    const double b5 = ps[nc], b6 = temp[nc], b7 = cson[nc];
    v[nd] = 0.5 * (v[ni] + b0);
    v[ld + nd] = 0.5 * (v[ld + ni] + b1);
    v[2 * ld + nd] = 0.5 * (v[2 * ld + ni] + b2);
    v[3 * ld + nd] = 0.5 * (v[3 * ld + ni] + b3);
    v[4 * ld + nd] = 0.5 * (v[4 * ld + ni] + b4);
    ps[nd] = 0.5 * (ps[ni] + b5);
    temp[nd] = 0.5 * (temp[ni] + b6);
    cson[nd] = 0.5 * (cson[ni] + b7);
  } else if (kind == BC_EXTR) {  // clextr.f90:23-37
    for (int a = 0; a < 5; ++a) v[a * ld + nd] = v[a * ld + ni];
    ps[nd] = ps[ni];
    temp[nd] = temp[ni];
    cson[nd] = cson[ni];
  } else if (kind == BC_PARA || kind == BC_LP2) {  // clpara.f90:24-40 (rbord.f90:374-388)
    const double v1 = v[ni], v2 = v[ld + ni], v3 = v[2 * ld + ni], v4 = v[3 * ld + ni];
    const double rhoe1 = v[4 * ld + ni] - 0.5 * (sq(v2) + sq(v3) + sq(v4)) / v1;
    v[nd] = v1;
    v[ld + nd] = 0.;
    v[2 * ld + nd] = 0.;
    v[3 * ld + nd] = 0.;
    v[4 * ld + nd] = rhoe1;
    ps[nd] = ps[ni];
    temp[nd] = temp[ni];
    cson[nd] = cson[ni];
  } else if (kind == BC_PRD) {  // rbve.f90 then clprd.f90:31-59
    const double gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl;
    const double pres = bd.bceqt[e];
    const double r1 = v[ni];
    const double qxs = v[ld + ni] / r1, qys = v[2 * ld + ni] / r1, qzs = v[3 * ld + ni] / r1;
    const double p = gam1 * (v[4 * ld + ni] - 0.5 * r1 * (sq(qxs) + sq(qys) + sq(qzs)) - pinfl);
    const double cs2 = gam * p / r1;
    const double roc0 = sqrt(gam * p * r1);
    const double dqn = (pres - p) / roc0;
    const double qx = qxs + dqn * bd.nxn[e];
    const double qy = qys + dqn * bd.nyn[e];
    const double qz = qzs + dqn * bd.nzn[e];
    const double drho = (pres - p) / cs2;
    const double rho = r1 + drho;
    v[nd] = rho;
    v[ld + nd] = rho * qx;
    v[2 * ld + nd] = rho * qy;
    v[3 * ld + nd] = rho * qz;
    v[4 * ld + nd] = pres / gam1 + pinfl + 0.5 * rho * (sq(qx) + sq(qy) + sq(qz));
    ps[nd] = pres;
    const double tt = gam * pres / rho;
    temp[nd] = tt;
    cson[nd] = sqrt(tt);
  }
}

// utidd.f90 + rbve.f90 + clidd.f90:50-170: injection at imposed total
// pressure, total temperature and flow direction.  The reference iterates a
// Newton method on the normal velocity of every boundary cell, sweep after
// sweep, until the largest relative update over the whole boundary is below
// 1e-7 (at most 20 sweeps).  Each cell's iterate depends on that cell only;
// only the number of sweeps is global.  So pass 1 runs every cell's 20 sweeps
// and ORs into a per-boundary word which sweeps still had an update above
// 1e-7; pass 2 reads the sweep count (the first sweep whose bit is clear) and
// replays exactly that many sweeps: the same values as the sequential loop.
struct IddCell {
  double usdn, usdn2, un, qn, roc0, am0, rpi, rti;
};

__device__ __forceinline__ void idd_setup(const Bnd& bd, const Phys& ph,
                                          const double* __restrict__ v,
                                          long long ld, long long e, IddCell& c) {
  const long long nl = bd.nlist, ni = bd.ncin[e];
  const double d0x = bd.bceqt[2 * nl + e], d0y = bd.bceqt[3 * nl + e],
               d0z = bd.bceqt[4 * nl + e];
  const double nx = bd.nxn[e], ny = bd.nyn[e], nz = bd.nzn[e];
  c.rpi = bd.bceqt[e];
  c.rti = bd.bceqt[nl + e];
  c.usdn = 1. / (d0x * nx + d0y * ny + d0z * nz);
  c.usdn2 = sq(c.usdn);
  c.un = ph.omg * (bd.ym[e] * nz - bd.zm[e] * ny);
  // the ghost cell holds the interior state (rbve) when clidd reads it
  const double r1 = v[ni], r2 = v[ld + ni], r3 = v[2 * ld + ni], r4 = v[3 * ld + ni];
  const double qxs = r2 / r1, qys = r3 / r1, qzs = r4 / r1;
  c.qn = qxs * nx + qys * ny + qzs * nz;
  const double p = ph.gam1 * (v[4 * ld + ni] - 0.5 * (qxs * r2 + qys * r3 + qzs * r4) - ph.pinfl);
  c.roc0 = -sqrt(ph.gam * p * r1);
  c.am0 = p + c.roc0 * c.qn;
}

// one Newton sweep of clidd.f90:96-113 on one cell; returns resi
__device__ __forceinline__ double idd_sweep(const Phys& ph, IddCell& c) {
  const double gam6 = ph.gam / ph.gam1;
  const double gamt = ph.gam / sq(ph.aa1);
  const double gam2t = 0.5 * ph.gam1 / sq(ph.aa1);
  const double b = 1. / (1. + gam2t / c.rti * c.usdn2 * sq(c.qn + c.un));
  const double p = ph.pa1 * c.rpi * cns_pow(b, gam6);
  const double ro = gamt * p / (b * c.rti);
  const double f = p + c.roc0 * c.qn - c.am0;
  const double df = c.roc0 - ro * (c.qn + c.un) * c.usdn2;
  const double dqn = -f / df;
  const double resi = fabs(dqn) / c.qn;
  c.qn = c.qn + dqn;
  return resi;
}

__global__ void __launch_bounds__(256) k_clidd_mask(Bnd bd, Phys ph, const long long* ents,
                                                   long long nent, const double* v,
                                                   long long ld, unsigned* masks) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nent) return;
  const long long e = ents[q];
  IddCell c;
  idd_setup(bd, ph, v, ld, e, c);
  unsigned bits = 0u;
  for (int t = 0; t < 20; ++t) {
    const double resi = idd_sweep(ph, c);
    if (resi > 0.0000001) bits |= 1u << t;
  }
  atomicOr(&masks[bd.ent_bnd[e]], bits);
}

__global__ void __launch_bounds__(256) k_clidd_apply(Bnd bd, Phys ph, const long long* ents,
                                                    long long nent, double* v, long long ld,
                                                    double* ps_, double* temp, double* cson,
                                                    const unsigned* masks) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nent) return;
  const long long e = ents[q], nl = bd.nlist, nc = bd.ncbd[e];
  const unsigned bits = masks[bd.ent_bnd[e]];
  int nsweep = 20;
  for (int t = 0; t < 20; ++t)
    if (!(bits & (1u << t))) {
      nsweep = t + 1;
      break;
    }
  IddCell c;
  idd_setup(bd, ph, v, ld, e, c);
  for (int t = 0; t < nsweep; ++t) idd_sweep(ph, c);
  const double gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl, omg = ph.omg;
  const double gam6 = gam / gam1;
  const double gamt = gam / sq(ph.aa1);
  const double gam2t = 0.5 * gam1 / sq(ph.aa1);
  const double d0x = bd.bceqt[2 * nl + e], d0y = bd.bceqt[3 * nl + e],
               d0z = bd.bceqt[4 * nl + e];
  const double ym = bd.ym[e], zm = bd.zm[e];
  const double b = 1. / (1. + gam2t / c.rti * c.usdn2 * sq(c.qn + c.un));
  const double p = ph.pa1 * c.rpi * cns_pow(b, gam6);
  const double ro = gamt * p / (b * c.rti);
  const double wn = c.qn + c.un;
  const double w = wn * c.usdn;
  const double m2 = ro * (w * d0x);
  const double m3 = ro * (w * d0y + zm * omg);
  const double m4 = ro * (w * d0z - ym * omg);
  v[nc] = ro;
  v[ld + nc] = m2;
  v[2 * ld + nc] = m3;
  v[3 * ld + nc] = m4;
  v[4 * ld + nc] = p / gam1 + pinfl + 0.5 * (sq(m2) + sq(m3) + sq(m4)) / ro;
  ps_[nc] = p;
  const double tt = gam * p / ro;
  temp[nc] = tt;
  cson[nc] = sqrt(tt);
}

// rbte.f90:15-31 (non-coincident boundaries: copy of the interior cell) and
// rbtc.f90:30-100 (coincident: average with the rotated partner)
__global__ void __launch_bounds__(256) k_tau_ghosts(Bnd bd, double* tau, long long ld) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= bd.nlist) return;
  const int bb = bd.ent_bnd[e];
  const long long nd = bd.ncbd[e], ndm = bd.ncin[e];
  if (bd.type[bb] != BC_RC) {
    for (int a = 0; a < 9; ++a) tau[a * ld + nd] = tau[a * ld + ndm];
    return;
  }
  const int p = bd.partner[bb];
  const long long nc = bd.ncin[bd.mpb[p] + (e - bd.mpb[bb])];
  const double sr = -bd.sinr[p], cr = bd.cosr[p];
  const double txx = tau[nc], txy = tau[ld + nc], txz = tau[2 * ld + nc],
               tyy = tau[3 * ld + nc], tyz = tau[4 * ld + nc], tzz = tau[5 * ld + nc];
  double bf[9];
  bf[0] = txx;
  bf[1] = cr * txy - sr * txz;
  bf[2] = cr * txz + sr * txy;
  bf[3] = cr * cr * tyy - 2. * cr * sr * tyz + sr * sr * tzz;
  bf[4] = -cr * sr * (tzz - tyy) + (2. * cr * cr - 1.) * tyz;
  bf[5] = sr * sr * tyy + 2. * cr * sr * tyz + cr * cr * tzz;
  bf[6] = tau[6 * ld + nc];
  bf[7] = cr * tau[7 * ld + nc] - sr * tau[8 * ld + nc];
  bf[8] = cr * tau[8 * ld + nc] + sr * tau[7 * ld + nc];
#pragma unroll
  for (int a = 0; a < 9; ++a) tau[a * ld + nd] = 0.5 * (tau[a * ld + ndm] + bf[a]);
}

// ---------------------------------------------------------------------------
// viscous gradients and stresses: zgrad2.f90 (unit weights, inivec.f90:110)
// then zfluto.f90:38-57, per real cell
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kTile) k_grad(const Blk* __restrict__ blks,
                                                Space sp, Phys ph,
                                                const double* __restrict__ s,
                                                const double* __restrict__ prim,
                                                long long ld,
                                                const double* __restrict__ mu,
                                                const double* __restrict__ mut,
                                                double* __restrict__ tau,
                                                const double* __restrict__ sn,
                                                const double* __restrict__ vol,
                                                const double* __restrict__ temp) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double g[12];
#pragma unroll
  for (int a = 0; a < 12; ++a) g[a] = 0.;
  (void)s;
  const double fc[4] = {prim[n], prim[ld + n], prim[2 * ld + n], temp[n]};
  // directions in the reference's order: k faces, then j, then i
#pragma unroll
  for (int oi = 0; oi < 3; ++oi) {
    const int dir = 2 - oi;
    const long long inc = ninc_of(B, dir);
    const int nd = nd_of(B, dir);
    const int p = dir == 0 ? i : (dir == 1 ? j : k);
    const double *s0 = sn_ptr(sn, B, dir, 0), *s1 = sn_ptr(sn, B, dir, 1),
                 *s2 = sn_ptr(sn, B, dir, 2);
    const long long nl = n - inc, nu = n + inc;
    const double fl[4] = {prim[nl], prim[ld + nl], prim[2 * ld + nl], temp[nl]};
    const double fu[4] = {prim[nu], prim[ld + nu], prim[2 * ld + nu], temp[nu]};
    const double sl[3] = {s0[n], s1[n], s2[n]};
    const double su[3] = {s0[nu], s1[nu], s2[nu]};
    const bool lower_bnd = (p == 1), upper_bnd = (p + 1 == nd);
    const bool upper_first = lower_bnd && nd >= 3;
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
      const bool do_upper = (pass == 0) == upper_first;
      if (!do_upper) {  // lower face of the cell
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (lower_bnd)
              g[3 * a + c] = g[3 * a + c] - sl[c] * 2 * fl[a];
            else
              g[3 * a + c] = g[3 * a + c] - (fc[a] + fl[a]) * sl[c];
          }
      } else {  // upper face
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            if (upper_bnd)
              g[3 * a + c] = g[3 * a + c] + su[c] * 2 * fu[a];
            else
              g[3 * a + c] = g[3 * a + c] + (fu[a] + fc[a]) * su[c];
          }
      }
    }
  }
  const double eps = 0.00001, ds3 = 2. / 3.;
  const double vn = vol[n];
  const double ts = copysign(0.5, -vn);
  const double vols = (0.5 + ts) * eps + (0.5 - ts) * vn;
  const double c0 = .5 / (vols + 2.2250738585072014e-308);
#pragma unroll
  for (int a = 0; a < 12; ++a) g[a] = g[a] * c0;
  const double dvxx = g[0], dvxy = g[1], dvxz = g[2], dvyx = g[3], dvyy = g[4],
               dvyz = g[5], dvzx = g[6], dvzy = g[7], dvzz = g[8];
  const double m = mu[n] + mut[n];
  tau[n] = ds3 * m * (2 * dvxx - dvyy - dvzz);
  tau[3 * ld + n] = ds3 * m * (2 * dvyy - dvxx - dvzz);
  tau[5 * ld + n] = ds3 * m * (2 * dvzz - dvxx - dvyy);
  tau[ld + n] = m * (dvxy + dvyx);
  tau[2 * ld + n] = m * (dvxz + dvzx);
  tau[4 * ld + n] = m * (dvyz + dvzy);
  const double kq = ph.cp * (mu[n] / ph.pr + mut[n] / ph.prt);
  tau[6 * ld + n] = kq * g[9];
  tau[7 * ld + n] = kq * g[10];
  tau[8 * ld + n] = kq * g[11];
}

// per real cell: coefdiag seed (vol/dt, or vol*(fact+1/dt) with fact = 0 or,
// with dual time stepping, 1.5/dt1min) and the viscous spectral factor rv
// (implimf_3d.f90:95-105, implimf_eu.f90:82-85, 124-134)
__global__ void __launch_bounds__(kTile) k_impl_cell0(
    const Blk* __restrict__ blks, Space sp, Phys ph, int eu, double fact,
    const double* __restrict__ v, const double* __restrict__ dt,
    const double* __restrict__ mu, const double* __restrict__ mut,
    const double* __restrict__ vol, double* coefdiag, double* rv) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  if (eu) {
    coefdiag[n] = vol[n] * (fact + 1. / dt[n]);
  } else {
    rv[n] = ph.gam * (mu[n] / ph.pr + mut[n] / ph.prt) / v[n];
    coefdiag[n] = vol[n] / dt[n];
  }
}

// per face: spectral radius coefe (implimf_eu.f90:141-159,
// implimf_3d.f90:110-190)
template <class TO>
__global__ void __launch_bounds__(kTile) k_impl_coefe(
    const Blk* __restrict__ blks, Space sp, int dir, int eu,
    const double* __restrict__ v, const double* __restrict__ prim, long long ld,
    const double* __restrict__ sn,
    const double* __restrict__ vol, const double* __restrict__ cson,
    const double* __restrict__ rv, double* coefe, TO* coefe_out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long inc = ninc_of(B, dir);
  const long long n = cell_index(B, i, j, k), nl = n - inc;
  const double sx = sn_ptr(sn, B, dir, 0)[n], sy = sn_ptr(sn, B, dir, 1)[n],
               sz = sn_ptr(sn, B, dir, 2)[n];
  const double cnds = sx * sx + sy * sy + sz * sz;
  const double cc = 0.5 * (cson[n] + cson[nl]);
  double ce;
  if (eu) {
    const double norm = 1. / v[n], norm1 = 1. / v[nl];
    const double uu = 0.5 * (v[ld + n] * norm + v[ld + nl] * norm1);
    const double vv = 0.5 * (v[2 * ld + n] * norm + v[2 * ld + nl] * norm1);
    const double ww = 0.5 * (v[3 * ld + n] * norm + v[3 * ld + nl] * norm1);
    ce = 0.5 * (fabs(uu * sx + vv * sy + ww * sz)) + sqrt(cnds) * cc;
  } else {
    const double uu = 0.5 * (prim[n] + prim[nl]);
    const double vv = 0.5 * (prim[ld + n] + prim[ld + nl]);
    const double ww = 0.5 * (prim[2 * ld + n] + prim[2 * ld + nl]);
    const double vn = uu * sx + vv * sy + ww * sz;
    ce = 0.5 * (fabs(vn) + sqrt(cnds) * cc) + (rv[n] + rv[nl]) * cnds / (vol[n] + vol[nl]);
  }
  coefe[(long long)dir * ld + n] = ce;
  if (coefe_out) coefe_out[(long long)dir * ld + n] = (TO)ce;
}

// per real cell: coefdiag += coefe of the six faces (implimf_eu.f90:161-170,
// implimf_3d.f90:192-203: the same left-to-right chain); dtpas > 0: then
// + 1.5*vol/dtpas, the physical time term of dual time stepping
// (implimf_3d.f90:213-224)
template <class TO>
__global__ void __launch_bounds__(kTile) k_impl_diag(const Blk* __restrict__ blks,
                                                     Space sp, long long ld,
                                                     const double* __restrict__ coefe,
                                                     const double* __restrict__ vol,
                                                     double dtpas,
                                                     double* coefdiag, TO* coefdiag_out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double c = coefdiag[n];
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    c = c + coefe[(long long)dir * ld + n];
    c = c + coefe[(long long)dir * ld + n + inc];
  }
  if (dtpas > 0.) c = c + 1.5 * vol[n] / dtpas;
  coefdiag[n] = c;
  if (coefdiag_out) coefdiag_out[n] = (TO)c;
}


// standalone residual partials from stored arrays (rscpsv.f90 called with u0)
__global__ void __launch_bounds__(kTile) k_norm_partials(
    const Blk* __restrict__ blks, Space sp, long long ld,
    const double* __restrict__ u0, const double* __restrict__ v,
    const double* __restrict__ dt, double* normpart) {
  int b, i, j, k;
  const bool valid = space_elem(sp, threadIdx.x, b, i, j, k);
  double res[5] = {0., 0., 0., 0., 0.};
  if (valid) {
    const long long n = cell_index(blks[b], i, j, k);
#pragma unroll
    for (int a = 0; a < 5; ++a) res[a] = (v[a * ld + n] - u0[a * ld + n]) / dt[n];
  }
  norm_tile_reduce(res, valid, normpart + (long long)(sp.tile0 + blockIdx.x) * 15);
}

// per-block sums of the tile partials in a fixed tree order (one CTA per
// block), then the rscpsv.f90:79-150 combination over blocks (one thread)
__global__ void __launch_bounds__(256) k_norm_blocks(const int* __restrict__ blk_tile0,
                                                    int b0, const double* __restrict__ normpart,
                                                    double* __restrict__ blocksum) {
  __shared__ double red[256][15];
  const int b = b0 + blockIdx.x;
  const int t0 = blk_tile0[b], t1 = blk_tile0[b + 1];
  double loc[15];
#pragma unroll
  for (int q = 0; q < 15; ++q) loc[q] = 0.;
  for (int t = t0 + (int)threadIdx.x; t < t1; t += blockDim.x)
#pragma unroll
    for (int q = 0; q < 15; ++q)
      loc[q] = (q >= 10) ? fmax(loc[q], normpart[(long long)t * 15 + q])
                         : loc[q] + normpart[(long long)t * 15 + q];
#pragma unroll
  for (int q = 0; q < 15; ++q) red[threadIdx.x][q] = loc[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int q = 0; q < 15; ++q)
        red[threadIdx.x][q] = (q >= 10) ? fmax(red[threadIdx.x][q], red[threadIdx.x + s][q])
                                        : red[threadIdx.x][q] + red[threadIdx.x + s][q];
    __syncthreads();
  }
  if (threadIdx.x < 15) blocksum[(long long)blockIdx.x * 15 + threadIdx.x] = red[0][threadIdx.x];
}

__global__ void k_norm_combine(const Blk* __restrict__ blks, int b0, int b1,
                               const double* __restrict__ blocksum, double* norms) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double g[15];
  for (int q = 0; q < 15; ++q) g[q] = 0.;
  long long npts = 0;
  for (int b = b0; b < b1; ++b) {
    const Blk& B = blks[b];
    const double* bs = blocksum + (long long)(b - b0) * 15;
    const long long nmax = (long long)(B.ni - 1) * (B.nj - 1) * (B.nk - 1);
    const double coef = 1. / (double)nmax;
    for (int a = 0; a < 5; ++a) {
      const double d1 = coef * bs[a];
      const double d2 = sqrt(coef * bs[5 + a]);
      g[a] = g[a] + (double)nmax * d1;
      g[5 + a] = g[5 + a] + (double)nmax * sq(d2);
      g[10 + a] = fmax(g[10 + a], fabs(bs[10 + a]));
    }
    npts += nmax;
  }
  for (int a = 0; a < 5; ++a) {
    norms[a] = g[a] / (double)npts;
    norms[5 + a] = sqrt(g[5 + a] / (double)npts);
    norms[10 + a] = g[10 + a];
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

cudaError_t launch_zpres(const Blk* blks, Space sp, Phys ph, int with_mu,
                         const double* v, long long ld, double* ps, double* temp,
                         double* cson, double* mu, int* status, cudaStream_t st) {
  if (sp.ntiles > 0)
    k_zpres<<<grid_of(sp), kTile, 0, st>>>(blks, sp, ph, with_mu, v, ld, ps, temp,
                                           cson, mu, status);
  return cudaGetLastError();
}

cudaError_t launch_zvismo(const Blk* blks, Space sp, Phys ph, double* mu,
                          const double* temp, int* status, cudaStream_t st) {
  if (sp.ntiles > 0)
    k_zvismo<<<grid_of(sp), kTile, 0, st>>>(blks, sp, ph, mu, temp, status);
  return cudaGetLastError();
}

cudaError_t launch_prim(long long n0, long long n1, const double* v, long long ld,
                        double* prim, cudaStream_t st) {
  if (n1 > n0)
    k_prim<false><<<(int)((n1 - n0 + 255) / 256), 256, 0, st>>>(n0, n1, v, ld, prim, nullptr,
                                                                PrimShadow{});
  return cudaGetLastError();
}

cudaError_t launch_prim_shadow(long long ncells, const double* v, long long ld, double* prim,
                               const double* ps, const PrimShadow& sh, cudaStream_t st) {
  if (ncells > 0)
    k_prim<true><<<(int)((ncells + 255) / 256), 256, 0, st>>>(0, ncells, v, ld, prim, ps, sh);
  return cudaGetLastError();
}

// chrono.f90:113-151 (kdtl = 0): the smallest local time step over the real
// cells of every block, min(dt1min, it) everywhere, and the reference's stop
// when it is below dt1min as status bit 2.  Min is exact in any order.
__global__ void __launch_bounds__(kTile) k_dt_partials(const Blk* __restrict__ blks, Space sp,
                                                       const double* __restrict__ dt,
                                                       double* __restrict__ part) {
  int b, i, j, k;
  double x = CUDART_INF;
  if (space_elem(sp, threadIdx.x, b, i, j, k)) x = dt[cell_index(blks[b], i, j, k)];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  __shared__ double wm[kTile / 32];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = wm[0];
    for (int q = 1; q < kTile / 32; ++q) m = fmin(m, wm[q]);
    part[blockIdx.x] = m;
  }
}

__global__ void __launch_bounds__(256) k_dt_reduce(const double* __restrict__ part, int n,
                                                  double dt1min, double* __restrict__ out,
                                                  int* status) {
  double x = CUDART_INF;
  for (int q = threadIdx.x; q < n; q += blockDim.x) x = fmin(x, part[q]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = wm[0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) m = fmin(m, wm[q]);
    const double dtmin = fmin(dt1min, m);
    if (dtmin < dt1min) atomicOr(status, 2);
    *out = dtmin;
  }
}

__global__ void __launch_bounds__(256) k_dt_set(long long ncells, const double* __restrict__ v,
                                               double* __restrict__ dt) {
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n < ncells) dt[n] = *v;
}

cudaError_t launch_chronos(const Blk* blks, Space sp, Phys ph, Scheme sc,
                           const double* mu, const double* mut, const double* v,
                           long long ld, double* dt, const double* sn,
                           const double* vol, const double* cson, cudaStream_t st) {
  if (sp.ntiles > 0)
    k_chronos<<<grid_of(sp), kTile, 0, st>>>(blks, sp, ph, sc, mu, mut, v, ld, dt,
                                             sn, vol, cson);
  return cudaGetLastError();
}

cudaError_t launch_zpres_chronos(const Blk* blks, Space sp, Phys ph, Scheme sc,
                                 const double* v, long long ld, double* ps, double* temp,
                                 double* cson, double* mu, const double* mut, double* dt,
                                 const double* sn, const double* vol, int* status,
                                 cudaStream_t st) {
  if (sp.ntiles > 0)
    k_zpres_chronos<<<grid_of(sp), kTile, 0, st>>>(blks, sp, ph, sc, v, ld, ps, temp, cson, mu,
                                                   mut, dt, sn, vol, status);
  return cudaGetLastError();
}

cudaError_t launch_dt_global(const Blk* blks, Space cells, long long ncells, double dt1min,
                             double* dt, double* part, double* scalar, int* status,
                             cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  k_dt_partials<<<grid_of(cells), kTile, 0, st>>>(blks, cells, dt, part);
  k_dt_reduce<<<1, 256, 0, st>>>(part, cells.ntiles, dt1min, scalar, status);
  k_dt_set<<<(int)((ncells + 255) / 256), 256, 0, st>>>(ncells, scalar, dt);
  return cudaGetLastError();
}

cudaError_t launch_rbord(const Bnd& bd, Phys ph, double* v, long long ld,
                         double* ps, double* temp, double* cson, long long n_idd_ent,
                         const long long* idd_ents, unsigned* masks, cudaStream_t st) {
  if (bd.nlist > 0)
    k_rbord<<<(int)((bd.nlist + 255) / 256), 256, 0, st>>>(bd, ph, v, ld, ps, temp, cson);
  if (n_idd_ent > 0) {
    cudaError_t e = cudaMemsetAsync(masks, 0, sizeof(unsigned) * bd.nbnd, st);
    if (e != cudaSuccess) return e;
    const int g = (int)((n_idd_ent + 255) / 256);
    k_clidd_mask<<<g, 256, 0, st>>>(bd, ph, idd_ents, n_idd_ent, v, ld, masks);
    k_clidd_apply<<<g, 256, 0, st>>>(bd, ph, idd_ents, n_idd_ent, v, ld, ps, temp, cson,
                                     masks);
  }
  return cudaGetLastError();
}

cudaError_t launch_tau_ghosts(const Bnd& bd, double* tau, long long ld,
                              cudaStream_t st) {
  if (bd.nlist > 0)
    k_tau_ghosts<<<(int)((bd.nlist + 255) / 256), 256, 0, st>>>(bd, tau, ld);
  return cudaGetLastError();
}

cudaError_t launch_grad(const Blk* blks, Space sp, Phys ph, const double* v,
                        const double* prim, long long ld, const double* mu,
                        const double* mut, double* tau, const double* sn,
                        const double* vol, const double* temp, cudaStream_t st) {
  if (sp.ntiles > 0)
    k_grad<<<grid_of(sp), kTile, 0, st>>>(blks, sp, ph, v, prim, ld, mu, mut, tau, sn,
                                          vol, temp);
  return cudaGetLastError();
}

template <>
cudaError_t launch_ratio_t<double>(const Blk* blks, const SpaceBuf* lines, int l0,
                                   const double* v, const double* prim, long long ld,
                                   const double* ps, double* R, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = lines[dir].view(l0);
    if (sp.ntiles > 0)
      k_ratio<double><<<dim3(grid_of(sp), 5), kTile, 0, st>>>(blks, sp, dir, v, prim, ld, ps, R);
  }
  return cudaGetLastError();
}

cudaError_t launch_residual_fused(const Blk* blks, Tiles tl, Phys ph, Scheme sc, const double* v,
                                  const double* prim, long long ld, const double* ps,
                                  const double* tau, const double* sn, const double* R,
                                  double* u, float* u32, cudaStream_t st) {
  return residual_fused_dispatch<double>(blks, tl, ph, sc, v, prim, ld, ps, tau, sn, R, u, u32,
                                         st);
}

template <>
cudaError_t launch_face_flux_t<double>(const Blk* blks, const SpaceBuf* faces, int l0,
                                       Phys ph, Scheme sc, const double* v,
                                       const double* prim, long long ld,
                                       const double* ps, const double* tau,
                                       const double* sn, const double* R, double* G,
                                       cudaStream_t st, double* V) {
  return face_flux_dispatch(blks, faces, l0, ph, sc, v, prim, ld, ps, tau, sn, R, G, V, st);
}

template <>
cudaError_t launch_accumulate_t<double>(const Blk* blks, Space sp, const double* G,
                                        long long ld, const double* corr, double* u,
                                        float* u32, cudaStream_t st, const double* V) {
  if (sp.ntiles > 0)
    k_accumulate<double><<<grid_of(sp), kTile, 0, st>>>(blks, sp, G, ld, corr, u, u32, V);
  return cudaGetLastError();
}

template <>
cudaError_t launch_jacobi_25d_t<double>(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                                        long long ld, const double* u, const double* v,
                                        const double* prim, const double* ps, const double* sn,
                                        const double* coefe, const double* coefdiag,
                                        const double* d_in, double* d_out, cudaStream_t st) {
  return jacobi_25d_dispatch<double, 0>(blks, tl, ph, qfix, eu, ld, u, v, prim, ps, sn, coefe,
                                        coefdiag, d_in, d_out, st);
}

cudaError_t init_jacobi_25d() {
  cudaError_t e = jacobi_25d_attr<double, 0>();
  if (e == cudaSuccess) e = init_jacobi_25d_float();
  return e;
}

// the FP64 sweeps: the first (zero previous iterate) per cell, the others
// 2.5D-blocked with the increments evaluated by the reference expressions
// (bit-identical to storing them, implimf_3d.f90:222-466)
template <>
cudaError_t launch_sweeps_t<double>(const Blk* blks, Space cells, Tiles tl, Phys ph,
                                    Scheme sc, int eu, int lmx, long long ld, const double* u,
                                    const double* v, const double* prim, const double* ps,
                                    const double* sn, const double* coefe,
                                    const double* coefdiag, double* const dpp[2],
                                    int* cur_out, cudaStream_t st) {
  const int g = grid_of(cells);
  int cur = 0;
  if (lmx == 0) {
    cudaError_t e0 = cudaMemsetAsync(dpp[0], 0, sizeof(double) * 5 * ld, st);
    if (e0 != cudaSuccess) return e0;
  }
  const int q = eu ? sc.qfix_dfez : 0;
  for (int ls = 1; ls <= lmx; ++ls) {
    const int nxt = (ls == 1) ? 0 : 1 - cur;
    const double* din = dpp[cur];
    double* dout = dpp[nxt];
    if (ls == 1) {
      if (g > 0) {
        if (eu)
          k_jacobi_rc<double, true, true><<<g, kTile, 0, st>>>(blks, cells, ph, q, ld, u, v,
                                                               prim, ps, sn, coefe, coefdiag,
                                                               din, dout);
        else
          k_jacobi_rc<double, false, true><<<g, kTile, 0, st>>>(blks, cells, ph, q, ld, u, v,
                                                                prim, ps, sn, coefe, coefdiag,
                                                                din, dout);
      }
    } else {
      cudaError_t e1 = launch_jacobi_25d_t<double>(blks, tl, ph, q, eu, ld, u, v, prim, ps, sn,
                                                   coefe, coefdiag, din, dout, st);
      if (e1 != cudaSuccess) return e1;
    }
    cur = nxt;
  }
  *cur_out = cur;
  return cudaGetLastError();
}

template <>
cudaError_t launch_update_t<double>(const Blk* blks, Space cells, long long ld,
                                    const double* d, double* v, const double* dt,
                                    double* d_out, double* normpart, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_update<double><<<grid_of(cells), kTile, 0, st>>>(blks, cells, ld, d, v, dt, d_out,
                                                       normpart);
  return cudaGetLastError();
}

// implicit coefficients computed in FP64 (coefdiag seed, face spectral radii,
// diagonal); TO copies for the reduced-precision sweeps when given
template <class TO>
static cudaError_t implicit_coefficients(const Blk* blks, Space cells,
                                         const SpaceBuf* faces, int l0, Phys ph, int eu,
                                         double dtpas, const double* dt, const double* v,
                                         const double* prim, const double* mu,
                                         const double* mut, const double* sn,
                                         const double* vol, const double* cson, Work& w,
                                         TO* coefe_out, TO* coefdiag_out, cudaStream_t st) {
  const long long ld = w.ld;
  const int g = grid_of(cells);
  // dtpas > 0: dual time stepping with physical step dtpas
  const double fact = dtpas > 0. ? 1.5 / dtpas : 0.;
  k_impl_cell0<<<g, kTile, 0, st>>>(blks, cells, ph, eu, fact, v, dt, mu, mut, vol,
                                    w.coefdiag, w.rv);
  for (int dir = 0; dir < 3; ++dir) {
    const Space fs = faces[dir].view(l0);
    if (fs.ntiles > 0)
      k_impl_coefe<TO><<<fs.ntiles, kTile, 0, st>>>(blks, fs, dir, eu, v, prim, ld, sn, vol,
                                                    cson, w.rv, w.coefe, coefe_out);
  }
  k_impl_diag<TO><<<g, kTile, 0, st>>>(blks, cells, ld, w.coefe, vol, eu ? 0. : dtpas,
                                       w.coefdiag, coefdiag_out);
  return cudaGetLastError();
}

cudaError_t launch_implicit_coefficients(const Blk* blks, Space cells,
                                         const SpaceBuf* faces, int l0, Phys ph, int eu,
                                         const double* dt, const double* v,
                                         const double* prim, const double* mu,
                                         const double* mut, const double* sn,
                                         const double* vol, const double* cson, Work& w,
                                         float* coefe32, float* coefdiag32,
                                         cudaStream_t st) {
  if (cells.ntiles == 0) return cudaSuccess;
  return implicit_coefficients<float>(blks, cells, faces, l0, ph, eu, 0., dt, v, prim, mu, mut,
                                      sn, vol, cson, w, coefe32, coefdiag32, st);
}

cudaError_t launch_implicit(const Blk* blks, Space cells, Tiles tl, const SpaceBuf* faces,
                            int l0, Phys ph, Scheme sc, int eu, int lmx,
                            const double* u, const double* dt, double* v,
                            double* d_out, const double* mu, const double* mut,
                            const double* sn, const double* vol,
                            const double* ps, const double* cson, Work& w,
                            int want_norms, cudaStream_t st) {
  const long long ld = w.ld;
  if (cells.ntiles == 0) return cudaSuccess;
  cudaError_t e = implicit_coefficients<double>(blks, cells, faces, l0, ph, eu,
                                                sc.kfmg == 3 ? sc.dt1min : 0., dt, v, w.prim,
                                                mu, mut, sn, vol, cson, w, nullptr, nullptr,
                                                st);
  int cur = 0;
  if (e == cudaSuccess)
    e = launch_sweeps_t<double>(blks, cells, tl, ph, sc, eu, lmx, ld, u, v, w.prim, ps, sn,
                                w.coefe, w.coefdiag, w.dpp, &cur, st);
  if (e == cudaSuccess)
    e = launch_update_t<double>(blks, cells, ld, w.dpp[cur], v, dt, d_out,
                                want_norms ? w.normpart : nullptr, st);
  return e;
}

// sch_dual.f90:18-52 / sch_dual2.f90:18-52: u += vol*dti*(fact*v + ptdual)
// on the real cells (the physical time term of dual time stepping); u32:
// the single-precision copy of u the FP32 sweeps read, refreshed
__global__ void __launch_bounds__(kTile) k_dual(const Blk* __restrict__ blks, Space sp,
                                                long long ld, double fact, double dti,
                                                const double* __restrict__ v,
                                                const double* __restrict__ vol,
                                                const double* __restrict__ ptdual,
                                                double* __restrict__ u, float* __restrict__ u32) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double c0 = vol[n] * dti;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const double r = u[a * ld + n] + c0 * (fact * v[a * ld + n] + ptdual[a * ld + n]);
    u[a * ld + n] = r;
    if (u32) u32[a * ld + n] = (float)r;
  }
}

// the physical-step arrays on the real cells: mode 0 = sch_duin.f90 after
// utinia.f90:140-160 (vdual = vdual1 = vdual2 = v, ptdual = -vdual); mode 1
// = sch_duup.f90 (vdual1 = vdual, vdual = v, ptdual = -2 vdual + 0.5 vdual1);
// mode 2 = sch_duup2.f90 (vdual2 = vdual1, vdual1 = vdual, vdual = v,
// ptdual = -3 vdual + 1.5 vdual1 - vdual2/3)
__global__ void __launch_bounds__(kTile) k_dual_update(const Blk* __restrict__ blks, Space sp,
                                                       long long ld, int mode,
                                                       const double* __restrict__ v,
                                                       double* ptdual, double* vdual,
                                                       double* vdual1, double* vdual2) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  const double c13 = 1. / 3.;
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    const long long q = a * ld + n;
    if (mode == 0) {
      vdual[q] = v[q];
      vdual1[q] = v[q];
      vdual2[q] = v[q];
      ptdual[q] = -vdual[q];
    } else if (mode == 1) {
      vdual1[q] = vdual[q];
      vdual[q] = v[q];
      ptdual[q] = -2. * vdual[q] + 0.5 * vdual1[q];
    } else {
      vdual2[q] = vdual1[q];
      vdual1[q] = vdual[q];
      vdual[q] = v[q];
      ptdual[q] = -3. * vdual[q] + 1.5 * vdual1[q] - c13 * vdual2[q];
    }
  }
}

cudaError_t launch_dual(const Blk* blks, Space cells, long long ld, double fact, double dti,
                        const double* v, const double* vol, const double* ptdual, double* u,
                        float* u32, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_dual<<<cells.ntiles, kTile, 0, st>>>(blks, cells, ld, fact, dti, v, vol, ptdual, u, u32);
  return cudaGetLastError();
}

cudaError_t launch_dual_update(const Blk* blks, Space cells, long long ld, int mode,
                               const double* v, double* ptdual, double* vdual, double* vdual1,
                               double* vdual2, cudaStream_t st) {
  if (cells.ntiles > 0)
    k_dual_update<<<cells.ntiles, kTile, 0, st>>>(blks, cells, ld, mode, v, ptdual, vdual,
                                                  vdual1, vdual2);
  return cudaGetLastError();
}

cudaError_t launch_norm_partials(const Blk* blks, Space cells, long long ld,
                                 const double* u0, const double* v,
                                 const double* dt, double* normpart,
                                 cudaStream_t st) {
  if (cells.ntiles > 0)
    k_norm_partials<<<cells.ntiles, kTile, 0, st>>>(blks, cells, ld, u0, v, dt, normpart);
  return cudaGetLastError();
}

cudaError_t launch_norm_finalize(const Blk* blks, const int* blk_tile0_dev,
                                 int b0, int b1, const double* normpart,
                                 double* blocksum, double* norms, cudaStream_t st) {
  if (b1 <= b0) return cudaSuccess;
  k_norm_blocks<<<b1 - b0, 256, 0, st>>>(blk_tile0_dev, b0, normpart, blocksum);
  k_norm_combine<<<1, 32, 0, st>>>(blks, b0, b1, blocksum, norms);
  return cudaGetLastError();
}

}  // namespace cns
