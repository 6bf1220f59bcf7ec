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
#include "cns_kernels.cuh"

namespace cns {

namespace {

inline int grid_of(const Space& s) { return s.ntiles; }

// ---------------------------------------------------------------------------
// thermodynamics
// ---------------------------------------------------------------------------

// zpres.f90:66-79 and, for the Navier-Stokes equations, zvismo.f90:77-104
__global__ void __launch_bounds__(kTile) k_zpres(const Blk* __restrict__ blks,
                                                 Space sp, Phys ph, int with_mu,
                                                 const double* __restrict__ v,
                                                 long long ld, double* ps,
                                                 double* temp, double* cson,
                                                 double* mu, int* status) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  const double v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n],
               v5 = v[4 * ld + n];
  const double rhoe = v5 - 0.5 * (sq(v2) + sq(v3) + sq(v4)) / v1;
  const double p = ph.gam1 * (rhoe - ph.pinfl);
  const double t = ph.gam * p / v1;
  ps[n] = p;
  temp[n] = t;
  cson[n] = sqrt(t);
  if (with_mu) {
    // the reference aborts on T <= 0 (zvismo.f90:123-127); here the status
    // word records it and the host turns it into an error code
    if (t <= 0.) {
      mu[n] = 0.;
      atomicOr(status, 1);
    } else {
      const double usrey = 1. / ph.reynz, a = ph.suth_a;
      mu[n] = usrey * t * sqrt(t) * (1. + a) / (t + a);
    }
  }
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
__global__ void __launch_bounds__(256) k_prim(long long n0, long long n1,
                                             const double* __restrict__ v,
                                             long long ld, double* __restrict__ prim) {
  const long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= n1) return;
  const double r = v[n];
  prim[n] = v[ld + n] / r;
  prim[ld + n] = v[2 * ld + n] / r;
  prim[2 * ld + n] = v[3 * ld + n] / r;
}

// chronos.f90:110-194 (kprec = 0)
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
  const double dte = dism / (q + cson[nc]);
  double d = sc.eta * dte;
  if (sc.ns) {
    const double rv1 = ph.gam * (mu[nc] / ph.pr + mut[nc] / ph.prt) / t[nc];
    const double rv = fmax(rv1, 4. / 3. * (mu[nc] + mut[nc]) / t[nc]);
    const double dtv = sc.eta * 0.25 * sq(dism) / rv;
    d = fmin(d, dtv);
  }
  dt[nc] = d;
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
  } else if (kind == BC_PARA) {  // clpara.f90:24-40
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
  const double p = ph.pa1 * c.rpi * pow(b, gam6);
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
  const double p = ph.pa1 * c.rpi * pow(b, gam6);
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

// ---------------------------------------------------------------------------
// Roe-MUSCL face flux
// ---------------------------------------------------------------------------

// slope-ratio recurrence of sch_roe.f90:146-194 along one grid line: the
// ratio at face m divides by the ALREADY UPDATED ratio at face m-1, with a
// reset to 1 when |r(m-1) r(m) r(m+1)| <= tiny.  One thread walks one line
// for one of the five variables (blockIdx.y: rho, u, v, w, p); lines of the
// j and k directions are adjacent in i, so those walks are coalesced.
__global__ void __launch_bounds__(kTile) k_ratio(const Blk* __restrict__ blks,
                                                 Space sp, int dir,
                                                 const double* __restrict__ v,
                                                 const double* __restrict__ prim,
                                                 long long ld,
                                                 const double* __restrict__ ps,
                                                 double* __restrict__ R) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const int nd = nd_of(B, dir);
  if (nd < 3) return;
  const long long inc = ninc_of(B, dir);
  const int a = blockIdx.y;
  const double* x = a == 0 ? v : (a == 4 ? ps : prim + (long long)(a - 1) * ld);
  double* Ra = R + ((long long)dir * 5 + a) * ld;
  // (i,j,k) is position 1 of the line: cells 0 .. nd along dir
  const long long n0 = cell_index(B, i, j, k) - inc;
  double x0 = x[n0], x1 = x[n0 + inc], x2 = x[n0 + 2 * inc];
  double rprev = x1 - x0;   // face 1 (never updated)
  double dcur = x2 - x1;    // face 2
  for (int f = 2; f <= nd - 1; ++f) {
    const long long n = n0 + (long long)f * inc;
    const double x3 = x[n + inc];
    const double dnext = x3 - x2;
    double r;
    if (fabs(rprev * dcur * dnext) <= 2.2250738585072014e-308)
      r = 1.;
    else
      r = dcur / rprev;
    Ra[n] = r;
    rprev = r;
    dcur = dnext;
    x2 = x3;
  }
}

__device__ __forceinline__ double phi_mm(double a) {  // sch_roe.f90:1500-1504
  const double m = (a < 1.) ? a : 1.;
  return (m > 0.) ? m : 0.;
}

// kappa-MUSCL without limiter (sch_roe_euler.f90:245-273); cells c[0..3] are
// n-2, n-1, n, n+1 as (rho, u, v, w, p)
__device__ __forceinline__ void muscl_plain(const double c[4][5], double c4,
                                            double xk, double WL[5],
                                            double WR[5]) {
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    WL[a] = c[1][a] + c4 * ((1. - xk) * (c[1][a] - c[0][a]) + (1. + xk) * (c[2][a] - c[1][a]));
    WR[a] = c[2][a] - c4 * ((1. + xk) * (c[2][a] - c[1][a]) + (1. - xk) * (c[3][a] - c[2][a]));
  }
}

// limited MUSCL (sch_roe.f90:196-227): rho and p use one product order,
// the velocities another; rm are the ratios at this face, rp at the next
__device__ __forceinline__ void muscl_limited(const double c[4][5], double c4,
                                              int muscl, double xk,
                                              const double rm[5],
                                              const double rp[5], double WL[5],
                                              double WR[5]) {
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    if (a == 0 || a == 4) {
      WL[a] = c[1][a] + c4 * phi_mm(rm[a]) * (1. - xk) * (c[1][a] - c[0][a]) +
              c4 * phi_mm(1. / rm[a]) * (1. + xk) * (c[2][a] - c[1][a]);
      WR[a] = c[2][a] - c4 * phi_mm(rp[a]) * (1. + xk) * (c[2][a] - c[1][a]) -
              c4 * phi_mm(1. / rp[a]) * (1. - xk) * (c[3][a] - c[2][a]);
    } else {
      WL[a] = c[1][a] + c4 * phi_mm(rm[a]) * (1. - xk) * (c[1][a] - c[0][a]) +
              (1. + xk) * (c[2][a] - c[1][a]) * 0.25 * muscl * phi_mm(1. / rm[a]);
      WR[a] = c[2][a] - c4 * phi_mm(rp[a]) * (1. + xk) * (c[2][a] - c[1][a]) -
              (1. - xk) * (c[3][a] - c[2][a]) * 0.25 * muscl * phi_mm(1. / rp[a]);
    }
  }
}

// row r of the right eigenvector matrix P at the Roe state
__device__ __forceinline__ void p_row(int r, double nx, double ny, double nz,
                                      double um, double vm, double wm,
                                      double hm, double am, double vn,
                                      double vitm2, double rhom, double rhoiam,
                                      double p[5]) {
  switch (r) {
    case 0:
      p[0] = nx; p[1] = ny; p[2] = nz;
      p[3] = 0.5 * rhoiam; p[4] = 0.5 * rhoiam;
      break;
    case 1:
      p[0] = um * nx; p[1] = um * ny - rhom * nz; p[2] = um * nz + rhom * ny;
      p[3] = 0.5 * rhoiam * (um + nx * am); p[4] = 0.5 * rhoiam * (um - nx * am);
      break;
    case 2:
      p[0] = vm * nx + rhom * nz; p[1] = vm * ny; p[2] = vm * nz - rhom * nx;
      p[3] = 0.5 * rhoiam * (vm + ny * am); p[4] = 0.5 * rhoiam * (vm - ny * am);
      break;
    case 3:
      p[0] = wm * nx - rhom * ny; p[1] = wm * ny + rhom * nx; p[2] = wm * nz;
      p[3] = 0.5 * rhoiam * (wm + nz * am); p[4] = 0.5 * rhoiam * (wm - nz * am);
      break;
    default:
      p[0] = vitm2 * nx + rhom * (vm * nz - wm * ny);
      p[1] = vitm2 * ny + rhom * (wm * nx - um * nz);
      p[2] = vitm2 * nz + rhom * (um * ny - vm * nx);
      p[3] = 0.5 * rhoiam * (hm + am * vn);
      p[4] = 0.5 * rhoiam * (hm - am * vn);
  }
}

// Roe dissipation |A|(W_R - W_L) of sch_roe_euler.f90:284-402 (di), plus the
// specific total energies el, er used by the centred part
__device__ __forceinline__ void roe_dissipation(const double WL[5],
                                                const double WR[5], double sx,
                                                double sy, double sz, bool absam,
                                                const Phys& ph, double di[5],
                                                double& el, double& er) {
  const double gam = ph.gam, gam1 = ph.gam1, pinfl = ph.pinfl;
  const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
  const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
  const double cnds = sqrt(sx * sx + sy * sy + sz * sz);
  const double nx = sx / cnds, ny = sy / cnds, nz = sz / cnds;
  const double al = sqrt(gam * pl / rhol);
  const double ar = sqrt(gam * prr / rhor);
  const double q2l = sq(ul) + sq(vl) + sq(wl);
  const double q2r = sq(ur) + sq(vr) + sq(wr);
  const double hl = al * al / gam1 + 0.5 * q2l;
  const double hr = ar * ar / gam1 + 0.5 * q2r;
  el = pl / (gam1 * rhol) + 0.5 * q2l + pinfl / rhol;
  er = prr / (gam1 * rhor) + 0.5 * q2r + pinfl / rhor;
  const double gd = sqrt(rhor / rhol);
  const double gd1 = 1. / (1. + gd);
  const double gd2 = gd * gd1;
  const double rhom = sqrt(rhol * rhor);
  const double rhomi = 1. / rhom;
  const double um = gd1 * ul + gd2 * ur;
  const double vm = gd1 * vl + gd2 * vr;
  const double wm = gd1 * wl + gd2 * wr;
  const double hm = gd1 * hl + gd2 * hr;
  const double vitm2 = 0.5 * (sq(um) + sq(vm) + sq(wm));
  const double am = absam ? sqrt(fabs(gam1 * (hm - vitm2))) : sqrt(gam1 * (hm - vitm2));
  const double am2i = 1. / (am * am);
  const double vn = um * nx + vm * ny + wm * nz;
  const double rhoiam = rhom / am;
  const double rhoami = am2i / rhoiam;
  const double lam1 = fabs(vn * cnds);
  const double lam4 = fabs(vn * cnds + am * cnds);
  const double lam5 = fabs(vn * cnds - am * cnds);
  double q[5][5];
  q[0][0] = (1. - gam1 * vitm2 * am2i) * nx - (vm * nz - wm * ny) * rhomi;
  q[0][1] = gam1 * um * nx * am2i;
  q[0][2] = gam1 * vm * nx * am2i + nz * rhomi;
  q[0][3] = gam1 * wm * nx * am2i - ny * rhomi;
  q[0][4] = -gam1 * nx * am2i;
  q[1][0] = (1. - gam1 * vitm2 * am2i) * ny - (wm * nx - um * nz) * rhomi;
  q[1][1] = gam1 * um * ny * am2i - nz * rhomi;
  q[1][2] = gam1 * vm * ny * am2i;
  q[1][3] = gam1 * wm * ny * am2i + nx * rhomi;
  q[1][4] = -gam1 * ny * am2i;
  q[2][0] = (1. - gam1 * vitm2 * am2i) * nz - (um * ny - vm * nx) * rhomi;
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
  double dw[5];
  dw[0] = rhor - rhol;
  dw[1] = rhor * ur - rhol * ul;
  dw[2] = rhor * vr - rhol * vl;
  dw[3] = rhor * wr - rhol * wl;
  dw[4] = rhor * er - rhol * el;
  const double lam[5] = {lam1, lam1, lam1, lam4, lam5};
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double p[5];
    p_row(r, nx, ny, nz, um, vm, wm, hm, am, vn, vitm2, rhom, rhoiam, p);
    double pl_[5];
#pragma unroll
    for (int kk = 0; kk < 5; ++kk) pl_[kk] = p[kk] * lam[kk];
    double acc = 0.;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double a = pl_[0] * q[0][c];
#pragma unroll
      for (int kk = 1; kk < 5; ++kk) a = a + pl_[kk] * q[kk][c];
      acc = (c == 0) ? a * dw[0] : acc + a * dw[c];
    }
    di[r] = acc;
  }
}

// primitive (rho, u, v, w, p) of cell n
__device__ __forceinline__ void load_prim(const double* __restrict__ v,
                                          const double* __restrict__ prim,
                                          const double* __restrict__ ps,
                                          long long ld, long long n,
                                          double c[5]) {
  c[0] = v[n];
  c[1] = prim[n];
  c[2] = prim[ld + n];
  c[3] = prim[2 * ld + n];
  c[4] = ps[n];
}

// one face per thread, direction dir: interior faces give 0.5*f (sch_roe*
// interior loops), boundary faces give the ghost-cell physical flux s
// (lower face 1, upper face nd).  Results go to G[dir][a][n] where n is the
// cell above the face.
template <bool NS>
__global__ void __launch_bounds__(kTile, 3) k_face_flux(
    const Blk* __restrict__ blks, Space sp, int dir, Phys ph, Scheme sc,
    const double* __restrict__ v, const double* __restrict__ prim, long long ld,
    const double* __restrict__ ps, const double* __restrict__ tau,
    const double* __restrict__ sn, const double* __restrict__ R,
    double* __restrict__ G) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long inc = ninc_of(B, dir);
  const int nd = nd_of(B, dir);
  const int p = dir == 0 ? i : (dir == 1 ? j : k);
  const long long n = cell_index(B, i, j, k);
  const double sx = sn_ptr(sn, B, dir, 0)[n], sy = sn_ptr(sn, B, dir, 1)[n],
               sz = sn_ptr(sn, B, dir, 2)[n];
  const double pinfl = ph.pinfl;
  double out[5];
  if (p == 1 || p == nd) {
    // boundary face: physical flux of the ghost cell (sch_roe_euler.f90:
    // 438-513, sch_roe.f90:497-580); the Euler j/k lower faces divide the
    // energy flux by the interior density (sch_roe_euler.f90:630-632)
    const long long ng = (p == 1) ? n - inc : n;
    const long long nrho = (!NS && p == 1 && dir > 0) ? n : ng;
    const double v1 = v[ng], v2 = v[ld + ng], v3 = v[2 * ld + ng],
                 v4 = v[3 * ld + ng], v5 = v[4 * ld + ng], pg = ps[ng];
    const double qu = prim[ng], qv = prim[ld + ng], qw = prim[2 * ld + ng];
    double fxx, fxy, fxz, fyy, fyz, fzz, fex, fey, fez;
    if (!NS) {
      const double rr = v[nrho];
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
      const double txx = tau[ng], txy = tau[ld + ng], txz = tau[2 * ld + ng],
                   tyy = tau[3 * ld + ng], tyz = tau[4 * ld + ng],
                   tzz = tau[5 * ld + ng], qx = tau[6 * ld + ng],
                   qy = tau[7 * ld + ng], qz = tau[8 * ld + ng];
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
    double c[4][5];
#pragma unroll
    for (int s = 0; s < 4; ++s) load_prim(v, prim, ps, ld, n + (long long)(s - 2) * inc, c[s]);
    double WL[5], WR[5];
    const double c4 = 0.25 * sc.muscl;
    if (NS && sc.ilim == 1 && p <= nd - 2) {
      const double* Rd = R + (long long)dir * 5 * ld;
      double rm[5], rp[5];
#pragma unroll
      for (int a = 0; a < 5; ++a) {
        rm[a] = Rd[a * ld + n];
        rp[a] = Rd[a * ld + n + inc];
      }
      muscl_limited(c, c4, sc.muscl, sc.xk, rm, rp, WL, WR);
    } else {
      muscl_plain(c, c4, sc.xk, WL, WR);
    }
    double di[5], el, er;
    roe_dissipation(WL, WR, sx, sy, sz, (!NS) && dir > 0, ph, di, el, er);
    const double rhol = WL[0], ul = WL[1], vl = WL[2], wl = WL[3], pl = WL[4];
    const double rhor = WR[0], ur = WR[1], vr = WR[2], wr = WR[3], prr = WR[4];
    double dfxx, dfxy, dfxz, dfyy, dfyz, dfzz, dfex, dfey, dfez;
    if (!NS) {
      dfxx = rhor * sq(ur) + prr - pinfl + rhol * sq(ul) + pl - pinfl;
      dfxy = rhor * ur * vr + rhol * ul * vl;
      dfxz = rhor * ur * wr + rhol * ul * wl;
      dfyy = rhor * sq(vr) + prr - pinfl + rhol * sq(vl) + pl - pinfl;
      dfyz = rhor * vr * wr + rhol * vl * wl;
      dfzz = rhor * sq(wr) + prr - pinfl + rhol * sq(wl) + pl - pinfl;
      dfex = (rhor * er + prr - pinfl) * ur + (rhol * el + pl - pinfl) * ul;
      dfey = (rhor * er + prr - pinfl) * vr + (rhol * el + pl - pinfl) * vl;
      dfez = (rhor * er + prr - pinfl) * wr + (rhol * el + pl - pinfl) * wl;
    } else {
      const long long nR = n, nL = n - inc;
      const double txxR = tau[nR], txyR = tau[ld + nR], txzR = tau[2 * ld + nR],
                   tyyR = tau[3 * ld + nR], tyzR = tau[4 * ld + nR],
                   tzzR = tau[5 * ld + nR];
      const double txxL = tau[nL], txyL = tau[ld + nL], txzL = tau[2 * ld + nL],
                   tyyL = tau[3 * ld + nL], tyzL = tau[4 * ld + nL],
                   tzzL = tau[5 * ld + nL];
      dfxx = rhor * sq(ur) + prr - pinfl - txxR + rhol * sq(ul) + pl - pinfl - txxL;
      dfxy = rhor * ur * vr - txyR + rhol * ul * vl - txyL;
      dfxz = rhor * ur * wr - txzR + rhol * ul * wl - txzL;
      dfyy = rhor * sq(vr) + prr - pinfl - tyyR + rhol * sq(vl) + pl - pinfl - tyyL;
      dfyz = rhor * vr * wr - tyzR + rhol * vl * wl - tyzL;
      dfzz = rhor * sq(wr) + prr - pinfl - tzzR + rhol * sq(wl) + pl - pinfl - tzzL;
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
    const double f1 = (rhor * ur + rhol * ul) * sx + (rhor * vr + rhol * vl) * sy +
                      (rhor * wr + rhol * wl) * sz - di[0];
    const double f2 = dfxx * sx + dfxy * sy + dfxz * sz - di[1];
    const double f3 = dfxy * sx + dfyy * sy + dfyz * sz - di[2];
    const double f4 = dfxz * sx + dfyz * sy + dfzz * sz - di[3];
    const double f5 = dfex * sx + dfey * sy + dfez * sz - di[4];
    out[0] = 0.5 * f1;
    out[1] = 0.5 * f2;
    out[2] = 0.5 * f3;
    out[3] = 0.5 * f4;
    out[4] = 0.5 * f5;
  }
  double* Gd = G + (long long)dir * 5 * ld;
#pragma unroll
  for (int a = 0; a < 5; ++a) Gd[a * ld + n] = out[a];
}

// u(n) from the six faces of the cell, in the reference's summation order
__global__ void __launch_bounds__(kTile) k_accumulate(const Blk* __restrict__ blks,
                                                      Space sp,
                                                      const double* __restrict__ G,
                                                      long long ld,
                                                      double* __restrict__ u) {
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
  for (int a = 0; a < 5; ++a) u[a * ld + n] = acc[a];
}

// ---------------------------------------------------------------------------
// implicit phase: matrix-free point Jacobi (implimf_eu.f90, implimf_3d.f90)
// ---------------------------------------------------------------------------

// per real cell: coefdiag seed (vol/dt or vol*(0+1/dt)) and the viscous
// spectral factor rv (implimf_3d.f90:95-105, implimf_eu.f90:124-134)
__global__ void __launch_bounds__(kTile) k_impl_cell0(
    const Blk* __restrict__ blks, Space sp, Phys ph, int eu,
    const double* __restrict__ v, const double* __restrict__ dt,
    const double* __restrict__ mu, const double* __restrict__ mut,
    const double* __restrict__ vol, double* coefdiag, double* rv) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
  if (eu) {
    const double fact = 0.;
    coefdiag[n] = vol[n] * (fact + 1. / dt[n]);
  } else {
    rv[n] = ph.gam * (mu[n] / ph.pr + mut[n] / ph.prt) / v[n];
    coefdiag[n] = vol[n] / dt[n];
  }
}

// per face: spectral radius coefe (implimf_eu.f90:141-159,
// implimf_3d.f90:110-190)
__global__ void __launch_bounds__(kTile) k_impl_coefe(
    const Blk* __restrict__ blks, Space sp, int dir, int eu,
    const double* __restrict__ v, const double* __restrict__ prim, long long ld,
    const double* __restrict__ sn,
    const double* __restrict__ vol, const double* __restrict__ cson,
    const double* __restrict__ rv, double* coefe) {
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
}

// per real cell: coefdiag += coefe of the six faces (implimf_eu.f90:161-170,
// implimf_3d.f90:192-203: the same left-to-right chain)
__global__ void __launch_bounds__(kTile) k_impl_diag(const Blk* __restrict__ blks,
                                                     Space sp, long long ld,
                                                     const double* __restrict__ coefe,
                                                     double* coefdiag) {
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
  coefdiag[n] = c;
}

// df index: 0 xx, 1 xy, 2 xz, 3 ex, 4 yy, 5 yz, 6 ey, 7 zz, 8 ez

// flux-increment projections tn(1..5) on the face between cells nu (above)
// and nl (below)
template <bool EU, bool FIRST>
__device__ __forceinline__ void jacobi_tn(const double* __restrict__ d,
                                          const double* __restrict__ df,
                                          long long ld, long long nu,
                                          long long nl, double sx, double sy,
                                          double sz, double tn[5]) {
  double a2, a3, a4, fxx, fxy, fxz, fex, fyy, fyz, fey, fzz, fez;
  if (FIRST) {
    a2 = a3 = a4 = 0. + 0.;
    fxx = fxy = fxz = fex = fyy = fyz = fey = fzz = fez = 0. + 0.;
  } else {
    a2 = d[ld + nu] + d[ld + nl];
    a3 = d[2 * ld + nu] + d[2 * ld + nl];
    a4 = d[3 * ld + nu] + d[3 * ld + nl];
    fxx = df[nu] + df[nl];
    fxy = df[ld + nu] + df[ld + nl];
    fxz = df[2 * ld + nu] + df[2 * ld + nl];
    fex = df[3 * ld + nu] + df[3 * ld + nl];
    fyy = df[4 * ld + nu] + df[4 * ld + nl];
    fyz = df[5 * ld + nu] + df[5 * ld + nl];
    fey = df[6 * ld + nu] + df[6 * ld + nl];
    fzz = df[7 * ld + nu] + df[7 * ld + nl];
    fez = df[8 * ld + nu] + df[8 * ld + nl];
  }
  if (EU) {
    tn[0] = 0.5 * (a2 * sx + a3 * sy + a4 * sz);
    tn[1] = 0.5 * (fxx * sx + fxy * sy + fxz * sz);
    tn[2] = 0.5 * (fxy * sx + fyy * sy + fyz * sz);
    tn[3] = 0.5 * (fxz * sx + fyz * sy + fzz * sz);
    tn[4] = 0.5 * (fex * sx + fey * sy + fez * sz);
  } else {
    tn[0] = 0.5 * a2 * sx + 0.5 * a3 * sy + 0.5 * a4 * sz;
    tn[1] = 0.5 * fxx * sx + 0.5 * fxy * sy + 0.5 * fxz * sz;
    tn[2] = 0.5 * fxy * sx + 0.5 * fyy * sy + 0.5 * fyz * sz;
    tn[3] = 0.5 * fxz * sx + 0.5 * fyz * sy + 0.5 * fzz * sz;
    tn[4] = 0.5 * fex * sx + 0.5 * fey * sy + 0.5 * fez * sz;
  }
}

// one Jacobi sub-iteration on one real cell: d2w = -u + sum over the faces,
// d = d2w / coefdiag, then the flux increments of v+d (implimf_eu.f90:
// 176-323, implimf_3d.f90:222-466).  Reads the previous iterate (d_in,
// df_in), writes the next one; FIRST: the previous iterate is zero.
template <bool EU, bool FIRST>
__global__ void __launch_bounds__(kTile) k_jacobi(
    const Blk* __restrict__ blks, Space sp, Phys ph, int qfix, long long ld,
    const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ prim,
    const double* __restrict__ ps, const double* __restrict__ sn,
    const double* __restrict__ coefe, const double* __restrict__ coefdiag,
    const double* __restrict__ d_in, const double* __restrict__ df_in,
    double* __restrict__ d_out, double* __restrict__ df_out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const Blk& B = blks[b];
  const long long n = cell_index(B, i, j, k);
  double d2w[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) d2w[a] = -u[a * ld + n];
#pragma unroll
  for (int dir = 0; dir < 3; ++dir) {
    const long long inc = ninc_of(B, dir);
    const double *s0 = sn_ptr(sn, B, dir, 0), *s1 = sn_ptr(sn, B, dir, 1),
                 *s2 = sn_ptr(sn, B, dir, 2);
    const double* ce = coefe + (long long)dir * ld;
    double tn[5];
    jacobi_tn<EU, FIRST>(d_in, df_in, ld, n, n - inc, s0[n], s1[n], s2[n], tn);
    const double cel = ce[n], ceu = ce[n + inc];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double dl = FIRST ? 0. : d_in[a * ld + n - inc];
      const double du = FIRST ? 0. : d_in[a * ld + n + inc];
      d2w[a] = d2w[a] + tn[a] + cel * dl + ceu * du;
    }
    const long long nu = n + inc;
    jacobi_tn<EU, FIRST>(d_in, df_in, ld, nu, n, s0[nu], s1[nu], s2[nu], tn);
#pragma unroll
    for (int a = 0; a < 5; ++a) d2w[a] = d2w[a] - tn[a];
  }
  const double cd = coefdiag[n];
  double dn[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) {
    dn[a] = d2w[a] / cd;
    d_out[a * ld + n] = dn[a];
  }
  const double gam1 = ph.gam1, pinfl = ph.pinfl;
  const double v1 = v[n], v2 = v[ld + n], v3 = v[2 * ld + n], v4 = v[3 * ld + n],
               v5 = v[4 * ld + n], p = ps[n];
  double f[9];
  if (EU) {
    const double wi1 = 1. / (v1 + dn[0]);
    const double ui = v2 + dn[1], vi = v3 + dn[2], wi = v4 + dn[3], wi5 = v5 + dn[4];
    const double pres = gam1 * (wi5 - .5 * wi1 * (sq(ui) + sq(vi) + sq(wi)) - pinfl);
    const double norm = 1. / v1;
    const double fxx = v2 * (v2 * norm) + p;
    const double fxy = v3 * (v2 * norm);
    const double fxz = v4 * (v2 * norm);
    const double fyy = v3 * (v3 * norm) + p;
    const double fyz = v4 * (v3 * norm);
    const double fzz = v4 * (v4 * norm) + p;
    const double fex = (v5 + p - pinfl) * v2 * norm;
    const double fey = (v5 + p - pinfl) * v3 * norm;
    const double fez = (v5 + p - pinfl) * v4 * norm;
    f[0] = wi1 * sq(ui) + pres - fxx;
    f[1] = wi1 * ui * vi - fxy;
    f[2] = wi1 * ui * wi - fxz;
    f[3] = wi1 * ui * (wi5 + pres - pinfl) - fex;
    f[4] = wi1 * sq(vi) + pres - fyy;
    f[5] = wi1 * vi * wi - fyz;
    f[6] = wi1 * vi * (wi5 + pres - pinfl) - fey;
    f[7] = wi1 * sq(wi) + pres - fzz;
    // implimf_eu.f90:312 lacks the *wi factor of the z energy increment; the
    // parity path keeps it, qfix (a flagged non-reference option) restores it
    f[8] = qfix ? wi1 * wi * (wi5 + pres - pinfl) - fez
                : wi1 * (wi5 + pres - pinfl) - fez;
  } else {
    const double wi1 = v1 + dn[0];
    const double ui = (v2 + dn[1]) / wi1, vi = (v3 + dn[2]) / wi1, wi = (v4 + dn[3]) / wi1;
    const double wi5 = v5 + dn[4];
    const double pres = gam1 * (wi5 - .5 * wi1 * (sq(ui) + sq(vi) + sq(wi)) - pinfl);
    const double qu = prim[n], qv = prim[ld + n], qw = prim[2 * ld + n];
    const double fxx = v2 * qu + p;
    const double fxy = v3 * qu;
    const double fxz = v4 * qu;
    const double fyy = v3 * qv + p;
    const double fyz = v4 * qv;
    const double fzz = v4 * qw + p;
    const double fex = (v5 + p - pinfl) * v2 / v1;
    const double fey = (v5 + p - pinfl) * v3 / v1;
    const double fez = (v5 + p - pinfl) * v4 / v1;
    f[0] = wi1 * sq(ui) + pres - fxx;
    f[1] = wi1 * ui * vi - fxy;
    f[2] = wi1 * ui * wi - fxz;
    f[3] = ui * (wi5 + pres - pinfl) - fex;
    f[4] = wi1 * sq(vi) + pres - fyy;
    f[5] = wi1 * vi * wi - fyz;
    f[6] = vi * (wi5 + pres - pinfl) - fey;
    f[7] = wi1 * sq(wi) + pres - fzz;
    f[8] = wi * (wi5 + pres - pinfl) - fez;
  }
#pragma unroll
  for (int a = 0; a < 9; ++a) df_out[a * ld + n] = f[a];
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

// v += d on the real cells (implimf_*.f90 final update), the residual norm
// partials and, when requested, the final increment copied to d_out
__global__ void __launch_bounds__(kTile) k_update(const Blk* __restrict__ blks,
                                                  Space sp, long long ld,
                                                  const double* __restrict__ d,
                                                  double* __restrict__ v,
                                                  const double* __restrict__ dt,
                                                  double* d_out, double* normpart) {
  int b, i, j, k;
  const bool valid = space_elem(sp, threadIdx.x, b, i, j, k);
  double res[5] = {0., 0., 0., 0., 0.};
  if (valid) {
    const long long n = cell_index(blks[b], i, j, k);
    const double t = dt[n];
#pragma unroll
    for (int a = 0; a < 5; ++a) {
      const double vo = v[a * ld + n], dd = d[a * ld + n];
      const double vn = vo + dd;
      v[a * ld + n] = vn;
      if (d_out) d_out[a * ld + n] = dd;
      res[a] = (vn - vo) / t;
    }
  }
  if (normpart) norm_tile_reduce(res, valid, normpart + (long long)(sp.tile0 + blockIdx.x) * 15);
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

// per-block sums of the tile partials in a fixed tree order, then the
// rscpsv.f90:79-150 combination over blocks; one CTA
__global__ void __launch_bounds__(256) k_norm_finalize(
    const Blk* __restrict__ blks, const int* __restrict__ blk_tile0, int b0,
    int b1, const double* __restrict__ normpart, double* norms) {
  __shared__ double red[256][15];
  __shared__ double blocksum[15];
  __shared__ double g[15];
  __shared__ long long npts;
  if (threadIdx.x < 15) g[threadIdx.x] = 0.;
  if (threadIdx.x == 0) npts = 0;
  __syncthreads();
  for (int b = b0; b < b1; ++b) {
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
    if (threadIdx.x < 15) blocksum[threadIdx.x] = red[0][threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
      const Blk& B = blks[b];
      const long long nmax = (long long)(B.ni - 1) * (B.nj - 1) * (B.nk - 1);
      const double coef = 1. / (double)nmax;
      for (int a = 0; a < 5; ++a) {
        const double d1 = coef * blocksum[a];
        const double d2 = sqrt(coef * blocksum[5 + a]);
        g[a] = g[a] + (double)nmax * d1;
        g[5 + a] = g[5 + a] + (double)nmax * sq(d2);
        g[10 + a] = fmax(g[10 + a], fabs(blocksum[10 + a]));
      }
      npts += nmax;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int a = 0; a < 5; ++a) {
      norms[a] = g[a] / (double)npts;
      norms[5 + a] = sqrt(g[5 + a] / (double)npts);
      norms[10 + a] = g[10 + a];
    }
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
    k_prim<<<(int)((n1 - n0 + 255) / 256), 256, 0, st>>>(n0, n1, v, ld, prim);
  return cudaGetLastError();
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

cudaError_t launch_ratio(const Blk* blks, const SpaceBuf* lines, int l0,
                         const double* v, const double* prim, long long ld,
                         const double* ps, double* R, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = lines[dir].view(l0);
    if (sp.ntiles > 0)
      k_ratio<<<dim3(grid_of(sp), 5), kTile, 0, st>>>(blks, sp, dir, v, prim, ld, ps, R);
  }
  return cudaGetLastError();
}

cudaError_t launch_face_flux(const Blk* blks, const SpaceBuf* faces, int l0,
                             Phys ph, Scheme sc, const double* v,
                             const double* prim, long long ld, const double* ps,
                             const double* tau, const double* sn, const double* R,
                             double* G, cudaStream_t st) {
  for (int dir = 0; dir < 3; ++dir) {
    const Space sp = faces[dir].view(l0);
    if (sp.ntiles == 0) continue;
    if (sc.ns)
      k_face_flux<true><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                       ld, ps, tau, sn, R, G);
    else
      k_face_flux<false><<<grid_of(sp), kTile, 0, st>>>(blks, sp, dir, ph, sc, v, prim,
                                                        ld, ps, tau, sn, R, G);
  }
  return cudaGetLastError();
}

cudaError_t launch_accumulate(const Blk* blks, Space sp, const double* G,
                              long long ld, double* u, cudaStream_t st) {
  if (sp.ntiles > 0) k_accumulate<<<grid_of(sp), kTile, 0, st>>>(blks, sp, G, ld, u);
  return cudaGetLastError();
}

cudaError_t launch_implicit(const Blk* blks, Space cells, const SpaceBuf* faces,
                            int l0, Phys ph, Scheme sc, int eu, int lmx,
                            const double* u, const double* dt, double* v,
                            double* d_out, const double* mu, const double* mut,
                            const double* sn, const double* vol,
                            const double* ps, const double* cson, Work& w,
                            int want_norms, cudaStream_t st) {
  const double* prim = w.prim;
  const long long ld = w.ld;
  if (cells.ntiles == 0) return cudaSuccess;
  const int g = grid_of(cells);
  k_impl_cell0<<<g, kTile, 0, st>>>(blks, cells, ph, eu, v, dt, mu, mut, vol,
                                    w.coefdiag, w.rv);
  for (int dir = 0; dir < 3; ++dir) {
    const Space fs = faces[dir].view(l0);
    if (fs.ntiles > 0)
      k_impl_coefe<<<fs.ntiles, kTile, 0, st>>>(blks, fs, dir, eu, v, prim, ld, sn,
                                                vol, cson, w.rv, w.coefe);
  }
  k_impl_diag<<<g, kTile, 0, st>>>(blks, cells, ld, w.coefe, w.coefdiag);
  int cur = 0;  // index of the buffer holding the latest iterate
  if (lmx == 0) {
    cudaError_t e0 = cudaMemsetAsync(w.dpp[0], 0, sizeof(double) * 5 * ld, st);
    if (e0 != cudaSuccess) return e0;
  }
  for (int ls = 1; ls <= lmx; ++ls) {
    const int nxt = (ls == 1) ? 0 : 1 - cur;
    const double* din = w.dpp[cur];
    const double* dfin = w.dfpp[cur];
    double* dout = w.dpp[nxt];
    double* dfout = w.dfpp[nxt];
    if (eu) {
      if (ls == 1)
        k_jacobi<true, true><<<g, kTile, 0, st>>>(blks, cells, ph, sc.qfix_dfez, ld, u, v,
                                                  prim, ps, sn, w.coefe, w.coefdiag, din,
                                                  dfin, dout, dfout);
      else
        k_jacobi<true, false><<<g, kTile, 0, st>>>(blks, cells, ph, sc.qfix_dfez, ld, u, v,
                                                   prim, ps, sn, w.coefe, w.coefdiag, din,
                                                   dfin, dout, dfout);
    } else {
      if (ls == 1)
        k_jacobi<false, true><<<g, kTile, 0, st>>>(blks, cells, ph, 0, ld, u, v, prim, ps,
                                                   sn, w.coefe, w.coefdiag, din,
                                                   dfin, dout, dfout);
      else
        k_jacobi<false, false><<<g, kTile, 0, st>>>(blks, cells, ph, 0, ld, u, v, prim, ps,
                                                    sn, w.coefe, w.coefdiag, din,
                                                    dfin, dout, dfout);
    }
    cur = nxt;
  }
  k_update<<<g, kTile, 0, st>>>(blks, cells, ld, w.dpp[cur], v, dt, d_out,
                                want_norms ? w.normpart : nullptr);
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
                                 double* norms, cudaStream_t st) {
  k_norm_finalize<<<1, 256, 0, st>>>(blks, blk_tile0_dev, b0, b1, normpart, norms);
  return cudaGetLastError();
}

}  // namespace cns
