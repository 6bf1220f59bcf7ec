/*
 * cns_abi.h -- C ABI of the B200 implementation of the CodeNS per-iteration
 * hot path (residual evaluation and matrix-free implicit update on
 * structured multi-block grids).
 *
 * The entry points keep the reference's call surface: one function per
 * reference subroutine, the same argument meaning and order, prefixed
 * "cns_", plus a context handle that carries what the reference reads from
 * its Fortran modules (maillage: block layout; proprieteflu/definition:
 * physical constants; schemanum: scheme keys; boundary: boundary lists).
 *
 * Data contract (identical to the reference's arrays, crdms.f90:125-158):
 *   - blocks l = 1..nblk with real nodes 1..ni, 1..nj, 1..nk and one ghost
 *     layer; nodes and cells share one flat index space; block l starts at
 *     npc(l) = sum of (ni+2)(nj+2)(nk+2) of the blocks before it;
 *   - cell (i,j,k) of block l is element npc(l) + i + j*(ni+2) + k*(ni+2)*(nj+2)
 *     (0-based storage of sch_roe.f90:1487-1491);
 *   - v, u, d are column-major (ld, 5) double arrays (ip11 x ip60, columns
 *     1..5 = rho, rho u, rho v, rho w, rho E); scalar cell arrays are (ld);
 *   - sn holds, for block l at offset 9*npc(l), sn(nnn, 3 face directions,
 *     3 components), the area vector of the lower face of each cell oriented
 *     towards increasing index (norm.f90);
 *   - tau is (ld, 9): toxx, toxy, toxz, toyy, toyz, tozz, qcx, qcy, qcz.
 * Per-routine entry points (zpres ... implimf_3d below) take the reference
 * routine's argument list in its order after the context handle: its
 * switches (ityprk, equat, lmx, dtpas, etal), its arrays, and its work
 * arrays (accepted for the drop-in and not used: the device recomputes what
 * the reference stores in them; they may be NULL).  As in the reference,
 * sn is the block's slice sn(npsn) with lgsnlt = nnn(lm) (sequence
 * association, atsch_num.f90:470-479); lm = 0 (every block in one launch, an
 * extension) takes the whole array with lgsnlt = ld.  equat is the
 * reference's character*7 (no terminating NUL): the equations 'eu' or 'ns'
 * in (1:2) and the three-dimensional form '3d' in (3:4); the
 * two-dimensional forms return CNS_EINVAL.  ityprk != 0 (multigrid forcing)
 * is honoured as in the reference: the flux routines subtract u from ff on
 * the real cells, the implicit routines solve with -u - ff.
 *
 * Array arguments of the per-routine entry points may be DEVICE pointers on
 * the context's device (the call only enqueues work on the context stream)
 * or HOST pointers, the reference's own arrays passed as they are: a host
 * array is copied to the device before the routine, copied back after it
 * when the routine writes it, and the call returns when the copies are done
 * (the copy-in/out parity mode; one call may mix both kinds).  The fast path
 * (cns_bind_state, cns_atsch_num_step) takes device arrays; the *_host
 * entry point host arrays.
 *
 * Errors: every function returns 0 on success or a CNS_E* code.  The
 * reference prints and stops instead (zvismo.f90:123-127, chrono.f90:134-142,
 * rbord.f90:417-421); a Fortran shim turns a nonzero code into that message
 * and STOP.
 *
 * Threading: a context is used from one host thread; work is ordered on the
 * context's CUDA stream (cns_set_stream).
 */
#ifndef CNS_ABI_H
#define CNS_ABI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CNS_OK = 0,
  CNS_EINVAL = 1,      /* bad argument (block number, sizes, pointers) */
  CNS_ECUDA = 2,       /* CUDA runtime error */
  CNS_ETEMP = 3,       /* non-positive temperature (zvismo.f90:123-127) */
  CNS_EDT = 4,         /* global time step below dt1min (chrono.f90:134-142) */
  CNS_EBC = 5,         /* unknown boundary condition (rbord.f90:417-421) */
  CNS_ENOTREADY = 6,   /* state arrays not bound / metric not computed */
  CNS_ENONFINITE = 7,  /* non-finite residual norm after a step */
  CNS_EIO = 8,         /* a file cannot be opened, read or written */
  CNS_EFORMAT = 9      /* a file's records do not match the layout (the
                          reference stops: readdg.f90:86-89) */
};

/* boundary kinds (rbord.f90:144-424); CNS_BC_LP2: the adiabatic wall with
 * the wall law ('lp2', rbord.f90:374-388): the ghosts of 'para', and with
 * the Navier-Stokes equations the wall stresses of lparoi1.f90 after zvisqc
 * (cllparoi1.f90, atsch_num.f90:579-604), with the Spalart-Allmaras step the
 * first cell's nu~ of lpsa1.f90 and no implicit increment there
 * (impli2_eqt_3d.f90:384-405); it needs the wall distance of cns_set_sa */
enum { CNS_BC_EXTR = 1, CNS_BC_RC = 2, CNS_BC_PARA = 3, CNS_BC_IDD = 4,
       CNS_BC_PRD = 5, CNS_BC_LP2 = 6 };

typedef struct cns_ctx cns_ctx;

/* maillage: block dimensions (ii2, jj2, kk2 = real node counts) */
typedef struct {
  int32_t nblk;
  const int32_t *dims;   /* [3*nblk]: ni, nj, nk of each block (each >= 2,
                            (ni+2)(nj+2)(nk+2) < 2^31, else CNS_EINVAL) */
  int64_t ld;            /* ip11: leading dimension of the state arrays */
} cns_layout_t;

/* proprieteflu / definition (dfph.f90, c_nzst.f90, zvismo.f90:79) */
typedef struct {
  double gam, pinfl, pr, prt, reynz;
  double suth_a;         /* Sutherland 110.4/tnz */
  double pa1, aa1, omg;  /* reference pressure, sound speed, rotation speed */
} cns_phys_t;

/* schemanum keys of the path (tcmd_dfnm.f90, defdf*.f90) */
typedef struct {
  int32_t ns;            /* equat(1:2) == 'ns' */
  int32_t muscl;
  double xk;
  int32_t ilim;          /* 1: minmod limiter with the in-place ratio recurrence */
  double eta;            /* CFL */
  int32_t kdtl;          /* 0: global time step (chrono.f90:113-151) */
  double dt1min;
  int32_t lmax;          /* Jacobi sub-iterations */
  int32_t qfix_dfez;     /* non-reference option: restore the missing *wi of
                            implimf_eu.f90:312 (0 = reference behaviour) */
  int32_t precision;     /* fused step: 0 = FP64 (bit-exact); 1 = mixed: FP64
                            residual, boundary conditions, update and norms,
                            FP32 Jacobi sweeps (same steady state as FP64);
                            2 = defect correction: FP32 face fluxes too, the
                            FP64 residual every kdefect iterations (stalls at
                            the FP32 rounding level of the fluxes) */
  int32_t kdefect;       /* precision 2: the FP64 residual and the correction
                            R64 - R32 are refreshed every kdefect iterations */
  int32_t ischema;       /* 7: Roe (sch_roe, sch_roe_euler); 14: HLLC; 9: Rusanov; 5: AUSM+;
                            12: WENO5 (sch_weno5_3d); 1: Jameson
                            (dissip_jameson + sch_jameson, kprec = 0) */
  double ki2, ki4;       /* Jameson 2nd/4th-difference coefficients (ki2(lm),
                            ki4(lm); one value for every block) */
  int32_t ncychro;       /* the fused iteration number n (1, 2, ... since the
                            state was bound) recomputes the time step when
                            n mod ncychro = 1 or n < icychr0, and otherwise keeps
                            the previous one (atsch_num.f90:173-178, 436);
                            ncychro <= 1: every iteration */
  int32_t icychr0;
  int32_t kfmg;          /* 0: steady; 3: dual time stepping (smg_num.f90:110,
                            atsch_num.f90:993-1003) with physical step dt1min */
  int32_t kdualns;       /* dual time: 0 or 1 second order (sch_dual, sch_duup),
                            2 third order (sch_dual2, sch_duup2) */
  const double *eta_l;   /* [nblk] eta(lm) of each block, or NULL: eta for all */
  const double *ki2_l;   /* [nblk] ki2(lm), or NULL: ki2 for all */
  const double *ki4_l;   /* [nblk] ki4(lm), or NULL: ki4 for all */
  int32_t weno_fix;      /* non-reference option of ischema 12 (0 = reference):
                            every characteristic flux sums its three weighted
                            candidates; the reference sums only the first two
                            in the j and k directions and in the z flux of the
                            i direction, which no uniform flow survives */
} cns_scheme_t;

/* boundary lists (boundary module: mpb, mmb, ncbd, ncin, bceqt, ...) */
typedef struct {
  int32_t nbnd;
  const int32_t *type;    /* [nbnd] CNS_BC_* */
  const int32_t *blk;     /* [nbnd] owning block, 1-based */
  const int32_t *face;    /* [nbnd] 0..5 = i1,i2,j1,j2,k1,k2 */
  const int64_t *mpb;     /* [nbnd] first list entry */
  const int32_t *mmb;     /* [nbnd] entry count */
  const int32_t *partner; /* [nbnd] coincident partner boundary (0-based), -1 */
  const double *cosr;     /* [nbnd] cos of the boundary's periodic angle */
  const double *sinr;     /* [nbnd] sin of the boundary's periodic angle */
  int64_t nlist;
  const int64_t *ncbd;    /* [nlist] ghost cell (0-based flat index) */
  const int64_t *ncin;    /* [nlist] adjacent interior cell */
  const double *bceqt;    /* [5*nlist] column-major: idd rpi,rti,d0x,d0y,d0z;
                             prd p */
} cns_bnd_t;

/* device-resident arrays of the fast path (all device pointers, same layout
 * as above); the context never frees them */
typedef struct {
  double *v, *u, *d, *dt, *sn, *vol;
  double *pression, *ztemp, *cson, *mu, *mut, *tau;
  /* dual time stepping only (else NULL): (ld, 5) arrays ptdual, vdual,
     vdual1, vdual2 of smg_num.f90 */
  double *ptdual, *vdual, *vdual1, *vdual2;
} cns_state_t;

/* ---- context ---------------------------------------------------------- */
int cns_create(const cns_layout_t *layout, const cns_phys_t *phys,
               const cns_scheme_t *scheme, const cns_bnd_t *bnd,
               cns_ctx **out);
int cns_destroy(cns_ctx *ctx);
int cns_set_stream(cns_ctx *ctx, void *cuda_stream);
int cns_set_scheme(cns_ctx *ctx, const cns_scheme_t *scheme);
const char *cns_last_error(cns_ctx *ctx);
int64_t cns_scratch_bytes(cns_ctx *ctx);

/* chrono.f90:113-151, the global time step (kdtl = 0) after the per-block
 * cns_chronos calls: dt = min(dt1min, smallest real-cell dt) on every cell;
 * CNS_EDT when that is below dt1min (the reference stops).  The fused step
 * applies it itself when kdtl = 0. */
int cns_chrono_global(cns_ctx *ctx, double *dt);

/* Jameson scheme.  rfve.f90 (ghost = interior on every non-coincident
 * boundary) and rfvc.f90 (coincident ghosts = partner cells) refresh the
 * ghosts the dissipation reads; dissip_jameson.f90:4-431 zeroes d over the
 * block(s) and accumulates the scalar dissipation; sch_jameson.f90:4-437
 * zeroes u, accumulates the centred fluxes (tau used for NS) and finishes
 * with u = 0.5 u - d on the real cells.  l = 0: every block. */
int cns_rfve(cns_ctx *ctx, double *v, double *pression, double *ztemp, double *cson);
int cns_rfvc(cns_ctx *ctx, double *v, double *pression, double *ztemp, double *cson);
/* dissip_jameson.f90:4-8 (snu: the sensor work array, not used) */
int cns_dissip_jameson(cns_ctx *ctx, int lm, const double *v, double *d, const char *equat,
                       const double *sn, int64_t lgsnlt, double *snu, const double *ps,
                       const double *cson);
/* sch_jameson.f90:4-11 (fxx..fez: the flux-density work arrays, not used;
 * toxx..qcz read when equat(1:2) = 'ns') */
int cns_sch_jameson(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v,
                    const double *d, double *ff, const double *toxx, const double *toxy,
                    const double *toxz, const double *toyy, const double *toyz,
                    const double *tozz, const double *qcx, const double *qcy,
                    const double *qcz, const char *equat, const double *sn, int64_t lgsnlt,
                    double *fxx, double *fyy, double *fzz, double *fxy, double *fxz,
                    double *fyz, double *fex, double *fey, double *fez, const double *ps);

/* Turbulence-transport terms on the mean-flow path.  cns_set_turbulence
 * sets the modeleturb / schemanum constants these routines read (alfak,
 * alfae: k-epsilon diffusion numbers; sigma: Spalart-Allmaras; epsroe:
 * Harten's parameter; defaults 1, 1.3, 2/3, 0).  t, s and d are the
 * reference's (ld, 7) arrays; fd* are per cell (ip12).
 *   cns_met_fludc   met_fludc.f90:4-87   fd5* *= mu + mut/alfak, fd6* *= mu + mut/alfae
 *   cns_met_fludcsa met_fludcsa.f90:4-106 fd5* *= (mu + s(:,6))/sigma, fd6* = 0
 *   cns_met_roe2o   met_roe2o.f90:4-297  TVD Roe dissipation of t(:,6:7) -> d(:,6:7)
 *   cns_met_roe2oh  met_roe2oh.f90        the same with Harten's entropy fix
 * l = 0: every block. */
int cns_set_turbulence(cns_ctx *ctx, double alfak, double alfae, double sigma, double epsroe);
/* met_fludc.f90:4-8 (s, t, dtdx, dtdy, dtdz: in its argument list, not read) */
int cns_met_fludc(cns_ctx *ctx, int l, const double *s, const double *mu, const double *mut,
                  const double *t, const double *dtdx, const double *dtdy,
                  const double *dtdz, double *fd5x, double *fd5y, double *fd5z,
                  double *fd6x, double *fd6y, double *fd6z);
/* met_fludcsa.f90:4-7 */
int cns_met_fludcsa(cns_ctx *ctx, int l, const double *s, const double *mu, double *fd5x,
                    double *fd5y, double *fd5z, double *fd6x, double *fd6y, double *fd6z);
/* met_roe2o.f90:4-7, met_roe2oh.f90:4-7 (vol, del6, del7: work, not used) */
int cns_met_roe2o(cns_ctx *ctx, int l, const double *t, double *d, const double *sn,
                  int64_t lgsnlt, const double *vol, double *del6, double *del7);
int cns_met_roe2oh(cns_ctx *ctx, int l, const double *t, double *d, const double *sn,
                   int64_t lgsnlt, const double *vol, double *del6, double *del7);
/* Spalart-Allmaras (constants of atlecdon.f90:193-204):
 *   cns_met_samut  met_samut.f90:4-58   mut = v(:,6) fv1 on the real cells
 *   cns_sch_turb   sch_turb.f90:4-290   centred fluxes of v(:,6:7) with the
 *                  diffusion densities fd5*, fd6*, then
 *                  u6 = 0.5 u6 - vol ts6 - d6 (and 7); u(:,6:7) zeroed over
 *                  the block(s) first; no wall-law branch (kparoi = 0) */
int cns_met_samut(cns_ctx *ctx, int l, const double *v, const double *mu, double *mut);
/*   cns_teq_gradv  teq_gradv.f90:4-170  dv (9 x ld: xx xy xz yx yy yz zx zy
 *                  zz) = Green-Gauss gradients of u, v, w on the real cells
 *                  (teq_grads.f90, unit weights)
 *   cns_met_smsa   met_smsa.f90:4-186 with met_difsa.f90: ts6 (qcxts5) =
 *                  the SA source, ts7 (qcyts6) = 0, cfke = |d source| on the
 *                  real cells, from dv, the diffusion densities fd5* and the
 *                  wall distance dist */
int cns_teq_gradv(cns_ctx *ctx, int l, const double *v, const double *sn, const double *vol,
                  double *dv);
/*   cns_impli2_eqt_3d  impli2_eqt_3d.f90:4-330 (no wall law): implicit phase
 *                  of the transport equations, two alternating-line sweeps
 *                  (tridiagonal solves) per direction i, j, k; v(:,6:7) += dw
 *                  on the real cells; cmt = the model's constant (1 for 1SA) */
int cns_impli2_eqt_3d(cns_ctx *ctx, int l, const double *u, const double *dt, double *v,
                      const double *mu, const double *mut, const double *cfke,
                      const double *sn, const double *vol, double cmt);
int cns_met_smsa(cns_ctx *ctx, int l, const double *v, const double *mu, const double *dist,
                 const double *sn, const double *vol, const double *dv, const double *fd5x,
                 const double *fd5y, const double *fd5z, double *ts6, double *ts7,
                 double *cfke);
int cns_sch_turb(cns_ctx *ctx, int l, double *u, const double *v, const double *d,
                 const double *fd5x, const double *fd5y, const double *fd5z,
                 const double *fd6x, const double *fd6y, const double *fd6z,
                 const double *ts6, const double *ts7, const double *sn, const double *vol);

/* The rest of the Spalart-Allmaras transport step (met_num.f90 for equat
 * '1SA ': kcutke 2, kfludis 2, ksecmb 2, kcmut 2, kditur 2, klroe 2 with
 * met_roe2oh when |epsroe| > tiny, kparoi 0), bit-exact in FP64:
 *   cns_atcaldis3   atcaldis3.f90 with the default attachment of every block
 *                   to every wall (atdist_3.f90:34-58): dist = the distance
 *                   from each real cell centre (atccc.f90) to the nearest
 *                   facet centre (atccfp.f90) of the adiabatic-wall ('para')
 *                   boundaries; x, y, z are the node coordinates in the cell
 *                   index space; CNS_EBC when there is no wall
 *   cns_met_bord    met_bord.f90:24-258 on v(:,6:7): coincident ghosts =
 *                   average with the partner cell (met_rbvc), injection =
 *                   (rokinf, roeinf), wall = 0, others = interior cell
 *   cns_met_gradtr  met_gradtr.f90:48-130: fd5* = grad(s6/s1), fd6* =
 *                   grad(s7/s1) (teq_grads) over the flat real-cell range
 *   cns_met_rbse    met_rbse.f90 + met_rbsc.f90: ghost diffusion densities
 *   cns_met_cutsa   met_cutsa.f90:35-48: s6 < 0 -> epsk, s7 = 0
 * cns_set_sa enables the whole step in the fused iteration (after rbord,
 * before zvisqc, as atsch_num.f90:541-559 calls met_num; the bound v, u, d
 * must then have 7 columns); cns_met_num runs it once on the bound state.
 * NULL disables it. */
typedef struct {
  const double *dist;    /* wall distance of the real cells (device, ip12) */
  double rokinf, roeinf; /* v(:,6), v(:,7) of the injection ghosts */
  double epsk;           /* met_cutsa floor of v(:,6) */
  int32_t stilde_fix;    /* non-reference option (0 = reference): met_smsa with the
                            modified vorticity of Allmaras, Johnson & Spalart
                            2012 (S~ >= 0.3 vort) and its derivative zero where
                            r is clipped.  The reference's S~ can reach zero,
                            where its source bound cfke becomes inf or NaN.
                            cns_met_smsa follows it too while set */
} cns_sa_t;
int cns_atcaldis3(cns_ctx *ctx, const double *x, const double *y, const double *z,
                  double *dist);
int cns_met_bord(cns_ctx *ctx, double *v, double rokinf, double roeinf);
int cns_met_gradtr(cns_ctx *ctx, int l, const double *s, const double *sn, const double *vol,
                   double *fd5x, double *fd5y, double *fd5z, double *fd6x, double *fd6y,
                   double *fd6z);
int cns_met_rbse(cns_ctx *ctx, double *fd5x, double *fd5y, double *fd5z, double *fd6x,
                 double *fd6y, double *fd6z);
int cns_met_cutsa(cns_ctx *ctx, int l, double *v, double epsk);
/* Wall law of the adiabatic wall-law walls (CNS_BC_LP2; air, no transition;
 * vkar 0.41, cllog 5.25, yp0 11.13 as rbord.f90:377-379 sets them).  Both
 * take the friction law of lpsa1.f90:111-160 / lparoi1.f90:111-160: the
 * first cell's tangential velocity, the Crocco wall temperature, Sutherland's
 * wall viscosity, Van Driest's transform, and the wall stress of the linear
 * law (rho u y / mu <= yp0^2) or ten passes of the log law.  Device arrays.
 *   cns_lpsa       lpsa.f90 -> lpsa1.f90 on the 'lp2' walls of block l in
 *                  boundary order: mut of the first cell from the mixing
 *                  length, rho nu~ there from mut = rho nu~ fv1 (floored at
 *                  the context's epsk, cns_sa_t), rho nu~ = 0 in the ghost;
 *                  v is (ld, 7)
 *   cns_cllparoi1  cllparoi1.f90 -> lparoi1.f90 on every 'lp2' wall: the
 *                  wall stress tensor in the ghost and the first cell, the
 *                  first cell's heat flux, none in the ghost; tau (ld, 9) as
 *                  cns_zvisqc writes it */
int cns_lpsa(cns_ctx *ctx, int l, double *v, const double *mu, double *mut, const double *dist,
             const double *ztemp);
int cns_cllparoi1(cns_ctx *ctx, const double *v, const double *dist, const double *mu,
                  const double *mut, double *tau, const double *ztemp);
int cns_set_sa(cns_ctx *ctx, const cns_sa_t *sa);
/* The k-epsilon transport step of Jones & Launder (met_num.f90 for equat
 * '2JL ': kcutke 1, kfludis 1, ksecmb 1, kcmut 1, kparoi 0, kesst 0; cke1
 * 1.55, cke2 2, cmu 0.09, atlecdon.f90:113-128; met_fludc with the alfak,
 * alfae of cns_set_turbulence; no wall law), bit-exact in FP64:
 *   cns_met_prod   met_prod.f90:41-66: tprod = the production of k from the
 *                  velocity gradients dv (9 x ld, cns_teq_gradv) and mut
 *   cns_met_smke   met_smke.f90:93-118: met_exgr on dv's ghosts (in place),
 *                  met_bark (-2 mu |grad sqrt(k)|^2), met_bare (2 mut mu /
 *                  rho times the squared gradients of dv), met_smkes:
 *                  qcxts5, qcyts6 = the sources of k and epsilon, cfke the
 *                  bound of their derivative, on the real cells
 *   cns_met_kemut  met_kemut.f90:52-65: mut = exp(-2.5 / (1 + Re_t / 50))
 *                  cmu rho k^2 / eps
 *   cns_met_cutke  met_cutke.f90:43-60: k < epsk or eps < epse resets both
 *                  (i = 1..ni: the upper i ghost too)
 * Arrays are device arrays with the global cell index (dv, tprod, cfke:
 * 9 ld, ld, ld).  cns_set_ke enables the whole step in the fused iteration
 * (after rbord, as cns_set_sa does; v, u, d with 7 columns) and disables the
 * Spalart-Allmaras one; NULL disables it.  cns_met_num runs the enabled
 * step once on the bound state. */
typedef struct {
  double rokinf, roeinf; /* v(:,6), v(:,7) of the injection ghosts */
  double epsk, epse;     /* met_cutke floors of v(:,6), v(:,7) */
} cns_ke_t;
int cns_set_ke(cns_ctx *ctx, const cns_ke_t *ke);
int cns_met_prod(cns_ctx *ctx, int l, int ncyc, const double *mut, const double *s,
                 const double *dv, double *tprod);
int cns_met_smke(cns_ctx *ctx, int l, const double *sn, const double *vol, const double *v,
                 const double *mu, const double *mut, const double *tprod, double *cfke,
                 double *dv, double *qcxts5, double *qcyts6);
int cns_met_kemut(cns_ctx *ctx, int l, const double *v, const double *mu, double *mut);
int cns_met_cutke(cns_ctx *ctx, int l, double *v, double epsk, double epse);
/* The first cycle's turbulence initialisation (atsch_num.f90:256-345), on
 * the real cells of block l (device arrays):
 *   cns_met_inisa  met_inisa.f90:36-44: v(:,6) = mut (Spalart-Allmaras)
 *   cns_met_inmut  met_inmut.f90: mut = mu / 10 (keinit = 2)
 *   cns_met_ini    met_ini.f90 (k-epsilon, kinke = 1): teq_gradv into dv
 *                  (9 x ld), then met_brad.f90:37-51: v(:,6) = mut |omega| /
 *                  sqrt(cmu), v(:,7) = mut |omega|^2 */
int cns_met_inisa(cns_ctx *ctx, int l, double *v, const double *mut, const double *mu);
int cns_met_inmut(cns_ctx *ctx, int l, const double *mu, double *mut);
int cns_met_ini(cns_ctx *ctx, int l, double *v, const double *mut, const double *mu,
                const double *sn, const double *vol, double *dv);
int cns_met_num(cns_ctx *ctx);

/* Discrete adjoint of the FP64 Euler Roe iteration (sch_roe_euler with
 * unlimited MUSCL + implimf_eu with qfix_dfez = 1) at the bound state, for a
 * caller that solves A^T lambda = dJ/dW (no counterpart in the reference).
 *   cns_adjoint_prepare  recomputes the iteration's inputs at the state
 *                        (zpres, chronos, rbord, coefficients) and stores
 *                        the exact face-flux Jacobians and the linearised
 *                        Jacobi-update blocks (forward-mode dual numbers);
 *   cns_adjoint_rt       wbar (6 x ld) = A^T lam for every cell of i 0..ni,
 *                        j 0..nj, k 0..nk, split into the conserved-variable
 *                        part (rows 0-4) and the pressure part (row 5; the
 *                        residual reads the pressure array), and, when sbar
 *                        is given, sbar (3 dirs x 3 x ld) = lam^T du/dS per
 *                        face (at the face's cell index); lam is zero on
 *                        ghost cells;
 *   cns_adjoint_lt       out = L^T y, L the primal's implicit phase
 *                        linearised at d = 0 (lmax sweeps). */
int cns_adjoint_prepare(cns_ctx *ctx);
int cns_adjoint_rt(cns_ctx *ctx, const double *lam, double *wbar, double *sbar);
int cns_adjoint_lt(cns_ctx *ctx, const double *y, double *out);

/* kernels launched by the fused-step graphs of this context so far (the
 * kernel nodes of each captured iteration times its launches) */
int64_t cns_kernels_launched(cns_ctx *ctx);

/* ---- set-up ------------------------------------------------------------ */
/* metric.f90 -> metrics.f90: ghost nodes (extmhg), sn (norm), vol (svol),
 * coincident ghost volumes (rfsc) and the boundary-entry geometry (initns,
 * clidd ghost centres) kept in the context.  x, y, z: node coordinates,
 * ghost nodes overwritten. */
int cns_metric(cns_ctx *ctx, double *x, double *y, double *z, double *sn,
               double *vol);
/* copy the boundary-entry geometry to host arrays of nlist doubles */
int cns_boundary_geom(cns_ctx *ctx, double *nxn, double *nyn, double *nzn,
                      double *ym, double *zm);

/* ---- per-routine entry points (l = 1..nblk; l = 0: every block) ---------- */
/* zpres.f90:4-101 */
int cns_zpres(cns_ctx *ctx, int l, const double *v, double *pression,
              double *ztemp, double *cson);
/* zvismo.f90:4-136 (iflu = 1) */
int cns_zvismo(cns_ctx *ctx, int l, double *mu, const double *v,
               const double *ztemp);
/* chronos.f90:4-11 (kprec = 0): local time step of block l with the CFL
 * number etal; the viscous limit when equat(1:2) = 'ns'; sfsi, sfsj, sfsk,
 * dism: work arrays, not used */
int cns_chronos(cns_ctx *ctx, int l, double etal, const double *mu, const double *mut,
                const double *t, double *dt, const char *equat, const double *sn,
                int64_t lgsnlt, const double *vol, double *sfsi, double *sfsj,
                double *sfsk, double *dism, const double *cson);
/* rbord.f90:4-433 restricted to extr, rc, para, idd, prd */
int cns_rbord(cns_ctx *ctx, double *v, double *pression, double *ztemp,
              double *cson);
/* sch_roe_euler.f90:4-10 (rhol..prr: the reconstructed-state work arrays,
 * not used) */
int cns_sch_roe_euler(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v,
                      double *ff, const char *equat, const double *sn, int64_t lgsnlt,
                      double *rhol, double *ul, double *vl, double *wl, double *pl,
                      double *rhor, double *ur, double *vr, double *wr, double *prr,
                      const double *ps);
/* sch_roe.f90:4-11 (toxx..qcz: the stresses and heat fluxes of zvisqc, nine
 * arrays of ip12; used in place when they are the columns of one (ld, 9)
 * array) */
int cns_sch_roe(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v, double *ff,
                const double *toxx, const double *toxy, const double *toxz,
                const double *toyy, const double *toyz, const double *tozz,
                const double *qcx, const double *qcy, const double *qcz, const char *equat,
                const double *sn, int64_t lgsnlt, double *rhol, double *ul, double *vl,
                double *wl, double *pl, double *rhor, double *ur, double *vr, double *wr,
                double *prr, const double *ps);
/* zvisqc.f90:4-210: zgrad2 + zfluto on every block, then rbte/rbtc */
/* other flux families (atsch_num.f90:628-983), selected in the fused
 * iteration by cns_scheme_t.ischema: 14 = HLLC (sch_hllc_euler.f90:4-891,
 * sch_hllc.f90:4-1403, with the minmod limiter of ilim = 1 in the NS form),
 * 9 = Rusanov (sch_rusanov.f90:4-791: plain MUSCL, the stresses tau enter
 * whatever the equations -- zero for Euler); the argument lists of
 * sch_hllc_euler.f90:4-10, sch_hllc.f90:4-11, sch_rusanov.f90:4-11 */
int cns_sch_hllc_euler(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v,
                       double *ff, const char *equat, const double *sn, int64_t lgsnlt,
                       double *rhol, double *ul, double *vl, double *wl, double *pl,
                       double *rhor, double *ur, double *vr, double *wr, double *prr,
                       const double *ps);
int cns_sch_hllc(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v, double *ff,
                 const double *toxx, const double *toxy, const double *toxz,
                 const double *toyy, const double *toyz, const double *tozz,
                 const double *qcx, const double *qcy, const double *qcz, const char *equat,
                 const double *sn, int64_t lgsnlt, double *rhol, double *ul, double *vl,
                 double *wl, double *pl, double *rhor, double *ur, double *vr, double *wr,
                 double *prr, const double *ps);
int cns_sch_rusanov(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v,
                    double *ff, const double *toxx, const double *toxy, const double *toxz,
                    const double *toyy, const double *toyz, const double *tozz,
                    const double *qcx, const double *qcy, const double *qcz,
                    const char *equat, const double *sn, int64_t lgsnlt, double *rhol,
                    double *ul, double *vl, double *wl, double *pl, double *rhor, double *ur,
                    double *vr, double *wr, double *prr, const double *ps);
/* ischema 12 = WENO5 (sch_weno5_3d.f90:4-12, the 'xx3d' form of
 * atsch_num.f90:898-919): Jiang & Shu's fifth-order reconstruction of the
 * characteristic fluxes on Roe-averaged eigenvectors, upwinded by the sign
 * of each eigenvalue, Henrick's mapped weights; the stresses tau enter
 * whatever the equations (zero for Euler), a boundary face takes the flux of
 * its ghost cell.  Near a block face the stencil reads the spare slots of
 * the cell arrays (i = ni + 1, j = nj + 1, k = nk + 1) as the reference
 * does; at the first interior k face its point k = -1 lies before the block,
 * where the reference reads out of bounds, and this build reads the ghost
 * plane k = 0 there.  fxx..fez: the reference's flux work arrays, not used */
int cns_sch_weno5_3d(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v, double *ff,
                     const double *toxx, const double *toxy, const double *toxz,
                     const double *toyy, const double *toyz, const double *tozz,
                     const double *qcx, const double *qcy, const double *qcz,
                     const char *equat, const double *sn, int64_t lgsnlt, double *fxx,
                     double *fyy, double *fzz, double *fxy, double *fxz, double *fyz,
                     double *fex, double *fey, double *fez, const double *ps);
/* ischema 5 = AUSM+ (sch_ausmp.f90:4-11; the reference runs it for the
 * Navier-Stokes equations only: with the minmod limiter of ilim = 1, the
 * work and heat-flux terms of sch_ausmp.f90:81-83 from tau on the fly; d is
 * in its argument list and not read) */
int cns_sch_ausmp(cns_ctx *ctx, int lm, int ityprk, double *u, const double *v, double *d,
                  double *ff, const double *toxx, const double *toxy, const double *toxz,
                  const double *toyy, const double *toyz, const double *tozz,
                  const double *qcx, const double *qcy, const double *qcz,
                  const char *equat, const double *sn, int64_t lgsnlt, double *rhol,
                  double *ul, double *vl, double *wl, double *pl, double *rhor, double *ur,
                  double *vr, double *wr, double *prr, const double *ps);
int cns_zvisqc(cns_ctx *ctx, const double *v, const double *mu,
               const double *mut, double *tau, const double *sn,
               const double *vol, const double *ztemp);
/* implimf_eu.f90:6-12: lmx point-Jacobi sweeps and v += d on block lm;
 * dtpas: the physical step of the dual-time diagonal (used when the
 * scheme's kfmg = 3); dfxx..dfez, coefdiag: work arrays, not used (the
 * increments are recomputed in the sweeps) */
int cns_implimf_eu(cns_ctx *ctx, int lm, const double *u, const double *dt, double *v,
                   double *d, const double *ff, const char *equat, int lmx,
                   const double *sn, int64_t lgsnlt, const double *vol, double dtpas,
                   int ityprk, double *dfxx, double *dfyy, double *dfzz, double *dfxy,
                   double *dfxz, double *dfyz, double *dfex, double *dfey, double *dfez,
                   double *coefdiag, const double *ps, const double *cson);
/* implimf_3d.f90:4-11 (dfxx..dfez, rv: work arrays, not used) */
int cns_implimf_3d(cns_ctx *ctx, int lm, const double *u, const double *dt, double *v,
                   double *d, const double *ff, const double *mu, const double *mut,
                   const char *equat, int lmx, const double *sn, int64_t lgsnlt,
                   const double *vol, double dtpas, int ityprk, double *dfxx,
                   double *dfyy, double *dfzz, double *dfxy, double *dfxz, double *dfyz,
                   double *dfex, double *dfey, double *dfez, double *rv, const double *ps,
                   const double *cson);
/* rscpsv.f90 + residu.f90: L1, L2, Linf of (v-u0)/dt over all blocks;
 * norms: host array of 15 doubles (L1[5], L2[5], Linf[5]) */
int cns_rscpsv(cns_ctx *ctx, const double *u0, const double *v,
               const double *dt, double *norms);

/* ---- fast path ---------------------------------------------------------- */
int cns_bind_state(cns_ctx *ctx, const cns_state_t *state);
/* nsteps pseudo-time iterations of atsch_num.f90 (Roe, implicit) on the bound
 * state; the step sequence is captured once in a CUDA graph and replayed.
 * norms (host, may be NULL): 15 doubles of the LAST step. */
int cns_atsch_num_step(cns_ctx *ctx, int nsteps, double *norms);
/* enqueue nsteps iterations without waiting (stream-ordered); the norms of
 * the last enqueued iteration are read back by cns_last_norms, which waits
 * for the stream and checks the device status word */
int cns_atsch_num_launch(cns_ctx *ctx, int nsteps);
int cns_last_norms(cns_ctx *ctx, double *norms);

/* Iteration counters of the fused step: the reference's ncyc (global) and
 * icyc (within the current run or physical step) of the LAST iteration done;
 * each fused iteration advances both before use.  They select the time-step
 * updates (ncychro, icychr0) and the Jameson first cycle (ncyc = 1).
 * cns_bind_state sets both to 0. */
int cns_set_cycle(cns_ctx *ctx, int64_t ncyc, int64_t icyc);

/* Dual time stepping (kfmg = 3).  cns_sch_duin: the start of the physical
 * time loop on the bound state (vdual = vdual1 = vdual2 = v as utinia.f90:
 * 140-160 / readda.f90:150-176 set them, then sch_duin.f90: ptdual = -vdual);
 * cns_set_dual_cycle: the physical step index icycle the fused step's
 * sch_dual uses (fact = 1 for icycle <= 1); cns_sch_duup: the end of a
 * physical step (sch_duup.f90 or sch_duup2.f90 by kdualns) on the bound
 * state; cns_sch_dual: sch_dual.f90 / sch_dual2.f90 on block l with the
 * caller's arrays.  The Spalart-Allmaras step and the adjoint do not run
 * with dual time stepping (CNS_EINVAL). */
int cns_sch_duin(cns_ctx *ctx);
int cns_sch_duup(cns_ctx *ctx);
int cns_set_dual_cycle(cns_ctx *ctx, int icycle);
int cns_sch_dual(cns_ctx *ctx, int l, double *u, const double *v, int icycle,
                 const double *vol, const double *ptdual);

/* Jacobi sweep tiling (no counterpart in the reference).  Every sweep after
 * the first runs 2.5D-blocked over patches of ti x tj cell columns, kc
 * planes deep.  The first fused iteration of each precision tunes the tiling
 * on its own data (no result depends on it: the FP32 sweeps round every
 * operation explicitly).  cns_sweep_tiles returns {ti, tj, kc, source} of
 * precision 0 (FP64) or 1/2 (FP32 sweeps), source 0 = the default or a tiling
 * set by cns_set_sweep_tiles, 1 = timed on the data, 2 = read from the tuning
 * cache; cns_set_sweep_tiles fixes a tiling (ti x tj one of 32x4, 32x8, 16x8,
 * 16x16; kc >= 1).  cns_set_tune_cache names a text file of tuned tilings,
 * one line "key ti tj kc" per (GPU name, SM count, sweep precision,
 * equations, log2 real cells, log2 blocks, log2 cells of the smallest block):
 * a configuration found there is used without timing (the same tiling on
 * every run with that file), a new one is timed and appended; NULL or ""
 * turns the cache off. */
int cns_sweep_tiles(cns_ctx *ctx, int precision, int32_t *cfg);
int cns_set_sweep_tiles(cns_ctx *ctx, int precision, int ti, int tj, int kc);
int cns_set_tune_cache(cns_ctx *ctx, const char *path);
/* How the FP32 sweeps (precision 1 and 2) stage each plane of a patch in
 * shared memory (no counterpart in the reference): mode 0 (the default)
 * copies it as tensor boxes (cp.async.bulk.tensor, one per array and plane,
 * completing on an mbarrier; a wait that gives up after about two seconds
 * makes the next status check return CNS_ECUDA), mode 1 with per-thread
 * cp.async element copies.  Both give the same bits. */
int cns_set_sweep_staging(cns_ctx *ctx, int mode);
int cns_sweep_staging(cns_ctx *ctx, int32_t *mode);
/* Residual kernel variant (no counterpart in the reference): ti = 0 selects
 * the face kernels (one launch per direction into a face buffer, then the
 * per-cell accumulation); ti x tj = 32 x 4 or 16 x 8 selects the fused kernel
 * (all three directions and the accumulation in one launch over 2.5D tiles
 * of kc planes).  Both give the same bits in FP64.  cns_residual_tiles
 * returns {ti, tj, kc} (zeros for the face kernels). */
int cns_set_residual_tiles(cns_ctx *ctx, int ti, int tj, int kc);
int cns_residual_tiles(cns_ctx *ctx, int32_t *cfg);
/* drop-in call with host arrays: copies the real+ghost state v (host, ld x 5)
 * in, runs nsteps iterations, copies v back and returns the last norms */
int cns_atsch_num_step_host(cns_ctx *ctx, double *v_host, int nsteps,
                            double *norms);

/* ---- reference grid and flow files ------------------------------------ */
/* The reference's Fortran unformatted sequential files (solve.f90:401-404),
 * every block in block order, each record one array over a block's (i, j, k)
 * box, i fastest, with gfortran's 4-byte record markers in the machine's
 * byte order (a record longer than 2147483639 bytes split into subrecords
 * with negated markers).  Arrays are device arrays in the layout above; the
 * calls return when the file is complete.  A read modifies nothing unless the
 * whole file matches the layout (else CNS_EFORMAT, or CNS_EIO when it cannot
 * be opened), where the reference stops.
 *
 * cns_readdg: fgv, x, y, z at the real nodes of every block (ingr.f90:49 ->
 *   readdg.f90:71-80).
 * cns_writdg: svgr.f90 (chdgcv.f90 -> writdg.f90:46-48) for every block; disc
 *   "cvcv" = the real nodes (fgv), "cvcc" = the real cell centres (fgc),
 *   "cvcf" = the cell centres with the ghost layer (fgcf); a centre is .125
 *   times the sum of the cell's 8 nodes (cvccg.f90), ghost nodes included.
 * cns_readda: fac (infw.f90:64 -> readda.f90:88-128): v(:,1..5) at the real
 *   cells, mut when equat(1:2) = 'ns', and with equat(6:7) = 'ke' v(:,6),
 *   v(:,7) (v is (ld, 7)) when keinit = 0, else those two are zeroed.  The
 *   utau records of kutau = 1 models and the dual-time copies of kfmg = 3 are
 *   not handled.
 * cns_writda: svfw.f90 (chdacc.f90 -> writda.f90:78-97) for every block; disc
 *   "cccc" = the real cells (fac), "cccf" = the cells with the ghost layer
 *   (facf); the node-averaged "cccv" is not handled.
 * cns_set_subrecord_length: the largest subrecord the writers produce
 *   (gfortran's -fmax-subrecord-length; default and maximum 2147483639). */
int cns_set_subrecord_length(cns_ctx *ctx, int64_t bytes);
int cns_readdg(cns_ctx *ctx, const char *path, double *x, double *y, double *z);
int cns_writdg(cns_ctx *ctx, const char *path, const char *disc, const double *x,
               const double *y, const double *z);
int cns_readda(cns_ctx *ctx, const char *path, const char *equat, int keinit,
               double *v, double *mut);
int cns_writda(cns_ctx *ctx, const char *path, const char *disc, const char *equat,
               const double *v, const double *mut);

/* ---- no-allocation variant -------------------------------------------- */
/* No counterpart in the reference.  The Euler Roe residual of ONE block
 * (what cns_sch_roe_euler(ctx, 1, ...) computes for a layout of a single
 * block starting at offset 0), for callers that cannot let the library
 * allocate device memory -- a driver that owns every device array in its own
 * pre-sized pool or runs under a hard memory cap.  Needs no context: the
 * intermediates live in a 20 MiB static device array that every GPU loading
 * the library holds until exit, which limits ld to 131072 (larger calls
 * return CNS_EINVAL and launch nothing).  The first call on a device looks up
 * that array's address; make it before any stream capture.  Calls share the
 * array: calls that overlap on the GPU race, so order them on one stream.
 * ni, nj, nk: real node counts; ld: leading dimension of u, v; gam, pinfl,
 * muscl, xk: as in cns_phys_t / cns_scheme_t; u, v, sn, ps: device arrays;
 * stream: CUDA stream (NULL = legacy default stream). */
int cns_sch_roe_euler_noalloc(int32_t ni, int32_t nj, int32_t nk, int64_t ld,
                              double gam, double pinfl, int32_t muscl,
                              double xk, double *u, const double *v,
                              const double *sn, const double *ps,
                              void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CNS_ABI_H */
