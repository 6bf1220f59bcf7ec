/*
 * cns_oracle.h -- CPU oracle (test infrastructure only).
 *
 * A plain-C restatement of the CodeNS per-iteration hot path, used by the
 * test-suite and by bench.py's CPU-baseline leg as the checker for the CUDA
 * product.  It is NOT part of the product: nothing in codens_b200/ links,
 * loads or calls it.
 *
 * Parity status: UNPINNED.  The reference is Fortran 90 with no tests, golden
 * vectors or sample decks, and no Fortran compiler exists in this image, so
 * the restatement cannot be checked against reference outputs.  It is pinned
 * instead by line-by-line review against the cited reference lines and by the
 * analytic invariants exercised in tests/ (freestream preservation, Roe
 * consistency F(W,W)=F(W).S, telescoping conservation, Jacobi fixed point).
 *
 * Conventions (mirroring the reference's Fortran module globals):
 *   - blocks are numbered l = 1..nblk;
 *   - node and cell arrays share one flat index space; block l starts at the
 *     0-based offset npc(l) (crdms.f90:150-157);
 *   - within a block, cell (i,j,k) with Fortran index values i=0..ni+1
 *     (ghost layer nfi=1, id1=0) sits at npc + i + j*nid + k*nid*njd
 *     (sch_roe.f90:1487-1491 with 0-based storage);
 *   - v/u/d are column-major (ld, ncol) arrays: v[c*ld + n];
 *   - the normals of block l occupy sn[9*npc(l) ...] viewed as
 *     sn(nnn, 3 face directions, 3 components) (atsch_num.f90:470-479).
 * Arithmetic follows the reference expressions left to right with all
 * literals in double precision (CMake build, -fdefault-real-8) and no FMA
 * contraction (built with -ffp-contract=off).
 */
#ifndef CNS_ORACLE_H
#define CNS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* boundary condition kinds (rbord.f90:144-424); ORC_BC_LP2: the adiabatic
 * wall with the wall law ('lp2') */
enum { ORC_BC_EXTR = 1, ORC_BC_RC = 2, ORC_BC_PARA = 3, ORC_BC_IDD = 4,
       ORC_BC_PRD = 5, ORC_BC_LP2 = 6 };

int  orc_setup(int nblk, const int32_t *dims /* 3*nblk: ni,nj,nk nodes */, int64_t ld);
int64_t orc_npc(int l);
int64_t orc_ncells(void);

void orc_set_phys(double gam, double pinfl, double pr, double prt,
                  double reynz, double suth_a, double pa1, double aa1,
                  double omg);
/* qfix_dfez: non-reference option restoring the *wi factor missing from
 * implimf_eu.f90:312 (0 keeps the reference behaviour) */
void orc_set_scheme(int ns, int muscl, double xk, int ilim, double eta,
                    int kdtl, double dt1min, int lmax, int qfix_dfez);

/* boundaries: per boundary b: type, block (1-based), face (0..5 = i1,i2,j1,j2,
 * k1,k2), first list entry mpb and count mmb, partner boundary (RC) and the
 * boundary's own periodic rotation (cos, sin).  Per list entry: ghost cell
 * ncbd, interior cell ncin (0-based global) and bc values (nlist x 5, column
 * major: idd rpi,rti,d0x,d0y,d0z; prd p). */
int orc_set_boundaries(int nbnd, const int32_t *type, const int32_t *blk,
                       const int32_t *face, const int64_t *mpb,
                       const int32_t *mmb, const int32_t *partner,
                       const double *cosr, const double *sinr,
                       int64_t nlist, const int64_t *ncbd, const int64_t *ncin,
                       const double *bceqt);

/* geometry (metrics.f90, extmhg.f90, norm.f90, svol.f90, rfsc.f90) and the
 * boundary-entry geometry: inward unit normals (initns.f90) and ghost-cell
 * centres (clidd.f90:64-71), stored internally and returned by
 * orc_boundary_geom */
void orc_metric(double *x, double *y, double *z, double *sn, double *vol);
void orc_boundary_geom(double *nxn, double *nyn, double *nzn, double *ym,
                       double *zm);

/* per-block kernels (l = 1..nblk) */
void orc_zpres(int l, const double *v, double *ps, double *temp, double *cson);
void orc_zvismo(int l, double *mu, const double *temp);
void orc_chronos(int l, const double *mu, const double *mut, const double *v,
                 double *dt, const double *sn, const double *vol,
                 const double *cson);
void orc_chrono_global(double *dt);
void orc_rbord(double *v, double *ps, double *temp, double *cson);
void orc_sch_roe_euler(int l, double *u, const double *v, const double *sn,
                       const double *ps);
void orc_zvisqc(const double *v, const double *mu, const double *mut,
                double *tau /* 9 x ld: toxx,toxy,toxz,toyy,toyz,tozz,qcx,qcy,qcz */,
                const double *sn, const double *vol, const double *temp);
void orc_sch_roe(int l, double *u, const double *v, const double *tau,
                 const double *sn, const double *ps);
void orc_implimf_eu(int l, const double *u, const double *dt, double *v,
                    double *d, const double *sn, const double *vol,
                    const double *ps, const double *cson, int lmx);
void orc_implimf_3d(int l, const double *u, const double *dt, double *v,
                    double *d, const double *mu, const double *mut,
                    const double *sn, const double *vol, const double *ps,
                    const double *cson, int lmx);
/* residual norms (residu.f90, rscpsv.f90): out[0..4]=L1, [5..9]=L2,
 * [10..14]=Linf over all blocks */
void orc_rscpsv(const double *u0, const double *v, const double *dt,
                double *out);

/* one pseudo-time iteration over all blocks (atsch_num.f90:245-1134 for the
 * ischema=7, kmf=1 Roe/implicit path); work holds ld*(9+5) doubles for
 * ps,temp,cson,mu,mut,dt,...; returns 0 */
/* threads of the per-block loops of an iteration (OpenMP) */
void orc_set_threads(int n);

/* Jameson scheme: ischema 1, ki2/ki4 of every block (schemanum) */
void orc_set_dissipation(int ischema, double ki2, double ki4);
void orc_rfve(double *v, double *ps, double *temp, double *cson);
void orc_rfvc(double *v, double *ps, double *temp, double *cson);
void orc_dissip_jameson(int l, const double *v, double *d, const double *sn,
                        const double *ps, const double *cson);
void orc_sch_jameson(int l, double *u, const double *v, const double *d,
                     const double *tau, const double *sn, const double *ps);
int orc_step_jameson(double *v, double *u, double *d, double *dis, double *dt,
                     const double *sn, const double *vol, double *ps, double *temp,
                     double *cson, double *mu, double *mut, double *tau, int first_cycle);

/* turbulence transport terms: met_fludc, met_fludcsa, met_roe2o(h); t, s, d
 * are (ld, 7) */
void orc_met_fludc(int l, const double *mu, const double *mut, double *fd5x, double *fd5y,
                   double *fd5z, double *fd6x, double *fd6y, double *fd6z, double alfak,
                   double alfae);
void orc_met_fludcsa(int l, const double *s, const double *mu, double *fd5x, double *fd5y,
                     double *fd5z, double *fd6x, double *fd6y, double *fd6z, double sigma);
void orc_met_roe2o(int l, const double *t, double *d, const double *sn, int harten,
                   double epsroe);

/* Spalart-Allmaras: met_samut, sch_turb (v, u, d are (ld, 7)) */
void orc_met_samut(int l, const double *v, const double *mu, double *mut);
void orc_sch_turb(int l, double *u, const double *v, const double *d, const double *fd5x,
                  const double *fd5y, const double *fd5z, const double *fd6x,
                  const double *fd6y, const double *fd6z, const double *ts6,
                  const double *ts7, const double *sn, const double *vol);

/* teq_gradv (dv: [9][nnn] block-local) and met_smsa (+ met_difsa) */
void orc_teq_gradv(int l, const double *sn, const double *vol, const double *v, double *dv);
void orc_met_smsa(int l, const double *sn, const double *vol, const double *v,
                  const double *mu, const double *dist, const double *dv,
                  const double *fd5x, const double *fd5y, const double *fd5z, double *ts6,
                  double *ts7, double *cfke);

void orc_impli2_eqt_3d(int l, const double *u, const double *dt, double *v, const double *mu,
                       const double *mut, const double *cfke, const double *sn,
                       const double *vol, double cmt);

/* Spalart-Allmaras transport step: wall distance (atcaldis3 / atdist_3),
 * turbulence ghosts (met_bord, kparoi 0), grad(s6/s1), grad(s7/s1)
 * (met_gradtr), diffusion-density ghosts (met_rbse + met_rbsc), the clip
 * (met_cutsa) and the whole chain (met_num for 1SA).  orc_set_sa(on, ...)
 * makes orc_step / orc_step_jameson run met_num after rbord; fd (6 ld), ts
 * (2 ld) and cfke (ld) are the caller's scratch. */
int orc_atcaldis3(const double *x, const double *y, const double *z, double *dist);
void orc_met_bord(double *v, double rokinf, double roeinf);
void orc_met_gradtr(int l, const double *sn, const double *vol, const double *s, double *fd5x,
                    double *fd5y, double *fd5z, double *fd6x, double *fd6y, double *fd6z);
void orc_met_rbse(double *fd5x, double *fd5y, double *fd5z, double *fd6x, double *fd6y,
                  double *fd6z);
void orc_met_cutsa(int l, double *s, double epsk);
void orc_set_sa(int on, const double *dist, double rokinf, double roeinf, double epsk,
                int harten, double epsroe, double sigma, double *fd, double *ts,
                double *cfke);
void orc_met_num(double *v, double *u, double *d, const double *dt, const double *mu,
                 double *mut, const double *sn, const double *vol, const double *temp);
/* k-epsilon of Jones & Launder ('2JL'): met_prod (dv, tprod block-local
 * [9][nnn], [nnn]), met_smke (dv's ghosts extrapolated in place; ts6, ts7,
 * cfke global), met_kemut, met_cutke, the whole met_num; orc_set_ke(on, ...)
 * makes orc_step run it after rbord (fd 6 ld, ts 2 ld, cfke ld scratch) */
void orc_met_prod(int l, const double *mut, const double *s, const double *dv, double *tprod);
void orc_met_smke(int l, const double *sn, const double *vol, const double *v,
                  const double *mu, const double *mut, const double *tprod, double *dv,
                  double *ts6, double *ts7, double *cfke);
void orc_met_kemut(int l, const double *v, const double *mu, double *mut);
void orc_met_cutke(int l, double *s, double epsk, double epse);
void orc_set_ke(int on, double rokinf, double roeinf, double epsk, double epse, double alfak,
                double alfae, int harten, double epsroe, double *fd, double *ts, double *cfke);
void orc_met_num_ke(double *v, double *u, double *d, const double *dt, const double *mu,
                    double *mut, const double *sn, const double *vol);
/* first-cycle initialisation: met_inisa, met_inmut, met_ini (teq_gradv +
 * met_brad; dv [9][nnn] block-local) */
void orc_met_inisa(int l, double *v, const double *mut);
void orc_met_inmut(int l, const double *mu, double *mut);
void orc_met_ini(int l, double *v, const double *mut, const double *sn, const double *vol,
                 double *dv);
/* wall law of the 'lp2' walls: lpsa.f90 -> lpsa1.f90 on block l (v is
 * (ld, 7); epsk the floor of rho nu~) and cllparoi1.f90 -> lparoi1.f90 on
 * every 'lp2' wall (tau (ld, 9)) */
void orc_lpsa(int l, double *v, const double *mu, double *mut, const double *dist,
              const double *temp, double epsk);
void orc_cllparoi1(const double *v, const double *dist, const double *mu, const double *mut,
                   double *tau, const double *temp);
double orc_asin(double x);
/* non-reference option of met_smsa: the modified vorticity of Allmaras,
 * Johnson & Spalart 2012 and a derivative guarded where r is clipped
 * (0 = reference) */
void orc_set_sa_fix(int on);

int orc_step(double *v, double *u, double *d, double *dt, const double *sn,
             const double *vol, double *ps, double *temp, double *cson,
             double *mu, double *mut, double *tau, int compute_dt);

/* per-block eta(lm), ki2(lm), ki4(lm) (NULL: the scalar for every block) */
void orc_set_block_scheme(const double *eta_l, const double *ki2_l, const double *ki4_l);

/* other flux families (atsch_num.f90:628-983): ischema 14 HLLC
 * (sch_hllc_euler, sch_hllc), ischema 9 Rusanov (sch_rusanov, with the
 * stresses tau whatever the equations: zero for Euler); orc_step selects by
 * the ischema of orc_set_dissipation */
void orc_sch_hllc_euler(int l, double *u, const double *v, const double *sn,
                        const double *ps);
void orc_sch_hllc(int l, double *u, const double *v, const double *tau, const double *sn,
                  const double *ps);
void orc_sch_rusanov(int l, double *u, const double *v, const double *tau, const double *sn,
                     const double *ps);
/* ischema 12, WENO5 (sch_weno5_3d.f90; tau read whatever the equations,
 * zero for Euler; the k = -1 stencil point, before the block, taken at the
 * ghost plane k = 0) */
void orc_sch_weno5_3d(int l, double *u, const double *v, const double *tau, const double *sn,
                      const double *ps);
/* non-reference option (0 = reference): every WENO5 characteristic flux
 * sums its three weighted candidates */
void orc_set_weno_fix(int on);
/* ischema 5, AUSM+ (sch_ausmp.f90; Navier-Stokes only) */
void orc_sch_ausmp(int l, double *u, const double *v, const double *tau, const double *sn,
                   const double *ps);

/* dual time stepping (kfmg = 3; dt1min of orc_set_scheme is the physical
 * time step): the fused step adds sch_dual after the residual with the
 * physical step index icycle and the array ptdual given here */
void orc_set_dual(int kfmg, int kdualns, int icycle, double *ptdual);
void orc_sch_dual(int l, double *u, const double *v, int icycle, const double *vol,
                  const double *ptdual);
void orc_sch_duin(const double *v, double *ptdual, double *vdual, double *vdual1,
                  double *vdual2);
void orc_sch_duup(const double *v, double *ptdual, double *vdual, double *vdual1,
                  double *vdual2);

/* reference grid and flow files (readdg.f90, svgr.f90 -> writdg.f90,
 * readda.f90, svfw.f90 -> writda.f90), every block in order, gfortran's
 * unformatted sequential records (4-byte markers, subrecords of at most
 * maxsub bytes); returns 0, 1 (bad disc), 8 (file error) or 9 (records do
 * not match the layout) */
int orc_writdg(const char *path, const char *disc, const double *x, const double *y,
               const double *z, int64_t maxsub);
int orc_readdg(const char *path, double *x, double *y, double *z);
int orc_writda(const char *path, const char *disc, const char *equat, const double *v,
               const double *mut, int64_t maxsub);
int orc_readda(const char *path, const char *equat, int keinit, double *v, double *mut);

/* cns_pmath.h's exp and pow (the injection condition's b**gam6 and the SA
   source), exported for the libm comparison tests */
double orc_pow(double x, double y);
double orc_exp(double t);

#ifdef __cplusplus
}
#endif
#endif
