// cns_kernels.cuh -- host-side launchers of the CodeNS hot-path kernels.
#pragma once
#include <string>
#include <vector>

#include "cns_common.cuh"

namespace cns {

__device__ __forceinline__ double* sn_wptr(double* sn, const Blk& B, int dir,
                                           int c) {
  return sn + 9 * B.npc + (long long)c * 3 * B.nnn + (long long)dir * B.nnn - B.npc;
}

constexpr int kTile = 128;  // elements per tile (= threads per CTA)
// patch shapes (TI x TJ columns) of the 2.5D Jacobi sweep; the autotuner
// picks one of them and the plane count kc per context
constexpr int kSweepShapes = 4;
constexpr int kSweepShape[kSweepShapes][2] = {{32, 4}, {32, 8}, {16, 8}, {16, 16}};

struct HostLayout {
  std::vector<Blk> blks;
  long long ld = 0, ncells = 0, nreal = 0;
  long long ldp = 0;  // cells of the padded layout (Blk::pid), a multiple of 4
};

// an index space with its tile work list on the device
struct SpaceBuf {
  int ntiles = 0;
  std::vector<int> blk_tile0;  // first tile of each block, size nblk+1
  int* d_tile_blk = nullptr;
  long long* d_tile_start = nullptr;
  int* d_ext = nullptr;
  Space view(int l0 = -1) const {  // l0 < 0: all blocks, else block l0 only
    Space s;
    s.tile_blk = d_tile_blk;
    s.tile_start = d_tile_start;
    s.ext = d_ext;
    if (l0 < 0) {
      s.tile0 = 0;
      s.ntiles = ntiles;
    } else {
      s.tile0 = blk_tile0[l0];
      s.ntiles = blk_tile0[l0 + 1] - blk_tile0[l0];
    }
    return s;
  }
};

// one record of a reference grid or flow file: nval values of the array arr
// over the (i, j, k) box lo .. lo + ext - 1 of block blk, i fastest; img is
// the record's first value in the file's data image (records back to back)
struct IoRec {
  long long img, nval;
  double* arr;
  int blk, centre;  // centre: the value is the centre of the cell's 8 nodes (writes)
  int lo[3], ext[3];
};
struct IoPlan {
  std::vector<IoRec> recs;
  long long nval = 0;
};
// the pinned host ring the file readers and writers stream through
struct IoStage {
  static constexpr int kSlots = 4;
  static constexpr size_t kSlotBytes = size_t(8) << 20;
  char* ring = nullptr;
  cudaEvent_t ev[kSlots] = {};
};
cudaError_t io_stage_init(IoStage& s);
void io_stage_free(IoStage& s);
void io_add(IoPlan& p, int b, double* arr, int centre, const int lo[3], const int hi[3]);
// read the records of plan p from the file into the arrays, then zero the
// boxes of plan zero; returns a CNS_* code and sets err
int io_read(IoStage& stage, const IoPlan& p, const IoPlan& zero, const Blk* d_blks,
            const char* path, cudaStream_t st, std::string& err);
int io_write(IoStage& stage, const IoPlan& p, const Blk* d_blks, const char* path,
             long long maxsub, cudaStream_t st, std::string& err);

// dual time stepping: sch_dual (u += vol*dti*(fact*v + ptdual), u32 refreshed
// when given) and the physical-step arrays (mode 0 sch_duin, 1 sch_duup,
// 2 sch_duup2)
cudaError_t launch_dual(const Blk* blks, Space cells, long long ld, double fact, double dti,
                        const double* v, const double* vol, const double* ptdual, double* u,
                        float* u32, cudaStream_t st);
cudaError_t launch_dual_update(const Blk* blks, Space cells, long long ld, int mode,
                               const double* v, double* ptdual, double* vdual, double* vdual1,
                               double* vdual2, cudaStream_t st);

// the 2.5D tile list of one sweep configuration
struct TileBuf {
  int ti = 0, tj = 0, kc = 0, ntiles = 0;
  std::vector<int> blk_tile0;  // first tile of each block, size nblk+1
  int4* d_tile = nullptr;
  int* sched = nullptr;  // persistent launch: tile counter pair (device), else null
  int grid = 0;          // persistent launch: resident CTAs of the whole GPU
  const float4* faces = nullptr;  // FP32 sweep face/coefficient pack (Tiles::faces)
  Tiles view(int l0 = -1) const {
    Tiles t;
    t.tile = d_tile;
    t.kc = kc;
    t.ti = ti;
    t.tj = tj;
    t.sched = sched;
    t.grid = grid;
    t.faces = faces;
    if (l0 < 0) {
      t.tile0 = 0;
      t.ntiles = ntiles;
    } else {
      t.tile0 = blk_tile0[l0];
      t.ntiles = blk_tile0[l0 + 1] - blk_tile0[l0];
    }
    return t;
  }
};

// per-step scratch (device)
struct Work {
  long long ld = 0;
  double* prim = nullptr;     // primitive velocities u, v, w, [3][ld]
  double* dis = nullptr;      // Jameson dissipation [5][ld] (allocated on first use)
  double* dtpart = nullptr;   // global time step: per-tile minima + the result
  double* G = nullptr;        // face fluxes, [3][5][ld]
  double* R = nullptr;        // limiter ratios, [3][5][ld]
  double* V = nullptr;        // viscous halves, [3][4][ld] (ischema 14 with ns, ischema 12)
  double* tau0 = nullptr;     // zero stresses [9][ld] (ischema 12 with the Euler equations)
  double* coefe = nullptr;    // [3][ld]
  double* coefdiag = nullptr; // [ld]
  double* rv = nullptr;       // [ld]
  double* dpp[2] = {nullptr, nullptr};   // Jacobi iterates, [5][ld] each
  double* normpart = nullptr; // per tile partial norms [ntiles][15]
  double* norms = nullptr;    // [16]
  double* blocksum = nullptr; // per block norm sums [nblk][15]
  int* status = nullptr;      // device status word
  // mixed precision (allocated on first use)
  bool mixed_ready = false;
  float *v32 = nullptr, *prim32 = nullptr, *ps32 = nullptr, *tau32 = nullptr;
  float *sn32 = nullptr, *G32 = nullptr, *R32 = nullptr, *u32 = nullptr;
  float *coefe32 = nullptr, *coefdiag32 = nullptr;
  float* d32pp[2] = {nullptr, nullptr};  // FP32 iterates, padded [5][ldp] each
  float* st32 = nullptr;      // the FP32 sweep's state, padded [6][ldp]
  float4* cq32 = nullptr;     // the FP32 coefficients' inputs (u, v, w, c) [ld]
  float2* cv32 = nullptr;     // and (vol, rv) [ld]
  void* sweep_maps = nullptr; // the box staging's tensor maps (device)
  double *corr = nullptr, *ur32 = nullptr;
  float4* snc32 = nullptr;  // [ld][3]: half lower-face areas and their coefficients
};

cudaError_t launch_metric(const HostLayout& lay, const Blk* dblks, const Bnd& bd,
                          double* x, double* y, double* z, double* sn,
                          double* vol, cudaStream_t st);

cudaError_t launch_zpres(const Blk* blks, Space sp, Phys ph, int with_mu,
                         const double* v, long long ld, double* ps,
                         double* temp, double* cson, double* mu, int* status,
                         cudaStream_t st);

cudaError_t launch_zvismo(const Blk* blks, Space sp, Phys ph, double* mu,
                          const double* temp, int* status, cudaStream_t st);

// launch_zpres (with mu for the Navier-Stokes equations) and launch_chronos
// in one pass over the real cells sp, the same values
cudaError_t launch_zpres_chronos(const Blk* blks, Space sp, Phys ph, Scheme sc,
                                 const double* v, long long ld, double* ps, double* temp,
                                 double* cson, double* mu, const double* mut, double* dt,
                                 const double* sn, const double* vol, int* status,
                                 cudaStream_t st);
cudaError_t launch_chronos(const Blk* blks, Space sp, Phys ph, Scheme sc,
                           const double* mu, const double* mut, const double* v,
                           long long ld, double* dt, const double* sn,
                           const double* vol, const double* cson,
                           cudaStream_t st);

// rbord: every list entry, then the injection entries (two passes)
cudaError_t launch_rbord(const Bnd& bd, Phys ph, double* v, long long ld,
                         double* ps, double* temp, double* cson, long long n_idd_ent,
                         const long long* idd_ents, unsigned* masks, cudaStream_t st);

cudaError_t launch_tau_ghosts(const Bnd& bd, double* tau, long long ld,
                              cudaStream_t st);

// primitive velocities of the flat cell range [n0, n1)
cudaError_t launch_prim(long long n0, long long n1, const double* v, long long ld,
                        double* prim, cudaStream_t st);

cudaError_t launch_grad(const Blk* blks, Space sp, Phys ph, const double* v,
                        const double* prim, long long ld, const double* mu,
                        const double* mut, double* tau, const double* sn,
                        const double* vol, const double* temp, cudaStream_t st);

// hot kernels templated on the real type T (double: cns_flow.cu, bit-exact;
// float: cns_mixed.cu, the reduced-precision half of the mixed form)
template <class T>
cudaError_t launch_ratio_t(const Blk* blks, const SpaceBuf* lines, int l0, const T* v,
                           const T* prim, long long ld, const T* ps, T* R,
                           cudaStream_t st);
// the face fluxes of the flux family sc.ischema selects (7 Roe, 14 HLLC,
// 9 Rusanov); V: the HLLC viscous halves (ischema 14 with ns, [3][4][ld])
template <class T>
cudaError_t launch_face_flux_t(const Blk* blks, const SpaceBuf* faces, int l0, Phys ph,
                               Scheme sc, const T* v, const T* prim, long long ld,
                               const T* ps, const T* tau, const T* sn, const T* R, T* G,
                               cudaStream_t st, T* V);
// u = FP64 sum of the face fluxes (+ corr); u32 an optional float copy; V as
// above or null
template <class T>
cudaError_t launch_accumulate_t(const Blk* blks, Space sp, const T* G, long long ld,
                                const double* corr, double* u, float* u32,
                                cudaStream_t st, const T* V);
// lmx Jacobi sweeps over the real cells; the final iterate is in dpp[*cur_out]
template <class T>
cudaError_t launch_sweeps_t(const Blk* blks, Space cells, Tiles tl, Phys ph, Scheme sc, int eu,
                            int lmx, long long ld, const T* u, const T* v, const T* prim,
                            const T* ps, const T* sn, const T* coefe, const T* coefdiag,
                            T* const dpp[2], int* cur_out,
                            cudaStream_t st);
template <class T>
cudaError_t launch_update_t(const Blk* blks, Space cells, long long ld, const T* d,
                            double* v, const double* dt, double* d_out, double* normpart,
                            cudaStream_t st);

// the two precisions are defined in cns_flow.cu (double) and cns_mixed.cu (float)
#define CNS_DECLARE_HOT(T)                                                                  \
  template <>                                                                               \
  cudaError_t launch_ratio_t<T>(const Blk*, const SpaceBuf*, int, const T*, const T*,      \
                                long long, const T*, T*, cudaStream_t);                     \
  template <>                                                                               \
  cudaError_t launch_face_flux_t<T>(const Blk*, const SpaceBuf*, int, Phys, Scheme,        \
                                    const T*, const T*, long long, const T*, const T*,     \
                                    const T*, const T*, T*, cudaStream_t, T*);              \
  template <>                                                                               \
  cudaError_t launch_accumulate_t<T>(const Blk*, Space, const T*, long long,               \
                                     const double*, double*, float*, cudaStream_t,         \
                                     const T*);
CNS_DECLARE_HOT(double)
CNS_DECLARE_HOT(float)
#undef CNS_DECLARE_HOT
template <>
cudaError_t launch_sweeps_t<double>(const Blk*, Space, Tiles, Phys, Scheme, int, int, long long,
                                    const double*, const double*, const double*, const double*,
                                    const double*, const double*, const double*,
                                    double* const[2], int*, cudaStream_t);
template <>
cudaError_t launch_update_t<double>(const Blk*, Space, long long, const double*, double*,
                                    const double*, double*, double*, cudaStream_t);

// The FP32 sweeps of the mixed forms (cns_mixed.cu).  The iterates and the
// sweep's per-cell state st (rho, rho E, p, u, v, w of the real cells, six
// components) are in the padded layout (pad_index, component stride
// Blk::pld); u and coefdiag in the flat one.  maps: the device tensor maps
// of encode_sweep32_maps (box staging), or null (cp.async staging).
struct Sweep32 {
  const float* u;
  const float* st;
  const float* coefdiag;
  const void* maps;    // [(shape * 3 + array) * nblk + block], array 0 st, 1 dpp[0], 2 dpp[1]
  const void* map_st;  // set per launch: the state maps of the launch's shape
  int nblk;
  int* status;         // bit 4: a box wait gave up
};
// sweeps 2..lmx, 2.5D over tl, after launch_coefficients32 has written the
// first iterate into dpp[0] (lmx = 0: dpp[0] is zeroed); the final iterate
// in dpp[*cur_out]; ldp: the padded arrays' component stride
cudaError_t launch_sweeps32(Tiles tl, const Blk* blks, Phys ph, Scheme sc, int eu, int lmx,
                            long long ld, long long ldp, const Sweep32& a,
                            float* const dpp[2], int* cur_out, cudaStream_t st);
// one 2.5D sweep d_in (= dpp[din_sel]) -> d_out over the tiles tl
cudaError_t launch_sweep32_25d(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                               long long ld, const Sweep32& a, int din_sel, const float* d_in,
                               float* d_out, cudaStream_t st);
// v += d (d padded FP32) and the norm partials
cudaError_t launch_update32(const Blk* blks, Space cells, long long ld, const float* d,
                            double* v, const double* dt, double* normpart, cudaStream_t st);
// the tensor maps of the box staging for every sweep shape and block (host
// bytes, kSweepShapes * 3 * nblk maps of 128 bytes)
cudaError_t encode_sweep32_maps(const std::vector<Blk>& blks, const float* st,
                                float* const dpp[2], std::vector<unsigned char>& out);

// one sweep of the 2.5D kernel over the tiles tl (d_in -> d_out); every
// sweep but the first of launch_sweeps_t runs through it
template <class T>
cudaError_t launch_jacobi_25d_t(const Blk* blks, Tiles tl, Phys ph, int qfix, int eu,
                                long long ld, const T* u, const T* v, const T* prim,
                                const T* ps, const T* sn, const T* coefe, const T* coefdiag,
                                const T* d_in, T* d_out, cudaStream_t st);
template <>
cudaError_t launch_jacobi_25d_t<double>(const Blk*, Tiles, Phys, int, int, long long,
                                        const double*, const double*, const double*,
                                        const double*, const double*, const double*,
                                        const double*, const double*, double*, cudaStream_t);
// chrono.f90:113-151 (kdtl = 0): dt = min(dt1min, min over real cells) on
// [0, ncells); status bit 2 when below dt1min; part: one double per cell tile
cudaError_t launch_dt_global(const Blk* blks, Space cells, long long ncells, double dt1min,
                             double* dt, double* part, double* scalar, int* status,
                             cudaStream_t st);

// the Jameson scheme (cns_jameson.cu): mode 1 rfve, mode 2 rfvc
cudaError_t launch_ghost_refresh(const Bnd& bd, int mode, double* v, long long ld, double* ps,
                                 double* temp, double* cson, cudaStream_t st);
// dissipation of the faces of block l0 (all: -1) into G, summed into d
cudaError_t launch_dissip_jameson(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                                  const double* v, long long ld,
                                  const double* ps, const double* cson, const double* sn,
                                  double* G, double* d, cudaStream_t st);
// centred fluxes into G, u = 0.5 sum - dis (u32: float copy when given)
cudaError_t launch_sch_jameson(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                               int ns, double pinfl, const double* v, long long ld,
                               const double* ps, const double* tau, const double* sn,
                               const double* dis, double* G, double* u, float* u32,
                               cudaStream_t st);

// turbulence-transport terms (cns_turb.cu): met_fludc / met_fludcsa over the
// flat range [n0, n1]; fd = {fd5x, fd5y, fd5z, fd6x, fd6y, fd6z}
cudaError_t launch_fludc(long long n0, long long n1, const double* mu, const double* mut,
                         double* const fd[6], double alfak, double alfae, cudaStream_t st);
cudaError_t launch_fludcsa(long long n0, long long n1, const double* s6, const double* mu,
                           double* const fd[6], double sigma, cudaStream_t st);
// met_roe2o / met_roe2oh (harten) of block l0 (all: -1): t, d are (ld, 7);
// cells_ext covers i 0..ni, j 0..nj, k 0..nk
cudaError_t launch_roe2o(const Blk* blks, const SpaceBuf* faces, Space cells_ext, int l0,
                         int harten, double epsroe, double gam, double gam1, const double* t,
                         long long ld, const double* sn, double* G, double* d,
                         cudaStream_t st);

// discrete adjoint of the FP64 Euler Roe iteration (cns_adjoint.cu)
// face-flux Jacobians J[3 dirs][27 seeds][5][ld] (4 stencil cells x (W, p),
// face normal) at the state v, ps
cudaError_t launch_face_jac(const Blk* blks, const SpaceBuf* faces, Phys ph, Scheme sc,
                            const double* v, const double* ps, long long ld, const double* sn,
                            double* J, cudaStream_t st);
// wbar[6][ld] = (A^T lambda) per cell of i 0..ni, j 0..nj, k 0..nk (W, p
// parts), sbar[3][3][ld] = lambda^T du/dS per face
cudaError_t launch_adj_gather(const Blk* blks, Space cells_ext, const double* J,
                              const double* lam, long long ld, double* wbar, double* sbar,
                              cudaStream_t st);
// out = L^T y over lmax transposed sweeps of the linearised Euler Jacobi
// update (implimf_eu with qfix), from the flux Jacobians of each cell's state
// (z0, z1: scratch [5][ld]; icd: scratch [ld] for 1 / cd); T = float: face
// areas, coefficients and the sweep iterates in FP32 (the reduced-precision
// forms)
template <class T>
cudaError_t launch_precond_ta(const Blk* blks, Space cells, long long ld, const double* v,
                              const double* ps, const T* sn, const T* coefe, const T* cd,
                              double gam1, double pinfl, int lmax, const double* y, T* z0,
                              T* z1, T* icd, double* out, cudaStream_t st);

// met_samut (real cells of block l0's space) and sch_turb (u, v, d: (ld, 7))
cudaError_t launch_samut(const Blk* blks, Space cells, const double* v6, const double* mu,
                         double* mut, cudaStream_t st);
cudaError_t launch_sch_turb(const Blk* blks, const SpaceBuf* faces, Space cells, int l0,
                            const double* v, long long ld, const double* const fd[6],
                            const double* ts6, const double* ts7, const double* d,
                            const double* sn, const double* vol, double* G, double* u,
                            cudaStream_t st);

// teq_grads over the cells of the space into out[3 nsc][ld]: mode 0 = the
// velocity (nsc 3), mode 1 = the fields f[q][ld], mode 2 = the transport
// variables per unit mass s6/s1, s7/s1 (nsc 2, met_gradtr), mode 3 =
// sqrt(s6/s1) (nsc 1, met_bark); modes 0, 2 and 3
// evaluate their scalars once into sc[nsc][ld] over the flat range [n0, n1)
// covering the cells of the space and their ghosts.  met_smsa with its
// gradients of rho nu~ (grt) and rho (grr)
cudaError_t launch_teq_grads(const Blk* blks, Space cells, int mode, int nsc,
                             const double* v, const double* f, long long ld, const double* sn,
                             const double* vol, double* out, double* sc, long long n0,
                             long long n1, cudaStream_t st);
cudaError_t launch_smsa(const Blk* blks, Space cells, long long ld, const double* v,
                        const double* mu, const double* dist, const double* dv,
                        const double* grt, const double* grr, const double* const fd5[3],
                        double* ts6, double* ts7, double* cfke, int fix, cudaStream_t st);
// impli2_eqt_3d of block l0 (-1: all): u, v are (ld, 7); w: 20 ld scratch;
// rcp = 1: one reciprocal per line step instead of three divisions (the
// reduced-precision forms; not bit-exact)
// wall_ni: the first cells of the wall-law walls (nwall of them), whose
// increments are zeroed before the update (impli2_eqt_3d.f90:384-405)
cudaError_t launch_impli2(const Blk* blks, const SpaceBuf* faces, const SpaceBuf* lines,
                          Space cells, int l0, long long ld, const double* u, const double* dt,
                          double* v, const double* mu, const double* mut, const double* cfke,
                          const double* sn, const double* vol, double cmt, double* w, int rcp,
                          const long long* wall_ni, long long nwall, cudaStream_t st);

// wall laws of the adiabatic wall-law walls 'lp2' (rbord.f90:377-379: vkar,
// cllog, yp0; the SA cv1 and the nu~ floor epsk) on the cnt list entries
// from e0 of one boundary: lpsa1 (first cell's mut and rho nu~, ghost rho
// nu~ = 0; v is (ld, 7)) and lparoi1 (wall stresses and heat flux in tau)
struct WallLaw {
  double vkar, cllog, yp0, cv1, epsk;
};
cudaError_t launch_lpsa1(const Bnd& bd, long long e0, int cnt, Phys ph, WallLaw wl,
                         long long ld, double* v, const double* mu, double* mut,
                         const double* dist, const double* temp, cudaStream_t st);
cudaError_t launch_lparoi1(const Bnd& bd, long long e0, int cnt, Phys ph, WallLaw wl,
                           long long ld, const double* v, const double* mu, const double* mut,
                           const double* dist, const double* temp, double* tau,
                           cudaStream_t st);

// wall distance of the real cells to the nearest facet centre of the nw wall
// entries went (atcaldis3 / atdist_3); par: 3 nw scratch
cudaError_t launch_wall_dist(const Bnd& bd, const Blk* blks, Space cells,
                             const long long* went, long long nw, const double* x,
                             const double* y, const double* z, double* par, double* dist,
                             cudaStream_t st);
// the k-epsilon model of Jones & Launder ('2JL'): met_prod (tprod [ld]),
// met_exgr on the nine velocity gradients dv [9][ld] of block B, met_smke
// (met_bark + met_bare + met_smkes: ts6, ts7, cfke; w: 14 ld scratch; the
// flat range [n0, n1) holds the block's cells), met_kemut, met_cutke
cudaError_t launch_met_prod(const Blk* blks, Space cells, long long ld, const double* mut,
                            const double* s, const double* dv, double* tprod, cudaStream_t st);
cudaError_t launch_exgr(const Blk& B, long long ld, double* dv, cudaStream_t st);
cudaError_t launch_smke(const Blk* blks, Space cells, long long ld, const double* s,
                        const double* mu, const double* mut, const double* sn,
                        const double* vol, const double* tprod, const double* dv, double* w,
                        double* ts6, double* ts7, double* cfke, long long n0, long long n1,
                        cudaStream_t st);
cudaError_t launch_kemut(const Blk* blks, Space cells, long long ld, const double* v,
                         const double* mu, double* mut, cudaStream_t st);
cudaError_t launch_cutke(const Blk* blks, Space cells, long long ld, double* v, double epsk,
                         double epse, cudaStream_t st);
// first-cycle turbulence initialisation on the real cells: mode 0 met_inisa
// (v6 = mut), 1 met_inmut (mut = mu / 10), 2 met_brad (v6, v7 from mut and
// the vorticity of dv [9][ld])
cudaError_t launch_turb_init(const Blk* blks, Space cells, int mode, long long ld, double* v,
                             double* mut, const double* mu, const double* dv, cudaStream_t st);

// met_bord (kparoi 0) on v(:,6:7); met_rbse + met_rbsc on fd[6][ld];
// met_cutsa on the real cells
cudaError_t launch_turb_bord(const Bnd& bd, double* v, long long ld, double rokinf,
                             double roeinf, cudaStream_t st);
cudaError_t launch_fd_ghosts(const Bnd& bd, double* const fd[6], cudaStream_t st);
cudaError_t launch_cutsa(const Blk* blks, Space cells, double* v, long long ld, double epsk,
                         cudaStream_t st);

// raise the dynamic shared-memory limit of every 2.5D instantiation (once
// per device, before the first launch)
cudaError_t init_jacobi_25d();
// resident CTAs per SM of the FP32 sweep kernel of patch ti x tj (persistent launch size)
int sweep_f32_blocks_per_sm(int ti, int tj, int eu, int box);
cudaError_t init_jacobi_25d_float();

inline cudaError_t launch_ratio(const Blk* blks, const SpaceBuf* lines, int l0,
                                const double* v, const double* prim, long long ld,
                                const double* ps, double* R, cudaStream_t st) {
  return launch_ratio_t<double>(blks, lines, l0, v, prim, ld, ps, R, st);
}
// The fused residual (the face fluxes of the three directions and their
// accumulation into u, and u32 when given, in one launch over the 32 x 4
// residual tiles) for every flux family that keeps one value per face: all
// but HLLC with the stresses (ischema 14 with ns) and the Jameson scheme.
// launch_residual_fused: FP64 without contraction (the bit-exact path);
// launch_residual_fused_fma: the same kernel compiled with contraction (the
// FP64 residual of the mixed form).
inline bool residual_fused_ok(const Scheme& sc) {
  return (sc.ischema == 7 || sc.ischema == 9 || sc.ischema == 5 || sc.ischema == 14) &&
         !(sc.ischema == 14 && sc.ns);
}
constexpr int kResTI = 32, kResTJ = 4, kResKC = 16;  // default fused tiles
// the patch shapes the fused residual is instantiated for
constexpr int kResShapes = 2;
constexpr int kResShape[kResShapes][2] = {{32, 4}, {16, 8}};
cudaError_t launch_residual_fused(const Blk* blks, Tiles tl, Phys ph, Scheme sc, const double* v,
                                  const double* prim, long long ld, const double* ps,
                                  const double* tau, const double* sn, const double* R,
                                  double* u, float* u32, cudaStream_t st);
cudaError_t launch_residual_fused_fma(const Blk* blks, Tiles tl, Phys ph, Scheme sc,
                                      const double* v, const double* prim, long long ld,
                                      const double* ps, const double* tau, const double* sn,
                                      const double* R, double* u, float* u32, cudaStream_t st);

inline cudaError_t launch_face_flux(const Blk* blks, const SpaceBuf* faces, int l0,
                                    Phys ph, Scheme sc, const double* v,
                                    const double* prim, long long ld, const double* ps,
                                    const double* tau, const double* sn, const double* R,
                                    double* G, cudaStream_t st, double* V = nullptr) {
  return launch_face_flux_t<double>(blks, faces, l0, ph, sc, v, prim, ld, ps, tau, sn, R, G,
                                    st, V);
}
// WENO5 residual (sch_weno5_3d.f90, ischema 12) over the real cells of the
// space: u = the flux balance (every real cell written); tau: the nine
// stress arrays (zero for the Euler equations); G [3][5][ld] and
// V [3][4][ld]: face scratch; u32 (optional): u rounded to FP32 for the
// mixed sweeps; fix: the non-reference option that sums all three weighted
// candidates in every direction and flux component
cudaError_t launch_weno5(const Blk* blks, Space cells, Phys ph, int fix, const double* v,
                         long long ld,
                         const double* ps, const double* tau, const double* sn, double* G,
                         double* V, double* u, float* u32, cudaStream_t st);

inline cudaError_t launch_accumulate(const Blk* blks, Space sp, const double* G,
                                     long long ld, double* u, cudaStream_t st,
                                     const double* V = nullptr) {
  return launch_accumulate_t<double>(blks, sp, G, ld, nullptr, u, nullptr, st, V);
}

// FP64 implicit coefficients with float copies for the mixed sweeps
cudaError_t launch_implicit_coefficients(const Blk* blks, Space cells,
                                         const SpaceBuf* faces, int l0, Phys ph, int eu,
                                         const double* dt, const double* v,
                                         const double* prim, const double* mu,
                                         const double* mut, const double* sn,
                                         const double* vol, const double* cson, Work& w,
                                         float* coefe32, float* coefdiag32,
                                         cudaStream_t st);

// The single-precision copies the primitive-velocity kernel writes for the
// reduced-precision forms, each value rounded once from FP64:
//  - st32: the FP32 sweep state rho, rho E, p, u, v, w (padded layout);
//  - cq32 = (u, v, w, c) and cv32 = (vol, rv) per cell: the inputs of the
//    FP32 implicit coefficients, rv = (gam/pr mu + gam/prt mut) / rho the
//    viscous factor of implimf_3d.f90:95-105 (0 for the Euler equations);
//  - when v32 is given (defect form), v32, prim32 and ps32 for the FP32
//    face fluxes.
struct PrimShadow {
  float *v32, *prim32, *ps32;
  const Blk* blks;
  int nblk;
  float* st32;
  float4* cq32;
  float2* cv32;
  const double *cson, *mu, *mut, *vol;
  float gp, gpt;  // gam / pr, gam / prt
  int eu;
};
// primitive velocities over the flat range [0, ncells) together with the
// copies of sh
cudaError_t launch_prim_shadow(long long ncells, const double* v, long long ld, double* prim,
                               const double* ps, const PrimShadow& sh, cudaStream_t st);
cudaError_t launch_to_float(const double* a, float* b, long long n, cudaStream_t st);
// corr = u64 - u_r32 on the real cells (defect correction)
cudaError_t launch_defect(const Blk* blks, Space cells, long long ld, const double* u64,
                          const double* ur32, double* corr, cudaStream_t st);
// the FP32 implicit coefficients (coefe32 per face, coefdiag32 per cell) of
// the mixed sweeps in one pass over the real cells
// (the per-cell inputs cq32, cv32 of PrimShadow)
cudaError_t launch_coefficients32(const Blk* blks, Space cells, int eu, long long ld,
                                  double dtpas, const double* dt, const double* vol,
                                  const float4* cq32, const float2* cv32, const float* sn32,
                                  float* coefe32, float* coefdiag32, float4* snc32,
                                  const float* u32, float* d1, cudaStream_t st);
// the face lanes of the FP32 sweep's pack: snc[3n + dir].xyz = S/2 of cell n's
// lower face in dir (exact halves of sn32), .w = 0 until k_coef32 writes it
cudaError_t launch_pack_faces32(const Blk* blks, int nblk, long long ncells, const float* sn32,
                                float4* snc32, cudaStream_t st);
// FP64 face fluxes with FMA contraction (the mixed form's residual; agrees
// with launch_face_flux_t<double> to FP64 rounding, not bit for bit)
cudaError_t launch_face_flux_fma(const Blk* blks, const SpaceBuf* faces, int l0, Phys ph,
                                 Scheme sc, const double* v, const double* prim,
                                 long long ld, const double* ps, const double* tau,
                                 const double* sn, const double* R, double* G,
                                 cudaStream_t st, double* V);

// the implicit phase of implimf_eu (eu = 1) or implimf_3d (eu = 0) on the
// cells of the space: coefficients, lmx Jacobi sweeps, v += d; d_out
// (optional) receives the final increment, want_norms stores per-tile
// residual partials in w.normpart
cudaError_t launch_implicit(const Blk* blks, Space cells, Tiles tl, const SpaceBuf* faces,
                            int l0, Phys ph, Scheme sc, int eu, int lmx,
                            const double* u, const double* dt, double* v,
                            double* d_out, const double* mu, const double* mut,
                            const double* sn, const double* vol,
                            const double* ps, const double* cson, Work& w,
                            int want_norms, cudaStream_t st);

cudaError_t launch_norm_partials(const Blk* blks, Space cells, long long ld,
                                 const double* u0, const double* v,
                                 const double* dt, double* normpart,
                                 cudaStream_t st);

cudaError_t launch_norm_finalize(const Blk* blks, const int* blk_tile0_dev,
                                 int b0, int b1, const double* normpart,
                                 double* blocksum, double* norms, cudaStream_t st);

}  // namespace cns
