// cns_abi.cu -- C ABI of the CodeNS hot path: context (the reference's module
// state), tile work lists, per-routine entry points and the graph-captured
// fused pseudo-time step.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cns_abi.h"
#include "cns_kernels.cuh"


using namespace cns;

struct cns_ctx {
  int device = 0;
  cudaStream_t st = nullptr;      // stream the work is issued on
  cudaStream_t own_st = nullptr;  // stream created by the context
  HostLayout lay;
  Blk* d_blks = nullptr;
  Phys ph{};
  Scheme sc{};
  SpaceBuf cells, faces[3], lines[3];
  SpaceBuf cells_ext;  // i 0..ni, j 0..nj, k 0..nk (met_roe2o's zeroed range)
  double alfak = 1.0, alfae = 1.3, sigma = 2.0 / 3.0, epsroe = 0.0;  // modeleturb, schemanum
  double* sa_gr = nullptr;   // gradients of rho nu~ and rho [6][ld]
  double* sa_sc = nullptr;   // gradient scalars (velocity, s6/s1, s7/s1) [3][ld]
  double* sa_w = nullptr;    // impli2_eqt_3d scratch [20][ld]
  // Spalart-Allmaras transport step of the fused iteration (cns_set_sa)
  bool sa_on = false;
  double sa_rokinf = 0., sa_roeinf = 0., sa_epsk = 1e-8;
  int sa_fix = 0;                   // flagged non-reference SA source fix (cns_sa_t)
  const double* sa_dist = nullptr;  // the caller's wall distance (device)
  double* sa_dv = nullptr;          // velocity gradients [9][ld]
  double* sa_fd = nullptr;          // diffusion densities fd5x..fd6z [6][ld]
  double* sa_ts = nullptr;          // sources ts6, ts7 [2][ld]
  double* sa_cfke = nullptr;        // source-derivative bound [ld]
  // k-epsilon transport step of the fused iteration (cns_set_ke); it shares
  // the SA step's gradient, diffusion-density, source and line scratch
  bool ke_on = false;
  double ke_rokinf = 0., ke_roeinf = 0., ke_epsk = 0., ke_epse = 0.;
  double* ke_tprod = nullptr;       // production of k [ld]
  double* ke_w = nullptr;           // met_smke scratch [14][ld]
  long long n_wall_ent = 0;
  long long* d_wall_ents = nullptr;  // list entries of the wall boundaries
  // the wall-law walls 'lp2' in list order: first list entry, count, block
  struct Lp2 {
    long long e0;
    int cnt, blk;
  };
  std::vector<Lp2> lp2;
  long long* d_lp2_ni = nullptr;  // their first cells (no SA increment there)
  long long n_lp2_ni = 0;
  double* wall_par = nullptr;        // wall facet centres [3][n_wall_ent]
  double* adj_J = nullptr;   // adjoint: face-flux Jacobians [3][27][5][ld]
  double* adj_z = nullptr;   // adjoint: transposed-sweep scratch [2][5][ld] + 1 / cd [ld]
  double* tau_pack = nullptr;  // nine separate stress arrays packed as (ld, 9)
  double* u_forced = nullptr;  // implimf right-hand side u + ff (ityprk != 0) [5][ld]
  int* sched32 = nullptr;      // tile counter pair of the persistent FP32 sweep
  int staging32 = 0;           // FP32 sweep staging: 0 tensor boxes (TMA), 1 cp.async
  std::string tune_cache;      // sweep-tiling cache file ("" = none)
  int tune_src64 = 0, tune_src32 = 0;  // tiling source: 0 default or set, 1 timed, 2 cache
  int nsm = 0;                 // streaming multiprocessors of the device
  bool adj_fp32 = false;     // L^T of the prepared adjoint in FP32 (precision != 0)
  TileBuf tiles64, tiles32;   // 2.5D tiles of the FP64 and the FP32 Jacobi sweeps
  TileBuf tiles_res;          // 2.5D tiles of the fused residual
  bool res_fused = false;     // residual: fused kernel (tiles_res) or face kernels + accumulate
  bool tuned64 = false, tuned32 = false;
  float tune_ms64 = 0.f, tune_ms32 = 0.f;  // the chosen configuration's sweep time
  int* d_cells_tile0 = nullptr;  // cells.blk_tile0 on the device
  // boundaries
  Bnd bd{};
  std::vector<int> h_btype;
  long long n_idd_ent = 0;
  long long* d_idd_ents = nullptr;  // list entries of injection boundaries
  unsigned* d_idd_masks = nullptr;  // per boundary sweep masks
  // scratch
  Work w;
  std::vector<void*> allocs;
  long long scratch_bytes = 0;
  double* h_norms = nullptr;  // pinned [16]
  int* h_status = nullptr;    // pinned
  // fast path
  cns_state_t state{};
  bool bound = false;
  bool metric_done = false;
  // iteration graphs [form][time step recomputed]: form kGraph64 = FP64,
  // kGraphRef = mixed or defect iteration with refresh, kGraphReg = defect
  // iteration without refresh; and the kernel nodes of each
  cudaGraphExec_t gexec[3][2] = {};
  int nk_graph[3][2] = {};
  long long kernels_launched = 0;        // kernels of every fused-step graph launched
  long long mixed_iter = 0;              // mixed iterations since the last reset
  long long ncyc = 0;                    // fused iterations since the state was bound
  long long cyc_n = 0, cyc_i = 0;        // the reference's ncyc, icyc of the last iteration
  int dual_icycle = 1;                   // physical step index of sch_dual (kfmg = 3)
  long long io_maxsub = 2147483639;      // bytes per subrecord of the files written
  IoStage io_stage;                      // pinned ring of the file readers and writers
  std::string err;
};

namespace {

int fail(cns_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_fail(cns_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return CNS_OK;
  return fail(c, CNS_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                   \
  do {                                                             \
    cudaError_t e__ = (call);                                      \
    if (e__ != cudaSuccess) return cuda_fail(c, e__, #call);       \
  } while (0)

template <typename T>
cudaError_t dev_alloc(cns_ctx* c, T** p, size_t n, bool zero = true) {
  void* q = nullptr;
  const size_t bytes = sizeof(T) * (n > 0 ? n : 1);
  cudaError_t e = cudaMalloc(&q, bytes);
  if (e != cudaSuccess) return e;
  c->allocs.push_back(q);
  c->scratch_bytes += (long long)bytes;
  if (zero) e = cudaMemset(q, 0, bytes);
  *p = static_cast<T*>(q);
  return e;
}

template <typename T>
void dev_free(cns_ctx* c, T* p) {
  if (!p) return;
  for (size_t q = 0; q < c->allocs.size(); ++q)
    if (c->allocs[q] == (void*)p) {
      c->allocs.erase(c->allocs.begin() + q);
      break;
    }
  cudaFree(p);
}

template <typename T>
cudaError_t upload(cns_ctx* c, T** p, const T* h, size_t n) {
  cudaError_t e = dev_alloc(c, p, n, false);
  if (e != cudaSuccess) return e;
  if (n > 0) e = cudaMemcpy(*p, h, sizeof(T) * n, cudaMemcpyHostToDevice);
  return e;
}

// index space with extent ext(B) per block and its tile work list
template <typename F>
cudaError_t build_space(cns_ctx* c, SpaceBuf& s, F ext_of) {
  std::vector<int> tb, ext;
  std::vector<long long> ts;
  s.blk_tile0.assign(c->lay.blks.size() + 1, 0);
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    int e[3];
    ext_of(c->lay.blks[b], e);
    ext.push_back(e[0]);
    ext.push_back(e[1]);
    ext.push_back(e[2]);
    const long long cnt = (long long)e[0] * e[1] * e[2];
    s.blk_tile0[b] = (int)tb.size();
    for (long long t = 0; t < cnt; t += kTile) {
      tb.push_back((int)b);
      ts.push_back(t);
    }
  }
  s.blk_tile0.back() = (int)tb.size();
  s.ntiles = (int)tb.size();
  cudaError_t e = upload(c, &s.d_tile_blk, tb.data(), tb.size());
  if (e == cudaSuccess) e = upload(c, &s.d_tile_start, ts.data(), ts.size());
  if (e == cudaSuccess) e = upload(c, &s.d_ext, ext.data(), ext.size());
  return e;
}

// the 2.5D sweep tiles: patches of ti x tj columns, kc planes deep, block by
// block
cudaError_t build_tiles(cns_ctx* c, TileBuf& t, int ti, int tj, int kc) {
  dev_free(c, t.d_tile);
  t.d_tile = nullptr;
  std::vector<int4> tl;
  t.blk_tile0.assign(c->lay.blks.size() + 1, 0);
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    const Blk& B = c->lay.blks[b];
    t.blk_tile0[b] = (int)tl.size();
    for (int k0 = 1; k0 <= B.nk - 1; k0 += kc)
      for (int j0 = 1; j0 <= B.nj - 1; j0 += tj)
        for (int i0 = 1; i0 <= B.ni - 1; i0 += ti) tl.push_back(make_int4((int)b, i0, j0, k0));
  }
  t.blk_tile0.back() = (int)tl.size();
  t.ntiles = (int)tl.size();
  t.ti = ti;
  t.tj = tj;
  t.kc = kc;
  return upload(c, &t.d_tile, tl.data(), tl.size());
}

// the FP32 sweep tiles run as a persistent launch: one CTA per resident slot
// of the GPU (every SM times the kernel's CTAs per SM), taking tiles in turn
void persistent_sweep32(cns_ctx* c) {
  const int per_sm =
      sweep_f32_blocks_per_sm(c->tiles32.ti, c->tiles32.tj, !c->sc.ns, c->staging32 == 0);
  c->tiles32.sched = (c->sched32 && per_sm > 0 && c->nsm > 0) ? c->sched32 : nullptr;
  c->tiles32.grid = per_sm * c->nsm;
  c->tiles32.faces = c->w.snc32;
}

bool bad_block(cns_ctx* c, int l) { return l < 0 || l > (int)c->lay.blks.size(); }

// [first, last) flat range of block l (0 = every block)
void block_range(cns_ctx* c, int l, long long& n0, long long& n1) {
  if (l == 0) {
    n0 = 0;
    n1 = c->lay.ncells;
  } else {
    const Blk& B = c->lay.blks[l - 1];
    n0 = B.npc;
    n1 = B.npc + B.nnn;
  }
}

cudaError_t zero_cols(cns_ctx* c, double* a, int ncol, int l) {
  long long n0, n1;
  block_range(c, l, n0, n1);
  for (int col = 0; col < ncol; ++col) {
    cudaError_t e = cudaMemsetAsync(a + col * c->lay.ld + n0, 0,
                                    sizeof(double) * (n1 - n0), c->st);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

enum { kGraph64 = 0, kGraphRef = 1, kGraphReg = 2 };

void drop_graphs(cns_ctx* c) {
  for (auto& form : c->gexec)
    for (cudaGraphExec_t& g : form)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  // the defect-correction refresh schedule (mixed_iter) is not touched: new
  // tiles, a new stream or recaptured graphs change no iteration's form
}

// atsch_num.f90:173-178, 436: whether the iteration with counters ncyc = n,
// icyc = i recomputes the time step
bool dt_due(const cns_ctx* c, long long n, long long i) {
  const int nc = c->sc.ncychro;
  return nc <= 1 || n % nc == 1 || i < c->sc.icychr0;
}

// sch_dual.f90:18-19, sch_dual2.f90:18-19
double dual_fact(const cns_ctx* c) {
  if (c->dual_icycle <= 1) return 1.;
  return c->sc.kdualns == 2 ? 11. / 6. : 1.5;
}

// the physical time term after the residual (atsch_num.f90:993-1003)
cudaError_t enqueue_dual(cns_ctx* c, float* u32) {
  const cns_state_t& s = c->state;
  return launch_dual(c->d_blks, c->cells.view(-1), c->lay.ld, dual_fact(c), 1. / c->sc.dt1min,
                     s.v, s.vol, s.ptdual, s.u, u32, c->st);
}

int check_status(cns_ctx* c) {
  CK(cudaMemcpyAsync(c->h_status, c->w.status, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const int bits = *c->h_status;
  if (bits) {
    *c->h_status = 0;
    CK(cudaMemsetAsync(c->w.status, 0, sizeof(int), c->st));
    if (bits & 1) return fail(c, CNS_ETEMP, "non-positive temperature (zvismo)");
    if (bits & 4) return fail(c, CNS_ECUDA, "FP32 sweep: a staged box did not arrive");
    return fail(c, CNS_EDT, "global time step below dt1min (chrono)");
  }
  return CNS_OK;
}

// primitive velocities of the cells of block l (0: every block)
cudaError_t prim_of(cns_ctx* c, int l, const double* v) {
  long long n0, n1;
  block_range(c, l, n0, n1);
  return launch_prim(n0, n1, v, c->lay.ld, c->w.prim, c->st);
}

// the residual of one block set: (optional) limiter ratios, face fluxes,
// accumulation into u; the primitive velocities must be current
cudaError_t residual(cns_ctx* c, int l0, double* u, const double* v,
                     const double* tau, const double* sn, const double* ps) {
  const long long ld = c->lay.ld;
  cudaError_t e = cudaSuccess;
  // WENO5 (no limiter) reads the stresses whatever the equations
  if (c->sc.ischema == 12)
    return launch_weno5(c->d_blks, c->cells.view(l0), c->ph, c->sc.weno_fix, v, ld, ps, tau, sn,
                        c->w.G, c->w.V, u, nullptr, c->st);
  if (c->sc.ns && c->sc.ilim == 1)
    e = launch_ratio(c->d_blks, c->lines, l0, v, c->w.prim, ld, ps, c->w.R, c->st);
  if (e == cudaSuccess && c->res_fused && residual_fused_ok(c->sc))
    return launch_residual_fused(c->d_blks, c->tiles_res.view(l0), c->ph, c->sc, v, c->w.prim,
                                 ld, ps, tau, sn, c->w.R, u, nullptr, c->st);
  if (e == cudaSuccess)
    e = launch_face_flux(c->d_blks, c->faces, l0, c->ph, c->sc, v, c->w.prim, ld, ps, tau,
                         sn, c->w.R, c->w.G, c->st, c->w.V);
  if (e == cudaSuccess)
    e = launch_accumulate(c->d_blks, c->cells.view(l0), c->w.G, ld, u, c->st, c->w.V);
  return e;
}

// ---------------------------------------------------------------------------
// The reference call surface of the per-routine entry points.
//
// Arrays may be host or device pointers.  A host array (the reference's own
// Fortran arrays, passed as they are) is copied into a device buffer before
// the routine and, when the routine writes it, back after it, and the call
// returns when the copies are done: the copy-in/out parity mode.  Device
// arrays pass through and the call only enqueues work on the context stream.
// ---------------------------------------------------------------------------
bool host_pointer(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();  // a pageable pointer the runtime does not know
    return true;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

struct Staging {
  explicit Staging(cns_ctx* ctx) : c(ctx) {}
  ~Staging() {
    for (void* b : bufs) cudaFree(b);
  }
  // n elements at p, read (in) and/or written (out) by the routine
  template <class T>
  T* map(T* p, size_t n, bool in, bool out) {
    if (!p || err != cudaSuccess || !host_pointer(p)) return p;
    void* q = nullptr;
    err = cudaMalloc(&q, sizeof(T) * (n > 0 ? n : 1));
    if (err != cudaSuccess) return p;
    bufs.push_back(q);
    if (in) err = cudaMemcpyAsync(q, p, sizeof(T) * n, cudaMemcpyHostToDevice, c->st);
    else err = cudaMemsetAsync(q, 0, sizeof(T) * n, c->st);
    if (out) outs.push_back({(void*)p, q, sizeof(T) * n});
    staged = true;
    return static_cast<T*>(q);
  }
  template <class T>
  T* in(T* p, size_t n) { return map(p, n, true, false); }
  template <class T>
  T* inout(T* p, size_t n) { return map(p, n, true, true); }
  // copy the outputs back; wait for the stream when anything was staged
  cudaError_t finish() {
    for (const Out& o : outs)
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(o.host, o.dev, o.bytes, cudaMemcpyDeviceToHost, c->st);
    if (err == cudaSuccess && staged) err = cudaStreamSynchronize(c->st);
    return err;
  }
  struct Out {
    void* host;
    void* dev;
    size_t bytes;
  };
  cns_ctx* c;
  std::vector<void*> bufs;
  std::vector<Out> outs;
  bool staged = false;
  cudaError_t err = cudaSuccess;
};

// equat (the reference's character*7, not NUL-terminated): the equations
// (1:2) 'eu' or 'ns' and the three-dimensional form (3:4) '3d'; the
// two-dimensional variants ('2dk', ...) are not provided
bool equat_ok(const char* e) {
  if (!e) return false;
  const bool eq = (e[0] == 'e' && e[1] == 'u') || (e[0] == 'n' && e[1] == 's');
  return eq && e[2] == '3' && e[3] == 'd';
}

// the reference passes sn(npsn), the block's slice (sequence association,
// atsch_num.f90:470-479), with lgsnlt = nnn(lm); l = 0 (every block) takes
// the whole array.  Elements of the slice, and the array base the kernels
// index from.
bool sn_slice_ok(cns_ctx* c, int l, long long lgsnlt) {
  return l == 0 ? lgsnlt == c->lay.ld : lgsnlt == c->lay.blks[l - 1].nnn;
}
size_t sn_elems(cns_ctx* c, int l) {
  return 9 * (size_t)(l == 0 ? c->lay.ld : c->lay.blks[l - 1].nnn);
}
const double* sn_base(cns_ctx* c, int l, const double* sn) {
  return l == 0 ? sn : sn - 9 * c->lay.blks[l - 1].npc;
}

// the reference's nine stress / heat-flux arrays toxx, toxy, toxz, toyy,
// toyz, tozz, qcx, qcy, qcz as one (ld, 9) array: used in place when they
// are the columns of one such array, else gathered into context scratch
cudaError_t tau_view(cns_ctx* c, Staging& sg, const double* const t[9], const double** out) {
  const long long ld = c->lay.ld;
  const double* d[9];
  for (int a = 0; a < 9; ++a) {
    d[a] = sg.in(t[a], (size_t)ld);
    if (sg.err != cudaSuccess) return sg.err;
  }
  bool packed = true;
  for (int a = 1; a < 9; ++a) packed = packed && d[a] == d[0] + a * ld;
  if (packed) {
    *out = d[0];
    return cudaSuccess;
  }
  if (!c->tau_pack) {
    cudaError_t e = dev_alloc(c, &c->tau_pack, (size_t)(9 * ld));
    if (e != cudaSuccess) return e;
  }
  for (int a = 0; a < 9; ++a) {
    cudaError_t e = cudaMemcpyAsync(c->tau_pack + a * ld, d[a], sizeof(double) * ld,
                                    cudaMemcpyDeviceToDevice, c->st);
    if (e != cudaSuccess) return e;
  }
  *out = c->tau_pack;
  return cudaSuccess;
}

// ityprk != 0 (multigrid forcing, sch_roe.f90:1466-1481 and the other flux
// routines): ff(n, 1:5) -= u(n, 1:5) on the real cells of block l
__global__ void __launch_bounds__(kTile) k_forcing_sub(const Blk* __restrict__ blks, Space sp,
                                                       long long ld,
                                                       const double* __restrict__ u,
                                                       double* __restrict__ ff) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
#pragma unroll
  for (int a = 0; a < 5; ++a) ff[a * ld + n] = ff[a * ld + n] - u[a * ld + n];
}

// ityprk != 0 in implimf_3d.f90:249-264 / implimf_eu: the right-hand side
// -u - ff; out = u + ff on the real cells (-(u + ff) = -u - ff exactly)
__global__ void __launch_bounds__(kTile) k_forcing_add(const Blk* __restrict__ blks, Space sp,
                                                       long long ld,
                                                       const double* __restrict__ u,
                                                       const double* __restrict__ ff,
                                                       double* __restrict__ out) {
  int b, i, j, k;
  if (!space_elem(sp, threadIdx.x, b, i, j, k)) return;
  const long long n = cell_index(blks[b], i, j, k);
#pragma unroll
  for (int a = 0; a < 5; ++a) out[a * ld + n] = u[a * ld + n] + ff[a * ld + n];
}

cudaError_t forcing_sub(cns_ctx* c, int l, const double* u, double* ff) {
  const Space sp = c->cells.view(l - 1);
  if (sp.ntiles > 0)
    k_forcing_sub<<<sp.ntiles, kTile, 0, c->st>>>(c->d_blks, sp, c->lay.ld, u, ff);
  return cudaGetLastError();
}

cudaError_t forcing_add(cns_ctx* c, int l, const double* u, const double* ff, double* out) {
  const Space sp = c->cells.view(l - 1);
  if (sp.ntiles > 0)
    k_forcing_add<<<sp.ntiles, kTile, 0, c->st>>>(c->d_blks, sp, c->lay.ld, u, ff, out);
  return cudaGetLastError();
}

// the viscous halves of the HLLC faces (sch_hllc with the stresses) and of
// the WENO5 faces, and WENO5's zero stresses for the Euler equations,
// allocated when the scheme first asks for them (never inside a graph
// capture)
cudaError_t ensure_hllc_v(cns_ctx* c) {
  const bool weno = c->sc.ischema == 12;
  if (!c->w.V && (weno || (c->sc.ischema == 14 && c->sc.ns))) {
    cudaError_t e = dev_alloc(c, &c->w.V, (size_t)(12 * c->lay.ld));
    if (e != cudaSuccess) return e;
  }
  if (!c->w.tau0 && weno && !c->sc.ns) return dev_alloc(c, &c->w.tau0, (size_t)(9 * c->lay.ld));
  return cudaSuccess;
}

// the fused iteration of WENO5 with the Euler equations reads the zero
// stresses the reference leaves there (inivec.f90:93; zvisqc does not run),
// not the bound stress array
bool weno_euler(const cns_ctx* c) { return c->sc.ischema == 12 && !c->sc.ns; }

cudaError_t ensure_dis(cns_ctx* c) {
  if (c->w.dis) return cudaSuccess;
  return dev_alloc(c, &c->w.dis, (size_t)(5 * c->lay.ld));
}

bool jameson(const cns_ctx* c) { return c->sc.ischema <= 4; }

cudaError_t ensure_dtpart(cns_ctx* c) {
  if (c->w.dtpart) return cudaSuccess;
  return dev_alloc(c, &c->w.dtpart, (size_t)(c->cells.ntiles + 1));
}

// the global time step of kdtl = 0 after the local ones (chrono.f90:113-151)
cudaError_t global_dt(cns_ctx* c) {
  if (c->sc.kdtl != 0) return cudaSuccess;
  return launch_dt_global(c->d_blks, c->cells.view(-1), c->lay.ncells, c->sc.dt1min,
                          c->state.dt, c->w.dtpart, c->w.dtpart + c->cells.ntiles, c->w.status,
                          c->st);
}

// the Jameson dissipation of the fused iteration: rfve on the first cycle,
// rfvc, then dissip_jameson into w.dis (atsch_num.f90:448-508, before rbord)
cudaError_t jameson_dissipation(cns_ctx* c, bool first) {
  const cns_state_t& s = c->state;
  const long long ld = c->lay.ld;
  cudaError_t e = cudaSuccess;
  if (first) e = launch_ghost_refresh(c->bd, 1, s.v, ld, s.pression, s.ztemp, s.cson, c->st);
  if (e == cudaSuccess)
    e = launch_ghost_refresh(c->bd, 2, s.v, ld, s.pression, s.ztemp, s.cson, c->st);
  if (e == cudaSuccess)
    e = launch_dissip_jameson(c->d_blks, c->faces, c->cells.view(-1), -1,
                              s.v, ld, s.pression, s.cson, s.sn, c->w.G, c->w.dis, c->st);
  return e;
}

// the Spalart-Allmaras scratch, allocated on first use
cudaError_t ensure_sa_step(cns_ctx* c) {
  const size_t ld = (size_t)c->lay.ld;
  cudaError_t e = cudaSuccess;
  if (!c->sa_gr) e = dev_alloc(c, &c->sa_gr, 6 * ld, false);
  if (e == cudaSuccess && !c->sa_sc) e = dev_alloc(c, &c->sa_sc, 3 * ld, false);
  if (e == cudaSuccess && !c->sa_w) e = dev_alloc(c, &c->sa_w, 20 * ld, false);
  if (e == cudaSuccess && !c->sa_dv) e = dev_alloc(c, &c->sa_dv, 9 * ld);
  if (e == cudaSuccess && !c->sa_fd) e = dev_alloc(c, &c->sa_fd, 6 * ld);
  if (e == cudaSuccess && !c->sa_ts) e = dev_alloc(c, &c->sa_ts, 2 * ld);
  if (e == cudaSuccess && !c->sa_cfke) e = dev_alloc(c, &c->sa_cfke, ld);
  return e;
}

// the flat range indc(1,1,1)..indc(ni-1,nj-1,nk-1) of block l (the whole
// span for l = 0 is the union: first block's start to last block's end)
void fludc_range(cns_ctx* c, int l, long long& n0, long long& n1) {
  const Blk& F = c->lay.blks[l == 0 ? 0 : l - 1];
  const Blk& L = c->lay.blks[l == 0 ? c->lay.blks.size() - 1 : l - 1];
  n0 = F.npc + 1 + F.nid + F.nijd;
  n1 = L.npc + (L.ni - 1) + (long long)(L.nj - 1) * L.nid + (long long)(L.nk - 1) * L.nijd;
}

// met_num.f90:145-790 for equat '1SA ' (kcutke 2, kfludis 2, ksecmb 2, kcmut
// 2, kditur 2, klroe 2, kparoi 0) on the bound (ld, 7) state, after rbord:
// turbulence ghosts; per block, in block order (met_smsa.f90:177 reads
// txxf5x at the block-local index, so a later block sees block 1's scaled
// densities), the velocity gradients, grad(s6/s1) and grad(s7/s1), the
// source and the diffusion densities; their ghosts; then over every block
// the Roe dissipation, the explicit balance, the implicit line Jacobi, the
// clip and mut = v6 fv1.  dt is this iteration's mean-flow time step.  The
// reduced-precision forms solve the line systems with one reciprocal per
// step (same fixed point); precision 0 is the bit-exact FP64 step.
// met_num.f90:628-641: met_roe2oh (Harten) when |epsroe| > tiny(1.)
int sa_harten(const cns_ctx* c) { return fabs(c->epsroe) > 1.17549435082228751e-38 ? 1 : 0; }

// the wall-law constants (rbord.f90:377-379) with the SA cv1
// (atlecdon.f90:193-204) and the nu~ floor of the step
WallLaw wall_law(const cns_ctx* c) { return WallLaw{0.41, 5.25, 11.13, 7.1, c->sa_epsk}; }

// lpsa.f90:70-100 for block b (0-based): lpsa1 on its 'lp2' walls in
// boundary order
cudaError_t enqueue_lpsa(cns_ctx* c, int b, double* v, const double* mu, double* mut,
                         const double* dist, const double* temp) {
  cudaError_t e = cudaSuccess;
  for (const auto& w : c->lp2)
    if (w.blk == b && e == cudaSuccess)
      e = launch_lpsa1(c->bd, w.e0, w.cnt, c->ph, wall_law(c), c->lay.ld, v, mu, mut, dist,
                       temp, c->st);
  return e;
}

// cllparoi1.f90:89-124 (atsch_num.f90:579-604, after zvisqc): lparoi1 on
// every 'lp2' wall in boundary order
cudaError_t enqueue_cllparoi1(cns_ctx* c, const double* v, const double* mu, const double* mut,
                              const double* dist, const double* temp, double* tau) {
  cudaError_t e = cudaSuccess;
  for (const auto& w : c->lp2)
    if (e == cudaSuccess)
      e = launch_lparoi1(c->bd, w.e0, w.cnt, c->ph, wall_law(c), c->lay.ld, v, mu, mut, dist,
                         temp, tau, c->st);
  return e;
}

// met_num.f90:145-790 for '2JL ' on the bound (ld, 7) state, after rbord:
// met_bord; per block teq_gradv, met_prod, met_gradtr, met_smke (met_exgr,
// met_bark, met_bare, met_smkes) and met_fludc; met_rbse + met_rbsc; then
// over all blocks met_roe2o(h), sch_turb, impli2_eqt_3d (cmt = 1,
// impli2_eqt_3d.f90:85), met_cutke; met_kemut
cudaError_t enqueue_met_num_ke(cns_ctx* c) {
  const cns_state_t& s = c->state;
  const long long ld = c->lay.ld;
  const int nb = (int)c->lay.blks.size();
  double* fd = c->sa_fd;
  double* const fdw[6] = {fd, fd + ld, fd + 2 * ld, fd + 3 * ld, fd + 4 * ld, fd + 5 * ld};
  const double* const fdr[6] = {fdw[0], fdw[1], fdw[2], fdw[3], fdw[4], fdw[5]};
  double* ts6 = c->sa_ts;
  double* ts7 = c->sa_ts + ld;
  cudaError_t e = launch_turb_bord(c->bd, s.v, ld, c->ke_rokinf, c->ke_roeinf, c->st);
  for (int b = 0; b < nb && e == cudaSuccess; ++b) {
    const Space cb = c->cells.view(b);
    long long b0, b1, n0, n1;
    block_range(c, b + 1, b0, b1);
    fludc_range(c, b + 1, n0, n1);
    e = launch_teq_grads(c->d_blks, cb, 0, 3, s.v, nullptr, ld, s.sn, s.vol, c->sa_dv, c->sa_sc,
                         b0, b1, c->st);
    if (e == cudaSuccess)
      e = launch_met_prod(c->d_blks, cb, ld, s.mut, s.v, c->sa_dv, c->ke_tprod, c->st);
    for (int q = 0; q < 6 && e == cudaSuccess; ++q)
      e = cudaMemsetAsync(fdw[q] + n0, 0, sizeof(double) * (size_t)(n1 - n0 + 1), c->st);
    if (e == cudaSuccess)
      e = launch_teq_grads(c->d_blks, cb, 2, 2, s.v, nullptr, ld, s.sn, s.vol, fd, c->sa_sc, b0,
                           b1, c->st);
    if (e == cudaSuccess) e = launch_exgr(c->lay.blks[b], ld, c->sa_dv, c->st);
    if (e == cudaSuccess)
      e = launch_smke(c->d_blks, cb, ld, s.v, s.mu, s.mut, s.sn, s.vol, c->ke_tprod, c->sa_dv,
                      c->ke_w, ts6, ts7, c->sa_cfke, b0, b1, c->st);
    if (e == cudaSuccess) e = launch_fludc(n0, n1, s.mu, s.mut, fdw, c->alfak, c->alfae, c->st);
  }
  if (e == cudaSuccess) e = launch_fd_ghosts(c->bd, fdw, c->st);
  const Space all = c->cells.view(-1);
  if (e == cudaSuccess)
    e = launch_roe2o(c->d_blks, c->faces, c->cells_ext.view(-1), -1, sa_harten(c), c->epsroe,
                     c->ph.gam, c->ph.gam1, s.v, ld, s.sn, c->w.G, s.d, c->st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s.u + 5 * ld, 0, sizeof(double) * c->lay.ncells, c->st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s.u + 6 * ld, 0, sizeof(double) * c->lay.ncells, c->st);
  if (e == cudaSuccess)
    e = launch_sch_turb(c->d_blks, c->faces, all, -1, s.v, ld, fdr, ts6, ts7, s.d, s.sn, s.vol,
                        c->w.G, s.u, c->st);
  if (e == cudaSuccess)
    e = launch_impli2(c->d_blks, c->faces, c->lines, all, -1, ld, s.u, s.dt, s.v, s.mu, s.mut,
                      c->sa_cfke, s.sn, s.vol, 1.0, c->sa_w, c->sc.precision != 0, nullptr, 0,
                      c->st);
  if (e == cudaSuccess) e = launch_cutke(c->d_blks, all, ld, s.v, c->ke_epsk, c->ke_epse, c->st);
  if (e == cudaSuccess) e = launch_kemut(c->d_blks, all, ld, s.v, s.mu, s.mut, c->st);
  return e;
}

cudaError_t enqueue_met_num(cns_ctx* c) {
  if (c->ke_on) return enqueue_met_num_ke(c);
  const cns_state_t& s = c->state;
  const long long ld = c->lay.ld;
  const int nb = (int)c->lay.blks.size();
  double* fd = c->sa_fd;
  double* const fdw[6] = {fd, fd + ld, fd + 2 * ld, fd + 3 * ld, fd + 4 * ld, fd + 5 * ld};
  const double* const fdr[6] = {fdw[0], fdw[1], fdw[2], fdw[3], fdw[4], fdw[5]};
  double* ts6 = c->sa_ts;
  double* ts7 = c->sa_ts + ld;
  cudaError_t e = launch_turb_bord(c->bd, s.v, ld, c->sa_rokinf, c->sa_roeinf, c->st);
  for (int b = 0; b < nb && e == cudaSuccess; ++b) {
    const Space cb = c->cells.view(b);
    long long b0, b1;
    block_range(c, b + 1, b0, b1);
    e = launch_teq_grads(c->d_blks, cb, 0, 3, s.v, nullptr, ld, s.sn, s.vol, c->sa_dv, c->sa_sc,
                         b0, b1, c->st);
    // met_num.f90:193-279: the wall law of the block's 'lp2' walls after
    // teq_gradv and met_prod, before met_gradtr reads rho nu~
    if (e == cudaSuccess) e = enqueue_lpsa(c, b, s.v, s.mu, s.mut, c->sa_dist, s.ztemp);
    // met_gradtr.f90:97-104 writes the whole flat range of the real cells,
    // zero on the ghost cells inside it (what the next block's met_smsa
    // reads there through its block-local index)
    long long n0, n1;
    fludc_range(c, b + 1, n0, n1);
    for (int q = 0; q < 6 && e == cudaSuccess; ++q)
      e = cudaMemsetAsync(fdw[q] + n0, 0, sizeof(double) * (size_t)(n1 - n0 + 1), c->st);
    if (e == cudaSuccess)
      e = launch_teq_grads(c->d_blks, cb, 2, 2, s.v, nullptr, ld, s.sn, s.vol, fd, c->sa_sc, b0,
                           b1, c->st);
    if (e == cudaSuccess)
      e = launch_teq_grads(c->d_blks, cb, 1, 1, s.v, s.v + 5 * ld, ld, s.sn, s.vol, c->sa_gr,
                           nullptr, 0, 0, c->st);
    if (e == cudaSuccess)
      e = launch_teq_grads(c->d_blks, cb, 1, 1, s.v, s.v, ld, s.sn, s.vol, c->sa_gr + 3 * ld,
                           nullptr, 0, 0, c->st);
    if (e == cudaSuccess)
      e = launch_smsa(c->d_blks, cb, ld, s.v, s.mu, c->sa_dist, c->sa_dv, c->sa_gr,
                      c->sa_gr + 3 * ld, fdr, ts6, ts7, c->sa_cfke, c->sa_fix, c->st);
    if (e == cudaSuccess) e = launch_fludcsa(n0, n1, s.v + 5 * ld, s.mu, fdw, c->sigma, c->st);
  }
  if (e == cudaSuccess) e = launch_fd_ghosts(c->bd, fdw, c->st);
  const Space all = c->cells.view(-1);
  if (e == cudaSuccess)
    e = launch_roe2o(c->d_blks, c->faces, c->cells_ext.view(-1), -1, sa_harten(c), c->epsroe,
                     c->ph.gam, c->ph.gam1, s.v, ld, s.sn, c->w.G, s.d, c->st);
  // sch_turb.f90:59-66 zeroes u(:,6:7) over every block
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s.u + 5 * ld, 0, sizeof(double) * c->lay.ncells, c->st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s.u + 6 * ld, 0, sizeof(double) * c->lay.ncells, c->st);
  if (e == cudaSuccess)
    e = launch_sch_turb(c->d_blks, c->faces, all, -1, s.v, ld, fdr, ts6, ts7, s.d, s.sn, s.vol,
                        c->w.G, s.u, c->st);
  if (e == cudaSuccess)
    e = launch_impli2(c->d_blks, c->faces, c->lines, all, -1, ld, s.u, s.dt, s.v, s.mu, s.mut,
                      c->sa_cfke, s.sn, s.vol, 1.0, c->sa_w, c->sc.precision != 0,
                      c->d_lp2_ni, c->n_lp2_ni, c->st);
  if (e == cudaSuccess) e = launch_cutsa(c->d_blks, all, s.v, ld, c->sa_epsk, c->st);
  if (e == cudaSuccess) e = launch_samut(c->d_blks, all, s.v + 5 * ld, s.mu, s.mut, c->st);
  return e;
}

// one pseudo-time iteration on the bound state (atsch_num.f90:245-1134 for
// ischema = 7, kmf = 1, steady; dt_on: the time step is recomputed, else
// the previous one is kept; ischema <= 4: the Jameson dissipation before
// rbord, sch_jameson for the residual)
cudaError_t enqueue_step(cns_ctx* c, bool first, bool dt_on) {
  const cns_state_t& s = c->state;
  const long long ld = c->lay.ld;
  const Space all = c->cells.view(-1);
  // zpres (+ zvismo), and chronos when the time step is recomputed, in one pass
  cudaError_t e =
      dt_on ? launch_zpres_chronos(c->d_blks, all, c->ph, c->sc, s.v, ld, s.pression, s.ztemp,
                                   s.cson, s.mu, s.mut, s.dt, s.sn, s.vol, c->w.status, c->st)
            : launch_zpres(c->d_blks, all, c->ph, c->sc.ns, s.v, ld, s.pression, s.ztemp,
                           s.cson, s.mu, c->w.status, c->st);
  if (e == cudaSuccess && dt_on) e = global_dt(c);
  if (e == cudaSuccess && jameson(c)) e = jameson_dissipation(c, first);
  if (e == cudaSuccess)
    e = launch_rbord(c->bd, c->ph, s.v, ld, s.pression, s.ztemp, s.cson, c->n_idd_ent,
                     c->d_idd_ents, c->d_idd_masks, c->st);
  if (e == cudaSuccess && (c->sa_on || c->ke_on)) e = enqueue_met_num(c);
  if (e == cudaSuccess) e = launch_prim(0, c->lay.ncells, s.v, ld, c->w.prim, c->st);
  if (e == cudaSuccess && c->sc.ns) {
    e = launch_grad(c->d_blks, all, c->ph, s.v, c->w.prim, ld, s.mu, s.mut, s.tau, s.sn,
                    s.vol, s.ztemp, c->st);
    if (e == cudaSuccess) e = launch_tau_ghosts(c->bd, s.tau, ld, c->st);
    if (e == cudaSuccess)
      e = enqueue_cllparoi1(c, s.v, s.mu, s.mut, c->sa_dist, s.ztemp, s.tau);
  }
  if (e == cudaSuccess) {
    if (jameson(c))
      e = launch_sch_jameson(c->d_blks, c->faces, all, -1, c->sc.ns, c->ph.pinfl, s.v, ld,
                             s.pression, s.tau, s.sn, c->w.dis, c->w.G, s.u, nullptr, c->st);
    else
      e = residual(c, -1, s.u, s.v, weno_euler(c) ? c->w.tau0 : s.tau, s.sn, s.pression);
  }
  if (e == cudaSuccess && c->sc.kfmg == 3) e = enqueue_dual(c, nullptr);
  if (e == cudaSuccess)
    e = launch_implicit(c->d_blks, all, c->tiles64.view(-1), c->faces, -1, c->ph, c->sc,
                        !c->sc.ns,
                        c->sc.lmax, s.u, s.dt, s.v, nullptr, s.mu, s.mut, s.sn, s.vol,
                        s.pression, s.cson, c->w, 1, c->st);
  if (e == cudaSuccess)
    e = launch_norm_finalize(c->d_blks, c->d_cells_tile0, 0, (int)c->lay.blks.size(),
                             c->w.normpart, c->w.blocksum, c->w.norms, c->st);
  return e;
}

// the FP32 sweep's arguments (box staging unless cp.async staging is selected)
Sweep32 sweep32_args(cns_ctx* c) {
  Sweep32 a{};
  a.u = c->w.u32;
  a.st = c->w.st32;
  a.coefdiag = c->w.coefdiag32;
  a.maps = c->staging32 == 0 ? c->w.sweep_maps : nullptr;
  a.map_st = nullptr;
  a.nblk = (int)c->lay.blks.size();
  a.status = c->w.status;
  return a;
}

// the single-precision scratch of the mixed form, allocated on first use
cudaError_t ensure_mixed(cns_ctx* c) {
  Work& w = c->w;
  if (w.mixed_ready) return cudaSuccess;
  const long long ld = c->lay.ld;
  cudaError_t e = dev_alloc(c, &w.v32, (size_t)(5 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.prim32, (size_t)(3 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.ps32, (size_t)ld);
  if (e == cudaSuccess) e = dev_alloc(c, &w.tau32, (size_t)(9 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.sn32, (size_t)(9 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.G32, (size_t)(15 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.R32, (size_t)(15 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.u32, (size_t)(5 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.coefe32, (size_t)(3 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.coefdiag32, (size_t)ld);
  // the sweep's padded arrays (zeroed: their padding and ghost cells are
  // never written, and the sweep masks them)
  const long long ldp = c->lay.ldp;
  for (int q = 0; q < 2 && e == cudaSuccess; ++q) e = dev_alloc(c, &w.d32pp[q], (size_t)(5 * ldp));
  if (e == cudaSuccess) e = dev_alloc(c, &w.st32, (size_t)(6 * ldp));
  if (e == cudaSuccess) e = dev_alloc(c, &w.cq32, (size_t)ld);
  if (e == cudaSuccess) e = dev_alloc(c, &w.cv32, (size_t)ld);
  if (e == cudaSuccess) {
    std::vector<unsigned char> maps;
    e = encode_sweep32_maps(c->lay.blks, w.st32, w.d32pp, maps);
    if (e == cudaSuccess) e = upload(c, reinterpret_cast<unsigned char**>(&w.sweep_maps),
                                     maps.data(), maps.size());
  }
  if (e == cudaSuccess) e = dev_alloc(c, &w.corr, (size_t)(5 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.ur32, (size_t)(5 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &w.snc32, (size_t)(3 * ld));
  if (e == cudaSuccess) w.mixed_ready = true;
  c->tiles32.faces = w.snc32;
  return e;
}

// the FP32 face areas of the bound state's sn and the face lanes of the FP32
// sweep's pack
cudaError_t refresh_sn32(cns_ctx* c, const double* sn) {
  cudaError_t e = launch_to_float(sn, c->w.sn32, 9 * c->lay.ld, c->st);
  if (e == cudaSuccess)
    e = launch_pack_faces32(c->d_blks, (int)c->lay.blks.size(), c->lay.ncells, c->w.sn32,
                            c->w.snc32, c->st);
  c->tiles32.faces = c->w.snc32;
  return e;
}

// one reduced-precision iteration on the bound state.  kMixed: FP64 residual
// (face fluxes with FMA contraction), FP32 sweeps (precision 1).  kDefectRefresh / kDefectRegular (precision 2):
// FP32 face fluxes; the refresh iteration also evaluates the FP64 residual,
// advances with it and stores corr = R64 - R32 for the regular iterations.
enum MixedMode { kMixed, kDefectRefresh, kDefectRegular };

cudaError_t enqueue_step_mixed(cns_ctx* c, MixedMode mode, bool first, bool dt_on) {
  const cns_state_t& s = c->state;
  Work& w = c->w;
  const long long ld = c->lay.ld;
  const Space all = c->cells.view(-1);
  const bool lim = c->sc.ns && c->sc.ilim == 1;
  // zpres (+ zvismo), and chronos when the time step is recomputed, in one pass
  cudaError_t e =
      dt_on ? launch_zpres_chronos(c->d_blks, all, c->ph, c->sc, s.v, ld, s.pression, s.ztemp,
                                   s.cson, s.mu, s.mut, s.dt, s.sn, s.vol, w.status, c->st)
            : launch_zpres(c->d_blks, all, c->ph, c->sc.ns, s.v, ld, s.pression, s.ztemp,
                           s.cson, s.mu, w.status, c->st);
  if (e == cudaSuccess && dt_on) e = global_dt(c);
  if (e == cudaSuccess && jameson(c)) e = jameson_dissipation(c, first);
  if (e == cudaSuccess)
    e = launch_rbord(c->bd, c->ph, s.v, ld, s.pression, s.ztemp, s.cson, c->n_idd_ent,
                     c->d_idd_ents, c->d_idd_masks, c->st);
  if (e == cudaSuccess && (c->sa_on || c->ke_on)) e = enqueue_met_num(c);
  if (e == cudaSuccess) {
    PrimShadow sh{};
    sh.v32 = mode == kMixed ? nullptr : w.v32;
    sh.prim32 = w.prim32;
    sh.ps32 = w.ps32;
    sh.blks = c->d_blks;
    sh.nblk = (int)c->lay.blks.size();
    sh.st32 = w.st32;
    sh.cq32 = w.cq32;
    sh.cv32 = w.cv32;
    sh.cson = s.cson;
    sh.mu = s.mu;
    sh.mut = s.mut;
    sh.vol = s.vol;
    sh.gp = (float)(c->ph.gam / c->ph.pr);
    sh.gpt = (float)(c->ph.gam / c->ph.prt);
    sh.eu = !c->sc.ns;
    e = launch_prim_shadow(c->lay.ncells, s.v, ld, w.prim, s.pression, sh, c->st);
  }
  if (e == cudaSuccess && c->sc.ns) {
    e = launch_grad(c->d_blks, all, c->ph, s.v, w.prim, ld, s.mu, s.mut, s.tau, s.sn, s.vol,
                    s.ztemp, c->st);
    if (e == cudaSuccess) e = launch_tau_ghosts(c->bd, s.tau, ld, c->st);
    if (e == cudaSuccess)
      e = enqueue_cllparoi1(c, s.v, s.mu, s.mut, c->sa_dist, s.ztemp, s.tau);
  }
  if (mode != kMixed) {
    // single-precision face fluxes
    if (e == cudaSuccess && c->sc.ns) e = launch_to_float(s.tau, w.tau32, 9 * ld, c->st);
    if (e == cudaSuccess && lim)
      e = launch_ratio_t<float>(c->d_blks, c->lines, -1, w.v32, w.prim32, ld, w.ps32, w.R32,
                                c->st);
    if (e == cudaSuccess)
      e = launch_face_flux_t<float>(c->d_blks, c->faces, -1, c->ph, c->sc, w.v32, w.prim32,
                                    ld, w.ps32, w.tau32, w.sn32, w.R32, w.G32, c->st,
                                    nullptr);
  }
  if (mode == kDefectRegular) {
    if (e == cudaSuccess)
      e = launch_accumulate_t<float>(c->d_blks, all, w.G32, ld, w.corr, s.u, w.u32, c->st,
                                     nullptr);
  } else {
    // the FP64 residual; the defect refresh also keeps R32 alone for corr
    if (e == cudaSuccess && mode == kDefectRefresh)
      e = launch_accumulate_t<float>(c->d_blks, all, w.G32, ld, nullptr, w.ur32, nullptr,
                                     c->st, nullptr);
    if (jameson(c)) {
      if (e == cudaSuccess)
        e = launch_sch_jameson(c->d_blks, c->faces, all, -1, c->sc.ns, c->ph.pinfl, s.v, ld,
                               s.pression, s.tau, s.sn, w.dis, w.G, s.u, w.u32, c->st);
    } else if (c->sc.ischema == 12) {
      if (e == cudaSuccess)
        e = launch_weno5(c->d_blks, all, c->ph, c->sc.weno_fix, s.v, ld, s.pression,
                         weno_euler(c) ? w.tau0 : s.tau, s.sn, w.G, w.V, s.u, w.u32, c->st);
    } else {
      if (e == cudaSuccess && lim)
        e = launch_ratio(c->d_blks, c->lines, -1, s.v, w.prim, ld, s.pression, w.R, c->st);
      if (c->res_fused && residual_fused_ok(c->sc)) {
        if (e == cudaSuccess)
          e = launch_residual_fused_fma(c->d_blks, c->tiles_res.view(-1), c->ph, c->sc, s.v,
                                        w.prim, ld, s.pression, s.tau, s.sn, w.R, s.u, w.u32,
                                        c->st);
      } else {
        if (e == cudaSuccess)
          e = launch_face_flux_fma(c->d_blks, c->faces, -1, c->ph, c->sc, s.v, w.prim, ld,
                                   s.pression, s.tau, s.sn, w.R, w.G, c->st, w.V);
        if (e == cudaSuccess)
          e = launch_accumulate_t<double>(c->d_blks, all, w.G, ld, nullptr, s.u, w.u32, c->st,
                                          w.V);
      }
    }
    if (e == cudaSuccess && mode == kDefectRefresh)
      e = launch_defect(c->d_blks, all, ld, s.u, w.ur32, w.corr, c->st);
  }
  if (e == cudaSuccess && c->sc.kfmg == 3) e = enqueue_dual(c, w.u32);
  // single-precision coefficients and implicit sweeps, FP64 update
  if (e == cudaSuccess)
    e = launch_coefficients32(c->d_blks, all, !c->sc.ns, ld,
                              c->sc.kfmg == 3 ? c->sc.dt1min : 0., s.dt, s.vol, w.cq32,
                              w.cv32, w.sn32, w.coefe32, w.coefdiag32, w.snc32, w.u32,
                              c->sc.lmax >= 1 ? w.d32pp[0] : nullptr, c->st);
  int cur = 0;
  if (e == cudaSuccess)
    e = launch_sweeps32(c->tiles32.view(-1), c->d_blks, c->ph, c->sc, !c->sc.ns, c->sc.lmax,
                        ld, c->lay.ldp, sweep32_args(c), w.d32pp, &cur, c->st);
  if (e == cudaSuccess)
    e = launch_update32(c->d_blks, all, ld, w.d32pp[cur], s.v, s.dt, w.normpart, c->st);
  if (e == cudaSuccess)
    e = launch_norm_finalize(c->d_blks, c->d_cells_tile0, 0, (int)c->lay.blks.size(),
                             w.normpart, w.blocksum, w.norms, c->st);
  return e;
}

// The sweep autotuner: times one 2.5D sweep of every patch shape and plane
// count on the current iteration's data (u, coefficients and iterate of the
// step that just ran; the sweep only writes the scratch iterate) and keeps
// the fastest tile list.  FP64 results do not depend on the tiling.
constexpr int kTuneKc[] = {2, 4, 8, 16, 32};

template <class T>
cudaError_t time_sweep(cns_ctx* c, Tiles tl, const T* u, const T* v, const T* prim,
                       const T* ps, const T* sn, const T* coefe, const T* coefdiag,
                       const T* din, T* dout, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
  const int q = c->sc.ns ? 0 : c->sc.qfix_dfez;
  const long long ld = c->lay.ld;
  cudaError_t e = launch_jacobi_25d_t<T>(c->d_blks, tl, c->ph, q, !c->sc.ns, ld, u, v, prim, ps,
                                         sn, coefe, coefdiag, din, dout, c->st);
  if (e == cudaSuccess) e = cudaEventRecord(e0, c->st);
  for (int r = 0; r < 3 && e == cudaSuccess; ++r)
    e = launch_jacobi_25d_t<T>(c->d_blks, tl, c->ph, q, !c->sc.ns, ld, u, v, prim, ps, sn,
                               coefe, coefdiag, din, dout, c->st);
  if (e == cudaSuccess) e = cudaEventRecord(e1, c->st);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  return e;
}

// the FP32 sweep timed the same way (iterate 0 -> iterate 1)
cudaError_t time_sweep32(cns_ctx* c, Tiles tl, cudaEvent_t e0, cudaEvent_t e1, float* ms) {
  const int q = c->sc.ns ? 0 : c->sc.qfix_dfez;
  const long long ld = c->lay.ld;
  const Sweep32 a = sweep32_args(c);
  float* const* d = c->w.d32pp;
  cudaError_t e = launch_sweep32_25d(c->d_blks, tl, c->ph, q, !c->sc.ns, ld, a, 0, d[0], d[1],
                                     c->st);
  if (e == cudaSuccess) e = cudaEventRecord(e0, c->st);
  for (int r = 0; r < 3 && e == cudaSuccess; ++r)
    e = launch_sweep32_25d(c->d_blks, tl, c->ph, q, !c->sc.ns, ld, a, 0, d[0], d[1], c->st);
  if (e == cudaSuccess) e = cudaEventRecord(e1, c->st);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
  return e;
}

// The tuning cache (cns_set_tune_cache): one line per tuned configuration,
//   <key> <ti> <tj> <kc>
// key = GPU name (blanks as '_') | SM count | sweep precision (f64 / f32) |
// equations (eu / ns) | floor(log2(real cells)) | floor(log2(blocks)) |
// floor(log2(cells of the smallest block)).  A key found in the file is used
// as it is, without timing, so a given cache file always gives the same
// tiling; a missing key is tuned on the data and appended.
std::string tune_key(cns_ctx* c, bool fp32) {
  cudaDeviceProp pr{};
  if (cudaGetDeviceProperties(&pr, c->device) != cudaSuccess) return "";
  std::string name(pr.name);
  for (char& ch : name)
    if (ch == ' ' || ch == '|') ch = '_';
  auto lg = [](long long x) {
    int r = 0;
    while (x > 1) {
      x >>= 1;
      ++r;
    }
    return r;
  };
  long long smallest = -1;
  for (const Blk& B : c->lay.blks) {
    const long long n = (long long)(B.ni - 1) * (B.nj - 1) * (B.nk - 1);
    if (smallest < 0 || n < smallest) smallest = n;
  }
  char buf[512];
  std::snprintf(buf, sizeof buf, "%s|%d|%s|%s|%d|%d|%d", name.c_str(), pr.multiProcessorCount,
                fp32 ? "f32" : "f64", c->sc.ns ? "ns" : "eu", lg(c->lay.nreal),
                lg((long long)c->lay.blks.size()), lg(smallest));
  return buf;
}

bool tune_cache_lookup(cns_ctx* c, const std::string& key, int* ti, int* tj, int* kc) {
  FILE* f = std::fopen(c->tune_cache.c_str(), "r");
  if (!f) return false;
  char k[512];
  int a, b, d;
  bool found = false;
  while (std::fscanf(f, "%511s %d %d %d", k, &a, &b, &d) == 4) {
    if (key == k) {  // the last entry of a key wins
      *ti = a;
      *tj = b;
      *kc = d;
      found = true;
    }
  }
  std::fclose(f);
  if (!found) return false;
  for (int sh = 0; sh < kSweepShapes; ++sh)
    if (kSweepShape[sh][0] == *ti && kSweepShape[sh][1] == *tj && *kc >= 1) return true;
  return false;  // an entry this build has no kernel for: tune again
}

cudaError_t tune_sweeps(cns_ctx* c, bool fp32) {
  const cns_state_t& s = c->state;
  Work& w = c->w;
  TileBuf& best = fp32 ? c->tiles32 : c->tiles64;
  const std::string key = c->tune_cache.empty() ? std::string() : tune_key(c, fp32);
  {
    int cti, ctj, ckc;
    if (!key.empty() && tune_cache_lookup(c, key, &cti, &ctj, &ckc)) {
      cudaError_t e = build_tiles(c, best, cti, ctj, ckc);
      if (e == cudaSuccess && fp32) persistent_sweep32(c);
      if (e == cudaSuccess) {
        (fp32 ? c->tuned32 : c->tuned64) = true;
        (fp32 ? c->tune_src32 : c->tune_src64) = 2;
      }
      return e;
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float best_ms = 1e30f;
  int bti = best.ti, btj = best.tj, bkc = best.kc;
  TileBuf cand;
  for (int sh = 0; sh < kSweepShapes && e == cudaSuccess; ++sh)
    for (int kc : kTuneKc) {
      e = build_tiles(c, cand, kSweepShape[sh][0], kSweepShape[sh][1], kc);
      if (e != cudaSuccess) break;
      if (fp32) {  // timed as it runs: the persistent launch
        const int per_sm =
            sweep_f32_blocks_per_sm(cand.ti, cand.tj, !c->sc.ns, c->staging32 == 0);
        cand.sched = per_sm > 0 && c->nsm > 0 ? c->sched32 : nullptr;
        cand.grid = per_sm * c->nsm;
        cand.faces = w.snc32;
      }
      float ms = 0.f;
      if (fp32)
        e = time_sweep32(c, cand.view(-1), e0, e1, &ms);
      else
        e = time_sweep<double>(c, cand.view(-1), s.u, s.v, w.prim, s.pression, s.sn, w.coefe,
                               w.coefdiag, w.dpp[0], w.dpp[1], e0, e1, &ms);
      if (e != cudaSuccess) break;
      if (ms < best_ms) {
        best_ms = ms;
        bti = cand.ti;
        btj = cand.tj;
        bkc = cand.kc;
      }
    }
  dev_free(c, cand.d_tile);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e == cudaSuccess) e = build_tiles(c, best, bti, btj, bkc);
  if (e == cudaSuccess && fp32) persistent_sweep32(c);
  if (e == cudaSuccess) {
    (fp32 ? c->tuned32 : c->tuned64) = true;
    (fp32 ? c->tune_ms32 : c->tune_ms64) = best_ms / 3.f;
    (fp32 ? c->tune_src32 : c->tune_src64) = 1;
    if (!key.empty()) {
      FILE* f = std::fopen(c->tune_cache.c_str(), "a");
      if (f) {
        std::fprintf(f, "%s %d %d %d\n", key.c_str(), bti, btj, bkc);
        std::fclose(f);
      }
    }
  }
  return e;
}

// the kernel nodes of a captured graph (the launch count of one iteration)
int kernel_nodes(cudaGraph_t g) {
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return 0;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
  int k = 0;
  for (size_t q = 0; q < n; ++q) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
  }
  return k;
}

template <class F>
cudaError_t capture(cns_ctx* c, cudaGraphExec_t* out, int* nkernels, F enqueue) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t e1 = enqueue();
  cudaError_t e2 = cudaStreamEndCapture(c->st, &g);
  if (e1 != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return e1;
  }
  if (e2 != cudaSuccess) return e2;
  *nkernels = kernel_nodes(g);
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  return e;
}

// the (i, j, k) box of a file record over block B: what 0 = the real nodes,
// 1 = the real cells, 2 = the cells with the ghost layer (chdgcv.f90,
// chdacc.f90: ii1..ii2, ii1..ii2-1, ii1-1..ii2)
void io_box(const Blk& B, int what, int lo[3], int hi[3]) {
  const int n[3] = {B.ni, B.nj, B.nk};
  for (int a = 0; a < 3; ++a) {
    lo[a] = what == 2 ? 0 : 1;
    hi[a] = what == 1 ? n[a] - 1 : n[a];
  }
}

// equat(1:2) = 'ns' and equat(6:7) = 'ke' of the reference's 7-character
// equation key (blank-padded)
void equat_keys(const char* equat, bool& ns, bool& ke) {
  char q[8] = "       ";
  for (int a = 0; a < 7 && equat[a]; ++a) q[a] = equat[a];
  ns = q[0] == 'n' && q[1] == 's';
  ke = q[5] == 'k' && q[6] == 'e';
}

}  // namespace

extern "C" {

int cns_create(const cns_layout_t* layout, const cns_phys_t* phys,
               const cns_scheme_t* scheme, const cns_bnd_t* bnd, cns_ctx** out) {
  if (!layout || !phys || !scheme || !bnd || !out || layout->nblk < 1 ||
      layout->nblk > kMaxBlocks || !layout->dims)
    return CNS_EINVAL;
  cns_ctx* c = new cns_ctx();
  *out = nullptr;
  if (cudaGetDevice(&c->device) != cudaSuccess) {
    delete c;
    return CNS_ECUDA;
  }
  // layout (crdms.f90:125-158), and the padded layout of the FP32 sweep
  // arrays (a multiple of four cells per row, so of 16 bytes per plane too)
  long long off = 0, nreal = 0, poff = 0;
  for (int l = 0; l < layout->nblk; ++l) {
    Blk B{};
    B.ni = layout->dims[3 * l];
    B.nj = layout->dims[3 * l + 1];
    B.nk = layout->dims[3 * l + 2];
    if (B.ni < 2 || B.nj < 2 || B.nk < 2) {
      delete c;
      return CNS_EINVAL;
    }
    B.nid = B.ni + 2;
    B.njd = B.nj + 2;
    B.nkd = B.nk + 2;
    B.nijd = (long long)B.nid * B.njd;
    B.nnn = B.nijd * B.nkd;
    // the kernels index a block's cells with 32-bit offsets
    if (B.nnn >= (1LL << 31)) {
      delete c;
      return CNS_EINVAL;
    }
    B.npc = off;
    off += B.nnn;
    B.pid = (B.nid + 3) / 4 * 4;
    B.pnijd = (long long)B.pid * B.njd;
    B.ppc = poff;
    poff += B.pnijd * B.nkd;
    nreal += (long long)(B.ni - 1) * (B.nj - 1) * (B.nk - 1);
    c->lay.blks.push_back(B);
  }
  c->lay.ncells = off;
  c->lay.nreal = nreal;
  c->lay.ldp = poff;
  for (Blk& B : c->lay.blks) B.pld = poff;
  c->lay.ld = layout->ld > 0 ? layout->ld : off;
  if (c->lay.ld < off) {
    delete c;
    return CNS_EINVAL;
  }
  c->ph.gam = phys->gam;
  c->ph.gam1 = phys->gam - 1.;
  c->ph.pinfl = phys->pinfl;
  c->ph.pr = phys->pr;
  c->ph.prt = phys->prt;
  c->ph.cp = 1. / (phys->gam - 1.);
  c->ph.reynz = phys->reynz;
  c->ph.suth_a = phys->suth_a;
  c->ph.pa1 = phys->pa1;
  c->ph.aa1 = phys->aa1;
  c->ph.omg = phys->omg;
  int rc = cns_set_scheme(c, scheme);
  if (rc) {
    delete c;
    return rc;
  }
  auto cleanup_fail = [&](cudaError_t e, const char* what) {
    int r = cuda_fail(c, e, what);
    cns_destroy(c);
    return r;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&c->own_st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cleanup_fail(e, "stream");
  c->st = c->own_st;
  e = upload(c, &c->d_blks, c->lay.blks.data(), c->lay.blks.size());
  if (e != cudaSuccess) return cleanup_fail(e, "blocks");
  e = build_space(c, c->cells, [](const Blk& B, int x[3]) {
    x[0] = B.ni - 1; x[1] = B.nj - 1; x[2] = B.nk - 1; });
  if (e == cudaSuccess)
    e = build_space(c, c->cells_ext, [](const Blk& B, int x[3]) {
      x[0] = B.ni + 1; x[1] = B.nj + 1; x[2] = B.nk + 1; });
  if (e == cudaSuccess) e = build_tiles(c, c->tiles64, 32, 8, 8);
  if (e == cudaSuccess) e = build_tiles(c, c->tiles32, 32, 8, 8);
  if (e == cudaSuccess) e = dev_alloc(c, &c->sched32, 2);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, c->device);
  if (e == cudaSuccess) persistent_sweep32(c);
  if (e == cudaSuccess) e = build_tiles(c, c->tiles_res, kResTI, kResTJ, kResKC);
  if (e == cudaSuccess) e = init_jacobi_25d();
  for (int dir = 0; dir < 3 && e == cudaSuccess; ++dir) {
    e = build_space(c, c->faces[dir], [dir](const Blk& B, int x[3]) {
      x[0] = dir == 0 ? B.ni : B.ni - 1;
      x[1] = dir == 1 ? B.nj : B.nj - 1;
      x[2] = dir == 2 ? B.nk : B.nk - 1; });
    if (e == cudaSuccess)
      e = build_space(c, c->lines[dir], [dir](const Blk& B, int x[3]) {
        x[0] = dir == 0 ? 1 : B.ni - 1;
        x[1] = dir == 1 ? 1 : B.nj - 1;
        x[2] = dir == 2 ? 1 : B.nk - 1; });
  }
  if (e != cudaSuccess) return cleanup_fail(e, "index spaces");
  e = upload(c, &c->d_cells_tile0, c->cells.blk_tile0.data(), c->cells.blk_tile0.size());
  if (e != cudaSuccess) return cleanup_fail(e, "tiles");
  // boundaries
  const int nb = bnd->nbnd;
  const long long nl = bnd->nlist;
  if (nb < 0 || nl < 0) {
    cns_destroy(c);
    return CNS_EINVAL;
  }
  std::vector<int> ent_bnd((size_t)nl), blk0(nb);
  std::vector<long long> idd_ents, wall_ents, lp2_ni;
  for (int b = 0; b < nb; ++b) {
    const int t = bnd->type[b];
    if (t < CNS_BC_EXTR || t > CNS_BC_LP2) {
      cns_destroy(c);
      return CNS_EBC;
    }
    if (bnd->blk[b] < 1 || bnd->blk[b] > layout->nblk || bnd->face[b] < 0 ||
        bnd->face[b] > 5 || bnd->mpb[b] < 0 || bnd->mpb[b] + bnd->mmb[b] > nl) {
      cns_destroy(c);
      return CNS_EINVAL;
    }
    if (t == CNS_BC_RC) {
      const int p = bnd->partner[b];
      if (p < 0 || p >= nb || bnd->mmb[p] != bnd->mmb[b]) {
        cns_destroy(c);
        return CNS_EINVAL;
      }
    }
    blk0[b] = bnd->blk[b] - 1;
    for (int m = 0; m < bnd->mmb[b]; ++m) {
      ent_bnd[(size_t)(bnd->mpb[b] + m)] = b;
      if (t == CNS_BC_IDD) idd_ents.push_back(bnd->mpb[b] + m);
      // atcaldis3.f90:171: 'pa' and 'lp' boundaries are walls
      if (t == CNS_BC_PARA || t == CNS_BC_LP2) wall_ents.push_back(bnd->mpb[b] + m);
      if (t == CNS_BC_LP2) lp2_ni.push_back(bnd->ncin[bnd->mpb[b] + m]);
    }
    if (t == CNS_BC_LP2 && bnd->mmb[b] > 0)
      c->lp2.push_back({(long long)bnd->mpb[b], bnd->mmb[b], bnd->blk[b] - 1});
    c->h_btype.push_back(t);
  }
  for (long long q = 0; q < nl; ++q) {
    if (bnd->ncbd[q] < 0 || bnd->ncbd[q] >= off || bnd->ncin[q] < 0 || bnd->ncin[q] >= off) {
      cns_destroy(c);
      return CNS_EINVAL;
    }
  }
  c->bd.nbnd = nb;
  c->bd.nlist = nl;
  c->n_idd_ent = (long long)idd_ents.size();
  c->n_wall_ent = (long long)wall_ents.size();
  {
    int *t_, *b_, *f_, *m_, *p_, *eb_;
    long long *mpb_, *ncbd_, *ncin_;
    double *cr_, *sr_, *bc_;
    e = upload(c, &t_, bnd->type, nb);
    if (e == cudaSuccess) e = upload(c, &b_, blk0.data(), nb);
    if (e == cudaSuccess) e = upload(c, &f_, bnd->face, nb);
    if (e == cudaSuccess) e = upload(c, &mpb_, (const long long*)bnd->mpb, nb);
    if (e == cudaSuccess) e = upload(c, &m_, bnd->mmb, nb);
    if (e == cudaSuccess) e = upload(c, &p_, bnd->partner, nb);
    if (e == cudaSuccess) e = upload(c, &cr_, bnd->cosr, nb);
    if (e == cudaSuccess) e = upload(c, &sr_, bnd->sinr, nb);
    if (e == cudaSuccess) e = upload(c, &eb_, ent_bnd.data(), (size_t)nl);
    if (e == cudaSuccess) e = upload(c, &ncbd_, (const long long*)bnd->ncbd, (size_t)nl);
    if (e == cudaSuccess) e = upload(c, &ncin_, (const long long*)bnd->ncin, (size_t)nl);
    if (e == cudaSuccess) e = upload(c, &bc_, bnd->bceqt, (size_t)(5 * nl));
    if (e == cudaSuccess) e = upload(c, &c->d_idd_ents, idd_ents.data(), idd_ents.size());
    if (e == cudaSuccess) e = upload(c, &c->d_wall_ents, wall_ents.data(), wall_ents.size());
    if (e == cudaSuccess) e = upload(c, &c->d_lp2_ni, lp2_ni.data(), lp2_ni.size());
    c->n_lp2_ni = (long long)lp2_ni.size();
    if (e == cudaSuccess) e = dev_alloc(c, &c->d_idd_masks, (size_t)nb);
    if (e == cudaSuccess) e = dev_alloc(c, &c->bd.nxn, (size_t)nl);
    if (e == cudaSuccess) e = dev_alloc(c, &c->bd.nyn, (size_t)nl);
    if (e == cudaSuccess) e = dev_alloc(c, &c->bd.nzn, (size_t)nl);
    if (e == cudaSuccess) e = dev_alloc(c, &c->bd.ym, (size_t)nl);
    if (e == cudaSuccess) e = dev_alloc(c, &c->bd.zm, (size_t)nl);
    if (e != cudaSuccess) return cleanup_fail(e, "boundary tables");
    c->bd.type = t_;
    c->bd.blk = b_;
    c->bd.face = f_;
    c->bd.mpb = mpb_;
    c->bd.mmb = m_;
    c->bd.partner = p_;
    c->bd.cosr = cr_;
    c->bd.sinr = sr_;
    c->bd.ent_bnd = eb_;
    c->bd.ncbd = ncbd_;
    c->bd.ncin = ncin_;
    c->bd.bceqt = bc_;
  }
  // scratch (zeroed: ghost entries of the Jacobi iterates and of rv stay 0)
  const long long ld = c->lay.ld;
  c->w.ld = ld;
  e = dev_alloc(c, &c->w.prim, (size_t)(3 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.G, (size_t)(15 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.R, (size_t)(15 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.coefe, (size_t)(3 * ld));
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.coefdiag, (size_t)ld);
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.rv, (size_t)ld);
  for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
    e = dev_alloc(c, &c->w.dpp[q], (size_t)(5 * ld));
  }
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.normpart, (size_t)(15 * c->cells.ntiles));
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.norms, 16);
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.blocksum, (size_t)(15 * c->lay.blks.size()));
  if (e == cudaSuccess) e = ensure_hllc_v(c);
  if (e == cudaSuccess) e = dev_alloc(c, &c->w.status, 1);
  if (e == cudaSuccess) e = cudaMallocHost(&c->h_norms, 16 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost(&c->h_status, sizeof(int));
  if (e != cudaSuccess) return cleanup_fail(e, "scratch");
  *c->h_status = 0;
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cleanup_fail(e, "create");
  *out = c;
  return CNS_OK;
}

int cns_destroy(cns_ctx* c) {
  if (!c) return CNS_OK;
  drop_graphs(c);
  if (c->st) cudaStreamSynchronize(c->st);
  for (void* p : c->allocs) cudaFree(p);
  if (c->h_norms) cudaFreeHost(c->h_norms);
  if (c->h_status) cudaFreeHost(c->h_status);
  io_stage_free(c->io_stage);
  if (c->own_st) cudaStreamDestroy(c->own_st);
  delete c;
  return CNS_OK;
}

int cns_set_stream(cns_ctx* c, void* stream) {
  if (!c) return CNS_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  // work is issued on the caller's stream from now on (NULL: back to the
  // context's own stream)
  c->st = stream ? (cudaStream_t)stream : c->own_st;
  drop_graphs(c);
  return CNS_OK;
}

int cns_set_scheme(cns_ctx* c, const cns_scheme_t* s) {
  if (!c || !s) return CNS_EINVAL;
  if (s->lmax < 0 || s->muscl < 0 || (s->ilim != 0 && s->ilim != 1) ||
      s->precision < 0 || s->precision > 2 || (s->precision == 2 && s->kdefect < 1) ||
      (s->ischema != 1 && s->ischema != 7 && s->ischema != 9 && s->ischema != 14 &&
       s->ischema != 5 && s->ischema != 12) ||
      (s->ischema == 5 && !s->ns) ||
      (s->ischema != 7 && s->precision == 2) ||
      (s->kfmg != 0 && s->kfmg != 3) ||
      (s->kfmg == 3 && (!(s->dt1min > 0.) || s->kdualns < 0 || s->kdualns > 2)))
    return fail(c, CNS_EINVAL,
                "scheme: lmax >= 0, muscl >= 0, ilim in {0,1}, precision in {0,1,2}, "
                "kdefect >= 1, ischema in {1,5,7,9,12,14} (5: ns only; defect correction: Roe "
                "only), kfmg in "
                "{0,3} (3: dt1min > 0, kdualns in {0,1,2})");
  c->sc.ns = s->ns;
  c->sc.muscl = s->muscl;
  c->sc.xk = s->xk;
  c->sc.ilim = s->ilim;
  c->sc.eta = s->eta;
  c->sc.kdtl = s->kdtl;
  c->sc.dt1min = s->dt1min;
  c->sc.lmax = s->lmax;
  c->sc.qfix_dfez = s->qfix_dfez;
  c->sc.precision = s->precision;
  c->sc.kdefect = s->kdefect;
  c->sc.ischema = s->ischema;
  c->sc.ki2 = s->ki2;
  c->sc.ki4 = s->ki4;
  c->sc.ncychro = s->ncychro;
  c->sc.icychr0 = s->icychr0;
  c->sc.kfmg = s->kfmg;
  c->sc.kdualns = s->kdualns;
  c->sc.weno_fix = s->weno_fix ? 1 : 0;
  // eta(lm), ki2(lm), ki4(lm): per block when given, else the scalars
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    Blk& B = c->lay.blks[b];
    B.eta = s->eta_l ? s->eta_l[b] : s->eta;
    B.ki2 = s->ki2_l ? s->ki2_l[b] : s->ki2;
    B.ki4 = s->ki4_l ? s->ki4_l[b] : s->ki4;
  }
  if (c->d_blks)
    CK(cudaMemcpy(c->d_blks, c->lay.blks.data(), sizeof(Blk) * c->lay.blks.size(),
                  cudaMemcpyHostToDevice));
  drop_graphs(c);
  persistent_sweep32(c);  // the Euler and Navier-Stokes instantiations differ
  c->mixed_iter = 0;  // a new scheme restarts the defect refresh schedule
  if (c->w.ld > 0) CK(ensure_hllc_v(c));
  return CNS_OK;
}

const char* cns_last_error(cns_ctx* c) { return c ? c->err.c_str() : "no context"; }

int64_t cns_scratch_bytes(cns_ctx* c) { return c ? c->scratch_bytes : 0; }

int64_t cns_kernels_launched(cns_ctx* c) { return c ? c->kernels_launched : 0; }

int cns_metric(cns_ctx* c, double* x, double* y, double* z, double* sn,
               double* vol) {
  if (!c || !x || !y || !z || !sn || !vol) return CNS_EINVAL;
  CK(launch_metric(c->lay, c->d_blks, c->bd, x, y, z, sn, vol, c->st));
  if (c->w.mixed_ready && c->bound && c->state.sn == sn)
    CK(refresh_sn32(c, sn));
  CK(cudaStreamSynchronize(c->st));
  c->metric_done = true;
  c->mixed_iter = 0;
  c->ncyc = 0;
  return CNS_OK;
}

int cns_boundary_geom(cns_ctx* c, double* nxn, double* nyn, double* nzn,
                      double* ym, double* zm) {
  if (!c) return CNS_EINVAL;
  if (!c->metric_done) return fail(c, CNS_ENOTREADY, "cns_metric has not run");
  const size_t n = sizeof(double) * (size_t)c->bd.nlist;
  if (n == 0) return CNS_OK;
  CK(cudaMemcpyAsync(nxn, c->bd.nxn, n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(nyn, c->bd.nyn, n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(nzn, c->bd.nzn, n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(ym, c->bd.ym, n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(zm, c->bd.zm, n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CNS_OK;
}

int cns_zpres(cns_ctx* c, int l, const double* v, double* ps, double* temp,
              double* cson) {
  if (!c || bad_block(c, l) || !v || !ps || !temp || !cson) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dv = sg.in(v, 5 * ld);
  double* dps = sg.inout(ps, ld);
  double* dtemp = sg.inout(temp, ld);
  double* dcson = sg.inout(cson, ld);
  CK(sg.err);
  CK(launch_zpres(c->d_blks, c->cells.view(l - 1), c->ph, 0, dv, ld, dps, dtemp, dcson,
                  nullptr, c->w.status, c->st));
  CK(sg.finish());
  return CNS_OK;
}

int cns_zvismo(cns_ctx* c, int l, double* mu, const double* v, const double* temp) {
  (void)v;
  if (!c || bad_block(c, l) || !mu || !temp) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  double* dmu = sg.inout(mu, ld);
  const double* dtemp = sg.in(temp, ld);
  CK(sg.err);
  CK(launch_zvismo(c->d_blks, c->cells.view(l - 1), c->ph, dmu, dtemp, c->w.status, c->st));
  CK(sg.finish());
  return check_status(c);
}

int cns_chrono_global(cns_ctx* c, double* dt) {
  if (!c || !dt) return CNS_EINVAL;
  CK(ensure_dtpart(c));
  CK(launch_dt_global(c->d_blks, c->cells.view(-1), c->lay.ncells, c->sc.dt1min, dt,
                      c->w.dtpart, c->w.dtpart + c->cells.ntiles, c->w.status, c->st));
  return check_status(c);
}

int cns_chronos(cns_ctx* c, int l, double etal, const double* mu, const double* mut,
                const double* t, double* dt, const char* equat, const double* sn,
                int64_t lgsnlt, const double* vol, double* sfsi, double* sfsj, double* sfsk,
                double* dism, const double* cson) {
  (void)sfsi;
  (void)sfsj;
  (void)sfsk;
  (void)dism;
  if (!c || bad_block(c, l) || !t || !dt || !sn || !vol || !cson) return CNS_EINVAL;
  if (!equat_ok(equat)) return fail(c, CNS_EINVAL, "equat: only 'eu3d' / 'ns3d' forms");
  if (!sn_slice_ok(c, l, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(l)");
  const int ns = equat[0] == 'n';
  if (ns && (!mu || !mut)) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dmu = sg.in(mu, ld);
  const double* dmut = sg.in(mut, ld);
  const double* dv = sg.in(t, 5 * ld);
  double* ddt = sg.inout(dt, ld);
  const double* dsn = sg.in(sn, sn_elems(c, l));
  const double* dvol = sg.in(vol, ld);
  const double* dcson = sg.in(cson, ld);
  CK(sg.err);
  // chronos.f90:138-141 zeroes dt from cell (1,1,1) to cell (ni,nj,nk)
  const int b0 = l == 0 ? 0 : l - 1, b1 = l == 0 ? (int)c->lay.blks.size() : l;
  bool same_eta = true;
  for (int b = b0; b < b1; ++b) {
    const Blk& B = c->lay.blks[b];
    const long long n1 = B.npc + 1 + B.nid + B.nijd;
    const long long n2 = B.npc + B.ni + (long long)B.nj * B.nid + (long long)B.nk * B.nijd;
    CK(cudaMemsetAsync(ddt + n1, 0, sizeof(double) * (n2 - n1 + 1), c->st));
    same_eta = same_eta && B.eta == etal;
  }
  // the kernels read eta(lm) from the block table: the call's etal for this
  // launch, the context's values again after it
  std::vector<Blk> tmp;
  if (!same_eta) {
    tmp = c->lay.blks;
    for (int b = b0; b < b1; ++b) tmp[b].eta = etal;
    CK(cudaMemcpyAsync(c->d_blks, tmp.data(), sizeof(Blk) * tmp.size(),
                       cudaMemcpyHostToDevice, c->st));
  }
  Scheme sc = c->sc;
  sc.ns = ns;
  cudaError_t e = launch_chronos(c->d_blks, c->cells.view(l - 1), c->ph, sc, dmu, dmut, dv, ld,
                                 ddt, sn_base(c, l, dsn), dvol, dcson, c->st);
  if (!same_eta) {
    const cudaError_t e2 = cudaMemcpyAsync(c->d_blks, c->lay.blks.data(),
                                           sizeof(Blk) * c->lay.blks.size(),
                                           cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);  // tmp stays alive until then
  }
  CK(e);
  CK(sg.finish());
  return CNS_OK;
}

int cns_rbord(cns_ctx* c, double* v, double* ps, double* temp, double* cson) {
  if (!c || !v || !ps || !temp || !cson) return CNS_EINVAL;
  if (!c->metric_done) return fail(c, CNS_ENOTREADY, "cns_metric has not run");
  const long long ld = c->lay.ld;
  Staging sg(c);
  double* dv = sg.inout(v, 5 * ld);
  double* dps = sg.inout(ps, ld);
  double* dtemp = sg.inout(temp, ld);
  double* dcson = sg.inout(cson, ld);
  CK(sg.err);
  CK(launch_rbord(c->bd, c->ph, dv, ld, dps, dtemp, dcson, c->n_idd_ent, c->d_idd_ents,
                  c->d_idd_masks, c->st));
  CK(sg.finish());
  return CNS_OK;
}

// the flux routines (sch_roe.f90, sch_roe_euler.f90, sch_hllc*.f90,
// sch_rusanov.f90, sch_ausmp.f90): u zeroed over the block(s), the residual
// of the family ischema accumulated; ityprk != 0 then forms the forcing
// function ff -= u on the real cells (sch_roe.f90:1466-1481).  tau9: the
// nine stress and heat-flux arrays, or NULL for the Euler routines.
static int flux_entry(cns_ctx* c, int l, int ityprk, int ischema, int ns, double* u,
                      const double* v, double* ff, const double* const* tau9,
                      const char* equat, const double* sn, int64_t lgsnlt, const double* ps) {
  if (!c || bad_block(c, l) || !u || !v || !sn || !ps) return CNS_EINVAL;
  if (!equat_ok(equat)) return fail(c, CNS_EINVAL, "equat: only 'eu3d' / 'ns3d' forms");
  if (!sn_slice_ok(c, l, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(lm)");
  if (ityprk != 0 && !ff) return fail(c, CNS_EINVAL, "ityprk != 0 needs ff");
  if (tau9)
    for (int a = 0; a < 9; ++a)
      if (!tau9[a]) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  double* du = sg.inout(u, 5 * ld);
  const double* dv = sg.in(v, 5 * ld);
  double* dff = ityprk ? sg.inout(ff, 5 * ld) : nullptr;
  const double* dsn = sg.in(sn, sn_elems(c, l));
  const double* dps = sg.in(ps, ld);
  CK(sg.err);
  const double* dtau = nullptr;
  if (tau9) CK(tau_view(c, sg, tau9, &dtau));
  const Scheme keep = c->sc;
  c->sc.ns = ns;
  c->sc.ischema = ischema;
  cudaError_t e = ensure_hllc_v(c);
  if (e == cudaSuccess) e = zero_cols(c, du, 5, l);
  if (e == cudaSuccess) e = prim_of(c, l, dv);
  if (e == cudaSuccess) e = residual(c, l - 1, du, dv, dtau, sn_base(c, l, dsn), dps);
  if (e == cudaSuccess && ityprk != 0) e = forcing_sub(c, l, du, dff);
  c->sc = keep;
  CK(e);
  CK(sg.finish());
  return CNS_OK;
}

#define CNS_TAU9 toxx, toxy, toxz, toyy, toyz, tozz, qcx, qcy, qcz
#define CNS_TAU9_ARGS                                                                     \
  const double *toxx, const double *toxy, const double *toxz, const double *toyy,         \
      const double *toyz, const double *tozz, const double *qcx, const double *qcy,       \
      const double *qcz
#define CNS_MUSCL_WORK                                                                    \
  double *rhol, double *ul, double *vl, double *wl, double *pl, double *rhor, double *ur,  \
      double *vr, double *wr, double *prr

int cns_sch_roe_euler(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                      const char* equat, const double* sn, int64_t lgsnlt, CNS_MUSCL_WORK,
                      const double* ps) {
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  return flux_entry(c, lm, ityprk, 7, 0, u, v, ff, nullptr, equat, sn, lgsnlt, ps);
}

int cns_sch_roe(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                CNS_TAU9_ARGS, const char* equat, const double* sn, int64_t lgsnlt,
                CNS_MUSCL_WORK, const double* ps) {
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  const double* t9[9] = {CNS_TAU9};
  return flux_entry(c, lm, ityprk, 7, 1, u, v, ff, t9, equat, sn, lgsnlt, ps);
}

int cns_sch_hllc_euler(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                       const char* equat, const double* sn, int64_t lgsnlt, CNS_MUSCL_WORK,
                       const double* ps) {
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  return flux_entry(c, lm, ityprk, 14, 0, u, v, ff, nullptr, equat, sn, lgsnlt, ps);
}

int cns_sch_hllc(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                 CNS_TAU9_ARGS, const char* equat, const double* sn, int64_t lgsnlt,
                 CNS_MUSCL_WORK, const double* ps) {
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  const double* t9[9] = {CNS_TAU9};
  return flux_entry(c, lm, ityprk, 14, 1, u, v, ff, t9, equat, sn, lgsnlt, ps);
}

int cns_sch_rusanov(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                    CNS_TAU9_ARGS, const char* equat, const double* sn, int64_t lgsnlt,
                    CNS_MUSCL_WORK, const double* ps) {
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  // sch_rusanov.f90 reads the stresses whatever the equations (zero for Euler)
  const double* t9[9] = {CNS_TAU9};
  return flux_entry(c, lm, ityprk, 9, equat && equat[0] == 'n', u, v, ff, t9, equat, sn,
                    lgsnlt, ps);
}

int cns_sch_weno5_3d(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* ff,
                     CNS_TAU9_ARGS, const char* equat, const double* sn, int64_t lgsnlt,
                     double* fxx, double* fyy, double* fzz, double* fxy, double* fxz, double* fyz,
                     double* fex, double* fey, double* fez, const double* ps) {
  (void)fxx, (void)fyy, (void)fzz, (void)fxy, (void)fxz, (void)fyz, (void)fex, (void)fey,
      (void)fez;
  const double* t9[9] = {CNS_TAU9};
  return flux_entry(c, lm, ityprk, 12, equat && equat[0] == 'n', u, v, ff, t9, equat, sn,
                    lgsnlt, ps);
}

int cns_sch_ausmp(cns_ctx* c, int lm, int ityprk, double* u, const double* v, double* d,
                  double* ff, CNS_TAU9_ARGS, const char* equat, const double* sn,
                  int64_t lgsnlt, CNS_MUSCL_WORK, const double* ps) {
  (void)d;  // in the argument list of sch_ausmp.f90:4-11; not read by the flux
  (void)rhol, (void)ul, (void)vl, (void)wl, (void)pl, (void)rhor, (void)ur, (void)vr, (void)wr,
      (void)prr;
  const double* t9[9] = {CNS_TAU9};
  return flux_entry(c, lm, ityprk, 5, 1, u, v, ff, t9, equat, sn, lgsnlt, ps);
}







int cns_rfve(cns_ctx* c, double* v, double* ps, double* temp, double* cson) {
  if (!c || !v || !ps || !temp || !cson) return CNS_EINVAL;
  CK(launch_ghost_refresh(c->bd, 1, v, c->lay.ld, ps, temp, cson, c->st));
  return CNS_OK;
}

int cns_rfvc(cns_ctx* c, double* v, double* ps, double* temp, double* cson) {
  if (!c || !v || !ps || !temp || !cson) return CNS_EINVAL;
  CK(launch_ghost_refresh(c->bd, 2, v, c->lay.ld, ps, temp, cson, c->st));
  return CNS_OK;
}

int cns_dissip_jameson(cns_ctx* c, int lm, const double* v, double* d, const char* equat,
                       const double* sn, int64_t lgsnlt, double* snu, const double* ps,
                       const double* cson) {
  (void)snu;  // the sensor is evaluated inline from the pressures along the line
  if (!c || bad_block(c, lm) || !v || !d || !sn || !ps || !cson) return CNS_EINVAL;
  if (!equat_ok(equat)) return fail(c, CNS_EINVAL, "equat: only 'eu3d' / 'ns3d' forms");
  if (!sn_slice_ok(c, lm, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(lm)");
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dv = sg.in(v, 5 * ld);
  double* dd = sg.inout(d, 5 * ld);
  const double* dsn = sg.in(sn, sn_elems(c, lm));
  const double* dps = sg.in(ps, ld);
  const double* dcson = sg.in(cson, ld);
  CK(sg.err);
  CK(zero_cols(c, dd, 5, lm));
  CK(launch_dissip_jameson(c->d_blks, c->faces, c->cells.view(lm - 1), lm - 1, dv, ld, dps,
                           dcson, sn_base(c, lm, dsn), c->w.G, dd, c->st));
  CK(sg.finish());
  return CNS_OK;
}

int cns_sch_jameson(cns_ctx* c, int lm, int ityprk, double* u, const double* v,
                    const double* d, double* ff, CNS_TAU9_ARGS, const char* equat,
                    const double* sn, int64_t lgsnlt, double* fxx, double* fyy, double* fzz,
                    double* fxy, double* fxz, double* fyz, double* fex, double* fey,
                    double* fez, const double* ps) {
  (void)fxx, (void)fyy, (void)fzz, (void)fxy, (void)fxz, (void)fyz, (void)fex, (void)fey,
      (void)fez;  // the reference's flux-density work arrays: fluxes are formed per face
  if (!c || bad_block(c, lm) || !u || !v || !d || !sn || !ps) return CNS_EINVAL;
  if (!equat_ok(equat)) return fail(c, CNS_EINVAL, "equat: only 'eu3d' / 'ns3d' forms");
  if (!sn_slice_ok(c, lm, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(lm)");
  if (ityprk != 0 && !ff) return fail(c, CNS_EINVAL, "ityprk != 0 needs ff");
  const int ns = equat[0] == 'n';  // sch_jameson.f90:85
  const long long ld = c->lay.ld;
  Staging sg(c);
  double* du = sg.inout(u, 5 * ld);
  const double* dv = sg.in(v, 5 * ld);
  const double* dd = sg.in(d, 5 * ld);
  double* dff = ityprk ? sg.inout(ff, 5 * ld) : nullptr;
  const double* dsn = sg.in(sn, sn_elems(c, lm));
  const double* dps = sg.in(ps, ld);
  CK(sg.err);
  const double* dtau = nullptr;
  if (ns) {
    const double* t9[9] = {CNS_TAU9};
    for (int a = 0; a < 9; ++a)
      if (!t9[a]) return CNS_EINVAL;
    CK(tau_view(c, sg, t9, &dtau));
  }
  CK(zero_cols(c, du, 5, lm));
  CK(launch_sch_jameson(c->d_blks, c->faces, c->cells.view(lm - 1), lm - 1, ns, c->ph.pinfl,
                        dv, ld, dps, dtau, sn_base(c, lm, dsn), dd, c->w.G, du, nullptr,
                        c->st));
  if (ityprk != 0) CK(forcing_sub(c, lm, du, dff));
  CK(sg.finish());
  return CNS_OK;
}

int cns_set_turbulence(cns_ctx* c, double alfak, double alfae, double sigma, double epsroe) {
  if (!c || !(alfak != 0.) || !(alfae != 0.) || !(sigma != 0.)) return CNS_EINVAL;
  c->alfak = alfak;
  c->alfae = alfae;
  c->sigma = sigma;
  c->epsroe = epsroe;
  return CNS_OK;
}


int cns_met_fludc(cns_ctx* c, int l, const double* s, const double* mu, const double* mut,
                  const double* t, const double* dtdx, const double* dtdy, const double* dtdz,
                  double* fd5x, double* fd5y, double* fd5z, double* fd6x, double* fd6y,
                  double* fd6z) {
  // s, t and the temperature gradients are in the argument list of
  // met_fludc.f90:4-8; the routine only scales the diffusion densities
  (void)s, (void)t, (void)dtdx, (void)dtdy, (void)dtdz;
  if (!c || bad_block(c, l) || !mu || !mut || !fd5x || !fd5y || !fd5z || !fd6x || !fd6y ||
      !fd6z)
    return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dmu = sg.in(mu, ld);
  const double* dmut = sg.in(mut, ld);
  double* const fd[6] = {sg.inout(fd5x, ld), sg.inout(fd5y, ld), sg.inout(fd5z, ld),
                         sg.inout(fd6x, ld), sg.inout(fd6y, ld), sg.inout(fd6z, ld)};
  CK(sg.err);
  const int l0 = l == 0 ? 1 : l, l1 = l == 0 ? (int)c->lay.blks.size() : l;
  for (int b = l0; b <= l1; ++b) {
    long long n0, n1;
    fludc_range(c, b, n0, n1);
    CK(launch_fludc(n0, n1, dmu, dmut, fd, c->alfak, c->alfae, c->st));
  }
  CK(sg.finish());
  return CNS_OK;
}

int cns_met_fludcsa(cns_ctx* c, int l, const double* s, const double* mu, double* fd5x,
                    double* fd5y, double* fd5z, double* fd6x, double* fd6y, double* fd6z) {
  if (!c || bad_block(c, l) || !s || !mu || !fd5x || !fd5y || !fd5z || !fd6x || !fd6y || !fd6z)
    return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* ds = sg.in(s, 7 * ld);
  const double* dmu = sg.in(mu, ld);
  double* const fd[6] = {sg.inout(fd5x, ld), sg.inout(fd5y, ld), sg.inout(fd5z, ld),
                         sg.inout(fd6x, ld), sg.inout(fd6y, ld), sg.inout(fd6z, ld)};
  CK(sg.err);
  const int l0 = l == 0 ? 1 : l, l1 = l == 0 ? (int)c->lay.blks.size() : l;
  for (int b = l0; b <= l1; ++b) {
    long long n0, n1;
    fludc_range(c, b, n0, n1);
    CK(launch_fludcsa(n0, n1, ds + 5 * ld, dmu, fd, c->sigma, c->st));
  }
  CK(sg.finish());
  return CNS_OK;
}

static int met_roe2o_common(cns_ctx* c, int l, const double* t, double* d, const double* sn,
                            int64_t lgsnlt, int harten) {
  if (!c || bad_block(c, l) || !t || !d || !sn) return CNS_EINVAL;
  if (!sn_slice_ok(c, l, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(l)");
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dt7 = sg.in(t, 7 * ld);
  double* dd = sg.inout(d, 7 * ld);
  const double* dsn = sg.in(sn, sn_elems(c, l));
  CK(sg.err);
  CK(launch_roe2o(c->d_blks, c->faces, c->cells_ext.view(l - 1), l - 1, harten, c->epsroe,
                  c->ph.gam, c->ph.gam1, dt7, ld, sn_base(c, l, dsn), c->w.G, dd, c->st));
  CK(sg.finish());
  return CNS_OK;
}

int cns_met_samut(cns_ctx* c, int l, const double* v, const double* mu, double* mut) {
  if (!c || bad_block(c, l) || !v || !mu || !mut) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dv = sg.in(v, 7 * ld);
  const double* dmu = sg.in(mu, ld);
  double* dmut = sg.inout(mut, ld);
  CK(sg.err);
  CK(launch_samut(c->d_blks, c->cells.view(l - 1), dv + 5 * ld, dmu, dmut, c->st));
  CK(sg.finish());
  return CNS_OK;
}

int cns_sch_turb(cns_ctx* c, int l, double* u, const double* v, const double* d,
                 const double* fd5x, const double* fd5y, const double* fd5z,
                 const double* fd6x, const double* fd6y, const double* fd6z, const double* ts6,
                 const double* ts7, const double* sn, const double* vol) {
  if (!c || bad_block(c, l) || !u || !v || !d || !fd5x || !fd5y || !fd5z || !fd6x || !fd6y ||
      !fd6z || !ts6 || !ts7 || !sn || !vol)
    return CNS_EINVAL;
  const long long ld = c->lay.ld;
  // sch_turb.f90:59-66 zeroes u(:,6:7) over the block(s)
  long long n0, n1;
  block_range(c, l, n0, n1);
  CK(cudaMemsetAsync(u + 5 * ld + n0, 0, sizeof(double) * (n1 - n0), c->st));
  CK(cudaMemsetAsync(u + 6 * ld + n0, 0, sizeof(double) * (n1 - n0), c->st));
  const double* fd[6] = {fd5x, fd5y, fd5z, fd6x, fd6y, fd6z};
  CK(launch_sch_turb(c->d_blks, c->faces, c->cells.view(l - 1), l - 1, v, ld, fd, ts6, ts7, d,
                     sn, vol, c->w.G, u, c->st));
  return CNS_OK;
}

static cudaError_t ensure_sa(cns_ctx* c) {
  cudaError_t e = cudaSuccess;
  if (!c->sa_gr) e = dev_alloc(c, &c->sa_gr, (size_t)6 * c->lay.ld, false);
  if (e == cudaSuccess && !c->sa_sc) e = dev_alloc(c, &c->sa_sc, (size_t)3 * c->lay.ld, false);
  return e;
}

int cns_teq_gradv(cns_ctx* c, int l, const double* v, const double* sn, const double* vol,
                  double* dv) {
  if (!c || bad_block(c, l) || !v || !sn || !vol || !dv) return CNS_EINVAL;
  CK(ensure_sa(c));
  long long n0, n1;
  block_range(c, l, n0, n1);
  CK(launch_teq_grads(c->d_blks, c->cells.view(l - 1), 0, 3, v, nullptr, c->lay.ld, sn, vol,
                      dv, c->sa_sc, n0, n1, c->st));
  return CNS_OK;
}

int cns_met_smsa(cns_ctx* c, int l, const double* v, const double* mu, const double* dist,
                 const double* sn, const double* vol, const double* dv, const double* fd5x,
                 const double* fd5y, const double* fd5z, double* ts6, double* ts7,
                 double* cfke) {
  if (!c || bad_block(c, l) || !v || !mu || !dist || !sn || !vol || !dv || !fd5x || !fd5y ||
      !fd5z || !ts6 || !ts7 || !cfke)
    return CNS_EINVAL;
  CK(ensure_sa(c));
  const long long ld = c->lay.ld;
  const Space cells = c->cells.view(l - 1);
  // met_difsa: grad(rho nu~); met_smsa: grad(rho)
  CK(launch_teq_grads(c->d_blks, cells, 1, 1, v, v + 5 * ld, ld, sn, vol, c->sa_gr, nullptr, 0,
                      0, c->st));
  CK(launch_teq_grads(c->d_blks, cells, 1, 1, v, v, ld, sn, vol, c->sa_gr + 3 * ld, nullptr, 0,
                      0, c->st));
  const double* fd5[3] = {fd5x, fd5y, fd5z};
  CK(launch_smsa(c->d_blks, cells, ld, v, mu, dist, dv, c->sa_gr, c->sa_gr + 3 * ld, fd5, ts6,
                 ts7, cfke, c->sa_fix, c->st));
  return CNS_OK;
}

int cns_impli2_eqt_3d(cns_ctx* c, int l, const double* u, const double* dt, double* v,
                      const double* mu, const double* mut, const double* cfke,
                      const double* sn, const double* vol, double cmt) {
  if (!c || bad_block(c, l) || !u || !dt || !v || !mu || !mut || !cfke || !sn || !vol ||
      !(cmt != 0.))
    return CNS_EINVAL;
  if (!c->sa_w) CK(dev_alloc(c, &c->sa_w, (size_t)20 * c->lay.ld, false));
  CK(launch_impli2(c->d_blks, c->faces, c->lines, c->cells.view(l - 1), l - 1, c->lay.ld, u, dt,
                   v, mu, mut, cfke, sn, vol, cmt, c->sa_w, 0, c->d_lp2_ni, c->n_lp2_ni,
                   c->st));
  return CNS_OK;
}

int cns_met_roe2o(cns_ctx* c, int l, const double* t, double* d, const double* sn,
                  int64_t lgsnlt, const double* vol, double* del6, double* del7) {
  (void)vol, (void)del6, (void)del7;  // met_roe2o.f90:4-7's volume and slope work arrays
  return met_roe2o_common(c, l, t, d, sn, lgsnlt, 0);
}

int cns_met_roe2oh(cns_ctx* c, int l, const double* t, double* d, const double* sn,
                   int64_t lgsnlt, const double* vol, double* del6, double* del7) {
  (void)vol, (void)del6, (void)del7;
  return met_roe2o_common(c, l, t, d, sn, lgsnlt, 1);
}

int cns_atcaldis3(cns_ctx* c, const double* x, const double* y, const double* z,
                  double* dist) {
  if (!c || !x || !y || !z || !dist) return CNS_EINVAL;
  if (c->n_wall_ent == 0)
    return fail(c, CNS_EBC, "no wall boundary to measure the distance to (atcaldis3 stops)");
  if (!c->wall_par) CK(dev_alloc(c, &c->wall_par, (size_t)(3 * c->n_wall_ent), false));
  CK(launch_wall_dist(c->bd, c->d_blks, c->cells.view(-1), c->d_wall_ents, c->n_wall_ent, x,
                      y, z, c->wall_par, dist, c->st));
  return CNS_OK;
}

int cns_met_bord(cns_ctx* c, double* v, double rokinf, double roeinf) {
  if (!c || !v) return CNS_EINVAL;
  CK(launch_turb_bord(c->bd, v, c->lay.ld, rokinf, roeinf, c->st));
  return CNS_OK;
}

int cns_met_gradtr(cns_ctx* c, int l, const double* s, const double* sn, const double* vol,
                   double* fd5x, double* fd5y, double* fd5z, double* fd6x, double* fd6y,
                   double* fd6z) {
  if (!c || bad_block(c, l) || !s || !sn || !vol || !fd5x || !fd5y || !fd5z || !fd6x || !fd6y ||
      !fd6z)
    return CNS_EINVAL;
  CK(ensure_sa_step(c));
  const long long ld = c->lay.ld;
  double* const out[6] = {fd5x, fd5y, fd5z, fd6x, fd6y, fd6z};
  const int b0 = l == 0 ? 0 : l - 1, b1 = l == 0 ? (int)c->lay.blks.size() : l;
  for (int b = b0; b < b1; ++b) {
    // met_gradtr.f90:97-104: the flat range of the real cells, ghost cells
    // inside it included (zero there)
    long long n0, n1;
    fludc_range(c, b + 1, n0, n1);
    const size_t cnt = (size_t)(n1 - n0 + 1);
    for (int q = 0; q < 6; ++q)
      CK(cudaMemsetAsync(c->sa_fd + q * ld + n0, 0, sizeof(double) * cnt, c->st));
    long long b0, b1;
    block_range(c, b + 1, b0, b1);
    CK(launch_teq_grads(c->d_blks, c->cells.view(b), 2, 2, s, nullptr, ld, sn, vol, c->sa_fd,
                        c->sa_sc, b0, b1, c->st));
    for (int q = 0; q < 6; ++q)
      CK(cudaMemcpyAsync(out[q] + n0, c->sa_fd + q * ld + n0, sizeof(double) * cnt,
                         cudaMemcpyDeviceToDevice, c->st));
  }
  return CNS_OK;
}

int cns_met_rbse(cns_ctx* c, double* fd5x, double* fd5y, double* fd5z, double* fd6x,
                 double* fd6y, double* fd6z) {
  if (!c || !fd5x || !fd5y || !fd5z || !fd6x || !fd6y || !fd6z) return CNS_EINVAL;
  double* const fd[6] = {fd5x, fd5y, fd5z, fd6x, fd6y, fd6z};
  CK(launch_fd_ghosts(c->bd, fd, c->st));
  return CNS_OK;
}

int cns_met_cutsa(cns_ctx* c, int l, double* v, double epsk) {
  if (!c || bad_block(c, l) || !v) return CNS_EINVAL;
  CK(launch_cutsa(c->d_blks, c->cells.view(l - 1), v, c->lay.ld, epsk, c->st));
  return CNS_OK;
}

int cns_lpsa(cns_ctx* c, int l, double* v, const double* mu, double* mut, const double* dist,
             const double* ztemp) {
  if (!c || bad_block(c, l) || !v || !mu || !mut || !dist || !ztemp) return CNS_EINVAL;
  CK(enqueue_lpsa(c, l - 1, v, mu, mut, dist, ztemp));
  return CNS_OK;
}

int cns_cllparoi1(cns_ctx* c, const double* v, const double* dist, const double* mu,
                  const double* mut, double* tau, const double* ztemp) {
  if (!c || !v || !dist || !mu || !mut || !tau || !ztemp) return CNS_EINVAL;
  CK(enqueue_cllparoi1(c, v, mu, mut, dist, ztemp, tau));
  return CNS_OK;
}

int cns_set_sa(cns_ctx* c, const cns_sa_t* sa) {
  if (!c) return CNS_EINVAL;
  drop_graphs(c);
  if (!sa) {
    c->sa_on = false;
    c->sa_fix = 0;
    c->sa_dist = nullptr;
    return CNS_OK;
  }
  if (!sa->dist) return CNS_EINVAL;
  if (!c->sc.ns)
    return fail(c, CNS_EINVAL, "the Spalart-Allmaras step needs the Navier-Stokes equations");
  CK(ensure_sa_step(c));
  c->sa_dist = sa->dist;
  c->sa_rokinf = sa->rokinf;
  c->sa_roeinf = sa->roeinf;
  c->sa_epsk = sa->epsk;
  c->sa_fix = sa->stilde_fix ? 1 : 0;
  c->sa_on = true;
  c->ke_on = false;
  return CNS_OK;
}

int cns_set_ke(cns_ctx* c, const cns_ke_t* ke) {
  if (!c) return CNS_EINVAL;
  drop_graphs(c);
  if (!ke) {
    c->ke_on = false;
    return CNS_OK;
  }
  if (!c->sc.ns)
    return fail(c, CNS_EINVAL, "the k-epsilon step needs the Navier-Stokes equations");
  if (!c->lp2.empty())
    return fail(c, CNS_EINVAL, "the k-epsilon step has no wall law ('lp2' walls)");
  if (!(ke->epsk > 0.) || !(ke->epse > 0.))
    return fail(c, CNS_EINVAL, "k-epsilon: epsk and epse must be positive");
  CK(ensure_sa_step(c));
  const size_t ld = (size_t)c->lay.ld;
  if (!c->ke_tprod) CK(dev_alloc(c, &c->ke_tprod, ld));
  if (!c->ke_w) CK(dev_alloc(c, &c->ke_w, 14 * ld));
  c->ke_rokinf = ke->rokinf;
  c->ke_roeinf = ke->roeinf;
  c->ke_epsk = ke->epsk;
  c->ke_epse = ke->epse;
  c->ke_on = true;
  c->sa_on = false;
  c->sa_dist = nullptr;
  return CNS_OK;
}

int cns_met_prod(cns_ctx* c, int l, int ncyc, const double* mut, const double* s,
                 const double* dv, double* tprod) {
  (void)ncyc;  // in met_prod.f90:4-8's argument list, not read
  if (!c || bad_block(c, l) || !mut || !s || !dv || !tprod) return CNS_EINVAL;
  CK(launch_met_prod(c->d_blks, c->cells.view(l - 1), c->lay.ld, mut, s, dv, tprod, c->st));
  return CNS_OK;
}

int cns_met_smke(cns_ctx* c, int l, const double* sn, const double* vol, const double* v,
                 const double* mu, const double* mut, const double* tprod, double* cfke,
                 double* dv, double* qcxts5, double* qcyts6) {
  if (!c || bad_block(c, l) || !sn || !vol || !v || !mu || !mut || !tprod || !cfke || !dv ||
      !qcxts5 || !qcyts6)
    return CNS_EINVAL;
  CK(ensure_sa(c));
  if (!c->ke_w) CK(dev_alloc(c, &c->ke_w, 14 * (size_t)c->lay.ld));
  long long b0, b1;
  block_range(c, l, b0, b1);
  CK(launch_exgr(c->lay.blks[l - 1], c->lay.ld, dv, c->st));
  CK(launch_smke(c->d_blks, c->cells.view(l - 1), c->lay.ld, v, mu, mut, sn, vol, tprod, dv,
                 c->ke_w, qcxts5, qcyts6, cfke, b0, b1, c->st));
  return CNS_OK;
}

int cns_met_kemut(cns_ctx* c, int l, const double* v, const double* mu, double* mut) {
  if (!c || bad_block(c, l) || !v || !mu || !mut) return CNS_EINVAL;
  CK(launch_kemut(c->d_blks, c->cells.view(l - 1), c->lay.ld, v, mu, mut, c->st));
  return CNS_OK;
}

int cns_met_cutke(cns_ctx* c, int l, double* v, double epsk, double epse) {
  if (!c || bad_block(c, l) || !v) return CNS_EINVAL;
  CK(launch_cutke(c->d_blks, c->cells.view(l - 1), c->lay.ld, v, epsk, epse, c->st));
  return CNS_OK;
}

int cns_met_inisa(cns_ctx* c, int l, double* v, const double* mut, const double* mu) {
  (void)mu;  // in met_inisa.f90:4's argument list, not read
  if (!c || bad_block(c, l) || !v || !mut) return CNS_EINVAL;
  CK(launch_turb_init(c->d_blks, c->cells.view(l - 1), 0, c->lay.ld, v, const_cast<double*>(mut),
                      nullptr, nullptr, c->st));
  return CNS_OK;
}

int cns_met_inmut(cns_ctx* c, int l, const double* mu, double* mut) {
  if (!c || bad_block(c, l) || !mu || !mut) return CNS_EINVAL;
  CK(launch_turb_init(c->d_blks, c->cells.view(l - 1), 1, c->lay.ld, nullptr, mut, mu, nullptr,
                      c->st));
  return CNS_OK;
}

int cns_met_ini(cns_ctx* c, int l, double* v, const double* mut, const double* mu,
                const double* sn, const double* vol, double* dv) {
  (void)mu;  // in met_ini.f90:4-8's argument list, not read
  if (!c || bad_block(c, l) || !v || !mut || !sn || !vol || !dv) return CNS_EINVAL;
  CK(ensure_sa(c));
  long long n0, n1;
  block_range(c, l, n0, n1);
  const Space cb = c->cells.view(l - 1);
  CK(launch_teq_grads(c->d_blks, cb, 0, 3, v, nullptr, c->lay.ld, sn, vol, dv, c->sa_sc, n0, n1,
                      c->st));
  CK(launch_turb_init(c->d_blks, cb, 2, c->lay.ld, v, const_cast<double*>(mut), nullptr, dv,
                      c->st));
  return CNS_OK;
}

int cns_met_num(cns_ctx* c) {
  if (!c) return CNS_EINVAL;
  if (!c->bound || !(c->sa_on || c->ke_on))
    return fail(c, CNS_ENOTREADY, "bind the state and enable a turbulence step first");
  CK(enqueue_met_num(c));
  return CNS_OK;
}

int cns_adjoint_prepare(cns_ctx* c) {
  if (!c) return CNS_EINVAL;
  if (!c->bound || !c->metric_done)
    return fail(c, CNS_ENOTREADY, "bind the state and run cns_metric first");
  if (c->sc.ns || c->sc.ischema != 7 || c->sc.muscl < 0 || c->sc.muscl > 1 ||
      c->sc.ilim != 0 || c->sc.kfmg == 3)
    return fail(c, CNS_EINVAL, "the adjoint covers the steady Euler Roe scheme (ns = 0, "
                               "ischema 7, kfmg 0, first order or unlimited MUSCL)");
  if (!c->sc.qfix_dfez)
    return fail(c, CNS_EINVAL, "the adjoint needs qfix_dfez = 1 (the reference Euler implicit "
                               "phase is not linear in the increment)");
  const cns_state_t& s = c->state;
  const long long ld = c->lay.ld;
  if (!c->adj_J) CK(dev_alloc(c, &c->adj_J, (size_t)(3 * 27 * 5) * ld, false));
  if (!c->adj_z) CK(dev_alloc(c, &c->adj_z, (size_t)(2 * 5 + 1) * ld));
  const Space all = c->cells.view(-1);
  // the iteration's inputs at the bound (converged) state: thermodynamics,
  // time steps, ghost cells, velocities, implicit coefficients
  CK(launch_zpres(c->d_blks, all, c->ph, 0, s.v, ld, s.pression, s.ztemp, s.cson, s.mu,
                  c->w.status, c->st));
  CK(launch_chronos(c->d_blks, all, c->ph, c->sc, s.mu, s.mut, s.v, ld, s.dt, s.sn, s.vol,
                    s.cson, c->st));
  CK(global_dt(c));
  CK(launch_rbord(c->bd, c->ph, s.v, ld, s.pression, s.ztemp, s.cson, c->n_idd_ent,
                  c->d_idd_ents, c->d_idd_masks, c->st));
  CK(launch_prim(0, c->lay.ncells, s.v, ld, c->w.prim, c->st));
  CK(launch_implicit_coefficients(c->d_blks, all, c->faces, -1, c->ph, 1, s.dt, s.v, c->w.prim,
                                  s.mu, s.mut, s.sn, s.vol, s.cson, c->w, nullptr, nullptr,
                                  c->st));
  CK(launch_face_jac(c->d_blks, c->faces, c->ph, c->sc, s.v, s.pression, ld, s.sn, c->adj_J,
                     c->st));
  if (c->sc.precision != 0) {
    // the reduced-precision form: L^T in FP32 (face areas and coefficients
    // rounded once); A^T lambda stays FP64
    CK(ensure_mixed(c));
    CK(refresh_sn32(c, s.sn));
    CK(launch_to_float(c->w.coefe, c->w.coefe32, 3 * ld, c->st));
    CK(launch_to_float(c->w.coefdiag, c->w.coefdiag32, ld, c->st));
  }
  c->adj_fp32 = c->sc.precision != 0;
  return check_status(c);
}

int cns_adjoint_rt(cns_ctx* c, const double* lam, double* wbar, double* sbar) {
  if (!c || !lam || !wbar) return CNS_EINVAL;
  if (!c->adj_J) return fail(c, CNS_ENOTREADY, "run cns_adjoint_prepare first");
  CK(launch_adj_gather(c->d_blks, c->cells_ext.view(-1), c->adj_J, lam, c->lay.ld, wbar, sbar,
                       c->st));
  return CNS_OK;
}

int cns_adjoint_lt(cns_ctx* c, const double* y, double* out) {
  if (!c || !y || !out) return CNS_EINVAL;
  if (!c->adj_z) return fail(c, CNS_ENOTREADY, "run cns_adjoint_prepare first");
  const long long ld = c->lay.ld;
  const int lmx = c->sc.lmax > 0 ? c->sc.lmax : 1;
  const cns_state_t& s = c->state;
  if (c->adj_fp32) {
    float* z = reinterpret_cast<float*>(c->adj_z);
    CK(launch_precond_ta<float>(c->d_blks, c->cells.view(-1), ld, s.v, s.pression, c->w.sn32,
                                c->w.coefe32, c->w.coefdiag32, c->ph.gam1, c->ph.pinfl, lmx, y,
                                z, z + 5 * ld, z + 10 * ld, out, c->st));
  } else {
    CK(launch_precond_ta<double>(c->d_blks, c->cells.view(-1), ld, s.v, s.pression, s.sn,
                                 c->w.coefe, c->w.coefdiag, c->ph.gam1, c->ph.pinfl, lmx, y,
                                 c->adj_z, c->adj_z + 5 * ld, c->adj_z + 10 * ld, out, c->st));
  }
  return CNS_OK;
}

int cns_zvisqc(cns_ctx* c, const double* v, const double* mu, const double* mut,
               double* tau, const double* sn, const double* vol,
               const double* temp) {
  if (!c || !v || !mu || !mut || !tau || !sn || !vol || !temp) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* dv = sg.in(v, 5 * ld);
  const double* dmu = sg.in(mu, ld);
  const double* dmut = sg.in(mut, ld);
  double* dtau = sg.inout(tau, 9 * ld);
  const double* dsn = sg.in(sn, 9 * ld);
  const double* dvol = sg.in(vol, ld);
  const double* dtemp = sg.in(temp, ld);
  CK(sg.err);
  CK(prim_of(c, 0, dv));
  CK(launch_grad(c->d_blks, c->cells.view(-1), c->ph, dv, c->w.prim, ld, dmu, dmut, dtau, dsn,
                 dvol, dtemp, c->st));
  CK(launch_tau_ghosts(c->bd, dtau, ld, c->st));
  CK(sg.finish());
  return CNS_OK;
}

// implimf_3d.f90 / implimf_eu.f90 on block(s) l: d zeroed, lmax point-Jacobi
// sweeps, v += d.  ityprk != 0: right-hand side -u - ff; dtpas: the
// physical step of the dual-time diagonal term when kfmg = 3.
static int implimf(cns_ctx* c, int l, int eu, const double* u, const double* dt, double* v,
                   double* d, const double* ff, const double* mu, const double* mut,
                   const char* equat, int lmx, const double* sn, int64_t lgsnlt,
                   const double* vol, double dtpas, int ityprk, const double* ps,
                   const double* cson) {
  if (!c || bad_block(c, l) || !u || !dt || !v || !d || !sn || !vol || !ps || !cson ||
      lmx < 0)
    return CNS_EINVAL;
  if (!eu && (!mu || !mut)) return CNS_EINVAL;
  if (!equat_ok(equat)) return fail(c, CNS_EINVAL, "equat: only 'eu3d' / 'ns3d' forms");
  if (!sn_slice_ok(c, l, lgsnlt)) return fail(c, CNS_EINVAL, "lgsnlt must be nnn(lm)");
  if (ityprk != 0 && !ff) return fail(c, CNS_EINVAL, "ityprk != 0 needs ff");
  if (c->sc.kfmg == 3 && !(dtpas > 0.)) return fail(c, CNS_EINVAL, "kfmg = 3 needs dtpas > 0");
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* du = sg.in(u, 5 * ld);
  const double* ddt = sg.in(dt, ld);
  double* dv = sg.inout(v, 5 * ld);
  double* dd = sg.inout(d, 5 * ld);
  const double* dff = ityprk ? sg.in(ff, 5 * ld) : nullptr;
  const double* dmu = eu ? nullptr : sg.in(mu, ld);
  const double* dmut = eu ? nullptr : sg.in(mut, ld);
  const double* dsn = sg.in(sn, sn_elems(c, l));
  const double* dvol = sg.in(vol, ld);
  const double* dps = sg.in(ps, ld);
  const double* dcson = sg.in(cson, ld);
  CK(sg.err);
  if (ityprk != 0) {
    if (!c->u_forced) CK(dev_alloc(c, &c->u_forced, (size_t)(5 * ld)));
    CK(forcing_add(c, l, du, dff, c->u_forced));
    du = c->u_forced;
  }
  CK(zero_cols(c, dd, 5, l));
  CK(prim_of(c, l, dv));
  Scheme sc = c->sc;
  if (sc.kfmg == 3) sc.dt1min = dtpas;
  CK(launch_implicit(c->d_blks, c->cells.view(l - 1), c->tiles64.view(l - 1), c->faces, l - 1,
                     c->ph, sc, eu, lmx, du, ddt, dv, dd, dmu, dmut, sn_base(c, l, dsn), dvol,
                     dps, dcson, c->w, 0, c->st));
  CK(sg.finish());
  return CNS_OK;
}

#define CNS_DF9                                                                           \
  double *dfxx, double *dfyy, double *dfzz, double *dfxy, double *dfxz, double *dfyz,     \
      double *dfex, double *dfey, double *dfez
int cns_implimf_eu(cns_ctx* c, int lm, const double* u, const double* dt, double* v,
                   double* d, const double* ff, const char* equat, int lmx, const double* sn,
                   int64_t lgsnlt, const double* vol, double dtpas, int ityprk, CNS_DF9,
                   double* coefdiag, const double* ps, const double* cson) {
  // the stored flux increments and the diagonal are recomputed on the device
  (void)dfxx, (void)dfyy, (void)dfzz, (void)dfxy, (void)dfxz, (void)dfyz, (void)dfex,
      (void)dfey, (void)dfez, (void)coefdiag;
  return implimf(c, lm, 1, u, dt, v, d, ff, nullptr, nullptr, equat, lmx, sn, lgsnlt, vol,
                 dtpas, ityprk, ps, cson);
}

int cns_implimf_3d(cns_ctx* c, int lm, const double* u, const double* dt, double* v,
                   double* d, const double* ff, const double* mu, const double* mut,
                   const char* equat, int lmx, const double* sn, int64_t lgsnlt,
                   const double* vol, double dtpas, int ityprk, CNS_DF9, double* rv,
                   const double* ps, const double* cson) {
  (void)dfxx, (void)dfyy, (void)dfzz, (void)dfxy, (void)dfxz, (void)dfyz, (void)dfex,
      (void)dfey, (void)dfez, (void)rv;
  return implimf(c, lm, 0, u, dt, v, d, ff, mu, mut, equat, lmx, sn, lgsnlt, vol, dtpas,
                 ityprk, ps, cson);
}



int cns_rscpsv(cns_ctx* c, const double* u0, const double* v, const double* dt,
               double* norms) {
  if (!c || !u0 || !v || !dt || !norms) return CNS_EINVAL;
  const long long ld = c->lay.ld;
  Staging sg(c);
  const double* du0 = sg.in(u0, 5 * ld);
  const double* dv = sg.in(v, 5 * ld);
  const double* ddt = sg.in(dt, ld);
  CK(sg.err);
  CK(launch_norm_partials(c->d_blks, c->cells.view(-1), ld, du0, dv, ddt, c->w.normpart, c->st));
  CK(launch_norm_finalize(c->d_blks, c->d_cells_tile0, 0, (int)c->lay.blks.size(),
                          c->w.normpart, c->w.blocksum, c->w.norms, c->st));
  CK(cudaMemcpyAsync(c->h_norms, c->w.norms, 15 * sizeof(double), cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  std::memcpy(norms, c->h_norms, 15 * sizeof(double));
  return CNS_OK;
}

int cns_bind_state(cns_ctx* c, const cns_state_t* s) {
  if (!c || !s || !s->v || !s->u || !s->d || !s->dt || !s->sn || !s->vol ||
      !s->pression || !s->ztemp || !s->cson || !s->mu || !s->mut || !s->tau)
    return CNS_EINVAL;
  c->state = *s;
  c->bound = true;
  c->ncyc = c->cyc_n = c->cyc_i = 0;
  c->mixed_iter = 0;
  drop_graphs(c);
  return CNS_OK;
}

int cns_atsch_num_launch(cns_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return CNS_EINVAL;
  if (!c->bound || !c->metric_done)
    return fail(c, CNS_ENOTREADY, "bind the state and run cns_metric first");
  if (c->sc.kfmg == 3) {
    const cns_state_t& s = c->state;
    if (!s.ptdual || !s.vdual || !s.vdual1 || !s.vdual2)
      return fail(c, CNS_ENOTREADY, "dual time stepping: bind ptdual, vdual, vdual1, vdual2");
    if (c->sa_on || c->ke_on)
      return fail(c, CNS_EINVAL, "dual time stepping with a turbulence step");
  }
  if (c->sc.ns && !c->lp2.empty() && !c->sa_dist)
    return fail(c, CNS_ENOTREADY, "the wall law of the 'lp2' walls needs the wall distance "
                                  "(cns_set_sa)");
  if (c->sc.kdtl == 0) CK(ensure_dtpart(c));
  if (nsteps == 0) return CNS_OK;
  const int prec = c->sc.precision;
  if (prec != 0 && !c->w.mixed_ready) {
    CK(ensure_mixed(c));
    CK(refresh_sn32(c, c->state.sn));
  }
  if (jameson(c)) CK(ensure_dis(c));
  // first iteration of a form whose sweeps are not tuned yet, and the first
  // Jameson cycle (rfve before the dissipation): run it eagerly (the
  // launches the graph would hold), tune the sweep tiles on its data, then
  // capture the steady-state iteration with the chosen tiles
  const bool first = c->cyc_n == 0;  // the next iteration is the reference's ncyc = 1
  const bool tuned = prec == 0 ? c->tuned64 : c->tuned32;
  const bool eager = !tuned || (jameson(c) && first);
  auto enqueue = [&](int form, bool fst, bool on) {
    if (form == kGraph64) return enqueue_step(c, fst, on);
    return enqueue_step_mixed(c, prec == 1 ? kMixed : (form == kGraphRef ? kDefectRefresh
                                                                          : kDefectRegular),
                              fst, on);
  };
  // the form of the next iteration (defect correction refreshes every
  // kdefect iterations), advancing the refresh counter
  auto next_form = [&]() {
    if (prec == 0) return (int)kGraph64;
    if (prec == 1) return (int)kGraphRef;
    return (c->mixed_iter++ % c->sc.kdefect) == 0 ? (int)kGraphRef : (int)kGraphReg;
  };
  std::vector<std::pair<int, bool>> plan;  // (form, time step recomputed) per iteration
  if (eager) {
    const int form = next_form();
    ++c->ncyc;
    const bool on = dt_due(c, ++c->cyc_n, ++c->cyc_i);
    CK(enqueue(form, first, on));
    if (!tuned) {
      CK(tune_sweeps(c, prec != 0));
      drop_graphs(c);
    }
    --nsteps;
    plan.emplace_back(form, on);  // counted below with the launches of its graph
  }
  const size_t replay0 = plan.size();
  c->ncyc += nsteps;
  for (int q = 0; q < nsteps; ++q) {
    const int form = next_form();
    plan.emplace_back(form, dt_due(c, ++c->cyc_n, ++c->cyc_i));
  }
  // capture the graphs these iterations need, then replay them in order
  for (const auto& fo : plan) {
    cudaGraphExec_t& g = c->gexec[fo.first][fo.second];
    if (!g)
      CK(capture(c, &g, &c->nk_graph[fo.first][fo.second],
                 [&] { return enqueue(fo.first, false, fo.second); }));
  }
  for (size_t q = 0; q < plan.size(); ++q) {
    const auto& fo = plan[q];
    if (q >= replay0) CK(cudaGraphLaunch(c->gexec[fo.first][fo.second], c->st));
    c->kernels_launched += c->nk_graph[fo.first][fo.second];
  }
  return CNS_OK;
}

int cns_sweep_tiles(cns_ctx* c, int precision, int32_t* cfg) {
  if (!c || !cfg || precision < 0 || precision > 2) return CNS_EINVAL;
  const TileBuf& t = precision == 0 ? c->tiles64 : c->tiles32;
  cfg[0] = t.ti;
  cfg[1] = t.tj;
  cfg[2] = t.kc;
  cfg[3] = precision == 0 ? c->tune_src64 : c->tune_src32;
  return CNS_OK;
}

int cns_set_tune_cache(cns_ctx* c, const char* path) {
  if (!c) return CNS_EINVAL;
  c->tune_cache = path ? path : "";
  return CNS_OK;
}

int cns_set_sweep_tiles(cns_ctx* c, int precision, int ti, int tj, int kc) {
  if (!c || precision < 0 || precision > 2 || kc < 1) return CNS_EINVAL;
  bool ok = false;
  for (int sh = 0; sh < kSweepShapes; ++sh)
    ok = ok || (kSweepShape[sh][0] == ti && kSweepShape[sh][1] == tj);
  if (!ok) return fail(c, CNS_EINVAL, "sweep patch shape not one of 32x4, 32x8, 16x8, 16x16");
  CK(cudaStreamSynchronize(c->st));
  CK(build_tiles(c, precision == 0 ? c->tiles64 : c->tiles32, ti, tj, kc));
  if (precision != 0) persistent_sweep32(c);
  (precision == 0 ? c->tuned64 : c->tuned32) = true;
  (precision == 0 ? c->tune_src64 : c->tune_src32) = 0;
  drop_graphs(c);
  return CNS_OK;
}

int cns_set_sweep_staging(cns_ctx* c, int mode) {
  if (!c || mode < 0 || mode > 1) return CNS_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  c->staging32 = mode;
  persistent_sweep32(c);
  drop_graphs(c);
  return CNS_OK;
}

int cns_sweep_staging(cns_ctx* c, int32_t* mode) {
  if (!c || !mode) return CNS_EINVAL;
  *mode = c->staging32;
  return CNS_OK;
}

int cns_set_residual_tiles(cns_ctx* c, int ti, int tj, int kc) {
  if (!c || ti < 0 || tj < 0 || kc < 0) return CNS_EINVAL;
  CK(cudaStreamSynchronize(c->st));
  if (ti == 0) {
    c->res_fused = false;
    drop_graphs(c);
    return CNS_OK;
  }
  bool ok = kc >= 1;
  bool shape = false;
  for (int sh = 0; sh < kResShapes; ++sh)
    shape = shape || (kResShape[sh][0] == ti && kResShape[sh][1] == tj);
  if (!ok || !shape)
    return fail(c, CNS_EINVAL, "residual patch shape not one of 32x4, 16x8, or kc < 1");
  CK(build_tiles(c, c->tiles_res, ti, tj, kc));
  c->res_fused = true;
  drop_graphs(c);
  return CNS_OK;
}

int cns_residual_tiles(cns_ctx* c, int32_t* cfg) {
  if (!c || !cfg) return CNS_EINVAL;
  cfg[0] = c->res_fused ? c->tiles_res.ti : 0;
  cfg[1] = c->res_fused ? c->tiles_res.tj : 0;
  cfg[2] = c->res_fused ? c->tiles_res.kc : 0;
  return CNS_OK;
}

int cns_last_norms(cns_ctx* c, double* norms) {
  if (!c) return CNS_EINVAL;
  CK(cudaMemcpyAsync(c->h_norms, c->w.norms, 15 * sizeof(double), cudaMemcpyDeviceToHost,
                     c->st));
  int rc = check_status(c);
  if (rc) return rc;
  if (norms) std::memcpy(norms, c->h_norms, 15 * sizeof(double));
  for (int q = 0; q < 15; ++q)
    if (!std::isfinite(c->h_norms[q])) return fail(c, CNS_ENONFINITE, "non-finite residual norm");
  return CNS_OK;
}

int cns_atsch_num_step(cns_ctx* c, int nsteps, double* norms) {
  int rc = cns_atsch_num_launch(c, nsteps);
  if (rc) return rc;
  if (nsteps == 0) return check_status(c);
  return cns_last_norms(c, norms);
}

int cns_atsch_num_step_host(cns_ctx* c, double* v_host, int nsteps, double* norms) {
  if (!c || !v_host) return CNS_EINVAL;
  if (!c->bound) return fail(c, CNS_ENOTREADY, "bind the state first");
  // the (ld, 5) state, or (ld, 7) with a turbulence step
  const size_t bytes = sizeof(double) * (c->sa_on || c->ke_on ? 7 : 5) * (size_t)c->lay.ld;
  CK(cudaMemcpyAsync(c->state.v, v_host, bytes, cudaMemcpyHostToDevice, c->st));
  int rc = cns_atsch_num_step(c, nsteps, norms);
  if (rc) return rc;
  CK(cudaMemcpyAsync(v_host, c->state.v, bytes, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CNS_OK;
}

/* ---- reference grid and flow files ------------------------------------ */

int cns_set_subrecord_length(cns_ctx* c, int64_t bytes) {
  if (!c || bytes < 1 || bytes > 2147483639) return CNS_EINVAL;
  c->io_maxsub = bytes;
  return CNS_OK;
}

int cns_readdg(cns_ctx* c, const char* path, double* x, double* y, double* z) {
  if (!c || !path || !x || !y || !z) return CNS_EINVAL;
  cns::IoPlan p, none;
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    int lo[3], hi[3];
    io_box(c->lay.blks[b], 0, lo, hi);
    for (double* a : {x, y, z}) cns::io_add(p, (int)b, a, 0, lo, hi);
  }
  return cns::io_read(c->io_stage, p, none, c->d_blks, path, c->st, c->err);
}

int cns_writdg(cns_ctx* c, const char* path, const char* disc, const double* x,
               const double* y, const double* z) {
  if (!c || !path || !disc || !x || !y || !z) return CNS_EINVAL;
  int what;
  if (!std::strncmp(disc, "cvcv", 4)) what = 0;
  else if (!std::strncmp(disc, "cvcc", 4)) what = 1;
  else if (!std::strncmp(disc, "cvcf", 4)) what = 2;
  else return fail(c, CNS_EINVAL, "disc must be cvcv, cvcc or cvcf");
  cns::IoPlan p;
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    int lo[3], hi[3];
    io_box(c->lay.blks[b], what, lo, hi);
    for (const double* a : {x, y, z})
      cns::io_add(p, (int)b, const_cast<double*>(a), what != 0, lo, hi);
  }
  return cns::io_write(c->io_stage, p, c->d_blks, path, c->io_maxsub, c->st, c->err);
}

int cns_readda(cns_ctx* c, const char* path, const char* equat, int keinit, double* v,
               double* mut) {
  if (!c || !path || !equat || !v) return CNS_EINVAL;
  bool ns, ke;
  equat_keys(equat, ns, ke);
  if (ns && !mut) return fail(c, CNS_EINVAL, "equat 'ns': mut is read too");
  const long long ld = c->lay.ld;
  cns::IoPlan p, zero;
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    int lo[3], hi[3];
    io_box(c->lay.blks[b], 1, lo, hi);
    for (int a = 0; a < 5; ++a) cns::io_add(p, (int)b, v + a * ld, 0, lo, hi);
    if (ns) cns::io_add(p, (int)b, mut, 0, lo, hi);
    for (int a = 5; a < 7 && ke; ++a)
      cns::io_add(keinit == 0 ? p : zero, (int)b, v + a * ld, 0, lo, hi);
  }
  return cns::io_read(c->io_stage, p, zero, c->d_blks, path, c->st, c->err);
}

int cns_writda(cns_ctx* c, const char* path, const char* disc, const char* equat,
               const double* v, const double* mut) {
  if (!c || !path || !disc || !equat || !v) return CNS_EINVAL;
  int what;
  if (!std::strncmp(disc, "cccc", 4)) what = 1;
  else if (!std::strncmp(disc, "cccf", 4)) what = 2;
  else return fail(c, CNS_EINVAL, "disc must be cccc or cccf");
  bool ns, ke;
  equat_keys(equat, ns, ke);
  if (ns && !mut) return fail(c, CNS_EINVAL, "equat 'ns': mut is written too");
  const long long ld = c->lay.ld;
  double* w = const_cast<double*>(v);
  cns::IoPlan p;
  for (size_t b = 0; b < c->lay.blks.size(); ++b) {
    int lo[3], hi[3];
    io_box(c->lay.blks[b], what, lo, hi);
    for (int a = 0; a < 5; ++a) cns::io_add(p, (int)b, w + a * ld, 0, lo, hi);
    if (ns) cns::io_add(p, (int)b, const_cast<double*>(mut), 0, lo, hi);
    for (int a = 5; a < 7 && ke; ++a) cns::io_add(p, (int)b, w + a * ld, 0, lo, hi);
  }
  return cns::io_write(c->io_stage, p, c->d_blks, path, c->io_maxsub, c->st, c->err);
}

/* ---- iteration counters and dual time stepping -------------------------- */

int cns_set_cycle(cns_ctx* c, int64_t ncyc, int64_t icyc) {
  if (!c || ncyc < 0 || icyc < 0) return CNS_EINVAL;
  c->cyc_n = ncyc;
  c->cyc_i = icyc;
  return CNS_OK;
}

int cns_set_dual_cycle(cns_ctx* c, int icycle) {
  if (!c) return CNS_EINVAL;
  const double before = dual_fact(c);
  c->dual_icycle = icycle;
  if (dual_fact(c) != before) drop_graphs(c);  // sch_dual's factor is a graph constant
  return CNS_OK;
}

int cns_sch_duin(cns_ctx* c) {
  if (!c) return CNS_EINVAL;
  const cns_state_t& s = c->state;
  if (!c->bound || !s.ptdual || !s.vdual || !s.vdual1 || !s.vdual2)
    return fail(c, CNS_ENOTREADY, "bind the state with its dual time arrays first");
  CK(launch_dual_update(c->d_blks, c->cells.view(-1), c->lay.ld, 0, s.v, s.ptdual, s.vdual,
                        s.vdual1, s.vdual2, c->st));
  return CNS_OK;
}

int cns_sch_duup(cns_ctx* c) {
  if (!c) return CNS_EINVAL;
  const cns_state_t& s = c->state;
  if (!c->bound || !s.ptdual || !s.vdual || !s.vdual1 || !s.vdual2)
    return fail(c, CNS_ENOTREADY, "bind the state with its dual time arrays first");
  CK(launch_dual_update(c->d_blks, c->cells.view(-1), c->lay.ld, c->sc.kdualns == 2 ? 2 : 1,
                        s.v, s.ptdual, s.vdual, s.vdual1, s.vdual2, c->st));
  return CNS_OK;
}

int cns_sch_dual(cns_ctx* c, int l, double* u, const double* v, int icycle, const double* vol,
                 const double* ptdual) {
  if (!c || bad_block(c, l) || l == 0 || !u || !v || !vol || !ptdual) return CNS_EINVAL;
  if (!(c->sc.dt1min > 0.)) return fail(c, CNS_EINVAL, "sch_dual needs dt1min > 0");
  double fact = c->sc.kdualns == 2 ? 11. / 6. : 1.5;
  if (icycle <= 1) fact = 1.;
  CK(launch_dual(c->d_blks, c->cells.view(l - 1), c->lay.ld, fact, 1. / c->sc.dt1min, v, vol,
                 ptdual, u, nullptr, c->st));
  return CNS_OK;
}

}  // extern "C"
