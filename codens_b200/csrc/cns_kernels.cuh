// cns_kernels.cuh -- host-side launchers of the CodeNS hot-path kernels.
#pragma once
#include <vector>

#include "cns_common.cuh"

namespace cns {

__device__ __forceinline__ double* sn_wptr(double* sn, const Blk& B, int dir,
                                           int c) {
  return sn + 9 * B.npc + (long long)c * 3 * B.nnn + (long long)dir * B.nnn - B.npc;
}

constexpr int kTile = 128;  // elements per tile (= threads per CTA)

struct HostLayout {
  std::vector<Blk> blks;
  long long ld = 0, ncells = 0, nreal = 0;
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

// per-step scratch (device)
struct Work {
  long long ld = 0;
  double* prim = nullptr;     // primitive velocities u, v, w, [3][ld]
  double* G = nullptr;        // face fluxes, [3][5][ld]
  double* R = nullptr;        // limiter ratios, [3][5][ld]
  double* coefe = nullptr;    // [3][ld]
  double* coefdiag = nullptr; // [ld]
  double* rv = nullptr;       // [ld]
  double* dpp[2] = {nullptr, nullptr};   // Jacobi iterates, [5][ld] each
  double* dfpp[2] = {nullptr, nullptr};  // flux increments, [9][ld] each
  double* normpart = nullptr; // per tile partial norms [ntiles][15]
  double* norms = nullptr;    // [16]
  int* status = nullptr;      // device status word
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

cudaError_t launch_ratio(const Blk* blks, const SpaceBuf* lines, int l0,
                         const double* v, const double* prim, long long ld,
                         const double* ps, double* R, cudaStream_t st);

cudaError_t launch_face_flux(const Blk* blks, const SpaceBuf* faces, int l0,
                             Phys ph, Scheme sc, const double* v,
                             const double* prim, long long ld, const double* ps,
                             const double* tau, const double* sn, const double* R,
                             double* G, cudaStream_t st);

cudaError_t launch_accumulate(const Blk* blks, Space sp, const double* G,
                              long long ld, double* u, cudaStream_t st);

// the implicit phase of implimf_eu (eu = 1) or implimf_3d (eu = 0) on the
// cells of the space: coefficients, lmx Jacobi sweeps, v += d; d_out
// (optional) receives the final increment, want_norms stores per-tile
// residual partials in w.normpart
cudaError_t launch_implicit(const Blk* blks, Space cells, const SpaceBuf* faces,
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
                                 double* norms, cudaStream_t st);

}  // namespace cns
