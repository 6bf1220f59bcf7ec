// cns_noalloc.cu -- the Euler Roe residual of one block without any device
// allocation.
//
// Why: some callers cannot let a library allocate device memory.  A Fortran
// solver that hands over device arrays from its own pre-sized memory pool, a
// host running under a hard device-memory cap, or a simulation loop that must
// not grow the device heap once it has started all need an entry point that
// works only in memory they already own plus a fixed, known amount held by
// the library.  cns_sch_roe_euler_noalloc is that entry point: it computes
// what cns_sch_roe_euler computes for a single block, and keeps its
// intermediates (primitive velocities, face fluxes, work lists) in the
// file-scope array below instead of in a context created with cudaMalloc.
//
// The array is kNoallocBytes (20 MiB).  Every GPU that loads the library
// reserves it for the life of the process.  It bounds the leading dimension
// of the caller's arrays to kNoallocMaxLd = 131072 cells (a block of about
// 48 x 48 x 48 cells with its ghost layer); larger calls are rejected with
// CNS_EINVAL before anything is launched.
//
// All calls share the array and it keeps the contents of the last call.
// Every value a call reads from it is written earlier in the same call, so
// nothing has to start at zero, but two calls that overlap on the GPU (on
// different streams, or from different host threads without ordering) race
// on it: order them on one stream.
//
// The first call on a device looks up the device address of the array
// (cudaGetSymbolAddress) with that device current and remembers it; make
// that first call before any stream capture.  The remembered address belongs
// to the device's current context: after cudaDeviceReset on that device it
// is stale, so a process that resets a device must not call this entry point
// on it again.
#include <cstdint>
#include <mutex>

#include "../../include/cns_abi.h"
#include "cns_kernels.cuh"

namespace cns {
namespace {

constexpr long long kNoallocMaxLd = 131072;
constexpr int kNoallocMaxDevices = 64;
constexpr long long kMaxTiles = kNoallocMaxLd / kTile + 1;

// byte offsets inside the static array (each 256-aligned)
constexpr long long align256(long long x) { return (x + 255) / 256 * 256; }
constexpr long long kOffBlk = 0;
constexpr long long kOffExt = align256(kOffBlk + (long long)sizeof(Blk));
constexpr long long kOffTileBlk = align256(kOffExt + 4 * 3 * (long long)sizeof(int));
constexpr long long kOffTileStart = align256(kOffTileBlk + kMaxTiles * (long long)sizeof(int));
constexpr long long kOffPrim = align256(kOffTileStart + kMaxTiles * (long long)sizeof(long long));
constexpr long long kOffG = align256(kOffPrim + 3 * kNoallocMaxLd * (long long)sizeof(double));
constexpr long long kNoallocBytes = align256(kOffG + 15 * kNoallocMaxLd * (long long)sizeof(double));
static_assert(kNoallocBytes <= 20LL * 1024 * 1024, "static scratch stays at 20 MiB");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

void* g_scratch_addr[kNoallocMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// the work lists of the single block: one tile list shared by the four index
// spaces (real cells and the faces of each direction); extents at ext[3s..3s+2]
__global__ void k_noalloc_setup(Blk B, Blk* blk, int* ext, int* tile_blk,
                                long long* tile_start, int ntiles) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    *blk = B;
    const int e[4][3] = {{B.ni - 1, B.nj - 1, B.nk - 1},
                         {B.ni, B.nj - 1, B.nk - 1},
                         {B.ni - 1, B.nj, B.nk - 1},
                         {B.ni - 1, B.nj - 1, B.nk}};
    for (int s = 0; s < 4; ++s)
      for (int q = 0; q < 3; ++q) ext[3 * s + q] = e[s][q];
  }
  if (t < ntiles) {
    tile_blk[t] = 0;
    tile_start[t] = (long long)t * kTile;
  }
}

}  // namespace
}  // namespace cns

using namespace cns;

extern "C" int cns_sch_roe_euler_noalloc(int32_t ni, int32_t nj, int32_t nk,
                                         int64_t ld, double gam, double pinfl,
                                         int32_t muscl, double xk, double* u,
                                         const double* v, const double* sn,
                                         const double* ps, void* stream) {
  if (ni < 2 || nj < 2 || nk < 2 || !u || !v || !sn || !ps || muscl < 0)
    return CNS_EINVAL;
  // each ghosted side (n + 2) must fit the static array on its own before
  // the block's extents are formed, so no product below can overflow
  if ((long long)ni + 2 > kNoallocMaxLd || (long long)nj + 2 > kNoallocMaxLd ||
      (long long)nk + 2 > kNoallocMaxLd)
    return CNS_EINVAL;
  Blk B{};
  B.ni = ni;
  B.nj = nj;
  B.nk = nk;
  B.nid = ni + 2;
  B.njd = nj + 2;
  B.nkd = nk + 2;
  B.nijd = (long long)B.nid * B.njd;
  B.nnn = B.nijd * B.nkd;
  B.npc = 0;
  // the block's cells must fit the caller's arrays and the static scratch
  if (B.nnn <= 0 || B.nnn > kNoallocMaxLd || ld < B.nnn || ld > kNoallocMaxLd)
    return CNS_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices)
    return CNS_ECUDA;
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
        return CNS_ECUDA;
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  unsigned char* s8 = static_cast<unsigned char*>(base);
  Blk* d_blk = reinterpret_cast<Blk*>(s8 + kOffBlk);
  int* d_ext = reinterpret_cast<int*>(s8 + kOffExt);
  int* d_tile_blk = reinterpret_cast<int*>(s8 + kOffTileBlk);
  long long* d_tile_start = reinterpret_cast<long long*>(s8 + kOffTileStart);
  double* prim = reinterpret_cast<double*>(s8 + kOffPrim);
  double* G = reinterpret_cast<double*>(s8 + kOffG);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  const long long counts[4] = {(long long)(ni - 1) * (nj - 1) * (nk - 1),
                               (long long)ni * (nj - 1) * (nk - 1),
                               (long long)(ni - 1) * nj * (nk - 1),
                               (long long)(ni - 1) * (nj - 1) * nk};
  long long maxc = 0;
  for (long long cnt : counts) maxc = cnt > maxc ? cnt : maxc;
  const int ntiles = (int)((maxc + kTile - 1) / kTile);
  k_noalloc_setup<<<(ntiles + 255) / 256, 256, 0, st>>>(B, d_blk, d_ext, d_tile_blk,
                                                        d_tile_start, ntiles);
  // four spaces sharing the tile list, each with its own extent and tile count
  SpaceBuf sp[4];
  for (int q = 0; q < 4; ++q) {
    sp[q].ntiles = (int)((counts[q] + kTile - 1) / kTile);
    sp[q].d_tile_blk = d_tile_blk;
    sp[q].d_tile_start = d_tile_start;
    sp[q].d_ext = d_ext + 3 * q;
  }
  Phys ph{};
  ph.gam = gam;
  ph.gam1 = gam - 1.;
  ph.pinfl = pinfl;
  Scheme sc{};
  sc.ns = 0;
  sc.muscl = muscl;
  sc.xk = xk;
  // sch_roe_euler zeroes u over the whole block, ghosts included
  for (int a = 0; a < 5; ++a)
    if (cudaMemsetAsync(u + (long long)a * ld, 0, sizeof(double) * B.nnn, st) != cudaSuccess)
      return CNS_ECUDA;
  cudaError_t e = launch_prim(0, B.nnn, v, ld, prim, st);
  if (e == cudaSuccess)
    e = launch_face_flux(d_blk, sp + 1, -1, ph, sc, v, prim, ld, ps, nullptr, sn, nullptr,
                         G, st);
  if (e == cudaSuccess) e = launch_accumulate(d_blk, sp[0].view(-1), G, ld, u, st);
  return e == cudaSuccess ? CNS_OK : CNS_ECUDA;
}
