// cns_common.cuh -- device-side layout, index spaces and shared helpers of
// the CodeNS hot path on sm_100a.
//
// Layout (the reference's per-block arrays, crdms.f90:125-158): every block
// has real nodes 1..ni (one ghost layer on each side, id1 = 0), nodes and
// cells share one flat index space, block l starts at npc(l).  Cell
// (i,j,k) is npc + i + j*nid + k*nid*njd.  State arrays are column-major
// (ld, ncol); the normals of a block sit at sn[9*npc ...] as
// sn(nnn, 3 directions, 3 components).
//
// Work decomposition: every kernel walks an "index space" (real cells, the
// faces of one direction, the lines of one direction, a boundary list)
// through a tile work list built once on the host: tile t covers elements
// [start, start+TILE) of one block, so uneven blocks and many independent
// cases share a single launch with no per-thread block search.
//
// Arithmetic: the parity build compiles with --fmad=false and evaluates the
// reference expressions in the reference's left-to-right order, so every
// FP64 result is bit-identical to the reference semantics (IEEE add, mul,
// div and sqrt are correctly rounded on both sides).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cns {

constexpr int kMaxBlocks = 4096;

struct Blk {
  int ni, nj, nk;           // real node counts (ii2, jj2, kk2)
  int nid, njd, nkd;        // with the ghost layer
  long long npc;            // flat offset of the block
  long long nijd, nnn;
  double eta, ki2, ki4;     // the block's eta(lm), ki2(lm), ki4(lm) (schemanum)
  // the padded layout of the mixed form's FP32 sweep arrays (this build's
  // own, never the caller's): rows of pid = nid rounded up to a multiple of
  // four cells, so that every row and plane starts on 16 bytes (the tensor
  // copies' rule); cell (i, j, k) at ppc + i + j pid + k pnijd
  int pid;
  long long pnijd, ppc;
  long long pld;  // the padded arrays' component stride (the same in every block)
};

__host__ __device__ __forceinline__ long long pad_index(const Blk& B, int i, int j, int k) {
  return B.ppc + (long long)i + (long long)j * B.pid + (long long)k * B.pnijd;
}

// index space over all blocks: element e of block b has extents ext[3b..3b+2]
// and maps to (i,j,k) = (1,1,1) + unflatten(e)
struct Space {
  const int* tile_blk;          // [ntiles]
  const long long* tile_start;  // [ntiles]
  const int* ext;               // [3*nblk]
  int tile0;                    // first tile of this launch
  int ntiles;
};

struct Phys {
  double gam, gam1, pinfl, pr, prt, cp, reynz, suth_a, pa1, aa1, omg;
};

struct Scheme {
  int ns, muscl, ilim, kdtl, lmax, qfix_dfez, precision, kdefect;
  double xk, eta, dt1min;
  int ischema;      // 7 Roe, 1 Jameson
  double ki2, ki4;  // Jameson dissipation coefficients
  int ncychro, icychr0;  // time-step update frequency of the fused iteration
  int kfmg, kdualns;     // 3: dual time stepping (dt1min = physical step); its order
  int weno_fix;          // WENO5: all three candidates in every direction (non-reference)
};

// 2.5D tiles of the implicit sweeps: tile t = (block, i0, j0, k0) covers
// the cells i0..i0+TI-1, j0..j0+TJ-1, k0..k0+kc-1 of the block (clipped to
// its real cells); the tiles of one block are contiguous
struct Tiles {
  const int4* tile;
  int tile0;
  int ntiles;
  int kc;
  int ti, tj;  // patch shape (selects the kernel instantiation)
  // persistent launch (kernels that support it): when sched is set, grid
  // CTAs (at most ntiles) pull tiles from the work list through the counter
  // pair sched[0..1], which the last CTA to finish resets to zero
  int* sched;
  int grid;
  // the FP32 sweep's per-cell pack (3 float4 per cell: half the area vector
  // of the cell's lower face of each direction, and that face's implicit
  // coefficient), or null
  const float4* faces;
};

// boundary tables (per boundary, then per list entry)
struct Bnd {
  int nbnd;
  long long nlist;
  const int* type;        // [nbnd]
  const int* blk;         // [nbnd] 0-based
  const int* face;        // [nbnd] 0..5 = i1,i2,j1,j2,k1,k2
  const long long* mpb;   // [nbnd]
  const int* mmb;         // [nbnd]
  const int* partner;     // [nbnd]
  const double* cosr;     // [nbnd]
  const double* sinr;     // [nbnd]
  const int* ent_bnd;     // [nlist] owning boundary of each entry
  const long long* ncbd;  // [nlist]
  const long long* ncin;  // [nlist]
  const double* bceqt;    // [5*nlist] column-major
  double* nxn;            // [nlist] filled by the metric
  double* nyn;
  double* nzn;
  double* ym;
  double* zm;
};

// BC_LP2: the adiabatic wall-law wall 'lp2', whose ghosts are those of 'para'
enum BcKind { BC_EXTR = 1, BC_RC = 2, BC_PARA = 3, BC_IDD = 4, BC_PRD = 5, BC_LP2 = 6 };

__device__ __forceinline__ double sq(double a) { return a * a; }

// element lane of tile t (counted from the launch's first tile); false
// when past the block end
__device__ __forceinline__ bool space_elem_at(const Space& sp, int tile, int lane, int& b,
                                              int& i, int& j, int& k) {
  const int t = sp.tile0 + tile;
  b = sp.tile_blk[t];
  const long long e = sp.tile_start[t] + lane;
  const int ex = sp.ext[3 * b], ey = sp.ext[3 * b + 1], ez = sp.ext[3 * b + 2];
  if (e >= (long long)ex * ey * ez) return false;
  const int ee = (int)e;
  i = ee % ex;
  const int r = ee / ex;
  j = r % ey;
  k = r / ey;
  i += 1;
  j += 1;
  k += 1;
  return true;
}

// element of the tile handled by this thread (a CTA per tile); false when
// past the block end
__device__ __forceinline__ bool space_elem(const Space& sp, int lane, int& b, int& i, int& j,
                                           int& k) {
  return space_elem_at(sp, blockIdx.x, lane, b, i, j, k);
}

__device__ __forceinline__ long long cell_index(const Blk& B, int i, int j, int k) {
  return B.npc + (long long)i + (long long)j * B.nid + (long long)k * B.nijd;
}
__device__ __forceinline__ long long ninc_of(const Blk& B, int dir) {
  return dir == 0 ? 1LL : (dir == 1 ? (long long)B.nid : B.nijd);
}
__device__ __forceinline__ int nd_of(const Blk& B, int dir) {
  return dir == 0 ? B.ni : (dir == 1 ? B.nj : B.nk);
}
// sn(m, dir, c) of the block (m local index = n - npc)
template <class T>
__device__ __forceinline__ const T* sn_ptr(const T* sn, const Blk& B, int dir, int c) {
  return sn + 9 * B.npc + (long long)c * 3 * B.nnn + (long long)dir * B.nnn - B.npc;
}

}  // namespace cns
