// cns_io.cu -- the reference's grid and flow files, read into and written
// from the device arrays.
//
// Files (opened by solve.f90:401-404; one block after another in block
// order, each block's records in the order listed; a record holds one array
// over an (i, j, k) range of the block, i fastest, then j, then k):
//   fgv  x, y, z at the real nodes (readdg.f90:71-80; svgr 'cvcv' ->
//        cvcvg.f90, writdg.f90:46-48)
//   fgc  x, y, z at the real cell centres (svgr 'cvcc' -> cvccg.f90)
//   fgcf x, y, z at the cell centres with the ghost layer (svgr 'cvcf')
//   fac  rho, rho u, rho v, rho w, rho E at the real cells, then mut when
//        equat(1:2) = 'ns', then v(:,6), v(:,7) when equat(6:7) = 'ke'
//        (readda.f90:88-113; svfw 'cccc' -> cccca.f90, writda.f90:78-97)
//   facf the same at the cells with the ghost layer (svfw 'cccf')
//
// Record layout: gfortran's unformatted sequential format with 4-byte
// markers in the machine's byte order.  A logical record is one or more
// subrecords; a subrecord is a leading marker, the data and a trailing
// marker.  A marker holds the subrecord's byte count, negated on the leading
// marker when another subrecord follows and on the trailing marker when one
// precedes.  A subrecord holds at most 2147483639 bytes unless the writer is
// given a smaller limit (gfortran's -fmax-subrecord-length).  A Fortran READ
// that takes fewer items than a record holds skips the rest of the record;
// one that needs more fails.
//
// Data path.  The file's data (markers dropped) is one image of doubles in
// device memory, records back to back.  A read streams the data through a
// small ring of pinned host slots: each slot is copied to its place in the
// image as soon as it is full, while the next slot fills from the file, so
// the file read and the transfer overlap; one kernel then scatters the image
// into the ghosted arrays, so nothing is modified unless the whole file
// parsed.  A write gathers the arrays into the image with one kernel (cell
// centres averaged on the fly), then streams the image back through the ring
// (copies of the next slots in flight while one slot is written to the
// file), framing the records on the way.  Host memory stays at the ring's
// size whatever the grid's.
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cns_abi.h"
#include "cns_kernels.cuh"

namespace cns {

namespace {

// value t of the image <-> its array element; mode 0: array = image,
// 1: image = array (or the centre of the cell's 8 nodes), 2: array = 0
__global__ void __launch_bounds__(256) k_io(const Blk* __restrict__ blks,
                                            const IoRec* __restrict__ recs, int nrec,
                                            long long nval, double* __restrict__ img, int mode) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nval; t += stride) {
    int a = 0, b = nrec - 1;
    while (a < b) {
      const int m = (a + b + 1) >> 1;
      if (recs[m].img <= t) a = m;
      else b = m - 1;
    }
    const IoRec& r = recs[a];
    const Blk& B = blks[r.blk];
    const long long e = t - r.img;
    const long long q = e / r.ext[0];
    const int i = r.lo[0] + (int)(e - q * r.ext[0]);
    const int j = r.lo[1] + (int)(q % r.ext[1]);
    const int k = r.lo[2] + (int)(q / r.ext[1]);
    const long long n = B.npc + i + (long long)j * B.nid + (long long)k * B.nijd;
    if (mode == 0) {
      r.arr[n] = img[t];
    } else if (mode == 2) {
      r.arr[n] = 0.0;
    } else if (!r.centre) {
      img[t] = r.arr[n];
    } else {
      // cvccg.f90: .125 * the sum of the 8 nodes of the cell, in its order
      const double* x = r.arr;
      const long long i1 = 1, i2 = B.nid, i3 = B.nijd;
      const double s = x[n] + x[n + i3] + x[n + i1] + x[n + i1 + i3] + x[n + i2] +
                       x[n + i2 + i3] + x[n + i1 + i2] + x[n + i1 + i2 + i3];
      img[t] = 0.125 * s;
    }
  }
}

int io_fail(std::string& err, int code, const std::string& msg) {
  err = msg;
  return code;
}

constexpr int kSlots = IoStage::kSlots;
constexpr size_t kSlotBytes = IoStage::kSlotBytes;

// file bytes -> device image through the ring
struct Upload {
  IoStage& s;
  char* dimg;
  cudaStream_t st;
  size_t dpos = 0, fill = 0;
  int cur = 0;
  bool used[kSlots] = {};
  cudaError_t e = cudaSuccess;
  char* slot() { return s.ring + (size_t)cur * kSlotBytes; }
  void flush() {
    if (fill == 0 || e != cudaSuccess) return;
    e = cudaMemcpyAsync(dimg + dpos, slot(), fill, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev[cur], st);
    used[cur] = true;
    dpos += fill;
    fill = 0;
    cur = (cur + 1) % kSlots;
    if (used[cur] && e == cudaSuccess) e = cudaEventSynchronize(s.ev[cur]);  // slot free again
  }
  // n bytes of the file into the image; false at the end of the file
  bool put(FILE* f, size_t n) {
    while (n > 0) {
      if (e != cudaSuccess) return false;
      const size_t m = n < kSlotBytes - fill ? n : kSlotBytes - fill;
      if (fread(slot() + fill, 1, m, f) != m) return false;
      fill += m;
      n -= m;
      if (fill == kSlotBytes) flush();
    }
    return true;
  }
};

// device image -> file bytes through the ring (kSlots slot copies in flight)
struct Download {
  IoStage& s;
  const char* dimg;
  size_t total;
  cudaStream_t st;
  size_t chunk = 0, off = 0;
  cudaError_t e = cudaSuccess;
  size_t len(size_t c) const {
    const size_t a = c * kSlotBytes;
    return a >= total ? 0 : (total - a < kSlotBytes ? total - a : kSlotBytes);
  }
  void issue(size_t c) {
    if (len(c) == 0 || e != cudaSuccess) return;
    char* dst = s.ring + (c % kSlots) * kSlotBytes;
    e = cudaMemcpyAsync(dst, dimg + c * kSlotBytes, len(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev[c % kSlots], st);
  }
  void start() {
    for (size_t c = 0; c < (size_t)kSlots; ++c) issue(c);
  }
  // the next n bytes of the image into the file
  bool give(FILE* f, size_t n) {
    while (n > 0) {
      if (e != cudaSuccess) return false;
      if (off == 0) e = cudaEventSynchronize(s.ev[chunk % kSlots]);
      if (e != cudaSuccess) return false;
      const size_t L = len(chunk);
      if (L == 0) return false;
      const size_t m = n < L - off ? n : L - off;
      if (fwrite(s.ring + (chunk % kSlots) * kSlotBytes + off, 1, m, f) != m) return false;
      off += m;
      n -= m;
      if (off == L) {  // slot written out: refill it with the chunk kSlots ahead
        issue(chunk + kSlots);
        ++chunk;
        off = 0;
      }
    }
    return true;
  }
};

// the data of one logical record into the image (want bytes; a longer
// record's remainder is skipped, a shorter one is an error)
int read_record(FILE* f, Upload& up, long long want, size_t r, std::string& err) {
  long long got = 0;
  bool first = true;
  char skip[4096];
  const std::string rec = std::to_string(r + 1);
  for (;;) {
    int32_t m1, m2;
    if (fread(&m1, 4, 1, f) != 1)
      return io_fail(err, CNS_EFORMAT, "file ends before record " + rec);
    const long long len = m1 < 0 ? -(long long)m1 : (long long)m1;
    const long long take = len < want - got ? len : want - got;
    if (take > 0 && !up.put(f, (size_t)take))
      return io_fail(err, CNS_EFORMAT, "file ends inside record " + rec);
    got += take;
    for (long long left = len - take; left > 0;) {
      const size_t s = left < (long long)sizeof(skip) ? (size_t)left : sizeof(skip);
      if (fread(skip, 1, s, f) != s)
        return io_fail(err, CNS_EFORMAT, "file ends inside record " + rec);
      left -= (long long)s;
    }
    if (fread(&m2, 4, 1, f) != 1)
      return io_fail(err, CNS_EFORMAT, "file ends inside record " + rec);
    const long long len2 = m2 < 0 ? -(long long)m2 : (long long)m2;
    if (len2 != len || (m2 < 0) == first)
      return io_fail(err, CNS_EFORMAT, "record markers of record " + rec + " do not match");
    first = false;
    if (m1 >= 0) break;
  }
  if (got < want)
    return io_fail(err, CNS_EFORMAT,
                   "record " + rec + " holds " + std::to_string(got) + " bytes, " +
                       std::to_string(want) + " expected");
  return CNS_OK;
}

// one logical record of n image bytes in subrecords of at most maxsub bytes
bool write_record(FILE* f, Download& dn, long long n, long long maxsub) {
  bool first = true;
  long long left = n;
  do {
    const long long len = left < maxsub ? left : maxsub;
    const bool more = left > len;
    const int32_t m1 = (int32_t)(more ? -len : len), m2 = (int32_t)(first ? len : -len);
    if (fwrite(&m1, 4, 1, f) != 1) return false;
    if (len > 0 && !dn.give(f, (size_t)len)) return false;
    if (fwrite(&m2, 4, 1, f) != 1) return false;
    left -= len;
    first = false;
  } while (left > 0);
  return true;
}

int grid_of(long long nval) {
  const long long g = (nval + 255) / 256;
  return (int)(g < 148 * 16 ? (g > 0 ? g : 1) : 148 * 16);
}

// the device image and the record table of one call
struct IoBufs {
  double* d = nullptr;
  IoRec* d_recs = nullptr;
  IoRec* d_zero = nullptr;
  ~IoBufs() {
    if (d) cudaFree(d);
    if (d_recs) cudaFree(d_recs);
    if (d_zero) cudaFree(d_zero);
  }
};

cudaError_t upload_recs(const IoPlan& p, IoRec** d) {
  if (p.recs.empty()) return cudaSuccess;
  cudaError_t e = cudaMalloc(d, sizeof(IoRec) * p.recs.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(*d, p.recs.data(), sizeof(IoRec) * p.recs.size(), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

cudaError_t io_stage_init(IoStage& s) {
  if (s.ring) return cudaSuccess;
  cudaError_t e = cudaHostAlloc(&s.ring, kSlots * kSlotBytes, cudaHostAllocDefault);
  for (int c = 0; c < kSlots && e == cudaSuccess; ++c)
    e = cudaEventCreateWithFlags(&s.ev[c], cudaEventDisableTiming);
  if (e != cudaSuccess) io_stage_free(s);
  return e;
}

void io_stage_free(IoStage& s) {
  for (int c = 0; c < kSlots; ++c)
    if (s.ev[c]) {
      cudaEventDestroy(s.ev[c]);
      s.ev[c] = nullptr;
    }
  if (s.ring) cudaFreeHost(s.ring);
  s.ring = nullptr;
}

void io_add(IoPlan& p, int b, double* arr, int centre, const int lo[3], const int hi[3]) {
  IoRec r{};
  r.img = p.nval;
  r.arr = arr;
  r.blk = b;
  r.centre = centre;
  long long n = 1;
  for (int a = 0; a < 3; ++a) {
    r.lo[a] = lo[a];
    r.ext[a] = hi[a] - lo[a] + 1;
    n *= r.ext[a];
  }
  r.nval = n;
  p.recs.push_back(r);
  p.nval += n;
}

int io_read(IoStage& stage, const IoPlan& p, const IoPlan& zero, const Blk* d_blks,
            const char* path, cudaStream_t st, std::string& err) {
  FILE* f = fopen(path, "rb");
  if (!f) return io_fail(err, CNS_EIO, std::string("cannot open ") + path);
  IoBufs bf;
  cudaError_t e = io_stage_init(stage);
  if (e == cudaSuccess) e = cudaMalloc(&bf.d, sizeof(double) * (size_t)(p.nval > 0 ? p.nval : 1));
  if (e == cudaSuccess) e = upload_recs(p, &bf.d_recs);
  if (e == cudaSuccess) e = upload_recs(zero, &bf.d_zero);
  if (e != cudaSuccess) {
    fclose(f);
    return io_fail(err, CNS_ECUDA, std::string("file buffers: ") + cudaGetErrorString(e));
  }
  Upload up{stage, reinterpret_cast<char*>(bf.d), st};
  int rc = CNS_OK;
  for (size_t r = 0; r < p.recs.size() && rc == CNS_OK && up.e == cudaSuccess; ++r)
    rc = read_record(f, up, 8 * p.recs[r].nval, r, err);
  fclose(f);
  up.flush();
  e = up.e;
  if (e != cudaSuccess) rc = CNS_OK;  // a failed copy, not the file, stopped the read
  if (rc == CNS_OK && e == cudaSuccess && p.nval > 0) {
    k_io<<<grid_of(p.nval), 256, 0, st>>>(d_blks, bf.d_recs, (int)p.recs.size(), p.nval, bf.d,
                                          0);
    e = cudaGetLastError();
  }
  if (rc == CNS_OK && e == cudaSuccess && zero.nval > 0) {
    k_io<<<grid_of(zero.nval), 256, 0, st>>>(d_blks, bf.d_zero, (int)zero.recs.size(),
                                             zero.nval, nullptr, 2);
    e = cudaGetLastError();
  }
  const cudaError_t es = cudaStreamSynchronize(st);  // the ring and the image are reused
  if (e == cudaSuccess) e = es;
  if (rc != CNS_OK) return rc;
  if (e != cudaSuccess)
    return io_fail(err, CNS_ECUDA, std::string("file read: ") + cudaGetErrorString(e));
  return CNS_OK;
}

int io_write(IoStage& stage, const IoPlan& p, const Blk* d_blks, const char* path,
             long long maxsub, cudaStream_t st, std::string& err) {
  IoBufs bf;
  cudaError_t e = io_stage_init(stage);
  if (e == cudaSuccess) e = cudaMalloc(&bf.d, sizeof(double) * (size_t)(p.nval > 0 ? p.nval : 1));
  if (e == cudaSuccess) e = upload_recs(p, &bf.d_recs);
  if (e == cudaSuccess && p.nval > 0) {
    k_io<<<grid_of(p.nval), 256, 0, st>>>(d_blks, bf.d_recs, (int)p.recs.size(), p.nval, bf.d,
                                          1);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    cudaStreamSynchronize(st);
    return io_fail(err, CNS_ECUDA, std::string("file write: ") + cudaGetErrorString(e));
  }
  FILE* f = fopen(path, "wb");
  if (!f) {
    cudaStreamSynchronize(st);
    return io_fail(err, CNS_EIO, std::string("cannot create ") + path);
  }
  Download dn{stage, reinterpret_cast<const char*>(bf.d), 8 * (size_t)p.nval, st};
  dn.start();
  bool ok = true;
  for (size_t r = 0; r < p.recs.size() && ok; ++r)
    ok = write_record(f, dn, 8 * p.recs[r].nval, maxsub);
  const bool closed = fclose(f) == 0;
  e = dn.e;
  const cudaError_t es = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess)
    return io_fail(err, CNS_ECUDA, std::string("file write: ") + cudaGetErrorString(e));
  if (!ok || !closed) return io_fail(err, CNS_EIO, std::string("cannot write ") + path);
  return CNS_OK;
}

}  // namespace cns
