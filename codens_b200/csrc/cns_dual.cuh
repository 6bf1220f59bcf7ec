// cns_dual.cuh -- a forward-mode dual number (value, one directional
// derivative) for the hot-path templates.  Instantiating a T-templated
// device function with Dual and seeding one input's derivative with 1 gives
// that function's exact partial derivative with respect to the input (the
// chain rule applied to the same operations), which is how the adjoint
// builds the flux and sweep Jacobians of the discrete FP64 scheme.
#pragma once
#include <cuda_runtime.h>

namespace cns {

// keep the real-valued overloads visible next to the Dual ones
using ::fabs;
using ::sqrt;

struct Dual {
  double v, d;
  __host__ __device__ Dual() : v(0.), d(0.) {}
  __host__ __device__ Dual(double x) : v(x), d(0.) {}
  __host__ __device__ Dual(float x) : v(x), d(0.) {}
  __host__ __device__ Dual(int x) : v(x), d(0.) {}
  __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
};

__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b) {
  return Dual(a.v * b.v, a.d * b.v + a.v * b.d);
}
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual sqrt(Dual a) {
  const double r = ::sqrt(a.v);
  return Dual(r, a.d / (2. * r));
}
__device__ __forceinline__ Dual fabs(Dual a) { return a.v < 0. ? -a : a; }

}  // namespace cns
