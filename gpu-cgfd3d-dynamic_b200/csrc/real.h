// real.h -- the arithmetic type of the device state and kernels.
//
// The solver computes in float, as the reference does (every hot-path
// value is float: src/forward/sv_curv_col_el_iso_gpu.cu,
// trial_slipweakening.cu).  The same sources built with -DCGFD_FP64 give
// libcgfd64.so, whose kernels compute and store in double; its C ABI is the
// same (float inputs widened on upload, float outputs narrowed on
// read-back), so that the float build's rounding error can be stated
// against a double build of the same kernels on the same inputs.
//
//   real    float / double
//   real4   a group of four components: float4 (16 bytes) / four doubles
//           (32 bytes, read as two 16-byte loads)
//   RL(x)   a literal of type real: x##f / x
#pragma once
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace cgfd {

#ifdef CGFD_FP64
typedef double real;
#define RL(x) x
#ifdef __CUDACC__
struct __align__(32) real4 { double x, y, z, w; };
__host__ __device__ __forceinline__ real4 make_real4(double x, double y, double z, double w) {
  real4 r; r.x = x; r.y = y; r.z = z; r.w = w; return r;
}
// read-only load of a group through the non-coherent path: two 16-byte loads
using ::__ldg;
__device__ __forceinline__ real4 __ldg(const real4 *p) {
  const double2 a = ::__ldg(reinterpret_cast<const double2 *>(p));
  const double2 b = ::__ldg(reinterpret_cast<const double2 *>(p) + 1);
  return make_real4(a.x, a.y, b.x, b.y);
}
#endif
#else
typedef float real;
#define RL(x) x##f
#ifdef __CUDACC__
typedef float4 real4;
__host__ __device__ __forceinline__ real4 make_real4(float x, float y, float z, float w) {
  return make_float4(x, y, z, w);
}
#endif
#endif

}  // namespace cgfd
