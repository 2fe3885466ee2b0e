// noalloc.cu -- the fixed device scratch of cgfd_run_noalloc.
//
// cgfd_run_noalloc advances a solver without allocating anything.  The one
// buffer a time step needs beyond the solver's own state is the per-stage
// traction scratch of the fault kernels (k_fault_trac writes it, the trial
// and slab-velocity kernels read it).  cgfd_run keeps a scratch allocated
// with the solver; the no-alloc entry point uses this file-scope device
// array instead.  Its size is fixed at build time (CGFD_NOALLOC_SCRATCH_FLOATS
// values: 32 MiB of float, 64 MiB in the double build of libcgfd64.so) and
// it is one array per device, shared by every solver in the process -- so
// two calls on the same device must not overlap.
#include <cuda_runtime.h>

#include "../../include/cgfd.h"
#include "real.h"

namespace cgfd {

namespace {
__device__ __align__(256) real g_noalloc_trac[CGFD_NOALLOC_SCRATCH_FLOATS];
}  // namespace

// device address of the array on the current device (looked up by the
// caller once per device)
cudaError_t noalloc_scratch_address(real **p) {
  return cudaGetSymbolAddress(reinterpret_cast<void **>(p), g_noalloc_trac);
}

}  // namespace cgfd
