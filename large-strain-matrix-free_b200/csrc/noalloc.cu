// Allocation-free residual norm: ||b - A x||_2 for an FP64 operator, with all
// scratch memory in a file-scope device array instead of cudaMalloc'd buffers.
//
// Who needs it: host applications that cannot call cudaMalloc once they are
// running - for example a code whose device memory is owned by another
// framework's caching allocator (PyTorch reserves and manages the pool), or a
// deployment with a no-allocation-after-start-up rule (real-time control
// loops, certified embedded builds).  They can still evaluate the true
// residual of an operator they set up earlier.
//
// The scratch holds A x (at most LSMF_NOALLOC_MAX_DOFS doubles, 16 MiB) and
// the per-block partial sums of the reduction.  Every GPU that loads this
// file's module keeps the array until the process exits.  With CUDA's lazy
// module loading (the default) the module, and with it the array, is placed
// in device memory the first time a device uses it: at the first call of the
// entry point on that device.  A caller whose memory pool is later taken by
// another allocator makes one call at start-up (or sets
// CUDA_MODULE_LOADING=EAGER), so that the 16 MiB are placed before the pool
// is reserved.
#include <cuda_runtime.h>

#include "lsmf_internal.h"

namespace lsmf {
lsmf_status launch_apply(const lsmf_op *op, void *dst, const void *src, unsigned mask, bool add);
}

namespace {

constexpr size_t NOALLOC_PARTIALS = 1024;  // reduction blocks (fixed grid)
constexpr int NOALLOC_THREADS = 256;

// [0, LSMF_NOALLOC_MAX_DOFS): A x; then NOALLOC_PARTIALS partial sums
static __device__ __align__(256) double g_scratch[LSMF_NOALLOC_MAX_DOFS + NOALLOC_PARTIALS];

__global__ void residual_partials_kernel(const double *__restrict__ ax, const double *__restrict__ b, size_t n,
                                         double *partial) {
  __shared__ double sh[NOALLOC_THREADS / 32];
  double s = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = b[i] - ax[i];
    s += r * r;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;  // every block writes its slot
  }
}

__global__ void sqrt_sum_kernel(const double *partial, int n, double *out) {
  __shared__ double sh[32];
  double s = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += partial[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *out = sqrt(s);
  }
}

// Device address of the scratch array for the operator's device.  Host code
// must not pass g_scratch itself to a kernel: on the host that name is only a
// stand-in, not a device address.  The address is looked up on every call (a
// host-side table lookup once the module is loaded), so it stays right after
// the device's context was reset and the module placed again.
lsmf_status scratch_address(const lsmf_op *op, double **out) {
  int dev = 0;
  LSMF_CUDA(cudaGetDevice(&dev));
  if (dev != op->device) {
    lsmf::set_error("the operator lives on device " + std::to_string(op->device) + " but device " +
                    std::to_string(dev) + " is current; make the operator's device current first");
    return LSMF_ERR_INVALID_ARG;
  }
  void *p = nullptr;
  LSMF_CUDA(cudaGetSymbolAddress(&p, g_scratch));
  *out = (double *)p;
  return LSMF_OK;
}

}  // namespace

extern "C" lsmf_status lsmf_residual_norm_noalloc(lsmf_op *op, const double *d_x, const double *d_b,
                                                  double *d_norm) {
  using namespace lsmf;
  if (!op || !d_x || !d_b || !d_norm) { set_error("null argument"); return LSMF_ERR_INVALID_ARG; }
  if (op->precision != LSMF_FP64) { set_error("the allocation-free residual norm needs an FP64 operator"); return LSMF_ERR_INVALID_ARG; }
  if (!op->cached) { set_error("cache() has not been called"); return LSMF_ERR_NOT_INITIALIZED; }
  const size_t n = (size_t)op->L().n_dofs();
  if (n > (size_t)LSMF_NOALLOC_MAX_DOFS) {
    set_error("operator has " + std::to_string(n) + " dofs; the allocation-free residual norm supports at most " +
              std::to_string((size_t)LSMF_NOALLOC_MAX_DOFS));
    return LSMF_ERR_INVALID_ARG;
  }
  double *scratch = nullptr;
  LSMF_TRY(scratch_address(op, &scratch));
  double *ax = scratch, *partial = scratch + LSMF_NOALLOC_MAX_DOFS;
  // A x into the scratch (the vmult overwrites every entry it owns: zero, cell
  // contributions, identity rows), then the fused (b - A x)^2 reduction
  LSMF_TRY(launch_apply(op, ax, d_x, LSMF_MASK_DEFAULT, false));
  residual_partials_kernel<<<(int)NOALLOC_PARTIALS, NOALLOC_THREADS, 0, op->stream>>>(ax, d_b, n, partial);
  sqrt_sum_kernel<<<1, 1024, 0, op->stream>>>(partial, (int)NOALLOC_PARTIALS, d_norm);
  LSMF_CUDA(cudaGetLastError());
  return LSMF_OK;
}
