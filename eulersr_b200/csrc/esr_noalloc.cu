// esr_noalloc.cu -- relative state change without any device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need this
// statistic: hosts whose device memory is entirely owned by their own
// allocator (a caching allocator that holds the whole budget, or a
// pre-sized arena in an embedded deployment that forbids allocation after
// start-up). The solver's own reduction (k_case_reduce) writes its per-block
// partial sums into a buffer the solver allocates; this variant keeps those
// partials in a fixed file-scope device array instead, so a call allocates
// nothing. The caller passes the two fields and the device output.
//
// Limits and sharing:
//   * at most kNoAllocMaxBlocks blocks of kNoAllocRowsPerBlock rows, i.e.
//     kNoAllocMaxRows rows; larger inputs are rejected with ESR_ERR_ARG;
//   * the partials array (kNoAllocMaxBlocks x 16 B = 16 KiB) lives on every
//     GPU that loads the library until the process exits;
//   * every call shares it and it keeps the last call's contents; each call
//     overwrites exactly the partials it reads, so nothing needs clearing,
//     but calls that overlap on the GPU (two streams at once) race on it;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current); make
//     that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "esr_device.cuh"
#include "esr_internal.h"

namespace {

constexpr int kNoAllocMaxBlocks = 1024;
constexpr int kNoAllocRowsPerBlock = 2048;
constexpr long long kNoAllocMaxRows = (long long)kNoAllocMaxBlocks * kNoAllocRowsPerBlock;
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_noalloc_partials[kNoAllocMaxBlocks];

std::mutex g_setup_mutex;
double2* g_partials_ptr[kMaxDevices] = {nullptr};

// errors go to the library's esr_last_error()
int noalloc_fail(int code, const std::string& msg) { return esr::report_error(code, msg); }

// block b sums rows [b*R, min(n,(b+1)*R)) of |A-B|^2 and |B|^2 in double
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads) k_relchange_partial(const esr::V4<T>* __restrict__ A,
                                                                        const esr::V4<T>* __restrict__ B, long long n,
                                                                        double2* __restrict__ part) {
  const long long r0 = (long long)blockIdx.x * kNoAllocRowsPerBlock;
  const long long r1 = min(n, r0 + kNoAllocRowsPerBlock);
  double s0 = 0.0, s1 = 0.0;
  for (long long r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const esr::V4<T> a = A[r], b = B[r];
    const double d0 = (double)a.x - (double)b.x, d1 = (double)a.y - (double)b.y;
    const double d2 = (double)a.z - (double)b.z, d3 = (double)a.w - (double)b.w;
    s0 += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
    s1 += (double)b.x * b.x + (double)b.y * b.y + (double)b.z * b.z + (double)b.w * b.w;
  }
  __shared__ double sh0[kNoAllocThreads], sh1[kNoAllocThreads];
  sh0[threadIdx.x] = s0;
  sh1[threadIdx.x] = s1;
  __syncthreads();
  for (int w = kNoAllocThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sh0[threadIdx.x] += sh0[threadIdx.x + w];
      sh1[threadIdx.x] += sh1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = make_double2(sh0[0], sh1[0]);
}

// fixed-order sum of the partials: ||A-B|| / (||B|| + 1e-16)
__global__ void k_relchange_final(const double2* __restrict__ part, int nb, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s0 = 0.0, s1 = 0.0;
  for (int i = 0; i < nb; ++i) {
    s0 += part[i].x;
    s1 += part[i].y;
  }
  *out = sqrt(s0) / (sqrt(s1) + 1e-16);
}

// A kernel of this file reads `p` (or writes it): it must be memory of the
// current GPU, or managed memory, aligned to `align` bytes. A host address or
// another GPU's memory is an argument error here, before any launch.
int check_device_ptr(const void* p, int dev, size_t align, const char* what) {
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();   // the failed query must not surface as a later launch's error
    return noalloc_fail(ESR_ERR_ARG, std::string("rel_change_noalloc: ") + what + ": not a device address (" +
                                         cudaGetErrorString(e) + ")");
  }
  const bool ok = (a.type == cudaMemoryTypeDevice && a.device == dev) || a.type == cudaMemoryTypeManaged;
  if (!ok) return noalloc_fail(ESR_ERR_ARG, std::string("rel_change_noalloc: ") + what + ": not device memory of the current GPU");
  if ((uintptr_t)p % align)
    return noalloc_fail(ESR_ERR_ARG, std::string("rel_change_noalloc: ") + what + " must be " + std::to_string(align) +
                                         "-byte aligned");
  return ESR_OK;
}

// device address of the partials array for the current device (set-up on first use)
int partials_for_current_device(double2** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(ESR_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(ESR_ERR_ARG, "rel_change_noalloc: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess)
      return noalloc_fail(ESR_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_partials_ptr[dev] = static_cast<double2*>(p);
  }
  *out = g_partials_ptr[dev];
  return ESR_OK;
}

}  // namespace

extern "C" {

int esr_rel_change_noalloc(const void* d_A, const void* d_B, int64_t n_rows, int32_t precision, double* d_out,
                           void* stream) {
  if (!d_A || !d_B || !d_out) return noalloc_fail(ESR_ERR_ARG, "rel_change_noalloc: null pointer");
  if (precision != ESR_PREC_F32 && precision != ESR_PREC_F64)
    return noalloc_fail(ESR_ERR_ARG, "rel_change_noalloc: precision must be ESR_PREC_F32 or ESR_PREC_F64");
  if (n_rows <= 0) return noalloc_fail(ESR_ERR_ARG, "rel_change_noalloc: n_rows must be > 0");
  if (n_rows > kNoAllocMaxRows)
    return noalloc_fail(ESR_ERR_ARG, "rel_change_noalloc: n_rows " + std::to_string(n_rows) + " exceeds the maximum " +
                                         std::to_string(kNoAllocMaxRows) + " of the fixed scratch array");
  int dev = 0;
  cudaError_t ge = cudaGetDevice(&dev);
  if (ge != cudaSuccess) return noalloc_fail(ESR_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ge));
  // the rows are read as 4-value vectors (16-byte loads), the result written as one double
  const size_t row_align = 16;
  int rc = check_device_ptr(d_A, dev, row_align, "d_A");
  if (rc == ESR_OK) rc = check_device_ptr(d_B, dev, row_align, "d_B");
  if (rc == ESR_OK) rc = check_device_ptr(d_out, dev, alignof(double), "d_out");
  if (rc != ESR_OK) return rc;
  double2* part = nullptr;
  rc = partials_for_current_device(&part);
  if (rc != ESR_OK) return rc;
  const int nb = (int)((n_rows + kNoAllocRowsPerBlock - 1) / kNoAllocRowsPerBlock);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == ESR_PREC_F64)
    k_relchange_partial<double><<<nb, kNoAllocThreads, 0, st>>>((const double4*)d_A, (const double4*)d_B, n_rows, part);
  else
    k_relchange_partial<float><<<nb, kNoAllocThreads, 0, st>>>((const float4*)d_A, (const float4*)d_B, n_rows, part);
  k_relchange_final<<<1, 32, 0, st>>>(part, nb, d_out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(ESR_ERR_CUDA, std::string("rel_change_noalloc launch: ") + cudaGetErrorString(e));
  return ESR_OK;
}

}  // extern "C"
