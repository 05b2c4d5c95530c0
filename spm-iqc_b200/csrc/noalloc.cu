// Allocation-free inner products: spm_inpfp_batch_noalloc.
//
// Some callers cannot allocate device memory at the moment they need an inner
// product: a host program whose device memory is already fully reserved by its
// own pool allocator (so any cudaMalloc would fail or fragment the pool), or a
// caller that must not let cudaMalloc's implicit device-wide synchronisation
// stall its other streams. This entry point needs no context and performs no
// allocation: the caller passes the input fields and a device output array,
// and the reduction's scratch (per-CTA partial sums and completion tickets)
// lives in the file-scope device array below.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxFields (16) field pairs per call; larger batches are
//    rejected with SPM_ERR_ARG before anything is enqueued;
//  * the scratch is one array per device, shared by every call on that device
//    and holding whatever the previous call left in it; the tickets are cleared
//    by the cudaMemsetAsync that each call enqueues ahead of its kernel (that
//    clear is what later calls rely on, also after a kernel that was aborted
//    half way), and the partials are always written before they are read;
//  * the stream and the pointers must belong to the device that is current
//    when the call is made: the scratch address is looked up for that device;
//  * two calls whose kernels overlap on the GPU (different streams, no ordering
//    between them) race on the scratch and give wrong results; order them;
//  * the first call on each device looks up the device address of the scratch
//    (cudaGetSymbolAddress, with that device current) and keeps it for the
//    life of the process. Make that first call before any stream capture
//    begins. After a cudaDeviceReset (or any teardown of the device's primary
//    context) the array may live at another address: do not use this entry
//    point on that device afterwards.
// The array stays resident on every device that loads this library until the
// process exits (about 77 KB).
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/spmiqc.h"
#include "fft_core.cuh"
#include "spm_internal.h"

namespace {

constexpr int kNoAllocMaxFields = 16;
constexpr int kNoAllocBlocks = 592;  // 4 CTAs of 256 threads per SM on 148 SMs
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocDoubles = kNoAllocMaxFields * kNoAllocBlocks + 64;  // partials, then tickets

// The scratch of the allocation-free reduction (see the file comment).
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

std::mutex g_mu;
void *g_scratch_addr[64] = {nullptr};  // device address per device ordinal

// partials: [field][block]; tickets: kNoAllocMaxFields unsigned after them.
template <class T>
__global__ void __launch_bounds__(kNoAllocThreads)
    inpfp_noalloc_kernel(const T *__restrict__ p, const T *__restrict__ q, size_t n, double inv_n,
                         double *scratch, double *out) {
  __shared__ double red[32];
  __shared__ int s_last;
  const int b = blockIdx.y;
  double *partials = scratch + (size_t)b * kNoAllocBlocks;
  unsigned *ticket = reinterpret_cast<unsigned *>(scratch + (size_t)kNoAllocMaxFields * kNoAllocBlocks) + b;
  const T *pb = p + (size_t)b * n;
  const T *qb = q + (size_t)b * n;
  double a[1] = {0.0};
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    a[0] += (double)__ldg(pb + i) * (double)__ldg(qb + i);
  spm::block_reduce<1, 0u>(a, red);
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = a[0];
    __threadfence();
    s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1u);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t[1] = {0.0};
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) t[0] += __ldcg(partials + i);
  spm::block_reduce<1, 0u>(t, red);
  if (threadIdx.x == 0) out[b] = t[0] * inv_n;
}

int scratch_address(void **addr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return spm_fail_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return spm_fail(SPM_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return spm_fail_cuda(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_addr[dev] = ptr;
  }
  *addr = g_scratch_addr[dev];
  return SPM_OK;
}

}  // namespace

extern "C" int spm_inpfp_batch_noalloc(size_t n, int nb, int precision, const void *p, const void *q,
                                       double *out, void *stream) {
  if (nb < 1 || nb > kNoAllocMaxFields)
    return spm_fail(SPM_ERR_ARG, "spm_inpfp_batch_noalloc: nb must be in [1, 16] (scratch is sized for 16 fields)");
  if (n == 0 || !p || !q || !out) return spm_fail(SPM_ERR_ARG, "spm_inpfp_batch_noalloc: empty field or NULL pointer");
  if (precision != SPM_FP64 && precision != SPM_FP32)
    return spm_fail(SPM_ERR_UNSUPPORTED, "spm_inpfp_batch_noalloc: precision");
  void *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != SPM_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  double *sd = reinterpret_cast<double *>(scratch);
  cudaError_t e = cudaMemsetAsync(sd + (size_t)kNoAllocMaxFields * kNoAllocBlocks, 0,
                                  sizeof(unsigned) * kNoAllocMaxFields, s);
  if (e != cudaSuccess) return spm_fail_cuda(e, "no-alloc ticket clear");
  const size_t want = (n + kNoAllocThreads - 1) / kNoAllocThreads;
  const int blocks = (int)(want < (size_t)kNoAllocBlocks ? want : (size_t)kNoAllocBlocks);
  const double inv_n = 1.0 / (double)n;
  if (precision == SPM_FP64)
    inpfp_noalloc_kernel<double><<<dim3(blocks, nb), kNoAllocThreads, 0, s>>>(
        (const double *)p, (const double *)q, n, inv_n, sd, out);
  else
    inpfp_noalloc_kernel<float><<<dim3(blocks, nb), kNoAllocThreads, 0, s>>>(
        (const float *)p, (const float *)q, n, inv_n, sd, out);
  e = cudaGetLastError();
  return e == cudaSuccess ? SPM_OK : spm_fail_cuda(e, "no-alloc inner product launch");
}
