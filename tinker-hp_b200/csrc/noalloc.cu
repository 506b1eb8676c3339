// noalloc.cu -- polarization energy without any device allocation.
//
// Some callers cannot allocate device memory when they need the energy: a
// host program whose GPU memory is reserved up front by another runtime (an
// OpenACC / CUDA-Fortran code that pools the device, as Tinker-HP's GPU build
// does), or a latency-critical loop where the implicit device synchronisation
// of cudaMalloc/cudaFree is unacceptable.
// thp_epolar_noalloc serves them: the caller passes device arrays in and a
// device scalar out, and the only scratch the reduction needs -- one partial
// sum per thread block and a completion counter -- lives in a fixed-size
// file-scope __device__ array that every GPU loading this library holds until
// the process exits.
//
// The scratch is shared by all calls on a device and keeps the last call's
// contents; the counter is cleared before every launch.  Calls that overlap
// on the GPU (on different streams, or from different host threads) race on
// the scratch and must be ordered by the caller.
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = THP_NOALLOC_MAX_ATOMS / kThreads;

struct NoallocScratch {
  double partial[kMaxBlocks];  // one partial sum per block
  unsigned counter;            // blocks finished; the last one sums the partials
};

// 128 KiB plus the counter, allocated with the module on every device.
static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// Epol = -1/2 electric sum_i uind_i . E_p,i (the epolar0c total), summed in
// a fixed order: per-block tree reduction, then the partials in block order.
__global__ void __launch_bounds__(kThreads) k_epol_noalloc(int n, const double* __restrict__ uind,
                                                           const double* __restrict__ ef, double* __restrict__ out,
                                                           NoallocScratch* __restrict__ s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (i < n) {
    const double* u = uind + (size_t)3 * i;
    const double* e = ef + (size_t)6 * i + 3;  // p field, ef(:,2,i)
    v[0] = u[0] * e[0] + u[1] * e[1] + u[2] * e[2];
  }
  thp::block_reduce<1>(v);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    s->partial[blockIdx.x] = v[0];
    __threadfence();
    last = atomicAdd(&s->counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t[1] = {0.0};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) t[0] += __ldcg(&s->partial[b]);
  thp::block_reduce<1>(t);
  if (threadIdx.x == 0) {
    *out = -0.5 * thp::kElectric * t[0];
    s->counter = 0;
  }
}

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
NoallocScratch* g_addr[kMaxDevices] = {nullptr};

}  // namespace

extern "C" int thp_epolar_noalloc(int n, const double* d_uind, const double* d_ef, double* d_epol, void* stream) {
  if (n <= 0 || n > THP_NOALLOC_MAX_ATOMS || !d_uind || !d_ef || !d_epol) return THP_E_INVALID;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return THP_E_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return THP_E_INVALID;
  NoallocScratch* s;
  {
    // set-up, once per device, with that device current: the symbol's name is
    // only a host-side stand-in, the kernel needs its device address
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return THP_E_CUDA;
      g_addr[dev] = static_cast<NoallocScratch*>(p);
    }
    s = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(&s->counter, 0, sizeof(unsigned), st) != cudaSuccess) return THP_E_CUDA;
  const int blocks = (n + kThreads - 1) / kThreads;
  k_epol_noalloc<<<blocks, kThreads, 0, st>>>(n, d_uind, d_ef, d_epol, s);
  return cudaGetLastError() == cudaSuccess ? THP_OK : THP_E_CUDA;
}
