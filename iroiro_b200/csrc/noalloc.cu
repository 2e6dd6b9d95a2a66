// Field norm that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host code that owns every byte of
// device memory through its own pool allocator with a fixed budget, or one
// that must not change its device-memory footprint once its fields are set
// up.  The context API allocates (contexts, staging buffers, workspaces), so
// those callers cannot use it.  iro_norm_noalloc() gives them the norm
// reduction of the solvers (Field::norm, include/field.h:74-78) on a device
// array they own: they pass the input and the output, and the only scratch
// the reduction needs -- one partial sum per block and the ticket counter of
// the last-block finish -- lives in a fixed file-scope __device__ array.
#include <cuda_runtime.h>

#include <mutex>

#include "iroiro_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 32;                       // doubles summed by one thread
constexpr int kMaxBlocks = 8192;                     // one partial per block
constexpr int64_t kPerBlock = int64_t(kThreads) * kPerThread;
constexpr int64_t kMaxDoubles = kPerBlock * kMaxBlocks;  // 67,108,864 doubles

// Scratch layout: kMaxBlocks per-block partial sums (64 KiB), then one
// 256-byte slot whose first word is the ticket counter of the last-block
// finish (blocks finished so far; it must be zero when a launch starts).
constexpr int kScratchDoubles = kMaxBlocks + 32;

// Every GPU that loads this library holds one copy of this array until the
// process exits.  In host code the name is only a stand-in: the device address
// comes from cudaGetSymbolAddress (see scratch_address).
static __device__ __align__(256) double g_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
double* g_address[kMaxDevices] = {};
unsigned long long g_context_id[kMaxDevices] = {};

__host__ __device__ inline unsigned* counter_of(double* scratch) {
  return reinterpret_cast<unsigned*>(scratch + kMaxBlocks);
}

// Driver API entry points, resolved through the runtime so that the library
// needs no link against libcuda: the ID of the current context, which is
// unique for the life of the process.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);

unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
    resolved = true;
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_scratch on the current device, looked up with that
// device current the first time, and again whenever the device's context is
// not the one the address was taken in (after a cudaDeviceReset the runtime
// makes a new context, in which the old address means nothing).
cudaError_t scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  // cudaGetSymbolAddress also makes the device's context current if needed
  if (!g_address[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_scratch);
    if (e != cudaSuccess) return e;
    g_address[dev] = p;
    g_context_id[dev] = current_context_id();
  } else {
    const unsigned long long id = current_context_id();
    if (id == 0 || id != g_context_id[dev]) {
      double* p = nullptr;
      e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_scratch);
      if (e != cudaSuccess) return e;
      g_address[dev] = p;
      g_context_id[dev] = current_context_id();
    }
  }
  *out = g_address[dev];
  return cudaSuccess;
}

// sqrt(sum x_i^2): each block sums a fixed tile in a fixed tree, the last block
// to finish sums the per-block partials in block order (deterministic).
__global__ void __launch_bounds__(kThreads) norm_noalloc_kernel(const double* __restrict__ x,
                                                                int64_t n, double* out,
                                                                double* scratch) {
  __shared__ double sm[kThreads];
  __shared__ bool last;
  const int t = threadIdx.x;
  const int64_t base = int64_t(blockIdx.x) * kPerBlock;
  double acc = 0.0;
#pragma unroll 8
  for (int k = 0; k < kPerThread; ++k) {
    const int64_t i = base + int64_t(k) * kThreads + t;
    if (i < n) {
      const double v = x[i];
      acc += v * v;
    }
  }
  sm[t] = acc;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (t < h) sm[t] += sm[t + h];
    __syncthreads();
  }
  if (t == 0) {
    scratch[blockIdx.x] = sm[0];
    __threadfence();
    last = atomicAdd(counter_of(scratch), 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a = 0.0;
  for (int b = t; b < int(gridDim.x); b += kThreads) a += __ldcg(&scratch[b]);
  sm[t] = a;
  __syncthreads();
  for (int h = kThreads / 2; h > 0; h >>= 1) {
    if (t < h) sm[t] += sm[t + h];
    __syncthreads();
  }
  if (t == 0) {
    *out = sqrt(sm[0]);
    *counter_of(scratch) = 0u;
  }
}

}  // namespace

extern "C" int iro_norm_noalloc(const double* d_in, int64_t n, double* d_out, void* stream) {
  if (!d_in || !d_out || n < 1) return IRO_BAD_ARG;
  if (n > kMaxDoubles) return IRO_BAD_ARG;  // more than the fixed scratch can reduce
  double* s = nullptr;
  if (scratch_address(&s) != cudaSuccess) return IRO_CUDA_ERROR;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the ticket counter must start at zero (an earlier call may have been cut short)
  if (cudaMemsetAsync(counter_of(s), 0, sizeof(unsigned), st) != cudaSuccess) return IRO_CUDA_ERROR;
  const int blocks = int((n + kPerBlock - 1) / kPerBlock);
  norm_noalloc_kernel<<<blocks, kThreads, 0, st>>>(d_in, n, d_out, s);
  return cudaGetLastError() == cudaSuccess ? IRO_OK : IRO_CUDA_ERROR;
}
