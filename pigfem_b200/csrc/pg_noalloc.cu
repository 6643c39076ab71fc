// pg_noalloc.cu -- a residual norm that allocates nothing (pg_norm2_noalloc).
//
// The norm's block partials live in one file-scope __device__ array of fixed size, so a call
// makes no device allocation at all.  Its address is looked up once per device with
// cudaGetSymbolAddress and then passed to the kernels as a plain pointer.  Two launches on the
// caller's stream: the block partials, then one block that sums them.  Stream order separates
// the two, so no completion counter (and no state that could outlive a call) is needed.
#include "../../include/pigfem_b200.h"

#include <cuda_runtime.h>

#include <mutex>

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 32;
constexpr long long kPerBlock = (long long)kThreads * kPerThread;  // 8192 values per block
constexpr int kMaxBlocks = PG_NORM_NOALLOC_MAX_N / kPerBlock;      // 4096 partials (32 KiB)
static_assert((long long)kMaxBlocks * kPerBlock == PG_NORM_NOALLOC_MAX_N, "max size is whole blocks");

// One partial sum of squares per block of the first launch.  Every call writes the partials it
// reads, so nothing has to start at zero.
__device__ __align__(256) double pg_norm_scratch[kMaxBlocks];

constexpr int kMaxDevices = 64;
double* g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Sum of squares in a fixed order: block b reduces values [b*8192, (b+1)*8192) with a fixed
// per-thread stride and a fixed tree into part[b].
__global__ void __launch_bounds__(kThreads) k_norm2_partials(const double* __restrict__ x, long long n, double* part) {
  __shared__ double sh[kThreads];
  const long long b0 = (long long)blockIdx.x * kPerBlock;
  const long long b1 = b0 + kPerBlock < n ? b0 + kPerBlock : n;
  double s = 0.0;
  for (long long i = b0 + threadIdx.x; i < b1; i += kThreads) s += x[i] * x[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// One block: the partials summed in a fixed tree order, then the square root.  The result
// depends on n and the data only, never on block scheduling.
__global__ void __launch_bounds__(kThreads) k_norm2_final(const double* __restrict__ part, int nb, double* out) {
  __shared__ double sh[kThreads];
  double t = 0.0;
  for (int i = threadIdx.x; i < nb; i += kThreads) t += part[i];
  sh[threadIdx.x] = t;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sqrt(sh[0]);
}

// Per-device set-up: the scratch address of the current device, looked up on the first call.
int scratch_for_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PG_ERR_DEVICE;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, pg_norm_scratch) != cudaSuccess || !p) return PG_ERR_DEVICE;
    g_scratch[dev] = static_cast<double*>(p);
  }
  *out = g_scratch[dev];
  return PG_OK;
}

}  // namespace

extern "C" int pg_norm2_noalloc(const double* d_x, int64_t n, double* d_out, void* stream) {
  if (!d_out || n < 0 || (n > 0 && !d_x)) return PG_ERR_INPUT;
  if (n > PG_NORM_NOALLOC_MAX_N) return PG_ERR_CAPACITY;
  double* scratch = nullptr;
  if (int rc = scratch_for_current_device(&scratch)) return rc;
  const int blocks = n == 0 ? 1 : (int)((n + kPerBlock - 1) / kPerBlock);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_norm2_partials<<<blocks, kThreads, 0, st>>>(d_x, (long long)n, scratch);
  k_norm2_final<<<1, kThreads, 0, st>>>(scratch, blocks, d_out);
  return cudaGetLastError() == cudaSuccess ? PG_OK : PG_ERR_DEVICE;
}
