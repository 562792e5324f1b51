// dgm_noalloc.cu -- the CFL time step without any device allocation.
//
// Some callers cannot call cudaMalloc: a host whose device memory is owned by another allocator
// (a framework's pool, an embedding runtime), code that runs while a CUDA stream is being
// captured into a graph, or a real-time loop that must not allocate.  They cannot create a
// dgm_ctx (dgm_create allocates), so dgm_compute_time_step_noalloc takes the state and the
// element heights in device buffers the caller already owns, writes the time step into a
// caller-owned device double, and keeps its only scratch -- one partial minimum per thread block
// -- in a fixed array that is part of the library image on every GPU that loads it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "dgm_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;
constexpr long long kElementsPerBlock = (long long)kThreads * kPerThread;    // 2,048
constexpr int kMaxPartials = 4096;                                            // 32 KiB of scratch
constexpr long long kMaxElements = (long long)kMaxPartials * kElementsPerBlock;  // 8,388,608
constexpr int kMaxDevices = 64;

// One partial minimum per block, as an order key of the double (see order_key).  In host code
// this name is only a host-side stand-in for the device array: its device address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned long long g_time_step_partials[kMaxPartials];

std::mutex g_mutex;
unsigned long long* g_partials_addr[kMaxDevices] = {};

// An unsigned key that orders like the double it encodes, for every finite or infinite value of
// either sign: the sign bit flipped for non-negative values, all bits flipped for negative ones.
// The minimum of the keys is the key of the minimum, so a time step that comes out negative (a
// negative minimum height) still wins the comparison the way the reference's `dt < time_step` does.
__device__ __forceinline__ unsigned long long order_key(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double key_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// TemperalDisc::compute_time_step (src/temporal_disc.rs:58-88) over the caller's state in the
// reference layout [element][variable][basis]: per element dt = cfl * h_min / (|u| + c) with the
// state taken as the sum of the modal coefficients; the block's minimum of the values below the
// reference's start value 1e10 goes to partials[blockIdx.x] (the key of +inf if none).
template <int NB>
__global__ void __launch_bounds__(kThreads) k_time_step_partials(const double* __restrict__ U,
                                                                 const double* __restrict__ hmin,
                                                                 long long ne, double cfl, double hcr,
                                                                 unsigned long long* __restrict__ partials) {
  unsigned long long best = 0xfff0000000000000ull;  // order_key(+inf)
  const long long first = (long long)blockIdx.x * kElementsPerBlock;
#pragma unroll
  for (int k = 0; k < kPerThread; ++k) {
    const long long e = first + (long long)k * kThreads + threadIdx.x;
    if (e >= ne) break;
    const double* u = &U[e * 4 * NB];
    double s[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double a = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) a += u[v * NB + b];
      s[v] = a;
    }
    const double rho = s[0];
    const double vx = s[1] / rho;
    const double vy = s[2] / rho;
    const double p = (hcr - 1.0) * (s[3] - 0.5 * rho * (vx * vx + vy * vy));
    const double c = sqrt(hcr * p / rho);
    const double speed = sqrt(vx * vx + vy * vy) + c;
    const double dt = cfl * hmin[e] / speed;
    if (dt < 1.0e10) {  // NaN never passes, like the reference's `if dt < time_step`
      const unsigned long long key = order_key(dt);
      best = key < best ? key : best;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other < best ? other : best;
  }
  __shared__ unsigned long long s_min[kThreads / 32];
  if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < kThreads / 32; ++i) best = s_min[i] < best ? s_min[i] : best;
    partials[blockIdx.x] = best;  // every used slot is rewritten by every call
  }
}

// Minimum over the partials, starting from the reference's 1e10 (temporal_disc.rs:61).
__global__ void __launch_bounds__(kThreads) k_time_step_final(const unsigned long long* __restrict__ partials,
                                                              int nparts, double* __restrict__ out) {
  unsigned long long best = order_key(1.0e10);
  for (int i = threadIdx.x; i < nparts; i += kThreads) best = partials[i] < best ? partials[i] : best;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other < best ? other : best;
  }
  __shared__ unsigned long long s_min[kThreads / 32];
  if ((threadIdx.x & 31) == 0) s_min[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < kThreads / 32; ++i) best = s_min[i] < best ? s_min[i] : best;
    out[0] = key_value(best);
  }
}

// Device address of the scratch array on the current device, looked up once per device and kept
// for the life of the process.  cudaDeviceReset destroys the context that holds the array, so the
// kept address is stale after it: this entry point must not be called after a cudaDeviceReset of
// a device it has already run on.
int scratch_address(unsigned long long** addr) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DGM_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_time_step_partials);
    if (rc != cudaSuccess || p == nullptr) {
      std::fprintf(stderr, "dgm_compute_time_step_noalloc: cudaGetSymbolAddress failed: %s\n",
                   cudaGetErrorString(rc));
      cudaGetLastError();
      return DGM_CUDA_ERROR;
    }
    g_partials_addr[dev] = static_cast<unsigned long long*>(p);
  }
  *addr = g_partials_addr[dev];
  return DGM_OK;
}

template <int NB>
void launch(const double* U, const double* hmin, long long ne, double cfl, double hcr, double* out,
            unsigned long long* partials, int nparts, cudaStream_t stream) {
  k_time_step_partials<NB><<<nparts, kThreads, 0, stream>>>(U, hmin, ne, cfl, hcr, partials);
  k_time_step_final<<<1, kThreads, 0, stream>>>(partials, nparts, out);
}

}  // namespace

extern "C" int32_t dgm_compute_time_step_noalloc(const double* solutions, const double* minimum_height,
                                                 int64_t n_elements, int32_t n_basis, double cfl, double hcr,
                                                 double* time_step, void* stream) {
  if (!solutions || !minimum_height || !time_step || n_elements <= 0) return DGM_BAD_ARG;
  if (n_basis != 3 && n_basis != 6 && n_basis != 10) return DGM_BAD_ARG;
  if (!(cfl > 0.0) || !(hcr > 1.0)) {  // NaN fails both tests
    std::fprintf(stderr, "dgm_compute_time_step_noalloc: cfl must be > 0 and hcr > 1 (got %g, %g)\n", cfl, hcr);
    return DGM_BAD_ARG;
  }
  if (n_elements > kMaxElements) {
    std::fprintf(stderr,
                 "dgm_compute_time_step_noalloc: %lld elements exceed the fixed scratch capacity of %lld "
                 "elements (%d partial minima of %lld elements each)\n",
                 (long long)n_elements, kMaxElements, kMaxPartials, kElementsPerBlock);
    return DGM_BAD_ARG;
  }
  // a runtime error left pending by earlier work of the caller would otherwise be read back below
  // as this call's launch failure: report it without launching and leave it pending
  const cudaError_t prior = cudaPeekAtLastError();
  if (prior != cudaSuccess) {
    std::fprintf(stderr, "dgm_compute_time_step_noalloc: an earlier CUDA error is pending: %s\n",
                 cudaGetErrorString(prior));
    return DGM_CUDA_ERROR;
  }
  unsigned long long* partials = nullptr;
  int st = scratch_address(&partials);
  if (st != DGM_OK) return st;
  const int nparts = (int)((n_elements + kElementsPerBlock - 1) / kElementsPerBlock);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (n_basis) {
    case 3: launch<3>(solutions, minimum_height, n_elements, cfl, hcr, time_step, partials, nparts, s); break;
    case 6: launch<6>(solutions, minimum_height, n_elements, cfl, hcr, time_step, partials, nparts, s); break;
    default: launch<10>(solutions, minimum_height, n_elements, cfl, hcr, time_step, partials, nparts, s); break;
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "dgm_compute_time_step_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return DGM_CUDA_ERROR;
  }
  return DGM_OK;
}
