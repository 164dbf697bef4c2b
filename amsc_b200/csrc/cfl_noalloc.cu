// CFL time step over particle arrays the caller holds on the device, with no
// device memory allocated by the call.
//
// The reference's GPU driver copies vpx, vpy and hp to the host every step
// to take their maxima and the CFL step (main/gpu_offload.cpp:284-300;
// main/optim_par.cpp:289-304).  dampm_cfl_dt_noalloc computes the same
// numbers on the device.  Its reduction scratch (one partial maximum triple
// per block) is a file-scope __device__ array, so a call makes no
// cudaMalloc/cudaFree: callers whose device memory is owned by someone else
// (an OpenMP `target data` region, a framework's memory pool) or whose step
// loop must not stall the device (cudaFree synchronises it) can call it on
// every step.
#include <climits>

#include <cuda_runtime.h>

#include "../../include/dampm_cuda.h"
#include "dampm_device.cuh"

namespace {

using dampm::ordered_key;
using dampm::ordered_value;

constexpr int kCflThreads = 256;
// Partial-maximum slots: up to 8 blocks per SM of a 148-SM B200; larger
// particle counts are covered by the grid-stride loop.
constexpr int kCflMaxBlocks = 8 * 148;

// 3 ordered keys (max |vpx|, max |vpy|, max hp) per block: 28,416 bytes.
// Every slot the final kernel reads was written by the same call's first
// kernel, so nothing here needs to start at zero.
static __device__ __align__(256) unsigned long long g_cfl_scratch[3 * kCflMaxBlocks];

__device__ __forceinline__ void block_max3(unsigned long long& m0,
                                           unsigned long long& m1,
                                           unsigned long long& m2) {
  __shared__ unsigned long long sm[3][kCflThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    m0 = max(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sm[0][w] = m0;
    sm[1][w] = m1;
    sm[2][w] = m2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kCflThreads / 32; ++k) {
      m0 = max(m0, sm[0][k]);
      m1 = max(m1, sm[1][k]);
      m2 = max(m2, sm[2][k]);
    }
  }
}

__global__ void __launch_bounds__(kCflThreads)
    k_cfl_partial(const double* __restrict__ vpx, const double* __restrict__ vpy,
                  const double* __restrict__ hp, long long np,
                  unsigned long long* __restrict__ part) {
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < np;
       i += stride) {
    m0 = max(m0, ordered_key(fabs(vpx[i])));
    m1 = max(m1, ordered_key(fabs(vpy[i])));
    m2 = max(m2, ordered_key(hp[i]));
  }
  block_max3(m0, m1, m2);
  if (threadIdx.x == 0) {
    part[3 * blockIdx.x + 0] = m0;
    part[3 * blockIdx.x + 1] = m1;
    part[3 * blockIdx.x + 2] = m2;
  }
}

// out: {dt, cel, max |vpx|, max |vpy|, max hp}, evaluated in the operand
// order of main/optim_par.cpp:289-304 (the same expressions as the step's
// own dt).
__global__ void __launch_bounds__(kCflThreads)
    k_cfl_final(const unsigned long long* __restrict__ part, int nb, double g,
                double CFL, double hx, double hy, double* __restrict__ out) {
  unsigned long long m0 = 0, m1 = 0, m2 = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    m0 = max(m0, part[3 * b + 0]);
    m1 = max(m1, part[3 * b + 1]);
    m2 = max(m2, part[3 * b + 2]);
  }
  block_max3(m0, m1, m2);
  if (threadIdx.x == 0) {
    const double mvx = ordered_value(m0);
    const double mvy = ordered_value(m1);
    const double hmax = ordered_value(m2);
    const double a = sqrt(g * hmax) + mvx;
    const double b = sqrt(g * hmax) + mvy;
    const double max_vel = (a < b) ? b : a;  // std::max
    const double cel = fabs(max_vel);
    const double hmin = (hy < hx) ? hy : hx;  // std::min
    out[0] = CFL * hmin / (1e-2 + cel);
    out[1] = cel;
    out[2] = mvx;
    out[3] = mvy;
    out[4] = hmax;
  }
}

// The scratch array's device address in the current context.  The address
// belongs to a CUDA context, not to a device number: it changes after
// cudaDeviceReset or when another context is made current on the device, so
// it is looked up on every call (a host-side query that allocates nothing).
// The first lookup in a context may load this library's kernels into it,
// which is why the first call should come before any stream capture.
int scratch_for_current_context(unsigned long long** out) {
  void* q = nullptr;
  if (cudaGetSymbolAddress(&q, g_cfl_scratch) != cudaSuccess || !q) {
    cudaGetLastError();  // the lookup's error is reported by the return code
    return DAMPM_ERR_CUDA;
  }
  *out = static_cast<unsigned long long*>(q);
  return DAMPM_OK;
}

// A stream created on another device than the current one would receive the
// current device's scratch address: refused.
int check_stream_device(cudaStream_t st) {
  if (st == nullptr) return DAMPM_OK;  // the legacy stream of the current device
  int dev = -1, sdev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return DAMPM_ERR_CUDA;
  if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) {
    cudaGetLastError();
    return DAMPM_ERR_CUDA;
  }
  return sdev == dev ? DAMPM_OK : DAMPM_ERR_DEVICE;
}

}  // namespace

extern "C" int dampm_cfl_dt_noalloc(const double* vpx, const double* vpy,
                                    const double* hp, long long np, double g,
                                    double CFL, double hx, double hy,
                                    double* out, void* cuda_stream) {
  if (!vpx || !vpy || !hp || !out) return DAMPM_ERR_ARG;
  if (!(hx > 0.0) || !(hy > 0.0)) return DAMPM_ERR_ARG;
  if (np < 1) return DAMPM_ERR_ARG;  // the maxima of no particles are undefined
  if (np > (long long)INT_MAX) return DAMPM_ERR_CAPACITY;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  int rc = check_stream_device(st);
  if (rc) return rc;
  unsigned long long* part = nullptr;
  rc = scratch_for_current_context(&part);
  if (rc) return rc;
  const long long want = (np + kCflThreads - 1) / kCflThreads;
  const int nb = (int)(want < kCflMaxBlocks ? want : kCflMaxBlocks);
  k_cfl_partial<<<nb, kCflThreads, 0, st>>>(vpx, vpy, hp, np, part);
  k_cfl_final<<<1, kCflThreads, 0, st>>>(part, nb, g, CFL, hx, hy, out);
  return cudaGetLastError() == cudaSuccess ? DAMPM_OK : DAMPM_ERR_CUDA;
}
