// caps_gpu_kinetic_noalloc (include/caps_gpu.h): the kinetic energy and kinetic tensor of a velocity set, computed
// without allocating device memory.
//
// Why it exists. Every other entry point of this library allocates its working buffers (pair list, grids, partial sums)
// with cudaMalloc when an engine is created or a run starts. Some callers cannot allow that: a host code whose memory
// manager owns all of the device's memory (an MD host that hands out pooled buffers and forbids allocations behind its
// back), or code that runs while the device is busy with a long stream-ordered pipeline, where cudaMalloc/cudaFree can
// synchronise the device and stall it. Those callers pass their own inputs and outputs; the only working memory is the
// fixed array below.
//
// The reduction is the one of the run loop's kinetic-energy kernel (k_ke, integrate.cu): per-block partial sums, then the
// last block to finish adds them in block order, so the result does not depend on block scheduling.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "caps_gpu.h"
#include "common.cuh"

namespace capsb {
void set_call_error(const std::string& text);   // engine.cu: the text caps_gpu_error(NULL) returns
}

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxAtoms = 1 << 20;                                   // 1,048,576 atoms per call
constexpr int kNoAllocMaxBlocks = kNoAllocMaxAtoms / kNoAllocThreads;       // 4096 blocks
constexpr double kAccNoAlloc = 4.184e-4;                                    // (kcal/mol/Å)/(g/mol) -> Å/fs², dynamics.cpp:23
constexpr int kMaxDevices = 64;

// The working memory of every call on one device: 4096 blocks × 7 partial sums + the finished-block counter, about
// 230 KB. Each GPU that loads the library holds one copy until the process exits.
struct NoAllocScratch {
  double part[kNoAllocMaxBlocks * 7];   // per block: sum m v², then sum m v_a v_b (xx yy zz xy xz yz)
  unsigned done;                        // blocks finished; must be 0 when a call's kernel starts
};
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

__global__ void __launch_bounds__(kNoAllocThreads) k_kinetic_noalloc(int n, const double* __restrict__ v, const double* __restrict__ m,
                                                                      double* __restrict__ out, NoAllocScratch* s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double t[7] = {0, 0, 0, 0, 0, 0, 0};
  if (i < n) {
    const double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2], mi = m[i];
    t[0] = mi * (vx * vx + vy * vy + vz * vz);
    t[1] = mi * vx * vx, t[2] = mi * vy * vy, t[3] = mi * vz * vz;
    t[4] = mi * vx * vy, t[5] = mi * vx * vz, t[6] = mi * vy * vz;
  }
  __shared__ double scratch[32];
  __shared__ bool last;
  for (int q = 0; q < 7; ++q) {
    const double b = capsb::block_sum(t[q], scratch);
    if (threadIdx.x == 0) s->part[7 * blockIdx.x + q] = b;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&s->done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int q = 0; q < 7; ++q) t[q] = 0;
  for (int b = threadIdx.x; b < int(gridDim.x); b += blockDim.x)
    for (int q = 0; q < 7; ++q) t[q] += __ldcg(s->part + 7 * b + q);
  double tot[7];
  for (int q = 0; q < 7; ++q) tot[q] = capsb::block_sum(t[q], scratch);
  if (threadIdx.x != 0) return;
  s->done = 0;
  out[0] = 0.5 * tot[0] / kAccNoAlloc;
  for (int q = 1; q < 7; ++q) out[q] = tot[q] / kAccNoAlloc;
}

std::mutex g_noalloc_mu;
NoAllocScratch* g_noalloc_addr[kMaxDevices] = {};   // device address of g_noalloc_scratch, per device

int32_t fail(int32_t code, const std::string& text) {
  capsb::set_call_error(text);
  return code;
}

}  // namespace

extern "C" int32_t caps_gpu_kinetic_noalloc(const double* d_v, const double* d_mass, int32_t n, double* d_out, void* stream) {
  if (!d_v || !d_mass || !d_out) return fail(CAPS_GPU_EINVAL, "caps_gpu_kinetic_noalloc: null argument");
  if (n < 1 || n > kNoAllocMaxAtoms)
    return fail(CAPS_GPU_EINVAL, "caps_gpu_kinetic_noalloc: n = " + std::to_string(n) + " atoms is outside [1, " +
                                     std::to_string(kNoAllocMaxAtoms) + "], the size of its fixed working memory");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(CAPS_GPU_ENODEV, "caps_gpu_kinetic_noalloc: no CUDA device");
  if (dev < 0 || dev >= kMaxDevices) return fail(CAPS_GPU_EINVAL, "caps_gpu_kinetic_noalloc: device index beyond 63");
  NoAllocScratch* s = nullptr;
  {
    // set-up, once per device with that device current: the host-side name of the array is not a device address
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return fail(CAPS_GPU_ECUDA, std::string("caps_gpu_kinetic_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_addr[dev] = static_cast<NoAllocScratch*>(p);
    }
    s = g_noalloc_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the finished-block counter must start at zero (a call that failed part-way may have left it set)
  cudaError_t e = cudaMemsetAsync(&s->done, 0, sizeof(unsigned), st);
  if (e != cudaSuccess) return fail(CAPS_GPU_ECUDA, std::string("caps_gpu_kinetic_noalloc: cudaMemsetAsync: ") + cudaGetErrorString(e));
  const int blocks = (n + kNoAllocThreads - 1) / kNoAllocThreads;
  k_kinetic_noalloc<<<blocks, kNoAllocThreads, 0, st>>>(n, d_v, d_mass, d_out, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CAPS_GPU_ECUDA, std::string("caps_gpu_kinetic_noalloc: launch: ") + cudaGetErrorString(e));
  return CAPS_GPU_OK;
}
