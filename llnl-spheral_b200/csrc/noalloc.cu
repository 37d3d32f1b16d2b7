// Conservation sums over caller-owned device arrays, with no allocation.
//
// sphgpu_conservation works on a problem handle, and creating a handle
// allocates the whole O(n) device state of a problem.  Some callers cannot
// allocate at the moment they want the sums: a driver whose node state
// already lives in its own device buffers and that charges every byte of
// HBM against a fixed admission budget (a serving loop), or code that runs
// where a cudaMalloc would synchronise the device or fail (a tight
// per-step diagnostic, a memory pool that is full by design).  This entry
// point reads their arrays directly and keeps its scratch in a fixed device
// array compiled into the library, so it calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// Scratch: g_noallocScratch, 8192 block partials of 8 doubles plus the 8
// results (512 KB + 64 B).  Each block sums a fixed chunk of 2048 nodes,
// so n is limited to 8192 * 2048 = 16,777,216 nodes; larger n is rejected.
// Nothing in the scratch has to start at zero: every partial the final pass
// reads is written by the partial pass earlier on the same stream.
// Calls that overlap in time on one device (two host threads, or two
// streams without ordering between them) share the scratch and race.
// The scratch address of a device is looked up on the first call there and
// kept for the life of the process; a cudaDeviceReset of that device reloads
// the module and leaves the kept address stale, so the entry point is not to
// be called on a device after it has been reset.
#include <mutex>

#include "problem.cuh"

namespace sphgpu {
namespace {

constexpr int kThreads = 256;
constexpr int kNodesPerBlock = 2048;
constexpr int kMaxBlocks = 8192;
constexpr int64_t kMaxNodes = (int64_t)kMaxBlocks*kNodesPerBlock;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noallocScratch[kMaxBlocks*8 + 8];

std::mutex g_setupMutex;
double* g_scratch[kMaxDevices] = {};

// Block b sums nodes [b*2048, min(n, (b+1)*2048)) in a fixed order.
__global__ void __launch_bounds__(kThreads) noalloc_partials_kernel(const double* mass, const double* vel,
                                                                    const double* eps, int64_t n,
                                                                    double* scratch) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int64_t lo = (int64_t)blockIdx.x*kNodesPerBlock;
  const int64_t hi = lo + kNodesPerBlock < n ? lo + kNodesPerBlock : n;
  for (int64_t i = lo + threadIdx.x; i < hi; i += kThreads) {
    const double m = mass[i];
    const double vx = vel[3*i], vy = vel[3*i + 1], vz = vel[3*i + 2];
    acc[0] += m;
    acc[1] += m*vx; acc[2] += m*vy; acc[3] += m*vz;
    acc[4] += 0.5*m*(vx*vx + vy*vy + vz*vz);
    acc[5] += m*eps[i];
  }
  __shared__ double sh[6][kThreads];
  for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = kThreads/2; s > 0; s >>= 1) {
    if (threadIdx.x < s) for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 8) scratch[blockIdx.x*8 + threadIdx.x] = threadIdx.x < 6 ? sh[threadIdx.x][0] : 0.0;
}

// One block folds the partials (fixed order) into the 8 results.
__global__ void __launch_bounds__(kThreads) noalloc_final_kernel(int nblocks, double* scratch) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += kThreads)
    for (int c = 0; c < 6; ++c) acc[c] += scratch[b*8 + c];
  __shared__ double sh[6][kThreads];
  for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int s = kThreads/2; s > 0; s >>= 1) {
    if (threadIdx.x < s) for (int c = 0; c < 6; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double* out = scratch + kMaxBlocks*8;
    for (int c = 0; c < 6; ++c) out[c] = sh[c][0];
    out[6] = sh[4][0] + sh[5][0];
    out[7] = 0.0;
  }
}

// Device address of the scratch array on the current device, looked up once.
int scratch_for_current_device(double** ptr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("sphgpu_conservation_noalloc: device ordinal out of range");
    return SPHGPU_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_setupMutex);
  if (g_scratch[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noallocScratch)");
    g_scratch[dev] = static_cast<double*>(p);
  }
  *ptr = g_scratch[dev];
  return SPHGPU_OK;
}

}  // namespace
}  // namespace sphgpu

using namespace sphgpu;

extern "C" int sphgpu_conservation_noalloc(const double* mass, const double* velocity,
                                           const double* specificThermalEnergy, int64_t n, void* stream,
                                           double out[8]) {
  if (out == nullptr || n < 0 || (n > 0 && (mass == nullptr || velocity == nullptr ||
                                            specificThermalEnergy == nullptr))) {
    set_error("sphgpu_conservation_noalloc: null pointer or negative node count");
    return SPHGPU_ERR_ARG;
  }
  if (n > kMaxNodes) {
    set_error("sphgpu_conservation_noalloc: n exceeds the fixed scratch limit of 16,777,216 nodes "
              "(use sphgpu_conservation on a problem handle)");
    return SPHGPU_ERR_CAPACITY;
  }
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc != SPHGPU_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nblocks = (int)((n + kNodesPerBlock - 1)/kNodesPerBlock);
  if (nblocks > 0)
    noalloc_partials_kernel<<<nblocks, kThreads, 0, st>>>(mass, velocity, specificThermalEnergy, n, scratch);
  noalloc_final_kernel<<<1, kThreads, 0, st>>>(nblocks, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "sphgpu_conservation_noalloc launch");
  e = cudaMemcpyAsync(out, scratch + kMaxBlocks*8, sizeof(double)*8, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_status(e, "sphgpu_conservation_noalloc copy");
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "sphgpu_conservation_noalloc");
  return SPHGPU_OK;
}
