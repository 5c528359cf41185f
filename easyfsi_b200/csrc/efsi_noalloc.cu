// Plan-free, allocation-free variant of the fluid-weighted dot product
// (fluid.py:4534-4546 _weighted_dot_kernel: the sum over fluid cells,
// obstacle == 0, of a * b * V with V = wx[i] wy[j] wz[k] in f64).
//
// Its reduction scratch is this file's static device array, not memory the
// caller or a plan provides, so the call needs no cudaMalloc, no plan and no
// allocating library call: it serves callers that may not allocate device
// memory where they run (a caching allocator's owner that must not re-enter
// it, or code holding no plan).  Limits:
//   * at most kMaxBlocks partial sums, hence at most kMaxCells cells; larger
//     grids are rejected with EFSI_ERR_ARG before anything is launched;
//   * the ticket counter must start at zero: every call clears it on its
//     stream (cudaMemsetAsync, which allocates nothing) before the launch, so
//     a call never depends on what an earlier call left in the scratch;
//   * the scratch is shared by all calls on a device, so calls must not
//     overlap (issue them on one stream, or synchronise between streams);
//   * the first call on each device resolves the scratch address with
//     cudaGetSymbolAddress, with that device current, and may load the
//     module; make that first call before any stream capture;
//   * the resolved address is kept for the life of the process, so the
//     library must not be used across a cudaDeviceReset of a device it has
//     already used (the reset unloads the module and the address goes stale).
#include <cuda_runtime.h>

#include <mutex>

#include "efsi_common.cuh"

namespace efsi {
namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocCellsPerThread = 16;
constexpr int kMaxBlocks = 65536;  // 512 KiB of partial sums
constexpr int64_t kMaxCells = (int64_t)kMaxBlocks * kNoAllocThreads * kNoAllocCellsPerThread;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dot_partials[kMaxBlocks];
static __device__ __align__(256) unsigned g_dot_ticket;  // cleared by every call before its launch

struct Scratch {
  double* partials = nullptr;
  unsigned* ticket = nullptr;
};

std::mutex g_scratch_mu;
Scratch g_scratch[kMaxDevices];

// Device addresses of the static scratch on the current device (resolved
// once per device).
int scratch_for_current_device(Scratch& out) {
  int dev = 0;
  EFSI_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("efsi_weighted_dot_noalloc: device index out of range");
    return EFSI_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  Scratch& s = g_scratch[dev];
  if (s.partials == nullptr) {
    void* p = nullptr;
    void* t = nullptr;
    EFSI_CUDA_CHECK(cudaGetSymbolAddress(&p, g_dot_partials));
    EFSI_CUDA_CHECK(cudaGetSymbolAddress(&t, g_dot_ticket));
    s.partials = static_cast<double*>(p);
    s.ticket = static_cast<unsigned*>(t);
  }
  out = s;
  return EFSI_OK;
}

// Each thread sums up to kNoAllocCellsPerThread cells (a block covers a
// contiguous range of cells); block partials and the ticket live in the
// static scratch; the last block writes the total to `result`.
__global__ void __launch_bounds__(kNoAllocThreads)
    k_weighted_dot_noalloc(int nx, int ny, int nz, const int32_t* __restrict__ obstacle,
                           const float* __restrict__ wx, const float* __restrict__ wy, const float* __restrict__ wz,
                           const double* __restrict__ a, const double* __restrict__ b, double* partials,
                           unsigned* ticket, double* result) {
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t first = (int64_t)blockIdx.x * kNoAllocThreads * kNoAllocCellsPerThread + threadIdx.x;
  double acc = 0.0;
#pragma unroll 4
  for (int q = 0; q < kNoAllocCellsPerThread; ++q) {
    const int64_t c = first + (int64_t)q * kNoAllocThreads;
    if (c >= n) break;
    if (__ldg(obstacle + c) != 0) continue;
    const int k = (int)(c % nz);
    const int64_t ij = c / nz;
    const int j = (int)(ij % ny), i = (int)(ij / ny);
    const double vol = (double)__ldg(wx + i) * (double)__ldg(wy + j) * (double)__ldg(wz + k);
    acc += __ldg(a + c) * __ldg(b + c) * vol;
  }
  double v[1] = {acc}, t[1];
  if (grid_sum<1>(v, partials, ticket, t)) {
    if (flat_tid() == 0) *result = t[0];
  }
}

}  // namespace
}  // namespace efsi

using namespace efsi;

extern "C" int efsi_weighted_dot_noalloc(int32_t nx, int32_t ny, int32_t nz, const int32_t* obstacle, const float* wx,
                                         const float* wy, const float* wz, const double* a, const double* b,
                                         double* result_device, void* stream) {
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "efsi_weighted_dot_noalloc: grid dimensions must be positive");
  const int64_t n = (int64_t)nx * ny * nz;
  EFSI_ARG_CHECK(n <= kMaxCells,
                 "efsi_weighted_dot_noalloc: grid exceeds the static scratch limit of 268435456 cells "
                 "(65536 blocks x 4096 cells)");
  EFSI_ARG_CHECK(obstacle && wx && wy && wz && a && b && result_device, "efsi_weighted_dot_noalloc: null pointer");
  Scratch sc;
  EFSI_TRY(scratch_for_current_device(sc));
  const int64_t per_block = (int64_t)kNoAllocThreads * kNoAllocCellsPerThread;
  const unsigned blocks = (unsigned)((n + per_block - 1) / per_block);
  EFSI_CUDA_CHECK(cudaMemsetAsync(sc.ticket, 0, sizeof(unsigned), as_stream(stream)));
  EFSI_COUNTED k_weighted_dot_noalloc<<<blocks, kNoAllocThreads, 0, as_stream(stream)>>>(
      nx, ny, nz, obstacle, wx, wy, wz, a, b, sc.partials, sc.ticket, result_device);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}
