// Shared helpers of the easyfsi_b200 CUDA library: error plumbing, launch
// shapes and the deterministic block / grid reductions used by every kernel
// that produces a scalar.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "easyfsi_b200.h"

namespace efsi {

void set_error(const std::string& msg);

#define EFSI_CUDA_CHECK(expr)                                                               \
  do {                                                                                      \
    cudaError_t _e = (expr);                                                                \
    if (_e != cudaSuccess) {                                                                \
      ::efsi::set_error(std::string(#expr " failed: ") + cudaGetErrorString(_e));          \
      return EFSI_ERR_CUDA;                                                                 \
    }                                                                                       \
  } while (0)

#define EFSI_LAUNCH_CHECK()                                                                 \
  do {                                                                                      \
    cudaError_t _e = cudaGetLastError();                                                    \
    if (_e != cudaSuccess) {                                                                \
      ::efsi::set_error(std::string("kernel launch failed: ") + cudaGetErrorString(_e));   \
      return EFSI_ERR_CUDA;                                                                 \
    }                                                                                       \
  } while (0)

#define EFSI_ARG_CHECK(cond, msg)        \
  do {                                   \
    if (!(cond)) {                       \
      ::efsi::set_error(msg);            \
      return EFSI_ERR_ARG;               \
    }                                    \
  } while (0)

#define EFSI_TRY(expr)            \
  do {                            \
    int _s = (expr);              \
    if (_s != EFSI_OK) return _s; \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Host-side count of every kernel this library launches (reported by the
// benchmark as its launch count).
void count_launch();
#define EFSI_COUNTED ::efsi::count_launch(),

// Optional CUDA-event timing of selected kernel families (benchmark use):
// when a family is enabled, its launches are bracketed by events on their own
// stream and their algorithmic byte counts accumulated.
enum KernelFamily : int {
  KF_SPMV_DIR = 0,
  KF_SWEEP_L0 = 1,
  KF_CG_UPDATE = 2,
  KF_RESTRICT_L0 = 3,
  KF_CG_DOTS = 4,
  KF_P2G = 5,
  KF_PREDICT = 6,
  KF_GRID_UPDATE = 7,
  KF_G2P = 8,
  KF_SCATTER = 9,
  KF_FEEDBACK = 10,
  KF_MPM_STEP = 11,  // the whole substep: clears, binning, P2G, grid update, G2P
  KF_SHELL_STEP = 12,  // the whole Mooney membrane step
  KF_COUNT = 13
};
bool timing_enabled(int family);
void timing_begin(int family, cudaStream_t s);
void timing_end(int family, cudaStream_t s, double bytes);
#define EFSI_TIMED(family, bytes, stream, ...)                    \
  do {                                                             \
    const bool _t = ::efsi::timing_enabled(family);                \
    if (_t) ::efsi::timing_begin(family, stream);                  \
    __VA_ARGS__;                                                   \
    if (_t) ::efsi::timing_end(family, stream, (double)(bytes));  \
  } while (0)

// Programmatic dependent launch.  Kernels of the PCG loop are launched with
// programmatic stream serialization (launch_pdl), so their launch and block
// set-up overlap the drain of the kernel before them; each of them calls
// pdl_wait() before its first global-memory access, which waits for the
// previous grid to complete and its writes to be visible.  For a kernel
// launched without the attribute pdl_wait() returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

bool pdl_enabled();  // false when EFSI_NO_PDL is set

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args... args) {
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

inline unsigned next_pow2(unsigned v) {
  unsigned p = 1;
  while (p < v) p <<= 1;
  return p;
}

// 3-D launch shape for a cell-per-thread kernel over an (nx, ny, nz) level:
// threads run along k (contiguous), then j, then i; 256 threads per block.
struct Shape3 {
  dim3 block;
  dim3 grid;
  unsigned nblocks() const { return grid.x * grid.y * grid.z; }
};

inline Shape3 shape3(int nx, int ny, int nz) {
  unsigned bx = next_pow2((unsigned)nz);
  if (bx > 32) bx = 32;
  unsigned by = next_pow2((unsigned)ny);
  if (by > 256 / bx) by = 256 / bx;
  unsigned bz = 256 / (bx * by);
  unsigned nxp = next_pow2((unsigned)nx);
  if (bz > nxp) bz = nxp;
  Shape3 s;
  s.block = dim3(bx, by, bz);
  s.grid = dim3((nz + bx - 1) / bx, (ny + by - 1) / by, (nx + bz - 1) / bz);
  return s;
}

inline unsigned blocks_1d(int64_t n, unsigned threads, unsigned cap) {
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

// ---------------------------------------------------------------------------
// Deterministic reductions.  Each block reduces its NV values in a fixed
// order (warp shuffles, then warps in index order) and stores them to
// partials[v * nblocks + block].  The last block to arrive (ticket counter)
// sums the partials of every value in block order and hands the totals to a
// finisher.  Given a launch shape the result is bitwise reproducible.
// ---------------------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned flat_tid() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ unsigned flat_bid() {
  return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}
__device__ __forceinline__ unsigned flat_nthreads() { return blockDim.x * blockDim.y * blockDim.z; }
__device__ __forceinline__ unsigned flat_nblocks() { return gridDim.x * gridDim.y * gridDim.z; }

// Block sum of NV doubles; the result is valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red[NV][32];
  const unsigned tid = flat_tid();
  const unsigned lane = tid & 31u, warp = tid >> 5;
  const unsigned nwarps = (flat_nthreads() + 31u) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = warp_sum(v[q]);
    if (lane == 0) red[q][warp] = s;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = lane < nwarps ? red[q][lane] : 0.0;
      v[q] = warp_sum(s);
    }
  }
  __syncthreads();
}

// Stores the block partials and returns true in the block that arrives last;
// that block then finds the NV grand totals in `total` (valid in all threads).
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double* partials, unsigned* ticket, double (&total)[NV]) {
  __shared__ bool am_last;
  __shared__ double tot[NV];
  block_sum<NV>(v);
  const unsigned tid = flat_tid();
  const unsigned nb = flat_nblocks(), bid = flat_bid();
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) partials[(size_t)q * nb + bid] = v[q];
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    am_last = (t == nb - 1);
  }
  __syncthreads();
  if (!am_last) return false;
  __threadfence();
  const unsigned nt = flat_nthreads();
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    // four independent L2 loads in flight per thread; fixed summation order
    const double* part = partials + (size_t)q * nb;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    unsigned b = tid;
    for (; b + 3 * nt < nb; b += 4 * nt) {
      s0 += __ldcg(part + b);
      s1 += __ldcg(part + b + nt);
      s2 += __ldcg(part + b + 2 * nt);
      s3 += __ldcg(part + b + 3 * nt);
    }
    for (; b < nb; b += nt) s0 += __ldcg(part + b);
    acc[q] = (s0 + s1) + (s2 + s3);
  }
  block_sum<NV>(acc);
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) tot[q] = acc[q];
    *ticket = 0u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NV; ++q) total[q] = tot[q];
  return true;
}

}  // namespace efsi
