// The learned preconditioner: a 3-D convolutional U-Net (4 levels, 16 / 32 /
// 48 / 64 channels, 15 3x3x3 convolutions, about 0.69 M parameters) that maps
// a residual r of the FV pressure system to an approximation of A^-1 r.  It has
// no counterpart in the reference; the flexible PCG it preconditions is the
// reference's (fluid.py:6535-6811), with the multigrid V-cycle as fallback.
//
// Activations are channels-last BF16 ([voxel][channel], channels a multiple of
// 16).  Convolutions run on the tensor cores (efsi_conv3d.cuh: tcgen05,
// FP32 accumulation in tensor memory): the forward pass and the input
// gradient, which is the same convolution with the taps flipped and the
// channel axes of the weights swapped.  The weight gradient, a reduction over
// the voxels, runs on the CUDA cores in FP32.  Master weights, gradients and
// the Adam moments are FP32; the BF16 weight copies are refreshed after every
// update.
//
// Layers (level l volume has ceil-halved extents of level l - 1):
//   encoder   e_la = relu(conv(in)), e_l = relu(conv(e_la)), in = pool(e_{l-1})
//   decoder   d_la = relu(conv([up(d_{l+1}), e_l])), d_l = relu(conv(d_la))
//   output    out = conv(d_0) (16 channels; channel 0 is the network output)
// with average pooling over the existing 2 x 2 x 2 children and
// nearest-neighbour upsampling, whose adjoints are used in the backward pass.
//
// Input channels (efsi_unet_pack_residual): 0 the residual scaled to unit RMS
// over the fluid cells, 1 the fluid mask, 2-4 log of the cell widths relative
// to the finest width of each axis; the rest are zero.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "efsi_common.cuh"
#include "efsi_conv3d.cuh"
#include "efsi_unet_internal.cuh"

using bf16 = __nv_bfloat16;

namespace efsi {
namespace {

constexpr int kLevels = 4;
constexpr int kCh[kLevels] = {16, 32, 48, 64};
constexpr int kInCh = 16;
constexpr int kOutCh = 16;
constexpr int kLayers = 15;

struct LayerSpec {
  int level, cin, cout, relu;
};

// Encoder l: 2l, 2l+1 (l = 0..3); decoder l: 8 + 2 (2 - l), + 1 (l = 2..0); output 14.
constexpr LayerSpec kSpec[kLayers] = {
    {0, kInCh, 16, 1}, {0, 16, 16, 1},            // e0a, e0
    {1, 16, 32, 1},    {1, 32, 32, 1},            // e1a, e1
    {2, 32, 48, 1},    {2, 48, 48, 1},            // e2a, e2
    {3, 48, 64, 1},    {3, 64, 64, 1},            // e3a, e3
    {2, 64 + 48, 48, 1}, {2, 48, 48, 1},          // d2a, d2
    {1, 48 + 32, 32, 1}, {1, 32, 32, 1},          // d1a, d1
    {0, 32 + 16, 16, 1}, {0, 16, 16, 1},          // d0a, d0
    {0, 16, kOutCh, 0},                           // out
};

int64_t weight_count(int l) { return (int64_t)kSpec[l].cout * 27 * kSpec[l].cin; }

// ---------------------------------------------------------------------------
// Element-wise and transfer kernels
// ---------------------------------------------------------------------------
#define UNET_STRIDE(q, n) \
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < (n); q += (int64_t)gridDim.x * blockDim.x)

struct Dims {
  int nx, ny, nz;
  __host__ __device__ int64_t n() const { return (int64_t)nx * ny * nz; }
};

__host__ __device__ inline Dims coarse_of(Dims d) { return Dims{(d.nx + 1) / 2, (d.ny + 1) / 2, (d.nz + 1) / 2}; }

__device__ __forceinline__ int64_t parent_of(const Dims& f, const Dims& c, int64_t v) {
  const int k = (int)(v % f.nz);
  const int64_t ij = v / f.nz;
  const int j = (int)(ij % f.ny), i = (int)(ij / f.ny);
  return ((int64_t)(i >> 1) * c.ny + (j >> 1)) * c.nz + (k >> 1);
}

// average over the existing children of each coarse voxel
__global__ void k_pool(Dims f, Dims c, int ch, const bf16* __restrict__ x, bf16* __restrict__ y) {
  UNET_STRIDE(q, c.n() * ch) {
    const int cc = (int)(q % ch);
    const int64_t v = q / ch;
    const int k = (int)(v % c.nz);
    const int64_t ij = v / c.nz;
    const int j = (int)(ij % c.ny), i = (int)(ij / c.ny);
    float s = 0.0f;
    int cnt = 0;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 2; ++d) {
          const int fi = 2 * i + a, fj = 2 * j + b, fk = 2 * k + d;
          if (fi < f.nx && fj < f.ny && fk < f.nz) {
            s += __bfloat162float(x[(((int64_t)fi * f.ny + fj) * f.nz + fk) * ch + cc]);
            ++cnt;
          }
        }
    y[q] = __float2bfloat16_rn(s / (float)cnt);
  }
}

// adjoint of k_pool, added into the fine gradient
__global__ void k_pool_back(Dims f, Dims c, int ch, const float* __restrict__ gc, float* __restrict__ gf) {
  UNET_STRIDE(q, f.n() * ch) {
    const int cc = (int)(q % ch);
    const int64_t v = q / ch;
    const int k = (int)(v % f.nz);
    const int64_t ij = v / f.nz;
    const int j = (int)(ij % f.ny), i = (int)(ij / f.ny);
    const int ci = i >> 1, cj = j >> 1, ck = k >> 1;
    const int cnt = (min(2 * ci + 2, f.nx) - 2 * ci) * (min(2 * cj + 2, f.ny) - 2 * cj) * (min(2 * ck + 2, f.nz) - 2 * ck);
    gf[q] += gc[(((int64_t)ci * c.ny + cj) * c.nz + ck) * ch + cc] / (float)cnt;
  }
}

// out[v] = [coarse[parent(v)] (ca channels), skip[v] (cb channels)]
__global__ void k_up_concat(Dims f, Dims c, int ca, int cb, const bf16* __restrict__ coarse,
                            const bf16* __restrict__ skip, bf16* __restrict__ out) {
  const int co = ca + cb;
  UNET_STRIDE(q, f.n() * co) {
    const int cc = (int)(q % co);
    const int64_t v = q / co;
    out[q] = cc < ca ? coarse[parent_of(f, c, v) * ca + cc] : skip[v * cb + (cc - ca)];
  }
}

// adjoint of k_up_concat: the first ca channels are summed over the children
// into the coarse gradient (written), the last cb added into the skip gradient
__global__ void k_up_concat_back_coarse(Dims f, Dims c, int ca, int cb, const float* __restrict__ g,
                                        float* __restrict__ gcoarse) {
  const int co = ca + cb;
  UNET_STRIDE(q, c.n() * ca) {
    const int cc = (int)(q % ca);
    const int64_t v = q / ca;
    const int k = (int)(v % c.nz);
    const int64_t ij = v / c.nz;
    const int j = (int)(ij % c.ny), i = (int)(ij / c.ny);
    float s = 0.0f;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int d = 0; d < 2; ++d) {
          const int fi = 2 * i + a, fj = 2 * j + b, fk = 2 * k + d;
          if (fi < f.nx && fj < f.ny && fk < f.nz) s += g[(((int64_t)fi * f.ny + fj) * f.nz + fk) * co + cc];
        }
    gcoarse[q] = s;
  }
}

__global__ void k_up_concat_back_skip(Dims f, int ca, int cb, const float* __restrict__ g, float* __restrict__ gskip) {
  const int co = ca + cb;
  UNET_STRIDE(q, f.n() * cb) {
    const int cc = (int)(q % cb);
    const int64_t v = q / cb;
    gskip[q] += g[v * co + ca + cc];
  }
}

// dpre = relu ? dy * (y > 0) : dy, as BF16; bias gradient summed per block
__global__ void k_relu_back(int64_t n, int ch, int relu, const float* __restrict__ dy, const bf16* __restrict__ y,
                            bf16* __restrict__ dpre, float* __restrict__ dbias) {
  __shared__ float sb[128];
  for (int c = threadIdx.x; c < ch; c += blockDim.x) sb[c] = 0.0f;
  __syncthreads();
  UNET_STRIDE(q, n * ch) {
    float g = dy[q];
    if (relu && !(__bfloat162float(y[q]) > 0.0f)) g = 0.0f;
    const bf16 gb = __float2bfloat16_rn(g);
    dpre[q] = gb;
    const float gr = __bfloat162float(gb);
    if (gr != 0.0f) atomicAdd(&sb[q % ch], gr);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ch; c += blockDim.x)
    if (sb[c] != 0.0f) atomicAdd(dbias + c, sb[c]);
}

// Weight gradient on the CUDA cores: dW[co][t][ci] += sum_v dpre[v][co] X[v + off(t)][ci]
// over this block's voxel chunk, staged 32 voxels at a time in shared memory.
constexpr int kWgThreads = 256;
constexpr int kWgChunk = 2048;
constexpr int kWgSub = 32;

__global__ void __launch_bounds__(kWgThreads) k_wgrad(Dims d, int cin, int cout, const bf16* __restrict__ x,
                                                      const bf16* __restrict__ dpre, float* __restrict__ dw) {
  extern __shared__ float wg_smem[];
  float* sg = wg_smem;                  // [kWgSub][cout]
  float* sx = wg_smem + kWgSub * cout;  // [kWgSub][cin]
  const int t = blockIdx.y;
  const int di = t / 9 - 1, dj = (t / 3) % 3 - 1, dk = t % 3 - 1;
  const int64_t n = d.n();
  const int64_t vbeg = (int64_t)blockIdx.x * kWgChunk, vend = min(n, vbeg + kWgChunk);
  const int nout = cout * cin;
  constexpr int kPer = 28;  // outputs per thread (cout * cin <= 256 * 28)
  float acc[kPer];
#pragma unroll
  for (int q = 0; q < kPer; ++q) acc[q] = 0.0f;
  for (int64_t s0 = vbeg; s0 < vend; s0 += kWgSub) {
    __syncthreads();
    for (int q = threadIdx.x; q < kWgSub * cout; q += kWgThreads) {
      const int r = q / cout, c = q - r * cout;
      const int64_t v = s0 + r;
      sg[q] = v < vend ? __bfloat162float(dpre[v * cout + c]) : 0.0f;
    }
    for (int q = threadIdx.x; q < kWgSub * cin; q += kWgThreads) {
      const int r = q / cin, c = q - r * cin;
      const int64_t v = s0 + r;
      float val = 0.0f;
      if (v < vend) {
        const int k = (int)(v % d.nz);
        const int64_t ij = v / d.nz;
        const int j = (int)(ij % d.ny), i = (int)(ij / d.ny);
        const int ii = i + di, jj = j + dj, kk = k + dk;
        if (ii >= 0 && ii < d.nx && jj >= 0 && jj < d.ny && kk >= 0 && kk < d.nz)
          val = __bfloat162float(x[(((int64_t)ii * d.ny + jj) * d.nz + kk) * cin + c]);
      }
      sx[q] = val;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      const int o = threadIdx.x + q * kWgThreads;
      if (o >= nout) break;
      const int co = o / cin, ci = o - co * cin;
      float a = acc[q];
      for (int r = 0; r < kWgSub; ++r) a += sg[r * cout + co] * sx[r * cin + ci];
      acc[q] = a;
    }
  }
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    const int o = threadIdx.x + q * kWgThreads;
    if (o >= nout) break;
    const int co = o / cin, ci = o - co * cin;
    if (acc[q] != 0.0f) atomicAdd(dw + ((int64_t)co * 27 + t) * cin + ci, acc[q]);
  }
}

// BF16 copy of the FP32 master weights, and the flipped / transposed copy for
// the input gradient: wt[ci][26 - t][co] = w[co][t][ci].
__global__ void k_weights_bf16(int cin, int cout, const float* __restrict__ w, bf16* __restrict__ wb,
                               bf16* __restrict__ wt) {
  UNET_STRIDE(q, (int64_t)cout * 27 * cin) {
    const int ci = (int)(q % cin);
    const int64_t r = q / cin;
    const int t = (int)(r % 27), co = (int)(r / 27);
    const bf16 b = __float2bfloat16_rn(w[q]);
    wb[q] = b;
    wt[((int64_t)ci * 27 + (26 - t)) * cout + co] = b;
  }
}

__global__ void k_adam(int64_t n, float* __restrict__ p, float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  UNET_STRIDE(q, n) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    g[q] = 0.0f;
  }
}

// masked mean-square loss of output channel 0 against the target, and its
// gradient dout (all 16 channels written; only channel 0 is non-zero)
__global__ void k_loss(int64_t n, const float* __restrict__ out, const float* __restrict__ target,
                       const float* __restrict__ mask, float inv_count, float* __restrict__ dout,
                       double* __restrict__ loss) {
  double part = 0.0;
  UNET_STRIDE(v, n) {
    const float m = mask[v];
    const float e = m * (out[v * kOutCh] - target[v]);
    part += (double)e * (double)e;
    dout[v * kOutCh] = 2.0f * e * inv_count;
#pragma unroll
    for (int c = 1; c < kOutCh; ++c) dout[v * kOutCh + c] = 0.0f;
  }
  double a[1] = {part};
  block_sum<1>(a);
  if (threadIdx.x == 0) atomicAdd(loss, a[0] * (double)inv_count);
}

#undef UNET_STRIDE

unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

}  // namespace
}  // namespace efsi

using namespace efsi;

// ---------------------------------------------------------------------------
// The network object
// ---------------------------------------------------------------------------
namespace efsi {
// Buffers of one volume size: layer outputs, decoder inputs, pooled inputs,
// the FP32 output and the backward pass's gradients.
struct UnetWorkspace {
  Dims dims[kLevels] = {};
  bf16* act[kLayers] = {};     // layer outputs
  bf16* cat[3] = {};           // decoder inputs [up, skip] at levels 2, 1, 0
  bf16* pooled[3] = {};        // encoder inputs at levels 1, 2, 3
  float* outf = nullptr;       // FP32 output of the last layer
  float* gbuf[2] = {};         // gradient ping-pong (FP32), sized for the largest layer input
  float* gskip[kLevels] = {};  // accumulated gradients of e_0 .. e_3
  float* gcoarse = nullptr;
  bf16* dpre = nullptr;
  float* dout = nullptr;
};
}  // namespace efsi

struct efsi_unet {
  // parameters (FP32 master, gradients, Adam moments) packed per layer:
  // weights [cout][27][cin] then bias [cout]
  int64_t nparams = 0;
  int64_t woff[kLayers], boff[kLayers];
  float* p = nullptr;
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  bf16* wb[kLayers] = {};
  bf16* wt[kLayers] = {};
  int adam_step = 0;
  // one workspace per volume size, kept until the network is destroyed (a
  // solver plan may have captured a workspace's buffers in its CUDA graphs);
  // `w` is the one of the current pass
  std::vector<efsi::UnetWorkspace*> spaces;
  efsi::UnetWorkspace* w = nullptr;
  double* loss = nullptr;
  int* error = nullptr;      // the network's own error word
  int* run_error = nullptr;  // where the convolutions of a run report (the PCG's fault word inside a solve)
};

namespace efsi {
namespace {

constexpr int kMaxWorkspaces = 8;

void free_workspace(UnetWorkspace* W) {
  for (auto& a : W->act) cudaFree(a), a = nullptr;
  for (auto& a : W->cat) cudaFree(a), a = nullptr;
  for (auto& a : W->pooled) cudaFree(a), a = nullptr;
  for (auto& a : W->gbuf) cudaFree(a), a = nullptr;
  for (auto& a : W->gskip) cudaFree(a), a = nullptr;
  cudaFree(W->outf);
  cudaFree(W->gcoarse);
  cudaFree(W->dpre);
  cudaFree(W->dout);
  W->outf = W->gcoarse = W->dout = nullptr;
  W->dpre = nullptr;
}

// Selects (allocating on first use) the workspace of a level-0 volume.
int ensure_workspace(efsi_unet* U, int nx, int ny, int nz) {
  for (UnetWorkspace* W : U->spaces)
    if (W->dims[0].nx == nx && W->dims[0].ny == ny && W->dims[0].nz == nz) {
      U->w = W;
      return EFSI_OK;
    }
  if ((int)U->spaces.size() >= kMaxWorkspaces) {
    set_error("the U-Net already holds workspaces for 8 volume sizes");
    return EFSI_ERR_ARG;
  }
  UnetWorkspace* W = new UnetWorkspace();
  const Dims d0{nx, ny, nz};
  W->dims[0] = d0;
  for (int l = 1; l < kLevels; ++l) W->dims[l] = coarse_of(W->dims[l - 1]);
  auto alloc_bf = [](bf16** p, int64_t n) { return cudaMalloc(p, (size_t)std::max<int64_t>(n, 1) * sizeof(bf16)); };
  auto alloc_f = [](float** p, int64_t n) { return cudaMalloc(p, (size_t)std::max<int64_t>(n, 1) * sizeof(float)); };
  int64_t gmax = 0;
  for (int l = 0; l < kLayers; ++l) {
    const int64_t n = W->dims[kSpec[l].level].n();
    if (alloc_bf(&W->act[l], n * kSpec[l].cout) != cudaSuccess) goto fail;
    gmax = std::max(gmax, n * std::max(kSpec[l].cin, kSpec[l].cout));
  }
  for (int q = 0; q < 3; ++q) {
    const int l = 2 - q;  // decoder levels 2, 1, 0
    const int64_t n = W->dims[l].n();
    if (alloc_bf(&W->cat[q], n * (kCh[l + 1] + kCh[l])) != cudaSuccess) goto fail;
    if (alloc_bf(&W->pooled[q], W->dims[q + 1].n() * kCh[q]) != cudaSuccess) goto fail;
  }
  for (int l = 0; l < kLevels; ++l)
    if (alloc_f(&W->gskip[l], W->dims[l].n() * kCh[l]) != cudaSuccess) goto fail;
  if (alloc_f(&W->gbuf[0], gmax) != cudaSuccess || alloc_f(&W->gbuf[1], gmax) != cudaSuccess ||
      alloc_f(&W->gcoarse, gmax) != cudaSuccess || alloc_bf(&W->dpre, gmax) != cudaSuccess ||
      alloc_f(&W->outf, d0.n() * kOutCh) != cudaSuccess || alloc_f(&W->dout, d0.n() * kOutCh) != cudaSuccess)
    goto fail;
  U->spaces.push_back(W);
  U->w = W;
  return EFSI_OK;
fail:
  free_workspace(W);
  delete W;
  set_error("cudaMalloc failed for the U-Net workspace");
  return EFSI_ERR_CUDA;
}

// Opt-in shared-memory limits of the convolution kernels, set once per
// process (before any graph capture: efsi_unet_create calls it).
int set_kernel_attributes() {
  static bool done = false;
  if (done) return EFSI_OK;
  EFSI_CUDA_CHECK(cudaFuncSetAttribute(conv::k_conv3d_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  EFSI_CUDA_CHECK(cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
  done = true;
  return EFSI_OK;
}

int conv_launch(const Dims& d, int cin, int cout, const bf16* x, const bf16* w, const float* bias, int relu, bf16* y,
                float* yf, int* error, cudaStream_t s) {
  conv::ConvArgs A{d.nx, d.ny, d.nz, cin, cout, x, w, bias, relu, y, yf, error};
  // enough shared memory per CTA that the CTAs resident on an SM never ask for
  // more than its 512 tensor-memory columns
  const int per_sm = 512 / (int)conv::tmem_columns(cout);
  const int smem = std::max(conv::conv_smem_bytes(cin, cout), 228 * 1024 / per_sm + 1024);
  EFSI_TRY(set_kernel_attributes());
  const unsigned blocks = (unsigned)((d.n() + conv::kTileM - 1) / conv::kTileM);
  EFSI_COUNTED conv::k_conv3d_tc<<<blocks, conv::kThreads, smem, s>>>(A);
  return EFSI_OK;
}

int wgrad_launch(const Dims& d, int cin, int cout, const bf16* x, const bf16* dpre, float* dw, cudaStream_t s) {
  EFSI_TRY(set_kernel_attributes());
  const dim3 grid((unsigned)((d.n() + kWgChunk - 1) / kWgChunk), 27);
  const int smem = kWgSub * (cin + cout) * (int)sizeof(float);
  EFSI_COUNTED k_wgrad<<<grid, kWgThreads, smem, s>>>(d, cin, cout, x, dpre, dw);
  return EFSI_OK;
}

int refresh_bf16(efsi_unet* U, cudaStream_t s) {
  for (int l = 0; l < kLayers; ++l) {
    const int64_t n = weight_count(l);
    EFSI_COUNTED k_weights_bf16<<<grid_for(n), 256, 0, s>>>(kSpec[l].cin, kSpec[l].cout, U->p + U->woff[l], U->wb[l],
                                                         U->wt[l]);
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

// Forward pass over the workspace volume; input [n0][16] BF16.
int forward(efsi_unet* U, const bf16* input, cudaStream_t s) {
  const bf16* x = input;
  int* err = U->run_error != nullptr ? U->run_error : U->error;
  // encoder
  for (int l = 0; l < kLevels; ++l) {
    const Dims& d = U->w->dims[l];
    if (l > 0) {
      EFSI_COUNTED k_pool<<<grid_for(d.n() * kCh[l - 1]), 256, 0, s>>>(U->w->dims[l - 1], d, kCh[l - 1], U->w->act[2 * l - 1],
                                                                    U->w->pooled[l - 1]);
      x = U->w->pooled[l - 1];
    }
    const int a = 2 * l, b = 2 * l + 1;
    EFSI_TRY(conv_launch(d, kSpec[a].cin, kSpec[a].cout, x, U->wb[a], U->p + U->boff[a], 1, U->w->act[a], nullptr,
                         err, s));
    EFSI_TRY(conv_launch(d, kSpec[b].cin, kSpec[b].cout, U->w->act[a], U->wb[b], U->p + U->boff[b], 1, U->w->act[b],
                         nullptr, err, s));
  }
  // decoder
  const bf16* coarse = U->w->act[7];
  for (int q = 0; q < 3; ++q) {
    const int l = 2 - q;
    const Dims& d = U->w->dims[l];
    const int ca = kCh[l + 1];
    EFSI_COUNTED k_up_concat<<<grid_for(d.n() * (ca + kCh[l])), 256, 0, s>>>(d, U->w->dims[l + 1], ca, kCh[l], coarse,
                                                                          U->w->act[2 * l + 1], U->w->cat[q]);
    const int a = 8 + 2 * q, b = 9 + 2 * q;
    EFSI_TRY(conv_launch(d, kSpec[a].cin, kSpec[a].cout, U->w->cat[q], U->wb[a], U->p + U->boff[a], 1, U->w->act[a],
                         nullptr, err, s));
    EFSI_TRY(conv_launch(d, kSpec[b].cin, kSpec[b].cout, U->w->act[a], U->wb[b], U->p + U->boff[b], 1, U->w->act[b],
                         nullptr, err, s));
    coarse = U->w->act[b];
  }
  EFSI_TRY(conv_launch(U->w->dims[0], kSpec[14].cin, kSpec[14].cout, U->w->act[13], U->wb[14], U->p + U->boff[14], 0,
                       U->w->act[14], U->w->outf, err, s));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

// Input of layer l during the forward pass.
const bf16* layer_input(efsi_unet* U, const bf16* input, int l) {
  if (l == 0) return input;
  if (l < 8) return (l % 2 == 1) ? U->w->act[l - 1] : U->w->pooled[l / 2 - 1];
  if (l < 14) return (l % 2 == 0) ? U->w->cat[(l - 8) / 2] : U->w->act[l - 1];
  return U->w->act[13];
}

// Backward of one layer: gy (FP32 [n][cout]) -> parameter gradients, and the
// input gradient into gx (FP32 [n][cin]) when gx is given.
int layer_backward(efsi_unet* U, const bf16* input, int l, const float* gy, float* gx, cudaStream_t s) {
  const LayerSpec& L = kSpec[l];
  const Dims& d = U->w->dims[L.level];
  const int64_t n = d.n();
  EFSI_COUNTED k_relu_back<<<grid_for(n * L.cout), 256, 0, s>>>(n, L.cout, L.relu, gy, U->w->act[l], U->w->dpre,
                                                             U->g + U->boff[l]);
  EFSI_TRY(wgrad_launch(d, L.cin, L.cout, layer_input(U, input, l), U->w->dpre, U->g + U->woff[l], s));
  if (gx != nullptr)
    EFSI_TRY(conv_launch(d, L.cout, L.cin, U->w->dpre, U->wt[l], nullptr, 0, nullptr, gx, U->error, s));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

// Backward pass from dout (FP32 [n0][16]); accumulates into U->g.
int backward(efsi_unet* U, const bf16* input, const float* dout, cudaStream_t s) {
  float* ga = U->w->gbuf[0];
  float* gb = U->w->gbuf[1];
  for (int l = 0; l < kLevels; ++l)
    EFSI_CUDA_CHECK(cudaMemsetAsync(U->w->gskip[l], 0, (size_t)U->w->dims[l].n() * kCh[l] * sizeof(float), s));
  // output layer and the decoder, level 0 up to level 2
  EFSI_TRY(layer_backward(U, input, 14, dout, ga, s));  // -> g(d0)
  const float* gcur = ga;
  for (int q = 2; q >= 0; --q) {
    const int l = 2 - q;  // decoder level of block q
    const int a = 8 + 2 * q, b = 9 + 2 * q;
    float* t1 = (gcur == ga) ? gb : ga;
    EFSI_TRY(layer_backward(U, input, b, gcur, t1, s));  // -> g(d_la)
    float* t2 = (t1 == ga) ? gb : ga;
    EFSI_TRY(layer_backward(U, input, a, t1, t2, s));  // -> g([up, skip])
    const int ca = kCh[l + 1], cb = kCh[l];
    EFSI_COUNTED k_up_concat_back_skip<<<grid_for(U->w->dims[l].n() * cb), 256, 0, s>>>(U->w->dims[l], ca, cb, t2,
                                                                                   U->w->gskip[l]);
    EFSI_COUNTED k_up_concat_back_coarse<<<grid_for(U->w->dims[l + 1].n() * ca), 256, 0, s>>>(
        U->w->dims[l], U->w->dims[l + 1], ca, cb, t2, U->w->gcoarse);
    // the coarse gradient is that of d_{l+1} (or e_3 for the deepest block)
    float* nxt = (t2 == ga) ? gb : ga;
    EFSI_CUDA_CHECK(cudaMemcpyAsync(nxt, U->w->gcoarse, (size_t)U->w->dims[l + 1].n() * ca * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s));
    gcur = nxt;
  }
  // gcur is g(e_3) from the decoder; the encoder from level 3 down to 0
  for (int l = kLevels - 1; l >= 0; --l) {
    const Dims& d = U->w->dims[l];
    float* gin;
    if (l == kLevels - 1) {
      gin = const_cast<float*>(gcur);
    } else {
      // e_l receives its skip gradient plus the pooled path's
      gin = U->w->gskip[l];
    }
    const int a = 2 * l, b = 2 * l + 1;
    float* t1 = (gin == ga) ? gb : ga;
    EFSI_TRY(layer_backward(U, input, b, gin, t1, s));  // -> g(e_la)
    if (l == 0) {
      EFSI_TRY(layer_backward(U, input, a, t1, nullptr, s));
      break;
    }
    float* t2 = (t1 == ga) ? gb : ga;
    EFSI_TRY(layer_backward(U, input, a, t1, t2, s));  // -> g(pooled e_{l-1})
    EFSI_COUNTED k_pool_back<<<grid_for(U->w->dims[l - 1].n() * kCh[l - 1]), 256, 0, s>>>(U->w->dims[l - 1], d, kCh[l - 1],
                                                                                     t2, U->w->gskip[l - 1]);
  }
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int check_error(efsi_unet* U, cudaStream_t s) {
  int h = 0;
  EFSI_CUDA_CHECK(cudaMemcpyAsync(&h, U->error, sizeof(int), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  if (h != 0) {
    set_error("a U-Net convolution's tensor-core pipeline did not complete in time");
    return EFSI_ERR_CUDA;
  }
  return EFSI_OK;
}

}  // namespace

int unet_prepare(efsi_unet* U, int nx, int ny, int nz) { return ensure_workspace(U, nx, ny, nz); }

int unet_run(efsi_unet* U, int nx, int ny, int nz, const void* input, int* error_word, const float** out,
             cudaStream_t s) {
  // the volume's workspace exists (unet_prepare), so this only selects it
  EFSI_TRY(ensure_workspace(U, nx, ny, nz));
  U->run_error = error_word;
  const int rc = forward(U, static_cast<const bf16*>(input), s);
  U->run_error = nullptr;
  *out = U->w->outf;
  return rc;
}

}  // namespace efsi

extern "C" {

int efsi_conv3d_bf16(int32_t nx, int32_t ny, int32_t nz, int32_t cin, int32_t cout, const void* x, const void* w,
                     const float* bias, int32_t relu, void* y, float* yf, int32_t* error_device, void* stream) {
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "volume extents must be positive");
  EFSI_ARG_CHECK(cin >= 16 && cin % 16 == 0 && cin <= 256, "cin must be a multiple of 16 in [16, 256]");
  EFSI_ARG_CHECK(cout >= 16 && cout % 16 == 0 && cout <= 256, "cout must be a multiple of 16 in [16, 256]");
  EFSI_ARG_CHECK(x != nullptr && w != nullptr && error_device != nullptr && (y != nullptr || yf != nullptr),
                 "null argument");
  EFSI_ARG_CHECK(conv::conv_smem_bytes(cin, cout) <= 200 * 1024, "cin x cout too large for the shared-memory stages");
  EFSI_TRY(conv_launch(Dims{nx, ny, nz}, cin, cout, static_cast<const bf16*>(x), static_cast<const bf16*>(w), bias,
                       relu, static_cast<bf16*>(y), yf, error_device, as_stream(stream)));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_conv3d_wgrad(int32_t nx, int32_t ny, int32_t nz, int32_t cin, int32_t cout, const void* x,
                      const void* dy, float* dw, void* stream) {
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "volume extents must be positive");
  EFSI_ARG_CHECK(cin >= 16 && cin % 16 == 0 && cout >= 16 && cout % 16 == 0 && cin * cout <= 256 * 28,
                 "unsupported channel counts for the weight gradient");
  EFSI_ARG_CHECK(x != nullptr && dy != nullptr && dw != nullptr, "null argument");
  EFSI_TRY(wgrad_launch(Dims{nx, ny, nz}, cin, cout, static_cast<const bf16*>(x), static_cast<const bf16*>(dy), dw,
                        as_stream(stream)));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

int efsi_unet_create(int32_t seed, efsi_unet** out) {
  EFSI_ARG_CHECK(out != nullptr, "null output");
  EFSI_TRY(set_kernel_attributes());
  efsi_unet* U = new efsi_unet();
  int64_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    U->woff[l] = off;
    off += weight_count(l);
    U->boff[l] = off;
    off += kSpec[l].cout;
  }
  U->nparams = off;
  bool ok = cudaMalloc(&U->p, off * sizeof(float)) == cudaSuccess && cudaMalloc(&U->g, off * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&U->m, off * sizeof(float)) == cudaSuccess && cudaMalloc(&U->v, off * sizeof(float)) == cudaSuccess &&
            cudaMalloc(&U->loss, sizeof(double)) == cudaSuccess && cudaMalloc(&U->error, sizeof(int)) == cudaSuccess;
  for (int l = 0; ok && l < kLayers; ++l)
    ok = cudaMalloc(&U->wb[l], weight_count(l) * sizeof(bf16)) == cudaSuccess &&
         cudaMalloc(&U->wt[l], weight_count(l) * sizeof(bf16)) == cudaSuccess;
  if (!ok) {
    efsi_unet_destroy(U);
    set_error("cudaMalloc failed for the U-Net parameters");
    return EFSI_ERR_CUDA;
  }
  // He-normal weights (fan-in 27 cin), zero biases; the output layer starts small
  std::vector<float> h((size_t)off, 0.0f);
  std::mt19937_64 rng((uint64_t)seed);
  for (int l = 0; l < kLayers; ++l) {
    const double sd = std::sqrt(2.0 / (27.0 * kSpec[l].cin)) * (l == kLayers - 1 ? 0.1 : 1.0);
    std::normal_distribution<double> nd(0.0, sd);
    for (int64_t q = 0; q < weight_count(l); ++q) h[(size_t)(U->woff[l] + q)] = (float)nd(rng);
  }
  if (cudaMemcpy(U->p, h.data(), off * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(U->g, 0, off * sizeof(float)) != cudaSuccess || cudaMemset(U->m, 0, off * sizeof(float)) != cudaSuccess ||
      cudaMemset(U->v, 0, off * sizeof(float)) != cudaSuccess || cudaMemset(U->error, 0, sizeof(int)) != cudaSuccess ||
      refresh_bf16(U, 0) != EFSI_OK || cudaDeviceSynchronize() != cudaSuccess) {
    efsi_unet_destroy(U);
    set_error("U-Net parameter initialisation failed");
    return EFSI_ERR_CUDA;
  }
  *out = U;
  return EFSI_OK;
}

int efsi_unet_destroy(efsi_unet* U) {
  if (U == nullptr) return EFSI_OK;
  for (UnetWorkspace* W : U->spaces) {
    free_workspace(W);
    delete W;
  }
  U->spaces.clear();
  cudaFree(U->p);
  cudaFree(U->g);
  cudaFree(U->m);
  cudaFree(U->v);
  cudaFree(U->loss);
  cudaFree(U->error);
  for (int l = 0; l < kLayers; ++l) {
    cudaFree(U->wb[l]);
    cudaFree(U->wt[l]);
  }
  delete U;
  return EFSI_OK;
}

int efsi_unet_param_count(efsi_unet* U, int64_t* count) {
  EFSI_ARG_CHECK(U != nullptr && count != nullptr, "null argument");
  *count = U->nparams;
  return EFSI_OK;
}

int efsi_unet_layer_offsets(efsi_unet* U, int64_t* weight_offsets, int64_t* bias_offsets, int32_t* shapes) {
  EFSI_ARG_CHECK(U != nullptr && weight_offsets != nullptr && bias_offsets != nullptr && shapes != nullptr,
                 "null argument");
  for (int l = 0; l < kLayers; ++l) {
    weight_offsets[l] = U->woff[l];
    bias_offsets[l] = U->boff[l];
    shapes[4 * l] = kSpec[l].level;
    shapes[4 * l + 1] = kSpec[l].cin;
    shapes[4 * l + 2] = kSpec[l].cout;
    shapes[4 * l + 3] = kSpec[l].relu;
  }
  return EFSI_OK;
}

int efsi_unet_get_params(efsi_unet* U, float* host_params, float* host_grads) {
  EFSI_ARG_CHECK(U != nullptr, "null network");
  if (host_params) EFSI_CUDA_CHECK(cudaMemcpy(host_params, U->p, U->nparams * sizeof(float), cudaMemcpyDeviceToHost));
  if (host_grads) EFSI_CUDA_CHECK(cudaMemcpy(host_grads, U->g, U->nparams * sizeof(float), cudaMemcpyDeviceToHost));
  return EFSI_OK;
}

int efsi_unet_set_params(efsi_unet* U, const float* host_params) {
  EFSI_ARG_CHECK(U != nullptr && host_params != nullptr, "null argument");
  EFSI_CUDA_CHECK(cudaMemcpy(U->p, host_params, U->nparams * sizeof(float), cudaMemcpyHostToDevice));
  EFSI_CUDA_CHECK(cudaMemset(U->m, 0, U->nparams * sizeof(float)));
  EFSI_CUDA_CHECK(cudaMemset(U->v, 0, U->nparams * sizeof(float)));
  U->adam_step = 0;
  EFSI_TRY(refresh_bf16(U, 0));
  EFSI_CUDA_CHECK(cudaDeviceSynchronize());
  return EFSI_OK;
}

int efsi_unet_forward(efsi_unet* U, int32_t nx, int32_t ny, int32_t nz, const void* input, float* output,
                      void* stream) {
  EFSI_ARG_CHECK(U != nullptr && input != nullptr, "null argument");
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "volume extents must be positive");
  cudaStream_t s = as_stream(stream);
  EFSI_TRY(ensure_workspace(U, nx, ny, nz));
  EFSI_TRY(forward(U, static_cast<const bf16*>(input), s));
  if (output != nullptr)
    EFSI_CUDA_CHECK(cudaMemcpyAsync(output, U->w->outf, (size_t)U->w->dims[0].n() * kOutCh * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s));
  return check_error(U, s);
}

int efsi_unet_accumulate_gradient(efsi_unet* U, int32_t nx, int32_t ny, int32_t nz, const void* input,
                                  const float* target, const float* mask, double* loss_host, void* stream) {
  EFSI_ARG_CHECK(U != nullptr && input != nullptr && target != nullptr && mask != nullptr && loss_host != nullptr,
                 "null argument");
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "volume extents must be positive");
  cudaStream_t s = as_stream(stream);
  EFSI_TRY(ensure_workspace(U, nx, ny, nz));
  const bf16* in = static_cast<const bf16*>(input);
  EFSI_TRY(forward(U, in, s));
  const int64_t n = U->w->dims[0].n();
  EFSI_CUDA_CHECK(cudaMemsetAsync(U->loss, 0, sizeof(double), s));
  EFSI_COUNTED k_loss<<<grid_for(n), 256, 0, s>>>(n, U->w->outf, target, mask, 1.0f / (float)n, U->w->dout, U->loss);
  EFSI_TRY(backward(U, in, U->w->dout, s));
  EFSI_CUDA_CHECK(cudaMemcpyAsync(loss_host, U->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
  return check_error(U, s);
}

int efsi_unet_backward_from(efsi_unet* U, int32_t nx, int32_t ny, int32_t nz, const void* input,
                            const float* dout, void* stream) {
  EFSI_ARG_CHECK(U != nullptr && input != nullptr && dout != nullptr, "null argument");
  cudaStream_t s = as_stream(stream);
  EFSI_TRY(ensure_workspace(U, nx, ny, nz));
  const bf16* in = static_cast<const bf16*>(input);
  EFSI_TRY(forward(U, in, s));
  EFSI_TRY(backward(U, in, dout, s));
  return check_error(U, s);
}

int efsi_unet_zero_grad(efsi_unet* U, void* stream) {
  EFSI_ARG_CHECK(U != nullptr, "null network");
  EFSI_CUDA_CHECK(cudaMemsetAsync(U->g, 0, U->nparams * sizeof(float), as_stream(stream)));
  return EFSI_OK;
}

int efsi_unet_adam_step(efsi_unet* U, float lr, float beta1, float beta2, float eps, void* stream) {
  EFSI_ARG_CHECK(U != nullptr, "null network");
  EFSI_ARG_CHECK(lr > 0.0f && beta1 >= 0.0f && beta1 < 1.0f && beta2 >= 0.0f && beta2 < 1.0f && eps > 0.0f,
                 "invalid Adam hyper-parameters");
  cudaStream_t s = as_stream(stream);
  U->adam_step += 1;
  const float c1 = 1.0f - std::pow(beta1, (float)U->adam_step), c2 = 1.0f - std::pow(beta2, (float)U->adam_step);
  EFSI_COUNTED k_adam<<<grid_for(U->nparams), 256, 0, s>>>(U->nparams, U->p, U->g, U->m, U->v, lr, beta1, beta2, eps,
                                                           c1, c2);
  EFSI_TRY(refresh_bf16(U, s));
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"
