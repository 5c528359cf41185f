// 3x3x3 convolutions of channels-last BF16 volumes on the sm_100a tensor cores
// (tcgen05), for the learned preconditioner's U-Net.
//
// Forward (and, with flipped / transposed weights, the input gradient) is an
// implicit GEMM: D[v][co] = sum_t sum_ci X[v + off(t)][ci] W[co][t][ci], with
// M = 128 consecutive voxels per CTA, N = Cout (16..256, a multiple of 16) and
// K = 27 taps x Cin (Cin a multiple of 16).  Per tap the 128 x Cin slice of
// the im2col matrix (zero outside the volume) and the Cout x Cin slice of the
// weights are copied by the CTA's threads (cp.async, 16 bytes each, zero
// filled outside the volume) into shared memory in the canonical no-swizzle
// K-major layout (8-row x 16-byte core matrices: SBO = 128 bytes between
// 8-row groups, LBO = rows x 16 bytes between 8-element K chunks), through a
// ring of kStages stages, so the copies of the next kAhead taps are in flight
// while one elected thread issues tcgen05.mma.kind::f16 (BF16
// operands, FP32 accumulator in tensor memory) per 16-channel K step of the
// current tap and commits to the stage's mbarrier.  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// lanes 32w..32w+31 = voxels), adds the bias, applies ReLU if asked and
// stores BF16 (and optionally FP32).
//
// Every mbarrier wait is bounded; a wait that gives up sets the caller's
// error word, waits (bounded) for the MMAs in flight and frees the tensor
// memory before returning.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace efsi {
namespace conv {

constexpr int kTileM = 128;          // voxels per CTA (MMA M)
constexpr int kThreads = 128;        // 4 warps: one TMEM lane quadrant each
constexpr int kStages = 4;           // taps in the shared-memory ring
constexpr int kLag = 2;              // a stage is refilled once the MMAs of kLag taps ago are done
constexpr int kAhead = kStages - kLag;  // taps whose copies are in flight ahead of the current one
constexpr long long kWaitLimit = 4000000000LL;  // ~2 s of clock64

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (SWIZZLE_NONE, K-major, version 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 D.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_test(bar, parity))
    if (clock64() - t0 > kWaitLimit) return false;
  return true;
}

// 16-byte asynchronous copy global -> shared; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

struct ConvArgs {
  int nx, ny, nz;
  int cin, cout;                 // multiples of 16; cout <= 256
  const __nv_bfloat16* x;        // [n][cin]
  const __nv_bfloat16* w;        // [cout][27][cin]
  const float* bias;             // [cout] or null
  int relu;                      // apply ReLU in the epilogue
  __nv_bfloat16* y;              // [n][cout] or null
  float* yf;                     // [n][cout] FP32 copy or null
  int* error;                    // set to 1 when a wait gives up
};

// Bytes of dynamic shared memory for one launch (kStages stages of A and B).
__host__ __device__ inline int conv_smem_bytes(int cin, int cout) {
  const int a = kTileM * cin * 2, b = cout * cin * 2;
  return kStages * (a + b) + 128;
}

__host__ __device__ inline uint32_t tmem_columns(int cout) {
  uint32_t c = 32;
  while ((int)c < cout) c <<= 1;
  return c;
}

__global__ void __launch_bounds__(kThreads) k_conv3d_tc(ConvArgs A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[kStages];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int cin = A.cin, cout = A.cout;
  const int a_bytes = kTileM * cin * 2, b_bytes = cout * cin * 2;
  const int stage_bytes = a_bytes + b_bytes;
  const uint32_t lbo_a = (kTileM / 8) * 128, lbo_b = (uint32_t)(cout / 8) * 128;
  const uint32_t ncols = tmem_columns(cout);
  const int64_t n = (int64_t)A.nx * A.ny * A.nz;
  const int64_t v0 = (int64_t)blockIdx.x * kTileM;

  if (tid == 0) {
    for (int q = 0; q < kStages; ++q) mbar_init(&bars[q]);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  // this thread's voxel row of the im2col slice
  const int64_t v = v0 + tid;
  int vi = 0, vj = 0, vk = 0;
  if (v < n) {
    vk = (int)(v % A.nz);
    const int64_t ij = v / A.nz;
    vj = (int)(ij % A.ny);
    vi = (int)(ij / A.ny);
  }
  const int kchunks = cin / 8;
  // copies of tap t into its stage: the thread's A row and a share of B
  auto issue = [&](int t) {
    unsigned char* sa = smem_raw + (t % kStages) * stage_bytes;
    unsigned char* sb = sa + a_bytes;
    const int di = t / 9 - 1, dj = (t / 3) % 3 - 1, dk = t % 3 - 1;
    const int ii = vi + di, jj = vj + dj, kk = vk + dk;
    const bool in = v < n && ii >= 0 && ii < A.nx && jj >= 0 && jj < A.ny && kk >= 0 && kk < A.nz;
    const __nv_bfloat16* src = in ? A.x + (((int64_t)ii * A.ny + jj) * A.nz + kk) * cin : A.x;
    unsigned char* dst = sa + (tid >> 3) * 128 + (tid & 7) * 16;
    for (int c = 0; c < kchunks; ++c) cp_async16(dst + c * lbo_a, src + (in ? c * 8 : 0), in ? 16 : 0);
    for (int q = tid; q < cout * kchunks; q += kThreads) {
      const int co = q / kchunks, c = q - co * kchunks;
      cp_async16(sb + c * lbo_b + (co >> 3) * 128 + (co & 7) * 16, A.w + ((int64_t)co * 27 + t) * cin + c * 8, 16);
    }
  };
  const uint32_t idesc = idesc_bf16(kTileM, cout);
  // prologue: taps 0 .. kAhead - 1 in flight (one commit group per tap)
  for (int t = 0; t < kAhead; ++t) {
    issue(t);
    cp_async_commit();
  }
  bool ok = true, good = true;
  for (int t = 0; t < 27; ++t) {
    // this thread's copies of tap t have landed once at most kAhead - 1
    // newer groups are pending; the block decides together whether to go on
    cp_async_wait<kAhead - 1>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (!__syncthreads_and(good)) {
      ok = false;
      break;
    }
    if (tid == 0) {
      tc_fence_after();
      const uint32_t a0 = smem_u32(smem_raw + (t % kStages) * stage_bytes);
      const uint32_t b0 = a0 + a_bytes;
      for (int ks = 0; ks < cin / 16; ++ks) {
        const uint64_t ad = umma_desc(a0 + ks * 2 * lbo_a, lbo_a, 128);
        const uint64_t bd = umma_desc(b0 + ks * 2 * lbo_b, lbo_b, 128);
        tc_mma(tmem, ad, bd, idesc, (t > 0 || ks > 0) ? 1 : 0);
      }
      tc_commit(&bars[t % kStages]);
    }
    // refill the stage of tap t - kLag with tap t + kAhead once the MMAs of
    // tap t - kLag have read it (issued kLag iterations ago, so the wait is
    // normally already over)
    const int tn = t + kAhead;
    if (tn < 27) {
      if (t >= kLag) good = mbar_wait_bounded(&bars[(t - kLag) % kStages], (unsigned)(((t - kLag) / kStages) & 1));
      if (good) issue(tn);
    }
    cp_async_commit();  // one group per iteration, possibly empty
  }
  cp_async_wait<0>();
  // the last commit covers every MMA issued before it
  ok = __syncthreads_and(ok && mbar_wait_bounded(&bars[26 % kStages], (unsigned)((26 / kStages) & 1)));
  tc_fence_after();
  if (ok) {
    const int64_t vr = v0 + warp * 32 + lane;
    for (int c0 = 0; c0 < cout; c0 += 16) {
      float acc[16];
      tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
      if (vr < n) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          float a = acc[q] + (A.bias != nullptr ? __ldg(A.bias + c0 + q) : 0.0f);
          acc[q] = A.relu ? fmaxf(a, 0.0f) : a;
        }
        if (A.y != nullptr) {
          __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) hb[q] = __float2bfloat16_rn(acc[q]);
          uint4* dst = reinterpret_cast<uint4*>(A.y + vr * cout + c0);
          dst[0] = reinterpret_cast<const uint4*>(hb)[0];
          dst[1] = reinterpret_cast<const uint4*>(hb)[1];
        }
        if (A.yf != nullptr) {
          float4* dst = reinterpret_cast<float4*>(A.yf + vr * cout + c0);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
        }
      }
    }
  } else {
    if (tid == 0) atomicExch(A.error, 1);
    // drain: give the MMAs in flight a bounded chance to finish
    for (int q = 0; q < kStages; ++q) mbar_wait_bounded(&bars[q], 0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
  }
}

}  // namespace conv
}  // namespace efsi
