// Neo-Hookean MLS/APIC-MPM substep, B200 path (replaces the fused Taichi
// _step_kernel of simulation_core/neo_hookean_mpm.py:696-959).
//
// The reference scatters every particle's 27-node stencil with 189 global f32
// atomics.  Here particles are first binned by the 4x4x4-node tile that holds
// their stencil base node (counting sort: histogram, scan, scatter), then one
// CTA per tile accumulates its particles' mass / momentum / force into a 6x6x6
// node block in shared memory and flushes it with one global atomic per
// non-zero node value.  Grid update and G2P are one pass each; G2P walks the
// particles in tile order so the 27-node gathers hit L1/L2.  The report
// diagnostics of the reference are reduced in the same passes (block sums, one
// f64 atomic per block).
#include <cuda_runtime.h>

#include <cmath>

#include "efsi_common.cuh"

namespace efsi {

constexpr int kTile = 4;             // nodes per tile edge
constexpr int kHalo = kTile + 2;     // node block touched by a tile's particles
constexpr int kHaloN = kHalo * kHalo * kHalo;
constexpr int kTileCells = kTile * kTile * kTile;  // nodes (and base cells) per tile

// Report accumulator slots (doubles), see k_mpm_finalize for the packing.
enum {
  R_MASS = 0,
  R_VOL,
  R_PMOM,       // 3
  R_GMOM = 5,   // 3
  R_FEXT = 8,   // 3
  R_TMOM = 11,  // 3 (transfer momentum)
  R_MOM2 = 14,
  R_MAXJ,
  R_MAXSPEED,
  R_ACTIVE,
  R_OOB,
  R_CLAMP,
  R_PDISP,       // 3
  R_PVEL = 23,   // 3
  R_SDISP = 26,  // 3
  R_SVEL = 29,   // 3
  R_PCOUNT = 32,
  R_SCOUNT,
  R_CSUM,        // 3 current centre sum
  R_RSUM = 37,   // 3 rest centre sum
  R_CCOUNT = 40,
  R_STRETCH,
  R_STRETCH_N,
  R_STRETCH_ERR,
  R_COUNT
};

}  // namespace efsi

struct efsi_mpm_plan {
  int capacity = 0;
  int nx = 0, ny = 0, nz = 0;
  int tx = 0, ty = 0, tz = 0;  // tile counts
  int ntiles = 0;              // + 1 bucket for out-of-stencil particles
  int32_t* key = nullptr;
  int32_t* sorted = nullptr;
  int32_t* count = nullptr;   // ntiles + 1
  int32_t* offset = nullptr;  // ntiles + 2
  int32_t* cursor = nullptr;  // ntiles + 1
  double* acc = nullptr;      // report accumulators
  // Tiles that hold particles (P2G runs only over them) and the tiles whose
  // nodes their stencils reach (cleared and updated).  The grid outside the
  // reached tiles stays zero: each step clears the tiles reached in this step
  // and in the previous one.
  int32_t* active = nullptr;     // ntiles + 1 tile ids
  uint8_t* reached_flag = nullptr;  // ntiles
  int32_t* reached[2] = {nullptr, nullptr};  // ntiles tile ids: this step's and the previous step's
  int32_t* counts = nullptr;     // [0] active, [1] reached now, [2] reached in the previous step,
                                 // [3] which reached list is this step's (flipped on the device)
};

namespace efsi {

__device__ __forceinline__ int64_t nidx(int i, int j, int k, int ny, int nz) { return ((int64_t)i * ny + j) * nz + k; }

__device__ __forceinline__ void grid_coord(const efsi_mpm_state& S, int p, float X[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) X[a] = __fdiv_rn(__fsub_rn(S.x[3 * p + a], S.bmin[a]), S.dx[a]);
}

__device__ __forceinline__ bool stencil_oob(const efsi_mpm_state& S, const float X[3]) {
  // neo_hookean_mpm.py:663-671 _particle_grid_stencil_out_of_bounds
  return X[0] < 0.5f || X[0] >= (float)S.nx - 1.5f || X[1] < 0.5f || X[1] >= (float)S.ny - 1.5f || X[2] < 0.5f ||
         X[2] >= (float)S.nz - 1.5f;
}

__device__ __forceinline__ void quad_w(float fx, float w[3]) {
  // neo_hookean_mpm.py:688-693 quadratic B-spline weights
  float a = 1.5f - fx, b = fx - 1.0f, c = fx - 0.5f;
  w[0] = 0.5f * a * a;
  w[1] = 0.75f - b * b;
  w[2] = 0.5f * c * c;
}

// ---------------------------------------------------------------------------
// Deformation clamp (neo_hookean_mpm.py:720-748).  A cheap sufficient test
// (sigma_max <= ||F||_F, sigma_min >= 2|det F| / ||F||_F^2) proves most
// particles unclamped; the rest get a one-sided Jacobi SVD in f64 (Hestenes;
// Demmel & Veselic 1992) with the reference's sign convention (U, V proper
// rotations, the smallest singular value carries the sign of det F).
// ---------------------------------------------------------------------------
__device__ double det3d(const double a[3][3]) {
  return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
         a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

__device__ void svd3(const double Ain[3][3], double U[3][3], double s[3], double V[3][3]) {
  double A[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i][j] = Ain[i][j];
      V[i][j] = (i == j) ? 1.0 : 0.0;
    }
  for (int sweep = 0; sweep < 30; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        double al = 0, be = 0, ga = 0;
        for (int i = 0; i < 3; ++i) {
          al += A[i][p] * A[i][p];
          be += A[i][q] * A[i][q];
          ga += A[i][p] * A[i][q];
        }
        if (ga == 0.0) continue;
        double scale = sqrt(al * be);
        if (scale > 0.0) off = fmax(off, fabs(ga) / scale);
        if (fabs(ga) <= 1.0e-15 * scale) continue;
        double zeta = (be - al) / (2.0 * ga);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        double c = 1.0 / sqrt(1.0 + t * t);
        double sn = c * t;
        for (int i = 0; i < 3; ++i) {
          double ap = A[i][p], aq = A[i][q];
          A[i][p] = c * ap - sn * aq;
          A[i][q] = sn * ap + c * aq;
          double vp = V[i][p], vq = V[i][q];
          V[i][p] = c * vp - sn * vq;
          V[i][q] = sn * vp + c * vq;
        }
      }
    if (off <= 1.0e-15) break;
  }
  double sv[3];
  for (int j = 0; j < 3; ++j) sv[j] = sqrt(A[0][j] * A[0][j] + A[1][j] * A[1][j] + A[2][j] * A[2][j]);
  int o[3] = {0, 1, 2};
  // sort descending (3-element network)
  if (sv[o[0]] < sv[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  if (sv[o[1]] < sv[o[2]]) { int t = o[1]; o[1] = o[2]; o[2] = t; }
  if (sv[o[0]] < sv[o[1]]) { int t = o[0]; o[0] = o[1]; o[1] = t; }
  double A2[3][3], V2[3][3];
  for (int j = 0; j < 3; ++j) {
    s[j] = sv[o[j]];
    for (int i = 0; i < 3; ++i) {
      A2[i][j] = A[i][o[j]];
      V2[i][j] = V[i][o[j]];
    }
  }
  if (det3d(V2) < 0.0)
    for (int i = 0; i < 3; ++i) {
      V2[i][2] = -V2[i][2];
      A2[i][2] = -A2[i][2];
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) V[i][j] = V2[i][j];
  for (int j = 0; j < 2; ++j)
    for (int i = 0; i < 3; ++i) U[i][j] = s[j] > 1.0e-300 ? A2[i][j] / s[j] : (i == j ? 1.0 : 0.0);
  if (s[2] > 1.0e-12 * fmax(s[0], 1.0e-300)) {
    for (int i = 0; i < 3; ++i) U[i][2] = A2[i][2] / s[2];
  } else {
    double sg = det3d(Ain) < 0.0 ? -1.0 : 1.0;
    U[0][2] = sg * (U[1][0] * U[2][1] - U[2][0] * U[1][1]);
    U[1][2] = sg * (U[2][0] * U[0][1] - U[0][0] * U[2][1]);
    U[2][2] = sg * (U[0][0] * U[1][1] - U[1][0] * U[0][1]);
  }
}

__device__ int clamp_deformation(const float F[9], float Fp[9]) {
  double A[3][3];
  double frob2 = 0.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      A[i][j] = (double)F[3 * i + j];
      frob2 += A[i][j] * A[i][j];
    }
  double det = det3d(A);
  if (det > 0.0 && frob2 <= 99.99 * 99.99 && 2.0 * det >= 0.0101 * frob2) {
    for (int a = 0; a < 9; ++a) Fp[a] = F[a];
    return 0;
  }
  double U[3][3], V[3][3], s[3];
  svd3(A, U, s, V);
  double sign3 = 1.0;
  if (det < 0.0) {
    sign3 = -1.0;
    for (int i = 0; i < 3; ++i) U[i][2] = -U[i][2];
  }
  float raw[3] = {(float)s[0], (float)s[1], (float)(sign3 * s[2])};
  int clamped = 0;
  double cv[3];
  for (int a = 0; a < 3; ++a) {
    float cs = fminf(fmaxf(fabsf(raw[a]), 1.0e-2f), 1.0e2f);
    if (fabsf(cs - raw[a]) > 1.0e-6f) clamped = 1;
    cv[a] = (double)cs;
  }
  float rawJ = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
  if (rawJ <= 0.0f) clamped = 1;
  if (!clamped) {
    for (int a = 0; a < 9; ++a) Fp[a] = F[a];
    return 0;
  }
  double Pm[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      Pm[i][j] = U[i][0] * cv[0] * V[j][0] + U[i][1] * cv[1] * V[j][1] + U[i][2] * cv[2] * V[j][2];
  if (det3d(Pm) <= 0.0)
    for (int i = 0; i < 3; ++i) Pm[i][2] = -Pm[i][2];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) Fp[3 * i + j] = (float)Pm[i][j];
  return 1;
}

// ---------------------------------------------------------------------------
// Binning
// ---------------------------------------------------------------------------
__global__ void k_bin_keys(efsi_mpm_state S, int tx, int ty, int tz, int ntiles, int32_t* key, int32_t* count,
                           uint8_t* reached) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= S.particle_count) return;
  float X[3];
  grid_coord(S, p, X);
  int kk = ntiles;  // out-of-stencil bucket
  if (!stencil_oob(S, X)) {
    int b0 = (int)floorf(X[0] - 0.5f), b1 = (int)floorf(X[1] - 0.5f), b2 = (int)floorf(X[2] - 0.5f);
    const int t0 = b0 / kTile, t1 = b1 / kTile, t2 = b2 / kTile;
    kk = (t0 * ty + t1) * tz + t2;
    // the stencil's nodes (base .. base + 2) lie in this tile and the next one per axis
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c)
          if (t0 + a < tx && t1 + b < ty && t2 + c < tz) reached[((t0 + a) * ty + (t1 + b)) * tz + (t2 + c)] = 1;
  }
  key[p] = kk;
  // warp-aggregated histogram increment
  unsigned peers = __match_any_sync(__activemask(), kk);
  int leader = __ffs(peers) - 1;
  if ((threadIdx.x & 31) == leader) atomicAdd(count + kk, __popc(peers));
}

// Exclusive scan of count[0..n) into offset[0..n] by one 1024-thread block.
// Each thread owns a run of `per` (a multiple of 4) consecutive counts, read
// and written as int4 (the runs start on 16-byte boundaries; count, offset
// and cursor are cudaMalloc'd), so the block issues all its loads at once.
__global__ void k_scan(const int32_t* count, int n, int32_t* offset, int32_t* cursor) {
  __shared__ int32_t part[1024];
  const int t = threadIdx.x;
  const int per = (((n + 1023) / 1024) + 3) & ~3;
  const int lo = min(n, t * per), hi = min(n, lo + per);
  int32_t s = 0;
  int q = lo;
  for (; q + 4 <= hi; q += 4) {
    const int4 c4 = *reinterpret_cast<const int4*>(count + q);
    s += c4.x + c4.y + c4.z + c4.w;
  }
  for (; q < hi; ++q) s += count[q];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int32_t v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int32_t run = part[t] - s;
  q = lo;
  for (; q + 4 <= hi; q += 4) {
    const int4 c4 = *reinterpret_cast<const int4*>(count + q);
    int4 o4;
    o4.x = run;
    o4.y = run + c4.x;
    o4.z = o4.y + c4.y;
    o4.w = o4.z + c4.z;
    run = o4.w + c4.w;
    *reinterpret_cast<int4*>(offset + q) = o4;
    *reinterpret_cast<int4*>(cursor + q) = make_int4(0, 0, 0, 0);
  }
  for (; q < hi; ++q) {
    offset[q] = run;
    cursor[q] = 0;
    run += count[q];
  }
  if (t == 1023) offset[n] = part[1023];
}

__global__ void k_bin_scatter(int P, const int32_t* key, const int32_t* offset, int32_t* cursor, int32_t* sorted) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  int kk = key[p];
  unsigned peers = __match_any_sync(__activemask(), kk);
  int leader = __ffs(peers) - 1;
  int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == leader) base = atomicAdd(cursor + kk, __popc(peers));
  base = __shfl_sync(peers, base, leader);
  int rank = __popc(peers & ((1u << lane) - 1u));
  sorted[offset[kk] + base + rank] = p;
}

__device__ __forceinline__ void block_add(double* acc, int slot, double v) {
  // block-sum then one atomic (called by every thread of the block)
  double a[1] = {v};
  block_sum<1>(a);
  if (flat_tid() == 0 && a[0] != 0.0) atomicAdd(acc + slot, a[0]);
}

__device__ __forceinline__ void block_max(double* acc, int slot, double v) {
  __shared__ double sm[32];
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  const unsigned tid = flat_tid();
  if ((tid & 31u) == 0) sm[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double b = 0.0;
    for (unsigned w = 0; w < (flat_nthreads() + 31u) / 32u; ++w) b = fmax(b, sm[w]);
    if (b > 0.0) atomicMax(reinterpret_cast<unsigned long long*>(acc + slot), (unsigned long long)__double_as_longlong(b));
  }
  __syncthreads();
}

// Lists of the occupied tiles (+ the out-of-stencil bucket when it holds
// particles) and of the reached tiles.
// The two reached-tile lists alternate between steps by a device-side parity
// (counts[3]), so a captured step replays with the same arguments:
// counts[0] occupied tiles, [1] this step's reached tiles, [2] the previous
// step's, [3] which of reached0 / reached1 is this step's list.
__device__ __forceinline__ int32_t* reached_now(int32_t* r0, int32_t* r1, const int32_t* counts) {
  return counts[3] ? r1 : r0;
}
__device__ __forceinline__ int32_t* reached_before(int32_t* r0, int32_t* r1, const int32_t* counts) {
  return counts[3] ? r0 : r1;
}

// Start of a step: the previous step's count moves to counts[2], the parity
// flips, the new counts start at zero.
__global__ void k_reached_flip(int32_t* counts) {
  if (threadIdx.x == 0) {
    counts[2] = counts[1];
    counts[3] ^= 1;
    counts[0] = 0;
    counts[1] = 0;
  }
}

__global__ void k_tile_lists(int ntiles, const int32_t* __restrict__ count, const uint8_t* __restrict__ reached_flag,
                             int32_t* active, int32_t* reached0, int32_t* reached1, int32_t* counts) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t > ntiles) return;
  int32_t* reached = reached_now(reached0, reached1, counts);
  if (count[t] > 0) active[atomicAdd(counts, 1)] = t;
  if (t < ntiles && reached_flag[t]) reached[atomicAdd(counts + 1, 1)] = t;
}

__device__ __forceinline__ bool tile_node(const efsi_mpm_state& S, int tile, int q, int ty, int tz, int64_t& g) {
  const int t2 = tile % tz, t1 = (tile / tz) % ty, t0 = tile / (tz * ty);
  const int g0 = t0 * kTile + q / (kTile * kTile), g1 = t1 * kTile + (q / kTile) % kTile, g2 = t2 * kTile + q % kTile;
  if (g0 >= S.nx || g1 >= S.ny || g2 >= S.nz) return false;
  g = nidx(g0, g1, g2, S.ny, S.nz);
  return true;
}

// Zeroes mass, momentum and force of the nodes of the tiles reached in this
// step and in the previous one (one warp-pair per tile, 64 nodes).
__global__ void __launch_bounds__(256) k_clear_reached(efsi_mpm_state S, int ty, int tz, int32_t* reached0,
                                                       int32_t* reached1, const int32_t* counts) {
  const int n_now = counts[1], n_before = counts[2];
  const int32_t* now = reached_now(reached0, reached1, counts);
  const int32_t* before = reached_before(reached0, reached1, counts);
  const int per_block = 256 / kTileCells;
  for (int w = blockIdx.x * per_block + threadIdx.x / kTileCells; w < n_now + n_before; w += gridDim.x * per_block) {
    const int tile = w < n_now ? now[w] : before[w - n_now];
    int64_t g;
    if (!tile_node(S, tile, threadIdx.x % kTileCells, ty, tz, g)) continue;
    S.grid_mass[g] = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      S.grid_velocity[3 * g + a] = 0.0f;
      S.grid_force[3 * g + a] = 0.0f;
    }
  }
}

// ---------------------------------------------------------------------------
// P2G (neo_hookean_mpm.py:712-801): one CTA per tile (+ one for the
// out-of-stencil bucket, which only clamps F and reports).
//
// The tile's particles are taken in chunks of kP2gChunk.  Each thread first
// forms its particle's transfer terms (weights, fractional offsets, mass,
// momentum, APIC/stress affine matrix, external force) and the particle is
// placed, by a counting sort in shared memory, in the run of its base cell
// (one of the tile's 4^3 cells).  Then the work is split by (base cell,
// stencil offset): the thread of item (c, o) sums the contributions of all
// particles of cell c to the node c + o in registers -- the threads of one
// cell read the same particle record together (shared-memory broadcast) -- and
// adds the sums to the 6^3 node block with one shared atomic per value.  The
// block is flushed to the grid with one global atomic per non-zero value.
// ---------------------------------------------------------------------------
constexpr int kP2gThreads = 256;
constexpr int kP2gChunk = 256;  // particles per chunk (one per thread)

struct P2gRecords {
  float w[9][kP2gChunk];   // w[3 a + o]: quadratic weight of offset o on axis a
  float fx[3][kP2gChunk];  // fractional offset from the base node, per axis
  float m[kP2gChunk];
  float mom[3][kP2gChunk];
  float aff[9][kP2gChunk];
  float fe[3][kP2gChunk];
};

__global__ void __launch_bounds__(kP2gThreads) k_p2g(efsi_mpm_state S, int tx, int ty, int tz, int ntiles,
                                                     const int32_t* __restrict__ sorted,
                                                     const int32_t* __restrict__ offset,
                                                     const int32_t* __restrict__ active,
                                                     const int32_t* __restrict__ counts, float dt, float mu,
                                                     float lam, double* acc) {
  __shared__ float sacc[7][kHaloN];
  __shared__ P2gRecords rec;
  __shared__ int cell_count[kTileCells];
  __shared__ int cell_start[kTileCells + 1];
  double rm = 0, rv = 0, rp0 = 0, rp1 = 0, rp2 = 0, rf0 = 0, rf1 = 0, rf2 = 0, rmom2 = 0, rmaxj = 0, roob = 0,
         rclamp = 0;
  const int n_active = counts[0];
  for (int a_idx = blockIdx.x; a_idx < n_active; a_idx += gridDim.x) {
  const int tile = active[a_idx];
  const int beg = offset[tile], end = offset[tile + 1];
  const bool in_stencil_bucket = tile < ntiles;
  int t0 = 0, t1 = 0, t2 = 0;
  if (in_stencil_bucket) {
    t2 = tile % tz;
    t1 = (tile / tz) % ty;
    t0 = tile / (tz * ty);
  }
  const int nb0 = t0 * kTile, nb1 = t1 * kTile, nb2 = t2 * kTile;
  for (int q = threadIdx.x; q < 7 * kHaloN; q += blockDim.x) (&sacc[0][0])[q] = 0.0f;
  const float inv4[3] = {(float)(4.0 / ((double)S.dx[0] * S.dx[0])), (float)(4.0 / ((double)S.dx[1] * S.dx[1])),
                         (float)(4.0 / ((double)S.dx[2] * S.dx[2]))};
  const float dxs[3] = {S.dx[0], S.dx[1], S.dx[2]};
  for (int c0 = beg; c0 < end; c0 += kP2gChunk) {
    for (int q = threadIdx.x; q < kTileCells; q += blockDim.x) cell_count[q] = 0;
    __syncthreads();
    const int q = c0 + threadIdx.x;
    const bool have = q < end;
    int lc = -1, rank = 0;
    float w[3][3], fx[3], mass = 0.0f, mom[3] = {0, 0, 0}, fe[3] = {0, 0, 0}, aff[9];
    if (have) {
      const int p = sorted[q];
      float X[3];
      grid_coord(S, p, X);
      int base[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        base[a] = (int)floorf(X[a] - 0.5f);
        fx[a] = X[a] - (float)base[a];
        quad_w(fx[a], w[a]);
      }
      float Fr[9], Fp[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) Fr[a] = S.F[9 * p + a];
      if (clamp_deformation(Fr, Fp)) {
        rclamp += 1.0;
#pragma unroll
        for (int a = 0; a < 9; ++a) S.F[9 * p + a] = Fp[a];
      }
      // J and log J in f64; F^-T = cofactor / J in f32.
      double J = (double)Fp[0] * ((double)Fp[4] * Fp[8] - (double)Fp[5] * Fp[7]) -
                 (double)Fp[1] * ((double)Fp[3] * Fp[8] - (double)Fp[5] * Fp[6]) +
                 (double)Fp[2] * ((double)Fp[3] * Fp[7] - (double)Fp[4] * Fp[6]);
      const float Jr = (float)J;
      float cof[9] = {Fp[4] * Fp[8] - Fp[5] * Fp[7], Fp[5] * Fp[6] - Fp[3] * Fp[8], Fp[3] * Fp[7] - Fp[4] * Fp[6],
                      Fp[2] * Fp[7] - Fp[1] * Fp[8], Fp[0] * Fp[8] - Fp[2] * Fp[6], Fp[1] * Fp[6] - Fp[0] * Fp[7],
                      Fp[1] * Fp[5] - Fp[2] * Fp[4], Fp[2] * Fp[3] - Fp[0] * Fp[5], Fp[0] * Fp[4] - Fp[1] * Fp[3]};
      const float lnJ = (float)log(J);
      float Pm[9];
#pragma unroll
      for (int a = 0; a < 9; ++a) {
        float finvT = cof[a] / Jr;
        Pm[a] = mu * (Fp[a] - finvT) + lam * lnJ * finvT;
      }
      mass = S.mass[p];
      const float vol = S.volume[p];
      const float sv = -dt * vol;
#pragma unroll
      for (int ii = 0; ii < 3; ++ii)
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
          float pf = Pm[3 * ii] * Fp[3 * jj] + Pm[3 * ii + 1] * Fp[3 * jj + 1] + Pm[3 * ii + 2] * Fp[3 * jj + 2];
          aff[3 * ii + jj] = sv * (pf * inv4[jj]) + mass * S.C[9 * p + 3 * ii + jj];
        }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mom[a] = mass * S.v[3 * p + a];
        fe[a] = S.fext[3 * p + a];
      }
      if (S.fixed[p] != 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) mom[a] = fe[a] = 0.0f;
#pragma unroll
        for (int a = 0; a < 9; ++a) aff[a] = 0.0f;
      }
      rm += mass;
      rv += vol;
      rp0 += mom[0];
      rp1 += mom[1];
      rp2 += mom[2];
      rf0 += fe[0];
      rf1 += fe[1];
      rf2 += fe[2];
      rmom2 += (double)(mom[0] * mom[0] + mom[1] * mom[1] + mom[2] * mom[2]);
      rmaxj = fmax(rmaxj, fabs((double)Jr));
      if (!in_stencil_bucket) {
        roob += 1.0;
      } else {
        // base - tile origin is in [0, kTile) on every axis (the bin key)
        lc = ((base[0] - nb0) * kTile + (base[1] - nb1)) * kTile + (base[2] - nb2);
        rank = atomicAdd(&cell_count[lc], 1);
      }
    }
    if (!in_stencil_bucket) continue;  // uniform per block
    __syncthreads();
    if (threadIdx.x < 32) {
      // exclusive scan of the 64 cell counts by one warp, two per lane
      const int l = threadIdx.x;
      const int a = cell_count[2 * l], b = cell_count[2 * l + 1];
      int v = a + b;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (l >= o) v += u;
      }
      cell_start[2 * l] = v - a - b;
      cell_start[2 * l + 1] = v - b;
      if (l == 31) cell_start[kTileCells] = v;
    }
    __syncthreads();
    if (lc >= 0) {
      const int slot = cell_start[lc] + rank;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 0; o < 3; ++o) rec.w[3 * a + o][slot] = w[a][o];
        rec.fx[a][slot] = fx[a];
        rec.mom[a][slot] = mom[a];
        rec.fe[a][slot] = fe[a];
      }
      rec.m[slot] = mass;
#pragma unroll
      for (int a = 0; a < 9; ++a) rec.aff[a][slot] = aff[a];
    }
    __syncthreads();
    for (int item = threadIdx.x; item < kTileCells * 27; item += blockDim.x) {
      const int c = item / 27, o = item - 27 * c;
      const int pb = cell_start[c], pe = cell_start[c + 1];
      if (pb == pe) continue;
      const int o0 = o / 9, o1 = (o / 3) % 3, o2 = o % 3;
      const float fo[3] = {(float)o0, (float)o1, (float)o2};
      float sm = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f, s4 = 0.0f, s5 = 0.0f, s6 = 0.0f;
      for (int r = pb; r < pe; ++r) {
        const float wt = rec.w[o0][r] * rec.w[3 + o1][r] * rec.w[6 + o2][r];
        const float d0 = (fo[0] - rec.fx[0][r]) * dxs[0], d1 = (fo[1] - rec.fx[1][r]) * dxs[1],
                    d2 = (fo[2] - rec.fx[2][r]) * dxs[2];
        sm += wt * rec.m[r];
        s1 += wt * (rec.mom[0][r] + (rec.aff[0][r] * d0 + rec.aff[1][r] * d1 + rec.aff[2][r] * d2));
        s2 += wt * (rec.mom[1][r] + (rec.aff[3][r] * d0 + rec.aff[4][r] * d1 + rec.aff[5][r] * d2));
        s3 += wt * (rec.mom[2][r] + (rec.aff[6][r] * d0 + rec.aff[7][r] * d1 + rec.aff[8][r] * d2));
        s4 += wt * rec.fe[0][r];
        s5 += wt * rec.fe[1][r];
        s6 += wt * rec.fe[2][r];
      }
      const int b0 = c / (kTile * kTile), b1 = (c / kTile) % kTile, b2 = c % kTile;
      const int ln = ((b0 + o0) * kHalo + (b1 + o1)) * kHalo + (b2 + o2);
      atomicAdd(&sacc[0][ln], sm);
      atomicAdd(&sacc[1][ln], s1);
      atomicAdd(&sacc[2][ln], s2);
      atomicAdd(&sacc[3][ln], s3);
      atomicAdd(&sacc[4][ln], s4);
      atomicAdd(&sacc[5][ln], s5);
      atomicAdd(&sacc[6][ln], s6);
    }
    __syncthreads();  // records and counts are reused by the next chunk
  }
  __syncthreads();
  if (in_stencil_bucket) {
    for (int ln = threadIdx.x; ln < kHaloN; ln += blockDim.x) {
      const int l2 = ln % kHalo, l1 = (ln / kHalo) % kHalo, l0 = ln / (kHalo * kHalo);
      const int g0 = nb0 + l0, g1 = nb1 + l1, g2 = nb2 + l2;
      if (g0 >= S.nx || g1 >= S.ny || g2 >= S.nz) continue;
      const int64_t g = nidx(g0, g1, g2, S.ny, S.nz);
      float mv = sacc[0][ln];
      if (mv != 0.0f) atomicAdd(S.grid_mass + g, mv);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        float vv = sacc[1 + a][ln];
        if (vv != 0.0f) atomicAdd(S.grid_velocity + 3 * g + a, vv);
        float ff = sacc[4 + a][ln];
        if (ff != 0.0f) atomicAdd(S.grid_force + 3 * g + a, ff);
      }
    }
  }
  __syncthreads();  // the node block is zeroed again for the next tile
  }
  if (acc != nullptr) {
    block_add(acc, R_MASS, rm);
    block_add(acc, R_VOL, rv);
    block_add(acc, R_PMOM + 0, rp0);
    block_add(acc, R_PMOM + 1, rp1);
    block_add(acc, R_PMOM + 2, rp2);
    block_add(acc, R_FEXT + 0, rf0);
    block_add(acc, R_FEXT + 1, rf1);
    block_add(acc, R_FEXT + 2, rf2);
    block_add(acc, R_MOM2, rmom2);
    block_add(acc, R_OOB, roob);
    block_add(acc, R_CLAMP, rclamp);
    block_max(acc, R_MAXJ, rmaxj);
  }
}

// Grid update (neo_hookean_mpm.py:803-817).
// Only the nodes of the reached tiles can carry mass; the rest of the grid is
// zero (k_clear_reached).
__global__ void __launch_bounds__(256) k_grid_update(efsi_mpm_state S, int ty, int tz, int32_t* reached0,
                                                     int32_t* reached1, const int32_t* counts, float dt,
                                                     float damping, double* acc) {
  double t0 = 0, t1 = 0, t2 = 0, m0 = 0, m1 = 0, m2 = 0, act = 0, spd = 0;
  const int n_reached = counts[1];
  const int32_t* reached = reached_now(reached0, reached1, counts);
  const int per_block = 256 / kTileCells;
  for (int w = blockIdx.x * per_block + threadIdx.x / kTileCells; w < n_reached; w += gridDim.x * per_block) {
    int64_t g;
    if (!tile_node(S, reached[w], threadIdx.x % kTileCells, ty, tz, g)) continue;
    const float m = S.grid_mass[g];
    if (m > 1.0e-20f) {
      float v[3], tv[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        v[a] = S.grid_velocity[3 * g + a] / m;
        v[a] += dt * S.grid_force[3 * g + a] / m;
        tv[a] = v[a];
        v[a] *= damping;
        S.grid_velocity[3 * g + a] = v[a];
      }
      t0 += m * tv[0];
      t1 += m * tv[1];
      t2 += m * tv[2];
      m0 += m * v[0];
      m1 += m * v[1];
      m2 += m * v[2];
      act += 1.0;
      spd = fmax(spd, (double)sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }
  }
  if (acc != nullptr) {
    block_add(acc, R_TMOM + 0, t0);
    block_add(acc, R_TMOM + 1, t1);
    block_add(acc, R_TMOM + 2, t2);
    block_add(acc, R_GMOM + 0, m0);
    block_add(acc, R_GMOM + 1, m1);
    block_add(acc, R_GMOM + 2, m2);
    block_add(acc, R_ACTIVE, act);
    block_max(acc, R_MAXSPEED, spd);
  }
}

// neo_hookean_mpm.py:674-685 Nanson update of area and normal.
__device__ void surface_geometry(const efsi_mpm_state& S, int p) {
  const float ra = S.rest_area[p];
  const float n0 = S.rest_normal[3 * p], n1 = S.rest_normal[3 * p + 1], n2 = S.rest_normal[3 * p + 2];
  if (!(ra > 0.0f && sqrtf(n0 * n0 + n1 * n1 + n2 * n2) > 1.0e-12f)) return;
  const float* F = S.F + 9 * p;
  float J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) + F[2] * (F[3] * F[7] - F[4] * F[6]);
  if (!(J > 1.0e-12f)) return;
  float cof[9] = {F[4] * F[8] - F[5] * F[7], F[5] * F[6] - F[3] * F[8], F[3] * F[7] - F[4] * F[6],
                  F[2] * F[7] - F[1] * F[8], F[0] * F[8] - F[2] * F[6], F[1] * F[6] - F[0] * F[7],
                  F[1] * F[5] - F[2] * F[4], F[2] * F[3] - F[0] * F[5], F[0] * F[4] - F[1] * F[3]};
  float av[3];
  for (int i = 0; i < 3; ++i) av[i] = cof[3 * i] * n0 + cof[3 * i + 1] * n1 + cof[3 * i + 2] * n2;
  float sc = sqrtf(av[0] * av[0] + av[1] * av[1] + av[2] * av[2]);
  if (sc > 1.0e-12f) {
    S.normal[3 * p] = av[0] / sc;
    S.normal[3 * p + 1] = av[1] / sc;
    S.normal[3 * p + 2] = av[2] / sc;
    S.area[p] = ra * sc;
  }
}

// G2P, F update, fixed particles, surface geometry and the region reports
// (neo_hookean_mpm.py:819-875), walking particles in tile order.
__global__ void __launch_bounds__(256) k_g2p(efsi_mpm_state S, const int32_t* __restrict__ sorted, float dt,
                                             int primary, int secondary, double* acc) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  double pd[3] = {0, 0, 0}, pv[3] = {0, 0, 0}, sd[3] = {0, 0, 0}, svv[3] = {0, 0, 0}, pc = 0, scn = 0;
  double cs[3] = {0, 0, 0}, rs[3] = {0, 0, 0}, cc = 0;
  if (q < S.particle_count) {
    const int p = sorted[q];
    float X[3];
    grid_coord(S, p, X);
    if (!stencil_oob(S, X)) {
      int base[3];
      float fx[3], w[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        base[a] = (int)floorf(X[a] - 0.5f);
        fx[a] = X[a] - (float)base[a];
        quad_w(fx[a], w[a]);
      }
      const float dx2[3] = {S.dx[0] * S.dx[0], S.dx[1] * S.dx[1], S.dx[2] * S.dx[2]};
      float nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int ox = 0; ox < 3; ++ox)
#pragma unroll
        for (int oy = 0; oy < 3; ++oy)
#pragma unroll
          for (int oz = 0; oz < 3; ++oz) {
            const float wt = w[0][ox] * w[1][oy] * w[2][oz];
            const float d[3] = {((float)ox - fx[0]) * S.dx[0], ((float)oy - fx[1]) * S.dx[1],
                                ((float)oz - fx[2]) * S.dx[2]};
            const int64_t g = nidx(base[0] + ox, base[1] + oy, base[2] + oz, S.ny, S.nz);
            const float gv[3] = {__ldg(S.grid_velocity + 3 * g), __ldg(S.grid_velocity + 3 * g + 1),
                                 __ldg(S.grid_velocity + 3 * g + 2)};
            const float qv[3] = {4.0f * d[0] / dx2[0], 4.0f * d[1] / dx2[1], 4.0f * d[2] / dx2[2]};
#pragma unroll
            for (int a = 0; a < 3; ++a) {
              nv[a] += wt * gv[a];
#pragma unroll
              for (int b = 0; b < 3; ++b) nC[3 * a + b] += wt * (gv[a] * qv[b]);
            }
          }
      if (S.fixed[p] == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          S.v[3 * p + a] = nv[a];
          S.x[3 * p + a] += dt * nv[a];
        }
        float Fo[9];
#pragma unroll
        for (int a = 0; a < 9; ++a) {
          S.C[9 * p + a] = nC[a];
          Fo[a] = S.F[9 * p + a];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            float s = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += (((i == k) ? 1.0f : 0.0f) + dt * nC[3 * i + k]) * Fo[3 * k + j];
            S.F[9 * p + 3 * i + j] = s;
          }
      }
    }
    if (S.fixed[p] != 0) {
#pragma unroll
      for (int a = 0; a < 3; ++a) S.v[3 * p + a] = 0.0f;
#pragma unroll
      for (int a = 0; a < 9; ++a) {
        S.C[9 * p + a] = 0.0f;
        S.F[9 * p + a] = (a % 4 == 0) ? 1.0f : 0.0f;
      }
    }
    surface_geometry(S, p);
    float Xn[3];
    grid_coord(S, p, Xn);
    if (!stencil_oob(S, Xn)) {
      const int r = S.region[p];
      if (r == primary) {
        for (int a = 0; a < 3; ++a) {
          pd[a] = S.x[3 * p + a] - S.rest_x[3 * p + a];
          pv[a] = S.v[3 * p + a];
        }
        pc = 1.0;
      } else if (r == secondary) {
        for (int a = 0; a < 3; ++a) {
          sd[a] = S.x[3 * p + a] - S.rest_x[3 * p + a];
          svv[a] = S.v[3 * p + a];
        }
        scn = 1.0;
      }
      for (int a = 0; a < 3; ++a) {
        cs[a] = S.x[3 * p + a];
        rs[a] = S.rest_x[3 * p + a];
      }
      cc = 1.0;
    }
  }
  if (acc != nullptr) {
    for (int a = 0; a < 3; ++a) {
      block_add(acc, R_PDISP + a, pd[a]);
      block_add(acc, R_PVEL + a, pv[a]);
      block_add(acc, R_SDISP + a, sd[a]);
      block_add(acc, R_SVEL + a, svv[a]);
      block_add(acc, R_CSUM + a, cs[a]);
      block_add(acc, R_RSUM + a, rs[a]);
    }
    block_add(acc, R_PCOUNT, pc);
    block_add(acc, R_SCOUNT, scn);
    block_add(acc, R_CCOUNT, cc);
  }
}

// Radial stretch diagnostics (neo_hookean_mpm.py:876-898).
__global__ void __launch_bounds__(256) k_radial(efsi_mpm_state S, double* acc) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  const double cnt = fmax(acc[R_CCOUNT], 1.0);
  double st = 0, stn = 0, err = 0;
  if (p < S.particle_count) {
    float X[3];
    grid_coord(S, p, X);
    if (!stencil_oob(S, X)) {
      double rr = 0, cr = 0;
      for (int a = 0; a < 3; ++a) {
        double d1 = S.rest_x[3 * p + a] - acc[R_RSUM + a] / cnt;
        double d2 = S.x[3 * p + a] - acc[R_CSUM + a] / cnt;
        rr += d1 * d1;
        cr += d2 * d2;
      }
      rr = sqrt(rr);
      if (rr > 1.0e-12) {
        double s = sqrt(cr) / rr;
        st = s;
        stn = 1.0;
        err = fabs(s - 1.0);
      }
    }
  }
  block_add(acc, R_STRETCH, st);
  block_add(acc, R_STRETCH_N, stn);
  block_max(acc, R_STRETCH_ERR, err);
}

// Packs the accumulators into the 34-value snapshot (neo_hookean_mpm.py:899-958).
__global__ void k_mpm_finalize(const double* acc, float dt, double* out) {
  if (threadIdx.x != 0) return;
  double expected[3], en = 0, tr = 0;
  for (int a = 0; a < 3; ++a) {
    expected[a] = acc[R_PMOM + a] + (double)dt * acc[R_FEXT + a];
    en += expected[a] * expected[a];
    tr += (acc[R_TMOM + a] - expected[a]) * (acc[R_TMOM + a] - expected[a]);
  }
  double denom = fmax(fmax(sqrt(en), sqrt(acc[R_MOM2])), 1.0e-20);
  out[0] = acc[R_MASS];
  out[1] = acc[R_VOL];
  for (int a = 0; a < 3; ++a) {
    out[2 + a] = acc[R_PMOM + a];
    out[5 + a] = acc[R_GMOM + a];
    out[8 + a] = acc[R_FEXT + a];
    out[16 + a] = acc[R_PDISP + a];
    out[19 + a] = acc[R_PVEL + a];
    out[22 + a] = acc[R_SDISP + a];
    out[25 + a] = acc[R_SVEL + a];
  }
  out[11] = sqrt(tr) / denom;
  out[12] = acc[R_MAXSPEED];
  out[13] = acc[R_MAXJ];
  out[14] = acc[R_STRETCH];
  out[15] = acc[R_STRETCH_ERR];
  out[28] = acc[R_ACTIVE];
  out[29] = acc[R_OOB];
  out[30] = acc[R_CLAMP];
  out[31] = acc[R_STRETCH_N];
  out[32] = acc[R_PCOUNT];
  out[33] = acc[R_SCOUNT];
}

}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_mpm_plan_create(int32_t capacity, int32_t nx, int32_t ny, int32_t nz, efsi_mpm_plan** out) {
  EFSI_ARG_CHECK(capacity > 0 && nx >= 4 && ny >= 4 && nz >= 4 && out != nullptr, "invalid MPM plan arguments");
  efsi_mpm_plan* P = new efsi_mpm_plan();
  P->capacity = capacity;
  P->nx = nx;
  P->ny = ny;
  P->nz = nz;
  P->tx = (nx + kTile - 1) / kTile;
  P->ty = (ny + kTile - 1) / kTile;
  P->tz = (nz + kTile - 1) / kTile;
  P->ntiles = P->tx * P->ty * P->tz;
  const size_t nb = (size_t)P->ntiles + 1;
  if (cudaMalloc(&P->key, capacity * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->sorted, capacity * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->count, nb * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->offset, (nb + 1) * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->cursor, nb * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->acc, R_COUNT * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&P->active, nb * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->reached_flag, nb) != cudaSuccess ||
      cudaMalloc(&P->reached[0], nb * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->reached[1], nb * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->counts, 4 * sizeof(int32_t)) != cudaSuccess ||
      cudaMemset(P->counts, 0, 4 * sizeof(int32_t)) != cudaSuccess) {
    efsi_mpm_plan_destroy(P);
    set_error("cudaMalloc failed for the MPM plan");
    return EFSI_ERR_CUDA;
  }
  *out = P;
  return EFSI_OK;
}

int efsi_mpm_plan_destroy(efsi_mpm_plan* P) {
  if (!P) return EFSI_OK;
  cudaFree(P->key);
  cudaFree(P->sorted);
  cudaFree(P->count);
  cudaFree(P->offset);
  cudaFree(P->cursor);
  cudaFree(P->acc);
  cudaFree(P->active);
  cudaFree(P->reached_flag);
  cudaFree(P->reached[0]);
  cudaFree(P->reached[1]);
  cudaFree(P->counts);
  delete P;
  return EFSI_OK;
}

int efsi_mpm_step(efsi_mpm_plan* P, const efsi_mpm_state* Sp, float dt, float mu, float lambda_,
                  float velocity_damping, int32_t primary_region, int32_t secondary_region, double* report_device,
                  void* stream) {
  EFSI_ARG_CHECK(P != nullptr && Sp != nullptr, "null MPM plan or state");
  const efsi_mpm_state& S = *Sp;
  EFSI_ARG_CHECK(S.nx == P->nx && S.ny == P->ny && S.nz == P->nz, "MPM state grid does not match the plan");
  EFSI_ARG_CHECK(S.particle_count > 0 && S.particle_count <= P->capacity, "particle_count out of range");
  cudaStream_t s = as_stream(stream);
  const int Pn = S.particle_count;
  double* acc = report_device != nullptr ? P->acc : nullptr;
  // algorithmic bytes of the substep: 216 per particle (read x, v, C, F, mass,
  // volume, f_ext, fixed; write x, v, C, F) and 68 per node of the reached
  // tiles (clear 28, update 40)
  const bool time_step = timing_enabled(KF_MPM_STEP);
  if (time_step) timing_begin(KF_MPM_STEP, s);
  // the previous step's reached list becomes "before"; this step's is rebuilt
  EFSI_COUNTED k_reached_flip<<<1, 32, 0, s>>>(P->counts);
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->count, 0, (P->ntiles + 1) * sizeof(int32_t), s));
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->reached_flag, 0, P->ntiles, s));
  if (acc) EFSI_CUDA_CHECK(cudaMemsetAsync(acc, 0, R_COUNT * sizeof(double), s));
  const unsigned pb = (Pn + 255) / 256;
  EFSI_COUNTED k_bin_keys<<<pb, 256, 0, s>>>(S, P->tx, P->ty, P->tz, P->ntiles, P->key, P->count, P->reached_flag);
  EFSI_COUNTED k_scan<<<1, 1024, 0, s>>>(P->count, P->ntiles + 1, P->offset, P->cursor);
  EFSI_COUNTED k_tile_lists<<<(P->ntiles + 256) / 256, 256, 0, s>>>(P->ntiles, P->count, P->reached_flag, P->active,
                                                                     P->reached[0], P->reached[1], P->counts);
  EFSI_COUNTED k_clear_reached<<<2 * 148, 256, 0, s>>>(S, P->ty, P->tz, P->reached[0], P->reached[1], P->counts);
  EFSI_COUNTED k_bin_scatter<<<pb, 256, 0, s>>>(Pn, P->key, P->offset, P->cursor, P->sorted);
  // P2G: 124 bytes per particle (read x, v, C, F, mass, volume, f_ext, fixed, sorted index)
  EFSI_TIMED(KF_P2G, 124.0 * Pn, s,
             EFSI_COUNTED k_p2g<<<4 * 148, kP2gThreads, 0, s>>>(S, P->tx, P->ty, P->tz, P->ntiles, P->sorted, P->offset,
                                                                P->active, P->counts, dt, mu, lambda_, acc));
  // grid update: 40 bytes per node of the reached tiles (read mass, momentum
  // and force, write velocity); the count is read back only while the
  // family is timed
  double reached_nodes = 0.0;
  if (timing_enabled(KF_GRID_UPDATE) || time_step) {
    int32_t h = 0;
    EFSI_CUDA_CHECK(cudaMemcpyAsync(&h, P->counts + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
    reached_nodes = (double)h * kTileCells;
  }
  EFSI_TIMED(KF_GRID_UPDATE, 40.0 * reached_nodes, s,
             EFSI_COUNTED k_grid_update<<<2 * 148, 256, 0, s>>>(S, P->ty, P->tz, P->reached[0], P->reached[1],
                                                                P->counts, dt, velocity_damping,
                                                                acc));
  // G2P: read x, F, fixed, region (56 bytes), write x, v, C, F (96 bytes)
  EFSI_TIMED(KF_G2P, 152.0 * Pn, s,
             EFSI_COUNTED k_g2p<<<pb, 256, 0, s>>>(S, P->sorted, dt, primary_region, secondary_region, acc));
  if (acc) {
    EFSI_COUNTED k_radial<<<pb, 256, 0, s>>>(S, acc);
    EFSI_COUNTED k_mpm_finalize<<<1, 32, 0, s>>>(acc, dt, report_device);
  }
  if (time_step) timing_end(KF_MPM_STEP, s, 216.0 * Pn + 68.0 * reached_nodes);
  EFSI_LAUNCH_CHECK();
  return EFSI_OK;
}

}  // extern "C"
