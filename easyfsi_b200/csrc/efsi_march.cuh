// Plane-marching stencil kernels of the graded-grid pressure solver: damped
// Jacobi sweeps of every level, the CG direction update + SpMV, and the
// residual restriction.
//
// A block of 32 (k) x 8 (j) threads owns a 32 x 8 column tile of a level and
// a chunk of planes [ib, ie) along i (the slowest-varying axis).  One elected
// thread streams every plane the chunk needs (ib-1 .. ie) into a ring of
// kStages shared-memory stages with TMA (cp.async.bulk.tensor, no multicast):
// the swept field as a (8 + 2) x (32 + 2 pad) tile with its one-cell halo,
// and the plane's right-hand side and stencil-mask tiles.  Each stage has an
// mbarrier that completes when its bytes have landed.  The block computes
// planes i and i+1 from the stages of planes i-1 .. i+2 while the copies of
// planes i+3 and i+4 are in flight, then releases the stages of i-1 and i at
// the iteration's block barrier and the elected thread refills them.  HBM is read once per
// value (halo rows come from L2); registers hold no prefetched data.
//
// The per-cell arithmetic is the same expression, in the same order, as the
// per-cell kernels (`stencil`, `row_residual`): open faces are selected from
// the stencil mask, closed faces contribute exact zeros.
//
// TMA rules honoured here: every copy starts at an x (k) coordinate that is a
// multiple of 16 bytes (the value tile starts 16 bytes left of the tile, the
// rhs / mask tiles at the tile edge, k0 a multiple of 32); rows outside the
// level read the zero fill value and are only used behind closed faces;
// destinations are 128-byte aligned.  The host only selects these kernels
// for levels whose row pitch is a multiple of 16 bytes for every field.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "efsi_fv_internal.cuh"

namespace efsi {

constexpr int kMK = 32;           // tile width along k (one warp)
constexpr int kTY = 8;            // thread rows per block
constexpr int kRows = 2;          // tile rows per thread row
constexpr int kMJ = kTY * kRows;  // tile height along j
constexpr int kStages = 6;
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s: a stage that never lands is reported, not waited on forever

// Launch configuration of the marching kernels of one level: `chunk` planes
// (even, so a plane pair of the restriction never straddles two blocks) per
// block, blocks = column tiles x ceil(nx / chunk).
struct MarchCfg {
  int chunk = 2;
  unsigned grid = 1;
};

inline MarchCfg march_cfg(int nx, int ny, int nz, int slots) {
  const int tiles = ((nz + kMK - 1) / kMK) * ((ny + kMJ - 1) / kMJ);
  int nsplit = slots / tiles;
  if (nsplit < 1) nsplit = 1;
  int chunk = (nx + nsplit - 1) / nsplit;
  if (chunk < 2) chunk = 2;
  chunk += chunk & 1;
  MarchCfg c;
  c.chunk = chunk;
  c.grid = (unsigned)(tiles * ((nx + chunk - 1) / chunk));
  return c;
}

// Thread (tx, ty) of a block owns the cells (j0 + ty + r * kTY, k0 + tx),
// r < kRows, of every plane of the block's chunk.
struct MarchGeom {
  int tx, ty;
  int j0, k0;             // tile origin
  int k, kc;              // this thread's k (may lie outside the level) and its clamp
  int ib, ie;             // planes of this block
  int j[kRows];           // the thread's rows
  bool active[kRows];     // (j, k) lies inside the level
  int off[kRows];         // in-plane offset of (j, k), clamped into the level
};

__device__ __forceinline__ bool march_geom(const LevelDev& L, int chunk, MarchGeom& g) {
  const int ntk = (L.nz + kMK - 1) / kMK, ntj = (L.ny + kMJ - 1) / kMJ;
  int b = (int)blockIdx.x;
  const int tk = b % ntk;
  b /= ntk;
  const int tj = b % ntj;
  const int sp = b / ntj;
  g.ib = sp * chunk;
  g.ie = min(L.nx, g.ib + chunk);
  g.tx = (int)threadIdx.x;
  g.ty = (int)threadIdx.y;
  g.k0 = tk * kMK;
  g.j0 = tj * kMJ;
  g.k = g.k0 + g.tx;
  g.kc = min(g.k, L.nz - 1);
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    g.j[r] = g.j0 + g.ty + r * kTY;
    g.active[r] = g.j[r] < L.ny && g.k < L.nz;
    g.off[r] = min(g.j[r], L.ny - 1) * L.nz + g.kc;
  }
  return g.ib < g.ie;
}

// Axis coefficients of one row that do not change along i.
struct RowCoef {
  double kym, kyp, kzm, kzp;
};

__device__ __forceinline__ RowCoef row_coef(const LevelDev& L, int j, int kc) {
  const int jc = min(j, L.ny - 1);
  RowCoef c;
  c.kym = __ldg(L.cym + jc);
  c.kyp = __ldg(L.cyp + jc);
  c.kzm = __ldg(L.czm + kc);
  c.kzp = __ldg(L.czp + kc);
  return c;
}

// Neighbour sum and denominator of row (i, j, k) (fluid.py:4080-4221): the
// mask selects the open faces in the order x-, x+, y-, y+, z-, z+; a closed
// face adds exact zeros.  kAux: the level may carry Dirichlet face weights
// (and an interface diagonal); without them the kernels skip those loads.
template <bool kAux>
__device__ __forceinline__ void stencil_sel(const LevelDev& L, const RowCoef& cc, double kxm, double kxp, int i,
                                            int j, int k, int64_t c, unsigned m, int outlet, double vxm, double vxp,
                                            double vym, double vyp, double vzm, double vzp, double& ns, double& den) {
  double kym = cc.kym, kyp = cc.kyp, kzm = cc.kzm, kzp = cc.kzp;
  if (kAux && L.fw != nullptr) {
    const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
    const double fc = (double)__ldg(L.fw + c);
    kxm *= fc;
    kxp *= (double)__ldg(L.fw + (i < L.nx - 1 ? c + sx : c));
    kym *= fc;
    kyp *= (double)__ldg(L.fw + (j < L.ny - 1 ? c + sy : c));
    kzm *= fc;
    kzp *= (double)__ldg(L.fw + (k < L.nz - 1 ? c + 1 : c));
  }
  const double axm = (m & M_XM) ? kxm : 0.0;
  const double axp = (m & M_XP) ? kxp : 0.0;
  const double aym = (m & M_YM) ? kym : 0.0;
  const double ayp = (m & M_YP) ? kyp : 0.0;
  const double azm = (m & M_ZM) ? kzm : 0.0;
  const double azp = (m & M_ZP) ? kzp : 0.0;
  ns = fma(axm, vxm, 0.0);
  ns = fma(axp, vxp, ns);
  ns = fma(aym, vym, ns);
  ns = fma(ayp, vyp, ns);
  ns = fma(azm, vzm, ns);
  ns = fma(azp, vzp, ns);
  den = 0.0 + axm;
  den += axp;
  den += aym;
  den += ayp;
  den += azm;
  den += azp;
  if (outlet && k == 0) den += L.oz;
}

// ---------------------------------------------------------------------------
// mbarrier / TMA primitives (inline PTX)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the phase with the given parity; false if it did not complete
// within kWaitCycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > kWaitCycles) return false;
  }
  return true;
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr int round128(int b) { return (b + 127) & ~127; }

// Shared-memory stage of the pipeline: NV value tiles of TV (with halo, the
// left pad is 16 bytes so the copy's x coordinate stays 16-byte aligned), an
// optional right-hand-side tile of TR and the mask tile.
template <typename TV, int NV, typename TR, bool kR>
struct StageLayout {
  static constexpr int kPad = 16 / (int)sizeof(TV);
  static constexpr int kW = kMK + 2 * kPad;  // value row width (elements)
  static constexpr int kVBytes = (kMJ + 2) * kW * (int)sizeof(TV);
  static constexpr int kRBytes = kR ? kMJ * kMK * (int)sizeof(TR) : 0;
  static constexpr int kMBytes = kMJ * kMK;
  static constexpr int kVStride = round128(kVBytes);
  static constexpr int kROff = NV * kVStride;
  static constexpr int kMOff = kROff + round128(kRBytes);
  static constexpr int kStage = round128(kMOff + kMBytes);
  static constexpr int kBarOff = kStages * kStage;
  static constexpr int kSmem = kBarOff + kStages * 8;
};

// The march, two planes per iteration.  Per plane i and owned row r,
// `Op::cell(i, j, k, c, t, slot, active, m, rhs, kxm, kxp, rc, val)` computes
// one cell (t: its index in the tile; slot = d * kRows + r for plane i + d of
// the iteration; an inactive row lies outside the level and must not store), reading the field through val(v, di, dj, dk) (value
// tile v at (i+di, j+dj, k+dk)); `Op::plane_end(g, i, np)` runs after the np
// planes i .. i+np-1 of an iteration, before its block barrier, and
// `Op::finish(g)` after the last plane.  `Op::prefetch(g, i, pbase, sx)`
// (and `prefetch_prologue(g)` for planes ib-1, ib) issue the op's own global
// loads of an iteration before its stage waits.  With Op::kPrepare, every
// stage is first passed to `Op::prepare(g, value_tile, mask_tile, plane,
// slot)` (all threads, in place; the mask tile is null for the halo planes;
// slot 0 / 1 for planes i+1 / i+2, or ib-1 / ib) once it has landed.  Returns false (in every thread) if a stage did not land in time;
// the kernel then reports it through `sc->fault`.
template <typename TV, int NV, typename TR, bool kR, class Op>
__device__ __forceinline__ bool march(const LevelDev& L, const MarchGeom& g, const CUtensorMap* const (&mv)[NV],
                                      const CUtensorMap* mr, const CUtensorMap* mm, Op& op) {
  extern __shared__ unsigned char dsmem[];  // launched with march_smem() bytes (128 of slack for the alignment)
  using Lay = StageLayout<TV, NV, TR, kR>;
  unsigned char* base = dsmem + ((128u - (smem_addr(dsmem) & 127u)) & 127u);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + Lay::kBarOff);
  const bool leader = g.tx == 0 && g.ty == 0;
  // Elected thread: copy plane p into stage s.  Halo planes (ib-1, ie) carry
  // only the value tiles.
  auto issue = [&](int p, int s) {
    unsigned char* st = base + s * Lay::kStage;
    const bool interior = p >= g.ib && p < g.ie;
    mbar_expect_tx(&bar[s], NV * Lay::kVBytes + (interior ? Lay::kRBytes + Lay::kMBytes : 0));
#pragma unroll
    for (int v = 0; v < NV; ++v) tma_load_3d(st + v * Lay::kVStride, mv[v], g.k0 - Lay::kPad, g.j0 - 1, p, &bar[s]);
    if (interior) {
      if (kR) tma_load_3d(st + Lay::kROff, mr, g.k0, g.j0, p, &bar[s]);
      tma_load_3d(st + Lay::kMOff, mm, g.k0, g.j0, p, &bar[s]);
    }
  };
  if (leader) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // plane p lives in stage (p - ib + 1) % kStages, phase ((p - ib + 1) / kStages) & 1
  int issued = min(g.ie, g.ib - 1 + kStages - 1);  // last plane in flight
  if (leader)
    for (int p = g.ib - 1; p <= issued; ++p) issue(p, p - g.ib + 1);
  auto vtile = [&](int s) { return reinterpret_cast<TV*>(base + s * Lay::kStage); };
  auto mtile = [&](int s) { return reinterpret_cast<const uint8_t*>(base + s * Lay::kStage + Lay::kMOff); };
  op.prefetch_prologue(g);  // the op's own loads for planes ib-1 and ib, ahead of the waits
  bool fail = !mbar_wait(&bar[0], 0u);
  if (!fail) fail = !mbar_wait(&bar[1], 0u);
  if (Op::kPrepare) {
    // planes ib-1 (a halo plane: no mask tile) and ib
    if (!fail) {
      op.prepare(g, vtile(0), nullptr, g.ib - 1, 0);
      op.prepare(g, vtile(1), mtile(1), g.ib, 1);
    }
    fence_proxy_async_smem();
    __syncthreads();
  }
  // Two planes per iteration: planes i-1 .. i+2 resident, the next two in
  // flight.  sb is the stage of plane i-1; plane p's phase parity is
  // ((p - ib + 1) / kStages) & 1.
  int sb = 0;
  auto stage_at = [&](int q) {  // stage of plane i - 1 + q
    const int st = sb + q;
    return st >= kStages ? st - kStages : st;
  };
  auto phase_of = [&](int p) { return (unsigned)(((p - g.ib + 1) / kStages) & 1); };
  const int64_t sx = (int64_t)L.ny * L.nz;
  const int col = g.tx + Lay::kPad, W = Lay::kW;
  RowCoef rc[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) rc[r] = row_coef(L, g.j[r], g.kc);
  int64_t pbase = (int64_t)g.ib * sx;
  for (int i = g.ib; i < g.ie; i += 2, pbase += 2 * sx) {
    const int np = min(2, g.ie - i);  // planes computed in this iteration
    // x-face coefficients of the iteration's planes, loaded ahead of the waits
    double kx[4];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
      const int ip = min(i + d, L.nx - 1);
      kx[2 * d] = __ldg(L.cxm + ip);
      kx[2 * d + 1] = __ldg(L.cxp + ip);
    }
    op.prefetch(g, i, pbase, sx);  // the op's own loads for this iteration, ahead of the waits
#pragma unroll
    for (int q = 1; q <= 2; ++q) {
      if (q > np) break;
      const int st = stage_at(q + 1);  // plane i + q
      if (!fail) fail = !mbar_wait(&bar[st], phase_of(i + q));
      if (Op::kPrepare && !fail) op.prepare(g, vtile(st), i + q < g.ie ? mtile(st) : nullptr, i + q, q - 1);
    }
    if (Op::kPrepare) {
      fence_proxy_async_smem();  // these generic writes precede the stages' next TMA refill
      __syncthreads();
    }
    if (!fail) {
      // all cells of the iteration in one branch-free block (inactive rows
      // compute on clamped data and only skip their stores)
      auto run = [&](auto planes) {
        constexpr int ND = decltype(planes)::value;
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          const int ip = i + d;
          const int sm = stage_at(d), s0 = stage_at(d + 1), sp = stage_at(d + 2);
          const TV* vt[3][NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            vt[0][v] = reinterpret_cast<const TV*>(base + sm * Lay::kStage + v * Lay::kVStride) + col;
            vt[1][v] = reinterpret_cast<const TV*>(base + s0 * Lay::kStage + v * Lay::kVStride) + col;
            vt[2][v] = reinterpret_cast<const TV*>(base + sp * Lay::kStage + v * Lay::kVStride) + col;
          }
          const TR* rt = reinterpret_cast<const TR*>(base + s0 * Lay::kStage + Lay::kROff);
          const uint8_t* mt = base + s0 * Lay::kStage + Lay::kMOff;
          const int64_t pb = pbase + d * sx;
#pragma unroll
          for (int r = 0; r < kRows; ++r) {
            const int t = (g.ty + r * kTY) * kMK + g.tx;
            const int row = (g.ty + r * kTY + 1) * W;
            op.cell(ip, g.j[r], g.k, pb + g.off[r], t, d * kRows + r, g.active[r], (unsigned)mt[t],
                    kR ? (double)rt[t] : 0.0, kx[2 * d], kx[2 * d + 1], rc[r],
                    [&](int v, int dp, int dj, int dk) -> double { return (double)vt[dp + 1][v][row + dj * W + dk]; });
          }
        }
      };
      if (np == 2)
        run(std::integral_constant<int, 2>{});
      else
        run(std::integral_constant<int, 1>{});
    }
    op.plane_end(g, i, np);
    if (__syncthreads_or(fail)) {
      // let the copies in flight land before the block exits
      if (leader)
        for (int p = i + np + 1; p <= issued; ++p)
          mbar_wait(&bar[(p - g.ib + 1) % kStages], ((p - g.ib + 1) / kStages) & 1u);
      __syncthreads();
      return false;
    }
    // planes i-1 and i are no longer needed: refill their stages
    if (leader) {
      fence_proxy_async_smem();
      if (i - 1 + kStages <= g.ie) issue(issued = i - 1 + kStages, stage_at(0));
      if (np == 2 && i + kStages <= g.ie) issue(issued = i + kStages, stage_at(1));
    }
    sb = stage_at(2);
  }
  op.finish(g);
  return true;
}

template <typename TV, int NV, typename TR, bool kR>
constexpr int march_smem() {
  return StageLayout<TV, NV, TR, kR>::kSmem + 128;
}

__device__ __forceinline__ void report_fault(CgScalars* sc) {
  if (flat_tid() == 0) atomicExch(&sc->fault, 1);
}

// ---------------------------------------------------------------------------
// Damped-Jacobi sweep (fluid.py:4224-4273), out of place, with the
// prolongation p += s * p_coarse of fluid cells fused in when kProlong
// (fluid.py:5391-5406) and, when `partials`, the fluid sum of out * V.
// ---------------------------------------------------------------------------
template <typename TP, bool kNegR, bool kProlong, bool kAux, bool kDots, bool kRd = false>
struct SweepOp {
  const LevelDev& L;
  TP* __restrict__ out;
  int outlet;
  double omega;
  ProlongSrc pr;
  bool want_sum;
  double zsum;
  // kDots (the V-cycle's last level-0 sweep inside the flexible PCG): the
  // sums behind <r, z'>_V and <delta, z'>_V with z' = z - mean_z, i.e.
  // sum r z V, sum r V, sum delta z V and sum delta V over fluid rows.
  const double* __restrict__ delta;
  double srz, sr, sdz, sd;
  double dl[2 * kRows];  // kDots: delta of the iteration's cells, prefetched
  // kRd: the rows' reciprocal denominators 1 / den (0 where den <= 0),
  // precomputed per plan, prefetched like delta
  const double* __restrict__ rden;
  double rdv[2 * kRows];

  // kProlong: every thread prolongs up to kPCells cells of each landed value
  // tile (the (kMJ + 2) x (kMK + 2) cells with halo, strided by the block);
  // their coarse values are loaded ahead of the stage waits.
  static constexpr int kCols = kMK + 2, kCells = (kMJ + 2) * kCols;
  static constexpr int kPCells = (kCells + kMK * kTY - 1) / (kMK * kTY);
  float pcv[2][kPCells];
  // per-thread constants of those cells: in-plane coarse offset, offset in
  // the value tile, and mask-tile index (-1: halo cell, prolonged always)
  int coff[kPCells], toff[kPCells], moff[kPCells];

  __device__ __forceinline__ void load_coarse(int plane, int slot) {
    const int64_t cplane = (int64_t)min(min(max(plane, 0), L.nx - 1) / 2, pr.cnx - 1) * pr.cny * pr.cnz;
#pragma unroll
    for (int q = 0; q < kPCells; ++q) pcv[slot][q] = __ldg(pr.pc + cplane + coff[q]);
  }
  __device__ __forceinline__ void prefetch_prologue(const MarchGeom& g) {
    if (kProlong) {
      using Lay = StageLayout<TP, 1, TP, true>;
#pragma unroll
      for (int q = 0; q < kPCells; ++q) {
        const int e = g.ty * kMK + g.tx + q * kMK * kTY;
        const int ec = min(e, kCells - 1);
        const int r = ec / kCols, cc = ec - r * kCols;
        const int cj = min(max(g.j0 - 1 + r, 0) / 2, pr.cny - 1), ck = min(max(g.k0 - 1 + cc, 0) / 2, pr.cnz - 1);
        coff[q] = cj * pr.cnz + ck;
        toff[q] = e < kCells ? r * Lay::kW + Lay::kPad - 1 + cc : -1;
        moff[q] = (r >= 1 && r <= kMJ && cc >= 1 && cc <= kMK) ? (r - 1) * kMK + cc - 1 : -1;
      }
      load_coarse(g.ib - 1, 0);
      load_coarse(g.ib, 1);
    }
  }
  __device__ __forceinline__ void prefetch(const MarchGeom& g, int i, int64_t pbase, int64_t sx) {
    if (kProlong) {
      load_coarse(i + 1, 0);
      load_coarse(i + 2, 1);
    }
    if (kDots) {
#pragma unroll
      for (int d = 0; d < 2; ++d)
#pragma unroll
        for (int r = 0; r < kRows; ++r)
          dl[d * kRows + r] = __ldg(delta + min(pbase + d * sx, (int64_t)(L.nx - 1) * sx) + g.off[r]);
    }
    if (kRd) {
#pragma unroll
      for (int d = 0; d < 2; ++d)
#pragma unroll
        for (int r = 0; r < kRows; ++r)
          rdv[d * kRows + r] = __ldg(rden + min(pbase + d * sx, (int64_t)(L.nx - 1) * sx) + g.off[r]);
    }
  }

  // The prolongation p + s * p_coarse (in the level's storage precision) is
  // applied to each landed value tile once: tile cells by their own mask,
  // halo cells (reached only through open faces, hence fluid)
  // unconditionally.  Coarse indices are clamped, so cells outside the level
  // take an in-level coarse value that is never used.
  static constexpr bool kPrepare = kProlong;
  __device__ __forceinline__ void prepare(const MarchGeom&, TP* tile, const uint8_t* mtile, int, int slot) const {
#pragma unroll
    for (int q = 0; q < kPCells; ++q) {
      if (toff[q] < 0) break;
      if (moff[q] >= 0 && mtile != nullptr && !(mtile[moff[q]] & M_FLUID)) continue;
      TP* v = tile + toff[q];
      const float corr = __fmul_rn(pr.scale, pcv[slot][q]);
      if (sizeof(TP) == 8)
        *v = (TP)__dadd_rn((double)*v, (double)corr);
      else
        *v = (TP)__fadd_rn((float)*v, corr);
    }
  }

  template <class V>
  __device__ __forceinline__ void cell(int i, int j, int k, int64_t c, int, int slot, bool active, unsigned m,
                                       double e, double kxm, double kxp, const RowCoef& rc, const V& val) {
    if (!active) return;
    TP res = (TP)0;
    if (!(m & M_SOLID)) {
      const double x0 = val(0, 0, 0, 0), xm = val(0, -1, 0, 0), xp = val(0, 1, 0, 0);
      const double ym = val(0, 0, -1, 0), yp = val(0, 0, 1, 0), zm = val(0, 0, 0, -1), zp = val(0, 0, 0, 1);
      double ns, den;
      stencil_sel<kAux>(L, rc, kxm, kxp, i, j, k, c, m, outlet, xm, xp, ym, yp, zm, zp, ns, den);
      if (kRd) {
        const double rd = rdv[slot];
        if (rd > 0.0) {
          const double rv = kNegR ? -e : e;
          const double jv = (ns - rv) * rd;
          res = (TP)(x0 + omega * (jv - x0));
        }
      } else {
        if (kAux) den += iface_at<TP>(L, c);
        if (den > 0.0) {
          const double rv = kNegR ? -e : e;
          const double jv = (ns - rv) / den;
          res = (TP)(x0 + omega * (jv - x0));
        }
      }
      if ((want_sum || kDots) && (m & M_FLUID)) {
        const double vol = vol64(L, i, j, k);
        zsum += (double)res * vol;
        if (kDots) {  // rhs e is r (level 0 of the PCG's V-cycle)
          const double dlc = dl[slot];
          srz += e * (double)res * vol;
          sr += e * vol;
          sdz += (double)res * dlc * vol;
          sd += dlc * vol;
        }
      }
    }
    out[c] = res;
  }
  __device__ __forceinline__ void plane_end(const MarchGeom&, int, int) {}
  __device__ __forceinline__ void finish(const MarchGeom&) {}
};

// Epilogue of a sweep that reduces: with kDots the z-mean and the flexible
// PCG's preconditioned dots of this iteration (what the dots kernel computes,
// fluid.py:4604-4611 / 4590-4601): rz_new = <r, z'>_V, beta_num = <delta,
// z'>_V and beta, from the five sums; otherwise (partials given) the z-mean.
template <bool kDots, class Op>
__device__ __forceinline__ void sweep_epilogue(const Op& op, double* partials, CgScalars* sc) {
  if (kDots) {
    double v[5] = {op.zsum, op.srz, op.sr, op.sdz, op.sd}, t[5];
    if (grid_sum<5>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        const double mz = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->mean_z = mz;
        sc->zproj = 1;
        const double rz_new = t[1] - mz * t[2];
        cg_beta_step(sc, rz_new, t[3] - mz * t[4], true);
        sc->rz = rz_new;
      }
    }
    return;
  }
  if (partials != nullptr) {
    double v[1] = {op.zsum}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_z = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->zproj = 1;
      }
    }
  }
}

// Three blocks per SM (the shared-memory ring allows three).
template <typename TP, bool kNegR, bool kProlong, bool kAux, bool kDots, bool kRd = false>
__global__ void __launch_bounds__(kMK* kTY, 3)
    km_sweep(LevelDev L, int chunk, const __grid_constant__ CUtensorMap map_p,
             const __grid_constant__ CUtensorMap map_r, const __grid_constant__ CUtensorMap map_m,
             TP* __restrict__ out, int outlet, double omega, ProlongSrc pr, double* partials, CgScalars* sc,
             const double* __restrict__ delta, const double* __restrict__ rden) {
  pdl_wait();
  using TR = typename std::conditional<kNegR, double, TP>::type;
  MarchGeom g;
  const bool any = march_geom(L, chunk, g);
  SweepOp<TP, kNegR, kProlong, kAux, kDots, kRd> op{L, out, outlet, omega, pr, partials != nullptr, 0.0,
                                                    delta, 0.0, 0.0, 0.0, 0.0, {}, rden};
  const CUtensorMap* const mv[1] = {&map_p};
  if (any && !march<TP, 1, TR, true>(L, g, mv, &map_r, &map_m, op)) report_fault(sc);
  sweep_epilogue<kDots>(op, partials, sc);
}

// ---------------------------------------------------------------------------
// Mixed-precision level-0 sweep of the fv_multigrid_mixed preconditioner: the
// iterate tiles are FP32 and the row arithmetic is FP32 (face coefficients
// rounded from the f64 tables); the right-hand side is the FP64 CG residual.
// The outer flexible CG, its inner products and scalars, and the z-mean /
// dot sums stay FP64.  No counterpart in the reference (its V-cycle is f64 on
// level 0); the outer CG still stops on its f64 true residual.  With out64
// the result is written as the f64 preconditioned residual z.
// ---------------------------------------------------------------------------
template <bool kAux>
__device__ __forceinline__ void stencil_sel32(const LevelDev& L, const RowCoef& cc, float kxm, float kxp, int i,
                                              int j, int k, int64_t c, unsigned m, int outlet, float vxm, float vxp,
                                              float vym, float vyp, float vzm, float vzp, float& ns, float& den) {
  float kym = (float)cc.kym, kyp = (float)cc.kyp, kzm = (float)cc.kzm, kzp = (float)cc.kzp;
  if (kAux && L.fw != nullptr) {
    const int64_t sx = (int64_t)L.ny * L.nz, sy = L.nz;
    const float fc = __ldg(L.fw + c);
    kxm *= fc;
    kxp *= __ldg(L.fw + (i < L.nx - 1 ? c + sx : c));
    kym *= fc;
    kyp *= __ldg(L.fw + (j < L.ny - 1 ? c + sy : c));
    kzm *= fc;
    kzp *= __ldg(L.fw + (k < L.nz - 1 ? c + 1 : c));
  }
  const float axm = (m & M_XM) ? kxm : 0.0f;
  const float axp = (m & M_XP) ? kxp : 0.0f;
  const float aym = (m & M_YM) ? kym : 0.0f;
  const float ayp = (m & M_YP) ? kyp : 0.0f;
  const float azm = (m & M_ZM) ? kzm : 0.0f;
  const float azp = (m & M_ZP) ? kzp : 0.0f;
  ns = axm * vxm;
  ns = fmaf(axp, vxp, ns);
  ns = fmaf(aym, vym, ns);
  ns = fmaf(ayp, vyp, ns);
  ns = fmaf(azm, vzm, ns);
  ns = fmaf(azp, vzp, ns);
  den = ((((axm + axp) + aym) + ayp) + azm) + azp;
  if (outlet && k == 0) den += (float)L.oz;
}

template <bool kProlong, bool kAux, bool kDots>
struct Sweep32Op : SweepOp<float, true, kProlong, kAux, kDots> {
  double* __restrict__ out64;  // when set, z is written here in f64 instead of the f32 output

  template <class V>
  __device__ __forceinline__ void cell(int i, int j, int k, int64_t c, int, int slot, bool active, unsigned m,
                                       double e, double kxm, double kxp, const RowCoef& rc, const V& val) {
    if (!active) return;
    const LevelDev& L = this->L;
    float res = 0.0f;
    if (!(m & M_SOLID)) {
      const float x0 = (float)val(0, 0, 0, 0);
      float ns, den;
      stencil_sel32<kAux>(L, rc, (float)kxm, (float)kxp, i, j, k, c, m, this->outlet, (float)val(0, -1, 0, 0),
                          (float)val(0, 1, 0, 0), (float)val(0, 0, -1, 0), (float)val(0, 0, 1, 0),
                          (float)val(0, 0, 0, -1), (float)val(0, 0, 0, 1), ns, den);
      if (kAux) den += (float)iface_at<double>(L, c);
      if (den > 0.0f) {
        const float jv = (ns + (float)e) / den;  // the level-0 rhs is -r
        res = x0 + (float)this->omega * (jv - x0);
      }
      if ((this->want_sum || kDots) && (m & M_FLUID)) {
        const double vol = vol64(L, i, j, k), rd = (double)res;
        this->zsum += rd * vol;
        if (kDots) {
          const double dlc = this->dl[slot];
          this->srz += e * rd * vol;
          this->sr += e * vol;
          this->sdz += rd * dlc * vol;
          this->sd += dlc * vol;
        }
      }
    }
    if (out64 != nullptr)
      out64[c] = (double)res;
    else
      this->out[c] = res;
  }
};

template <bool kProlong, bool kAux, bool kDots>
__global__ void __launch_bounds__(kMK* kTY, 3)
    km_sweep32(LevelDev L, int chunk, const __grid_constant__ CUtensorMap map_p,
               const __grid_constant__ CUtensorMap map_r, const __grid_constant__ CUtensorMap map_m,
               float* __restrict__ out, double* __restrict__ out64, int outlet, double omega, ProlongSrc pr,
               double* partials, CgScalars* sc, const double* __restrict__ delta) {
  pdl_wait();
  MarchGeom g;
  const bool any = march_geom(L, chunk, g);
  Sweep32Op<kProlong, kAux, kDots> op{{L, out, outlet, omega, pr, partials != nullptr, 0.0, delta, 0.0, 0.0, 0.0, 0.0},
                                      out64};
  const CUtensorMap* const mv[1] = {&map_p};
  if (any && !march<float, 1, double, true>(L, g, mv, &map_r, &map_m, op)) report_fault(sc);
  sweep_epilogue<kDots>(op, partials, sc);
}

// First sweep from a zero iterate: out = omega * (0 - rhs) / den per row; no
// neighbour values are needed, so this is a plain streaming pass: a 32 x 8
// block per (k, j) tile and four planes, every thread's loads issued before
// its arithmetic.
constexpr int kSweep0Planes = 4;

inline dim3 sweep0_grid(int nx, int ny, int nz) {
  return dim3((unsigned)((nz + kMK - 1) / kMK), (unsigned)((ny + kTY - 1) / kTY),
              (unsigned)((nx + kSweep0Planes - 1) / kSweep0Planes));
}

// rden (level 0, may be null): the rows' precomputed reciprocal denominators.
template <typename TP, bool kNegR, bool kAux>
__global__ void __launch_bounds__(kMK* kTY)
    km_sweep0(LevelDev L, const void* rhs, TP* __restrict__ out, int outlet, double omega, double* partials,
              CgScalars* sc, const double* __restrict__ rden) {
  pdl_wait();
  const int k = (int)(blockIdx.x * kMK + threadIdx.x), j = (int)(blockIdx.y * kTY + threadIdx.y);
  const int i0 = (int)blockIdx.z * kSweep0Planes;
  double zsum = 0.0;
  if (j < L.ny && k < L.nz) {
    const int64_t sx = (int64_t)L.ny * L.nz;
    const int64_t c0 = (int64_t)i0 * sx + (int64_t)j * L.nz + k;
    const RowCoef rc = row_coef(L, j, k);
    const int n = min(kSweep0Planes, L.nx - i0);
    unsigned m[kSweep0Planes];
    double e[kSweep0Planes], rd[kSweep0Planes];
#pragma unroll
    for (int q = 0; q < kSweep0Planes; ++q) {
      if (q >= n) break;
      m[q] = __ldg(L.mask + c0 + q * sx);
      e[q] = kNegR ? __ldg(reinterpret_cast<const double*>(rhs) + c0 + q * sx)
                   : (double)__ldg(reinterpret_cast<const TP*>(rhs) + c0 + q * sx);
      rd[q] = rden != nullptr ? __ldg(rden + c0 + q * sx) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kSweep0Planes; ++q) {
      if (q >= n) break;
      const int i = i0 + q;
      const int64_t c = c0 + q * sx;
      TP res = (TP)0;
      if (!(m[q] & M_SOLID)) {
        if (rden != nullptr) {
          if (rd[q] > 0.0) {
            const double rv = kNegR ? -e[q] : e[q];
            res = (TP)(0.0 + omega * ((0.0 - rv) * rd[q] - 0.0));
          }
        } else {
          double ns, den;
          stencil_sel<kAux>(L, rc, __ldg(L.cxm + i), __ldg(L.cxp + i), i, j, k, c, m[q], outlet, 0.0, 0.0, 0.0,
                            0.0, 0.0, 0.0, ns, den);
          if (kAux) den += iface_at<TP>(L, c);
          if (den > 0.0) {
            const double rv = kNegR ? -e[q] : e[q];
            const double jv = (ns - rv) / den;
            res = (TP)(0.0 + omega * (jv - 0.0));
          }
        }
        if (partials != nullptr && (m[q] & M_FLUID)) zsum += (double)res * vol64(L, i, j, k);
      }
      out[c] = res;
    }
  }
  if (partials != nullptr) {
    double v[1] = {zsum}, t[1];
    if (grid_sum<1>(v, partials, &sc->ticket, t)) {
      if (flat_tid() == 0) {
        sc->mean_z = sc->free_vol > 0.0 ? 1.0 * t[0] / sc->free_vol : 0.0;
        sc->zproj = 1;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// CG direction and SpMV: d_new = z' (copy) or z' + beta d_old (fluid.py:
// 4604-4611, masked; z' the zero-mean projected z of fluid.py:4716-4722),
// Ad = A d_new (fluid.py:4312-4345), <d, Ad>_V and alpha (fluid.py:4567-4574).
// The direction of every stencil point is formed from the z and d_old tiles.
// ---------------------------------------------------------------------------
template <bool kCopy, bool kAux>
struct SpmvOp {
  static constexpr bool kPrepare = false;
  template <typename T>
  __device__ __forceinline__ void prepare(const MarchGeom&, T*, const uint8_t*, int, int) const {}
  __device__ __forceinline__ void prefetch_prologue(const MarchGeom&) {}
  __device__ __forceinline__ void prefetch(const MarchGeom&, int, int64_t, int64_t) {}
  const LevelDev& L;
  double* __restrict__ d_new;
  double* __restrict__ Ad;
  int outlet;
  double beta, mz;
  int zproj;
  double part;

  // direction at a neighbour behind an open face (a fluid cell)
  template <class V>
  __device__ __forceinline__ double dir(const V& val, int dp, int dj, int dk) const {
    double zz = val(0, dp, dj, dk);
    if (zproj) zz = zz - mz;
    return kCopy ? zz : zz + beta * val(1, dp, dj, dk);
  }

  template <class V>
  __device__ __forceinline__ void cell(int i, int j, int k, int64_t c, int, int, bool active, unsigned m, double,
                                       double kxm, double kxp, const RowCoef& rc, const V& val) {
    const bool solid = (m & M_SOLID) != 0;
    double x0 = dir(val, 0, 0, 0);
    if (!(m & M_FLUID) && zproj) x0 = kCopy ? 0.0 : 0.0 + beta * val(1, 0, 0, 0);
    if (solid) x0 = 0.0;
    double ns, den;
    stencil_sel<kAux>(L, rc, kxm, kxp, i, j, k, c, m, outlet, dir(val, -1, 0, 0), dir(val, 1, 0, 0),
                      dir(val, 0, -1, 0), dir(val, 0, 1, 0), dir(val, 0, 0, -1), dir(val, 0, 0, 1), ns, den);
    const double o = solid ? 0.0 : (den + (kAux ? iface_at<double>(L, c) : 0.0)) * x0 - ns;
    if (active) {
      d_new[c] = x0;
      Ad[c] = o;
      if (m & M_FLUID) part += x0 * o * vol64(L, i, j, k);
    }
  }
  __device__ __forceinline__ void plane_end(const MarchGeom&, int, int) {}
  __device__ __forceinline__ void finish(const MarchGeom&) {}
};

template <bool kCopy, bool kAux>
// Two blocks per SM with up to 128 registers a thread: measured faster for
// this kernel (two value tiles per stage) than three blocks at 85.
__global__ void __launch_bounds__(kMK* kTY, 2)
    km_spmv_dir(LevelDev L, int chunk, const __grid_constant__ CUtensorMap map_z,
                const __grid_constant__ CUtensorMap map_d, const __grid_constant__ CUtensorMap map_m,
                double* __restrict__ d_new, double* __restrict__ Ad, int outlet, double* partials, CgScalars* sc) {
  pdl_wait();
  MarchGeom g;
  const bool any = march_geom(L, chunk, g);
  SpmvOp<kCopy, kAux> op{L, d_new, Ad, outlet, kCopy ? 0.0 : sc->beta, sc->mean_z, sc->zproj, 0.0};
  bool ok = true;
  if (any) {
    if (kCopy) {
      const CUtensorMap* const mv[1] = {&map_z};
      ok = march<double, 1, double, false>(L, g, mv, nullptr, &map_m, op);
    } else {
      const CUtensorMap* const mv[2] = {&map_z, &map_d};
      ok = march<double, 2, double, false>(L, g, mv, nullptr, &map_m, op);
    }
  }
  if (!ok) report_fault(sc);
  double v[1] = {op.part}, t[1];
  if (grid_sum<1>(v, partials, &sc->ticket, t)) {
    if (flat_tid() == 0) {
      spmv_alpha(sc, t[0]);
    }
  }
}

// ---------------------------------------------------------------------------
// Residual restriction (fluid.py:5262-5388): the fine residual of every row
// is formed in the march and staged in shared memory (one buffer per plane of
// the iteration's pair); the threads owning a coarse cell then accumulate its
// 2 x 2 x 2 children in the reference's order (i-pair outer, then j, then k)
// with the f32 volume weights.
// ---------------------------------------------------------------------------
// The zero-guess damped-Jacobi sweep of one coarse row (km_sweep0<float,
// kNegR = false> / k_sweep<float, false, true>: the neighbours are zero, so
// ns = 0 and only the row's own denominator and rhs enter), evaluated by the
// restriction that produced the row's rhs value v.
__device__ __forceinline__ float coarse_zero_sweep(const LevelDev& C, int ci, int cj, int ck, int64_t cc, float v,
                                                   int outlet, double omega) {
  const unsigned m = __ldg(C.mask + cc);
  float res = 0.0f;
  if (!(m & M_SOLID)) {
    double ns, den;
    stencil_sel<true>(C, row_coef(C, cj, ck), __ldg(C.cxm + ci), __ldg(C.cxp + ci), ci, cj, ck, cc, m, outlet, 0.0,
                      0.0, 0.0, 0.0, 0.0, 0.0, ns, den);
    den += iface_at<float>(C, cc);
    if (den > 0.0) {
      const double jv = (ns - (double)v) / den;
      res = (float)(0.0 + omega * (jv - 0.0));
    }
  }
  return res;
}

template <typename TP, bool kNegR, bool kAux>
struct RestrictOp {
  static constexpr bool kPrepare = false;
  template <typename T>
  __device__ __forceinline__ void prepare(const MarchGeom&, T*, const uint8_t*, int, int) const {}
  __device__ __forceinline__ void prefetch_prologue(const MarchGeom&) {}
  __device__ __forceinline__ void prefetch(const MarchGeom&, int, int64_t, int64_t) {}
  const LevelDev& L;
  int outlet;
  int cnx, cny, cnz;
  float* __restrict__ crhs;
  double (*rs)[kMJ * kMK];          // [2][tile]: fine residuals of planes by parity
  unsigned char (*rsolid)[kMJ * kMK];
  float wres, free_vol;
  int ocount;
  // with cpa: the coarse level's first pre-sweep from a zero iterate, which
  // reads only its own row's rhs, is formed too (in finish, over the
  // block's coarse cells once the march is done)
  const LevelDev& C;
  float* __restrict__ cpa;
  double omega;

  template <class V>
  __device__ __forceinline__ void cell(int i, int j, int k, int64_t c, int t, int, bool, unsigned m, double e,
                                       double kxm, double kxp, const RowCoef& rc, const V& val) {
    if (m & M_SOLID) {
      rsolid[i & 1][t] = 1;
      rs[i & 1][t] = 0.0;
      return;
    }
    double ns, den;
    stencil_sel<kAux>(L, rc, kxm, kxp, i, j, k, c, m, outlet, val(0, -1, 0, 0), val(0, 1, 0, 0), val(0, 0, -1, 0),
                      val(0, 0, 1, 0), val(0, 0, 0, -1), val(0, 0, 0, 1), ns, den);
    if (kAux) den += iface_at<TP>(L, c);
    const double applied = ns - den * val(0, 0, 0, 0);
    const double rv = kNegR ? -e : e;
    rsolid[i & 1][t] = 0;
    rs[i & 1][t] = (double)(TP)(rv - applied);
  }
  float wy[2], wz[2];  // the owner's fine widths along j and k (0 outside the level)

  __device__ __forceinline__ void load_widths(const MarchGeom& g) {
    const int fj0 = g.j0 + 2 * g.ty, fk0 = g.k0 + 2 * g.tx;
#pragma unroll
    for (int o = 0; o < 2; ++o) {
      wy[o] = fj0 + o < L.ny ? __ldg(L.wy + fj0 + o) : 0.0f;
      wz[o] = fk0 + o < L.nz ? __ldg(L.wz + fk0 + o) : 0.0f;
    }
  }

  // Owners (tx < 16, every thread row) fold fine plane q into their coarse cell.
  __device__ __forceinline__ void accumulate(const MarchGeom& g, int q) {
    if (g.tx >= kMK / 2) return;
    const int fj0 = g.j0 + 2 * g.ty, fk0 = g.k0 + 2 * g.tx;
    const float wxq = __ldg(L.wx + q);
#pragma unroll
    for (int oj = 0; oj < 2; ++oj)
#pragma unroll
      for (int ok = 0; ok < 2; ++ok) {
        const int fj = fj0 + oj, fk = fk0 + ok;
        if (fj < L.ny && fk < L.nz) {
          const int t = (2 * g.ty + oj) * kMK + 2 * g.tx + ok;
          if (rsolid[q & 1][t]) {
            ocount += 1;
          } else {
            const float vol = __fmul_rn(__fmul_rn(wxq, wy[oj]), wz[ok]);
            const double r = rs[q & 1][t];
            if (sizeof(TP) == 8)
              wres = (float)__dadd_rn((double)wres, __dmul_rn(r, (double)vol));
            else
              wres = __fadd_rn(wres, __fmul_rn((float)r, vol));
            free_vol = __fadd_rn(free_vol, vol);
          }
        }
      }
    if ((q & 1) || q == L.nx - 1) {
      const int ci = q >> 1, cj = fj0 >> 1, ck = fk0 >> 1;
      if (ci < cnx && cj < cny && ck < cnz)
        crhs[cidx(ci, cj, ck, cny, cnz)] = ocount > 0 ? 0.0f : __fdiv_rn(wres, fmaxf(free_vol, 1.0e-30f));
      wres = 0.0f;
      free_vol = 0.0f;
      ocount = 0;
    }
  }
  // An iteration's planes are the pair (2c, 2c+1) of coarse plane c (ib and
  // the chunk are even): fold them in order once both are staged.
  __device__ __forceinline__ void plane_end(const MarchGeom& g, int i, int np) {
    __syncthreads();
    accumulate(g, i);
    if (np == 2) accumulate(g, i + 1);
  }
  // The block's coarse cells (8 x 16 per coarse plane of its chunk, each
  // written by exactly one owner of this block) get their zero-guess sweep,
  // all threads sharing them: off the march's per-plane path.
  __device__ __forceinline__ void finish(const MarchGeom& g) {
    if (cpa == nullptr) return;
    __syncthreads();  // the owners' crhs stores are visible to the block
    constexpr int kCJ = kMJ / 2, kCK = kMK / 2;
    const int ci0 = g.ib >> 1, nci = ((g.ie + 1) >> 1) - ci0;
    const int cj0 = g.j0 >> 1, ck0 = g.k0 >> 1;
    for (int e = flat_tid(); e < nci * kCJ * kCK; e += kMK * kTY) {
      const int ci = ci0 + e / (kCJ * kCK), rem = e % (kCJ * kCK);
      const int cj = cj0 + rem / kCK, ck = ck0 + rem % kCK;
      if (ci < cnx && cj < cny && ck < cnz) {
        const int64_t cc = cidx(ci, cj, ck, cny, cnz);
        cpa[cc] = coarse_zero_sweep(C, ci, cj, ck, cc, crhs[cc], outlet, omega);
      }
    }
  }
};

template <typename TP, bool kNegR, bool kAux>
__global__ void __launch_bounds__(kMK* kTY, 3)
    km_restrict(LevelDev F, int chunk, const __grid_constant__ CUtensorMap map_p,
                const __grid_constant__ CUtensorMap map_r, const __grid_constant__ CUtensorMap map_m, int outlet,
                int cnx, int cny, int cnz, float* __restrict__ crhs, CgScalars* sc, LevelDev C,
                float* __restrict__ cpa, double omega) {
  pdl_wait();
  using TR = typename std::conditional<kNegR, double, TP>::type;
  __shared__ double rs[2][kMJ * kMK];
  __shared__ unsigned char rsolid[2][kMJ * kMK];
  MarchGeom g;
  const bool any = march_geom(F, chunk, g);
  RestrictOp<TP, kNegR, kAux> op{F,   outlet, cnx, cny, cnz, crhs,        rs,          rsolid, 0.0f, 0.0f,
                                 0,   C,      cpa, omega, {0.0f, 0.0f}, {0.0f, 0.0f}};
  op.load_widths(g);
  const CUtensorMap* const mv[1] = {&map_p};
  if (any && !march<TP, 1, TR, true>(F, g, mv, &map_r, &map_m, op)) report_fault(sc);
}

}  // namespace efsi
