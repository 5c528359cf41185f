// z-min outlet pressure reachability and the unreached fluid components
// (CartesianFluidSolver.mark_hibm_pressure_outlet_disconnected_nonprojectable_cells,
// fluid.py:1614-1876 and 4764-4910).
//
// The reference floods reachability from the outlet with Jacobi sweeps (up to
// 32 (nx + ny + nz) launches), then labels the unreached cells by min-label
// sweeps.  Both describe one undirected graph: fluid, non-barrier cells,
// joined through faces whose upper cell has no Dirichlet row and no barrier
// (fluid.py:1649-1698 / 4776-4845 read the same rule in both directions).  A
// cell is reached iff its connected component holds a seed (a fluid,
// non-barrier, row-free cell at k = 0), and an unreached component's label is
// its smallest linear cell index.  So here one connected-components labelling
// of the open faces (rounds of hooking and pointer jumping; every component
// ends labelled by its smallest index) gives both; the components are then
// ranked by their root as the reference ranks its labels (up to 256, the rest
// keep their raw label).
#include <algorithm>
#include <vector>

#include "efsi_common.cuh"

struct efsi_reach_plan {
  int32_t* roots = nullptr;  // unreached component roots, appended
  int64_t roots_cap = 0;
  int32_t* counters = nullptr;  // [0] roots, [1] unreached cells, [2] a hook changed a label this round
  int32_t* table = nullptr;     // the ranked roots (256)
  int32_t* host_counters = nullptr;
};

namespace efsi {
namespace {

constexpr int32_t kNoLabel = 1 << 30;
constexpr int kComponentCapacity = 256;  // HIBM_PRESSURE_COMPONENT_CAPACITY (fluid.py:17)
constexpr int kMaxRounds = 4096;  // hook-and-jump rounds before giving up

struct ReachArgs {
  int nx, ny, nz;
  int64_t n;
  const int32_t* obs;
  const int32_t* vdir;     // may be null
  const int32_t* barrier;  // may be null
  int32_t* reach;
  int32_t* label;  // component labels (smallest cell index) while labelling
};

__device__ __forceinline__ int32_t at(const int32_t* a, int64_t c) { return a == nullptr ? 0 : __ldg(a + c); }

__device__ __forceinline__ bool node(const ReachArgs& A, int64_t c) {
  return __ldg(A.obs + c) == 0 && at(A.barrier, c) == 0;
}

// the face below the upper cell u is open
__device__ __forceinline__ bool face_open(const ReachArgs& A, int64_t u) {
  return at(A.vdir, u) == 0 && at(A.barrier, u) == 0;
}

// node_kind -> barrier (fluid.py:1618-1627), or clear it
__global__ void k_reach_barrier(int64_t n, const int32_t* __restrict__ kind, int32_t code, int32_t* barrier) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) barrier[c] = (kind != nullptr && kind[c] == code) ? 1 : 0;
}

__global__ void k_reach_init(ReachArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n) return;
  A.label[c] = node(A, c) ? (int32_t)c : kNoLabel;
  A.reach[c] = 0;
}

// Connected components by rounds of hooking and pointer jumping.  Every label
// is a cell of the same component with an index no larger than its own.  A
// round first hooks: for every open face whose two cells carry different
// labels, the larger label's cell is pointed (atomicMin) at the smaller label.
// Then it jumps: every cell follows its labels to the end of the chain, where
// the label points to itself.  Labels only decrease, and a round whose hooks
// change nothing leaves every face with equal labels at both ends (the jump of
// the previous round made every label a chain end), so then each component is
// labelled by its smallest cell index.  Nothing here depends on the order in
// which the device's threads see each other's writes.
__global__ void k_reach_hook(ReachArgs A, int32_t* changed) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n || !node(A, c)) return;
  const int k = (int)(c % A.nz), j = (int)((c / A.nz) % A.ny), i = (int)(c / ((int64_t)A.ny * A.nz));
  const int64_t up[3] = {i < A.nx - 1 ? c + (int64_t)A.ny * A.nz : -1, j < A.ny - 1 ? c + A.nz : -1,
                         k < A.nz - 1 ? c + 1 : -1};
  bool any = false;
  for (int d = 0; d < 3; ++d) {
    const int64_t u = up[d];
    if (u < 0 || !node(A, u) || !face_open(A, u)) continue;
    const int32_t a = atomicAdd(A.label + c, 0), b = atomicAdd(A.label + u, 0);
    if (a == b) continue;
    const int32_t hi = a > b ? a : b, lo = a > b ? b : a;
    if (atomicMin(A.label + hi, lo) > lo) any = true;
  }
  if (any) atomicOr(changed, 1);
}

__global__ void k_reach_jump(ReachArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n) return;
  int32_t l = A.label[c];
  if (l == kNoLabel) return;
  // labels strictly decrease along a chain, so the walk ends
  int32_t next = atomicAdd(A.label + l, 0);
  while (next < l) {
    l = next;
    next = atomicAdd(A.label + l, 0);
  }
  atomicMin(A.label + c, l);
}

// seeds (fluid.py:1714-1725) mark their component's root
__global__ void k_reach_seed(ReachArgs A) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n || A.label[c] == kNoLabel) return;
  if (c % A.nz == 0 && at(A.vdir, c) == 0) atomicOr(A.reach + A.label[c], 1);
}

// every node takes its root's flag; unreached roots are collected
__global__ void k_reach_spread(ReachArgs A, int32_t* roots, int32_t* counters) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n || A.label[c] == kNoLabel) return;
  const int32_t r = A.label[c];
  const int32_t reached = A.reach[r];
  if (r != (int32_t)c) A.reach[c] = reached;
  if (!reached) {
    atomicAdd(counters + 1, 1);
    if (r == (int32_t)c) roots[atomicAdd(counters, 1)] = r;
  }
}

// reached and non-node cells carry no label; unreached cells of the first
// 256 components by root take -(rank + 1), the rest keep their root
__global__ void k_reach_label(ReachArgs A, const int32_t* __restrict__ table, int count) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n || A.label[c] == kNoLabel) return;
  if (A.reach[c]) {
    A.label[c] = kNoLabel;
    return;
  }
  const int32_t r = A.label[c];
  int lo = 0, hi = count;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (table[mid] < r)
      lo = mid + 1;
    else
      hi = mid;
  }
  if (lo < count && table[lo] == r) A.label[c] = -(lo + 1);
}

}  // namespace
}  // namespace efsi

using namespace efsi;

extern "C" {

int efsi_reach_plan_create(efsi_reach_plan** out) {
  EFSI_ARG_CHECK(out != nullptr, "null plan pointer");
  efsi_reach_plan* P = new efsi_reach_plan();
  if (cudaMalloc(&P->counters, 4 * sizeof(int32_t)) != cudaSuccess ||
      cudaMalloc(&P->table, kComponentCapacity * sizeof(int32_t)) != cudaSuccess ||
      cudaMallocHost(&P->host_counters, 4 * sizeof(int32_t)) != cudaSuccess) {
    cudaFree(P->counters);
    cudaFree(P->table);
    delete P;
    set_error("allocation failed for the reachability plan");
    return EFSI_ERR_CUDA;
  }
  *out = P;
  return EFSI_OK;
}

int efsi_reach_plan_destroy(efsi_reach_plan* P) {
  if (P == nullptr) return EFSI_OK;
  cudaFree(P->roots);
  cudaFree(P->counters);
  cudaFree(P->table);
  cudaFreeHost(P->host_counters);
  delete P;
  return EFSI_OK;
}

int efsi_outlet_reachability(efsi_reach_plan* P, int32_t nx, int32_t ny, int32_t nz, const int32_t* obstacle,
                             const int32_t* velocity_dirichlet_active, int32_t* barrier, const int32_t* node_kind,
                             int32_t barrier_code, int32_t update_barrier, int32_t* reachable, int32_t* label,
                             efsi_reach_report* report, void* stream) {
  EFSI_ARG_CHECK(P != nullptr && report != nullptr, "null argument");
  EFSI_ARG_CHECK(nx > 0 && ny > 0 && nz > 0, "grid_nodes must be positive");
  EFSI_ARG_CHECK(obstacle && barrier && reachable && label, "null field");
  const int64_t n = (int64_t)nx * ny * nz;
  EFSI_ARG_CHECK(n < (int64_t)kNoLabel, "the grid has too many cells for int32 labels");
  cudaStream_t s = as_stream(stream);
  const unsigned grid = (unsigned)((n + 255) / 256);
  if (update_barrier) EFSI_COUNTED k_reach_barrier<<<grid, 256, 0, s>>>(n, node_kind, barrier_code, barrier);
  if (P->roots_cap < n) {
    cudaFree(P->roots);
    P->roots = nullptr;
    P->roots_cap = 0;
    EFSI_CUDA_CHECK(cudaMalloc(&P->roots, (size_t)n * sizeof(int32_t)));
    P->roots_cap = n;
  }
  EFSI_CUDA_CHECK(cudaMemsetAsync(P->counters, 0, 4 * sizeof(int32_t), s));
  ReachArgs A{nx, ny, nz, n, obstacle, velocity_dirichlet_active, barrier, reachable, label};
  EFSI_COUNTED k_reach_init<<<grid, 256, 0, s>>>(A);
  int rounds = 0;
  for (;;) {
    EFSI_CUDA_CHECK(cudaMemsetAsync(P->counters + 2, 0, sizeof(int32_t), s));
    EFSI_COUNTED k_reach_hook<<<grid, 256, 0, s>>>(A, P->counters + 2);
    EFSI_COUNTED k_reach_jump<<<grid, 256, 0, s>>>(A);
    EFSI_LAUNCH_CHECK();
    EFSI_CUDA_CHECK(cudaMemcpyAsync(P->host_counters + 2, P->counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
    ++rounds;
    if (P->host_counters[2] == 0) break;
    EFSI_ARG_CHECK(rounds < kMaxRounds, "the component labels did not settle");
  }
  EFSI_COUNTED k_reach_seed<<<grid, 256, 0, s>>>(A);
  EFSI_COUNTED k_reach_spread<<<grid, 256, 0, s>>>(A, P->roots, P->counters);
  EFSI_LAUNCH_CHECK();
  EFSI_CUDA_CHECK(cudaMemcpyAsync(P->host_counters, P->counters, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  const int32_t nroots = P->host_counters[0], unreached = P->host_counters[1];
  int count = 0;
  if (nroots > 0) {
    std::vector<int32_t> roots((size_t)nroots);
    EFSI_CUDA_CHECK(cudaMemcpy(roots.data(), P->roots, (size_t)nroots * sizeof(int32_t), cudaMemcpyDeviceToHost));
    std::sort(roots.begin(), roots.end());
    count = std::min(nroots, kComponentCapacity);
    EFSI_CUDA_CHECK(cudaMemcpyAsync(P->table, roots.data(), (size_t)count * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  }
  EFSI_COUNTED k_reach_label<<<grid, 256, 0, s>>>(A, P->table, count);
  EFSI_LAUNCH_CHECK();
  EFSI_CUDA_CHECK(cudaStreamSynchronize(s));
  report->unreached_cells = unreached;
  report->components = count;
  report->overflow = nroots > kComponentCapacity ? 1 : 0;
  return EFSI_OK;
}

}  // extern "C"
