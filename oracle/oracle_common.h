// CPU oracle for the EasyFsi coupled-step hot path -- TEST INFRASTRUCTURE ONLY.
//
// This file and the sources beside it restate, in plain C++ on the host, the
// reference algorithms of lizhuoh9/EasyFsi for the per-step hot path
// (simulation_core/fluid.py, neo_hookean_mpm.py, hibm_mpm.py).  They are the
// checker that the CUDA path is compared against.  Only tests/, the smoke()
// entry of __graft_entry__.py and the cpu_baseline / reference arm of bench.py
// load this library; the product path (easyfsi_b200/) never does.
//
// The same source is compiled twice:
//   * liboracle_mirror.so : R32 = float.  Quantities the reference stores and
//     computes in f32 (velocity, divergence, coarse multigrid levels, MPM state,
//     marker geometry) stay f32; everything the reference keeps in f64
//     (pressure, CG vectors and scalars, marker tractions/forces) is f64.  This
//     is the precision mix of the reference's Taichi kernels, so the CUDA path
//     must match it to round-off.
//   * liboracle_fp64.so   : R32 = double.  The same algorithm entirely in FP64;
//     used to state the error of the f32 quantities against an FP64 solution.
//
// Parity pins: the reference's own known-answer tests are ported onto this
// library in tests/test_oracle_*.py, and the host-side grid metrics it consumes
// are pinned by fixtures generated from the reference's pure-Python grid builder
// (tests/golden/make_golden.py).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifndef EFO_R32
#define EFO_R32 float
#endif

typedef EFO_R32 r32;

#define EFO_API extern "C" __attribute__((visibility("default")))

static inline int64_t efo_idx(int i, int j, int k, int ny, int nz) {
  return ((int64_t)i * ny + j) * nz + k;
}

// One multigrid level: the f32 axis metric arrays the reference loads into
// cell_width_*_m / center_distance_*_m (fluid.py:1013-1024, 1161-1199).
typedef struct efo_level {
  int32_t nx, ny, nz;
  const r32* wx;
  const r32* wy;
  const r32* wz;
  const r32* cdx;
  const r32* cdy;
  const r32* cdz;
} efo_level;

// Full fluid grid: level metrics plus faces / centres (fluid.py:1003-1024).
typedef struct efo_grid {
  efo_level l0;
  const r32* fx;  // faces, nx+1
  const r32* fy;
  const r32* fz;
  const r32* cx;  // centres, nx
  const r32* cy;
  const r32* cz;
} efo_grid;
