// grid.cuh -- uniform-grid cell hash and stable counting sort.
//
// Replaces update_particle_grid (runner.hpp:1840-1867).  The reference
// appends particles to fixed-capacity buckets in atomicAdd order; the engine
// builds a compact cell-sorted permutation in canonical (cell, index) order:
//   1. hash:    cell id per particle, arrival rank within the cell
//   2. scan:    exclusive prefix sum of cell counts (3 passes, no waits)
//   3. scatter: slot = cell_start + arrival rank
//   4. order:   each cell's members sorted by original index (makes the
//               permutation independent of atomic arrival order)
// Particles outside the grid land in a tail bucket after all cells.
#pragma once

#include "common.cuh"
#include "engine.hpp"

namespace alb {

struct GridState {
  uint32_t n = 0;
  uint32_t ncells = 0;
  uint32_t* cell = nullptr;        // [n] cell of original particle (kNoCell outside)
  uint32_t* perm = nullptr;        // [n] sorted slot -> original index
  uint32_t* inv = nullptr;         // [n] original index -> sorted slot
  uint32_t* cell_start = nullptr;  // [ncells + 2]; [ncells] = in-grid count, [ncells+1] = n
  uint32_t* count = nullptr;       // [ncells + 1]; last = out-of-grid count
  uint32_t* flags = nullptr;       // [4] grid_anomaly[0..2] + spare (device)
};

// Kernels one grid_build launches (hash, three scan passes, scatter, the two
// per-cell orderings, gather).
constexpr int kGridBuildKernels = 8;

// Hashes, sorts and gathers positions into `xs` (sorted order, w = 0).
// particle_x is the caller's [n][3] array.  `flags` must be zeroed by the
// caller (it is also used by later passes).
template <class TF>
int grid_build(al_engine* e, const Cn<TF>& c, const GridDims& g, const TF* particle_x,
               uint32_t n, vec4<TF>* xs, uint32_t* flags, GridState& gs, cudaStream_t st);

// One scene of a fused batch's sort: its positions (the caller's [n][3]),
// grid, first cell in the batch's concatenated cells (its ncells cells, then
// its out-of-grid tail bucket, then a padding bucket that holds the `pad`
// slots up to the next scene's start), its slots [s0, s0 + n) of the
// batch's arena and its anomaly flags.
template <class TF>
struct SortScene {
  const TF* x;
  GridDims g;
  uint32_t cell0, s0, n, pad;
  uint32_t* flags;
};

// Every scene of a fused batch in one counting sort over the concatenated
// cells (ncells in all, tails and padding included): the scene of each
// 128-slot block in blk_scene (nscenes past every scene), the arena of
// `narena` slots.  gs.perm maps a sorted arena slot to the arena slot
// s0 + i of the scene's particle i, gs.cell_start holds arena slots; the
// cells' members, the out-of-grid tails included, are ordered by index.
// Anomalies go to each scene's flags.
template <class TF>
int grid_build_fused(al_engine* e, TF h, const uint32_t* blk_scene, const SortScene<TF>* scenes,
                     uint32_t nscenes, uint32_t narena, uint32_t ncells, GridState& gs,
                     cudaStream_t st);
// Kernels one grid_build_fused launches.
uint32_t grid_fused_kernels(uint32_t ncells);

// Scratch for grid_sort_into, all supplied by the caller.
struct GridSortScratch {
  uint32_t* rank;   // [n]
  uint32_t* count;  // [ncells + 1], zeroed by grid_sort_into
  uint32_t* start;  // [ncells + 2]
  uint32_t* sums;   // [grid_scan_tiles(ncells + 1)]
  uint32_t* flags;  // [4], zeroed by grid_sort_into
};

// Number of scan tiles for `len` entries.
uint32_t grid_scan_tiles(uint32_t len);

// The same hash / scan / scatter / per-cell ordering as grid_build, writing
// the per-particle cell and the permutation straight into cell / perm and
// using only the given scratch: no allocation of any kind.
template <class TF>
int grid_sort_into(const Cn<TF>& c, const GridDims& g, const TF* particle_x, uint32_t n,
                   uint32_t* cell, uint32_t* perm, const GridSortScratch& sc, cudaStream_t st);

}  // namespace alb
