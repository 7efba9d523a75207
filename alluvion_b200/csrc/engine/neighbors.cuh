// neighbors.cuh -- compact neighbor lists over the cell-sorted order.
//
// Replaces make_neighbor_list<0> (runner.hpp:1869-1911) and compute_density
// (runner.hpp:2052-2072).  The reference stores [N][cap] float4 entries
// {x_i - x_j, j} per particle row; the engine stores 32-bit sorted slots in
// slot-major layout nbr[k * N + s], so that the k-th neighbor of 32
// consecutive particles is one coalesced 128-byte line, and recomputes
// x_i - x_j from the cell-sorted positions (L1/L2 resident) in every pass.
//
// Candidate order: the 27 cells in ascending linear cell index; the three
// cells of a (dx, dy) row are contiguous in sorted order, so each row is one
// contiguous slot range and the list comes out in ascending slot order,
// i.e. canonical (cell, index) order.
#pragma once

#include "common.cuh"
#include "grid.cuh"

namespace alb {

// Boundary kernel terms {grad W * V, W * V} in the reference's
// [nb][N][4] layout (original particle order); used by the standalone
// update_particle_neighbors entry point.
template <class TF>
struct RefBoundaryKernel {
  const TF* bk;
  const uint32_t* perm;
  uint32_t n, nb;
  __device__ __forceinline__ TF density_term(uint32_t s) const {
    TF sum = 0;
    if (bk) {
      const uint32_t i = perm[s];
      for (uint32_t b = 0; b < nb; ++b) sum += bk[(size_t(b) * n + i) * 4 + 3];
    }
    return sum;
  }
  __device__ __forceinline__ vec3<TF> grad_term(uint32_t s) const {
    vec3<TF> g{0, 0, 0};
    if (bk) {
      const uint32_t i = perm[s];
      for (uint32_t b = 0; b < nb; ++b) {
        const TF* e = bk + (size_t(b) * n + i) * 4;
        g += vec3<TF>{e[0], e[1], e[2]};
      }
    }
    return g;
  }
};

// The engine's sparse boundary state in sorted order: only bodies whose bit
// is set in mask[s] contribute (their volume is non-zero; the others'
// terms are exactly zero).  Bodies are visited in ascending order, as the
// reference's boundary loops do.
template <class TF>
struct SortedBoundaryKernel {
  const uint32_t* mask;
  const vec4<TF>* bk;
  uint32_t n;
  __device__ __forceinline__ TF density_term(uint32_t s) const {
    TF sum = 0;
    for (uint32_t m = mask[s]; m; m &= m - 1) sum += bk[size_t(__ffs(m) - 1) * n + s].w;
    return sum;
  }
  __device__ __forceinline__ vec3<TF> grad_term(uint32_t s) const {
    vec3<TF> g{0, 0, 0};
    for (uint32_t m = mask[s]; m; m &= m - 1) g += xyz(bk[size_t(__ffs(m) - 1) * n + s]);
    return g;
  }
};

// Builds nbr / ncount for all n sorted slots and the density
// rho_s = rho0 (V W(0) + sum_j V W(x_sj) + boundary).  When `alpha` is
// non-null also the DFSPH factor of compute_dfsph_factor
// (runner.hpp:3123-3154).  Raises flags[2] on neighbor overflow.
template <class TF, class BK>
int build_neighbors_density(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                            const vec4<TF>* xs, const BK& bk, uint32_t* nbr, uint32_t* ncount,
                            TF* rho, TF* alpha, cudaStream_t st);

// ----------------------------------------------------------- compact lists
// The step's neighbor lists.  In canonical order the neighbors of a
// particle lie in the 9 (dx, dy) cell rows around its cell, each row one
// contiguous range of sorted slots starting at cell_start of the row's
// first cell.  A particle's list is stored as
//   desc[s]          9 row counts of 7 bits each (row r = 3 * (dx + 1) + (dy + 1))
//   off[k * N + s]   offset of the k-th neighbor from its row's first slot
// so a neighbor costs 1 byte instead of 4 and the list is rebuilt from the
// particle's own cell coordinates.  Rows hold at most 3 cells; an offset
// above 255 (only possible when cells overflow their capacity) is dropped
// and raises the cell-overflow flag.
constexpr int kRowBits = 7;
constexpr uint32_t kMaxRowOffset = 255;

struct NeighborRows {
  const uint64_t* desc;
  const uint8_t* off;
  const uint32_t* cell_start;
  uint32_t n;
  GridDims g;
};

__device__ __forceinline__ uint32_t row_count(uint64_t desc, int r) {
  return uint32_t(desc >> (kRowBits * r)) & ((1u << kRowBits) - 1u);
}
__device__ __forceinline__ uint32_t neighbor_total(uint64_t desc) {
  uint32_t c = 0;
#pragma unroll
  for (int r = 0; r < 9; ++r) c += row_count(desc, r);
  return c;
}

// Calls f(t) for every neighbor slot t of sorted particle s (position xi),
// in canonical order.
template <class TF, class F>
__device__ __forceinline__ void for_each_neighbor(const NeighborRows& L, TF h, uint32_t s,
                                                  vec3<TF> xi, uint64_t desc, F&& f) {
  int ip[3];
  cell_coords(h, L.g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  uint32_t k = 0;
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const uint32_t cr = row_count(desc, r);
    if (cr == 0) continue;
    const uint32_t base =
        __ldg(L.cell_start + cell_linear(L.g, ip[0] + r / 3 - 1, ip[1] + r % 3 - 1, z0));
    for (uint32_t j = 0; j < cr; ++j, ++k)
      f(base + uint32_t(__ldg(L.off + size_t(k) * L.n + s)));
  }
}

// Builds the compact lists of all n sorted slots, the density and, when
// `alpha` is non-null, the DFSPH factor (same arithmetic and order as
// build_neighbors_density).
template <class TF, class BK>
int build_compact_neighbors(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                            const vec4<TF>* xs, const BK& bk, uint64_t* desc, uint8_t* off,
                            TF* rho, TF* alpha, cudaStream_t st);

// Writes reference-layout outputs in original particle order:
// particle_neighbors [N][cap][4] {x_i - x_j, bits(j)} (if non-null),
// particle_num_neighbors [N], particle_density [N] (if non-null).
template <class TF>
int export_neighbors(const GridDims& g, const GridState& gs, const vec4<TF>* xs,
                     const uint32_t* nbr, const uint32_t* ncount, const TF* rho_sorted,
                     TF* particle_neighbors, uint32_t* particle_num_neighbors,
                     TF* particle_density, cudaStream_t st);

}  // namespace alb
