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

// Spare entries after the n sorted positions that the build reads: its scan
// loads candidates in rounds of up to 8 and may read past a row's last
// candidate (the extra bits are masked off), so every sorted-position
// buffer passed to the build holds n + kSortedPad entries.
constexpr uint32_t kSortedPad = 8;

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
  uint32_t n;  // row stride of bk
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

// Element stride of the density copy `rho_rec` (the step's particle
// records hold 8 reals per particle).
constexpr size_t kRecStride = 8;

// Builds nbr / ncount for all n sorted slots and the density
// rho_s = rho0 (V W(0) + sum_j V W(x_sj) + boundary).  When `alpha` is
// non-null also the DFSPH factor of compute_dfsph_factor
// (runner.hpp:3123-3154); when `rho_rec` is non-null also writes the
// density to rho_rec[s * kRecStride].  Raises flags[2] on neighbor overflow.
template <class TF, class BK>
int build_neighbors_density(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                            const vec4<TF>* xs, const BK& bk, uint32_t* nbr, uint32_t* ncount,
                            TF* rho, TF* alpha, TF* rho_rec, cudaStream_t st);

// Writes reference-layout outputs in original particle order:
// particle_neighbors [N][cap][4] {x_i - x_j, bits(j)} (if non-null),
// particle_num_neighbors [N], particle_density [N] (if non-null).
template <class TF>
int export_neighbors(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                     const vec4<TF>* xs,
                     const uint32_t* nbr, const uint32_t* ncount, const TF* rho_sorted,
                     TF* particle_neighbors, uint32_t* particle_num_neighbors,
                     TF* particle_density, cudaStream_t st);

}  // namespace alb
