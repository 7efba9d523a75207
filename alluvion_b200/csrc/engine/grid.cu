// grid.cu -- cell hash, 3-pass exclusive scan, stable counting sort.
#include "grid.cuh"

namespace alb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class TF>
__global__ void k_hash(const TF* __restrict__ x, uint32_t n, TF h, GridDims g,
                       uint32_t* __restrict__ cell, uint32_t* __restrict__ rank,
                       uint32_t* __restrict__ count, uint32_t* __restrict__ flags) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vec3<TF> p = ld3(x, i);
  int ip[3];
  cell_coords(h, g, p, ip);
  uint32_t c;
  if (in_grid(g, ip)) {
    c = cell_linear(g, ip[0], ip[1], ip[2]);
    cell[i] = c;
  } else {
    c = g.ncells;  // tail bucket
    cell[i] = kNoCell;
    flags[0] = 1u;
  }
  rank[i] = atomicAdd(&count[c], 1u);
}

// Phase 1: per-tile exclusive scan; tile totals to `sums`.  Also raises the
// cell-overflow flag (count > cap) for the first `ncells` entries.
__global__ void k_scan_tiles(const uint32_t* __restrict__ count, uint32_t* __restrict__ start,
                             uint32_t len, uint32_t* __restrict__ sums, uint32_t ncells,
                             uint32_t cap, uint32_t* __restrict__ flags) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t local = 0;
  bool over = false;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint32_t idx = base + k;
    uint32_t c = idx < len ? count[idx] : 0u;
    if (idx < ncells && c > cap) over = true;
    v[k] = local;
    local += c;
  }
  if (over) flags[1] = 1u;
  // inclusive warp scan of per-thread totals
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;  // exclusive warp offsets
    if (lane == kScanThreads / 32 - 1) sums[blockIdx.x] = wi;
  }
  __syncthreads();
  const uint32_t offset = warp_tot[warp] + (incl - local);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    uint32_t idx = base + k;
    if (idx < len) start[idx] = offset + v[k];
  }
}

// Phase 2: one block scans the tile totals in place (exclusive) and writes
// the grand total to start[len].
__global__ void k_scan_sums(uint32_t* __restrict__ sums, uint32_t ntiles,
                            uint32_t* __restrict__ start, uint32_t len) {
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  for (uint32_t base = 0; base < ntiles; base += blockDim.x) {
    uint32_t idx = base + threadIdx.x;
    uint32_t v = idx < ntiles ? sums[idx] : 0u;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < nw ? warp_tot[lane] : 0u;
      uint32_t wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      if (lane < nw) warp_tot[lane] = wi - w;
    }
    __syncthreads();
    uint32_t excl = carry + warp_tot[warp] + (incl - v);
    if (idx < ntiles) sums[idx] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) start[len] = carry;
}

__global__ void k_scan_add(uint32_t* __restrict__ start, uint32_t len,
                           const uint32_t* __restrict__ sums) {
  uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < len) start[idx] += sums[idx / kScanTile];
}

__global__ void k_scatter(const uint32_t* __restrict__ cell, const uint32_t* __restrict__ rank,
                          const uint32_t* __restrict__ start, uint32_t n, uint32_t ncells,
                          uint32_t* __restrict__ perm) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t c = cell[i];
  if (c == kNoCell) c = ncells;
  perm[start[c] + rank[i]] = i;
}

// Sorts every bucket's members by original index: one thread per cell,
// insertion sort in a local array (buckets hold ~8 particles at rest
// density and at most max_num_particles_per_cell = 64 without a
// cell-overflow report).  Larger cells are left to k_order_crowded.  The
// tail bucket of out-of-grid particles is left in arrival order.
constexpr uint32_t kOrderLocal = 64;

__global__ void k_order_cells(const uint32_t* __restrict__ start, uint32_t ncells,
                              uint32_t* __restrict__ perm) {
  uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const uint32_t b = start[c], e = start[c + 1];
  if (e - b < 2 || e - b > kOrderLocal) return;
  uint32_t a[kOrderLocal];
  const uint32_t m = e - b;
  for (uint32_t k = 0; k < m; ++k) {
    uint32_t v = perm[b + k];
    uint32_t j = k;
    while (j > 0 && a[j - 1] > v) {
      a[j] = a[j - 1];
      --j;
    }
    a[j] = v;
  }
  for (uint32_t k = 0; k < m; ++k) perm[b + k] = a[k];
}

// Cells above kOrderLocal members (an overflow the sort reports, but whose
// outputs are still written in canonical order): each block walks the cells
// in chunks of its width, and sorts each crowded cell it finds with all its
// threads, by a bitonic sort in shared memory for up to kCrowdedSmem
// members (indices are distinct, so the order is total).  Beyond that one
// thread sorts in place (a degenerate pile of thousands of particles in one
// cell).
constexpr uint32_t kCrowdedThreads = 256;
constexpr uint32_t kCrowdedSmem = 4096;
constexpr uint32_t kCrowdedBlocks = 256;

__global__ void __launch_bounds__(kCrowdedThreads)
    k_order_crowded(const uint32_t* __restrict__ start, uint32_t ncells,
                    uint32_t* __restrict__ perm) {
  __shared__ uint32_t v[kCrowdedSmem];
  __shared__ uint32_t crowded[kCrowdedThreads];
  __shared__ uint32_t ncrowded;
  for (uint32_t base = blockIdx.x * kCrowdedThreads; base < ncells;
       base += gridDim.x * kCrowdedThreads) {
    if (threadIdx.x == 0) ncrowded = 0;
    __syncthreads();
    const uint32_t c = base + threadIdx.x;
    if (c < ncells && start[c + 1] - start[c] > kOrderLocal)
      crowded[atomicAdd(&ncrowded, 1u)] = c;
    __syncthreads();
    const uint32_t nc = ncrowded;
    for (uint32_t q = 0; q < nc; ++q) {
      const uint32_t cc = crowded[q];
      const uint32_t b = start[cc], m = start[cc + 1] - b;
      if (m <= kCrowdedSmem) {
        uint32_t len = 1;
        while (len < m) len <<= 1;
        for (uint32_t k = threadIdx.x; k < len; k += kCrowdedThreads)
          v[k] = k < m ? perm[b + k] : 0xffffffffu;
        __syncthreads();
        for (uint32_t size = 2; size <= len; size <<= 1) {
          for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t k = threadIdx.x; k < len; k += kCrowdedThreads) {
              const uint32_t partner = k ^ stride;
              if (partner > k) {
                const bool up = (k & size) == 0;
                const uint32_t x = v[k], y = v[partner];
                if ((x > y) == up) {
                  v[k] = y;
                  v[partner] = x;
                }
              }
            }
            __syncthreads();
          }
        }
        for (uint32_t k = threadIdx.x; k < m; k += kCrowdedThreads) perm[b + k] = v[k];
        __syncthreads();
      } else if (threadIdx.x == 0) {
        for (uint32_t k = b + 1; k < b + m; ++k) {
          const uint32_t x = perm[k];
          uint32_t j = k;
          while (j > b && perm[j - 1] > x) {
            perm[j] = perm[j - 1];
            --j;
          }
          perm[j] = x;
        }
      }
      __syncthreads();
    }
  }
}

inline uint32_t crowded_blocks(uint32_t ncells) {
  const uint32_t chunks = (ncells + kCrowdedThreads - 1) / kCrowdedThreads;
  return chunks < kCrowdedBlocks ? (chunks ? chunks : 1u) : kCrowdedBlocks;
}

template <class TF>
__global__ void k_gather_x(const TF* __restrict__ x, const uint32_t* __restrict__ perm,
                           uint32_t n, vec4<TF>* __restrict__ xs, uint32_t* __restrict__ inv) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = perm[s];
  vec3<TF> p = ld3(x, i);
  xs[s] = vec4<TF>{p.x, p.y, p.z, TF(0)};
  inv[i] = s;
}

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

// k_hash over the arena of a fused batch: slot g of a 128-slot block holds
// particle g - s0 of the block's scene, or padding (no cell).
template <class TF>
__global__ void k_hash_fused(TF h, const uint32_t* __restrict__ blk_scene,
                             const SortScene<TF>* __restrict__ scenes, uint32_t nscenes,
                             uint32_t* __restrict__ cell, uint32_t* __restrict__ rank,
                             uint32_t* __restrict__ count) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t k = blk_scene[blockIdx.x];
  const SortScene<TF>* sc = k < nscenes ? scenes + k : nullptr;
  const uint32_t i = sc ? g - sc->s0 : 0u;
  if (!sc || i >= sc->n) {
    cell[g] = kNoCell;
    return;
  }
  const GridDims& gd = sc->g;
  const vec3<TF> p = ld3(sc->x, i);
  int ip[3];
  cell_coords(h, gd, p, ip);
  uint32_t lc;
  if (in_grid(gd, ip)) {
    lc = cell_linear(gd, ip[0], ip[1], ip[2]);
  } else {
    lc = gd.ncells;  // the scene's tail bucket
    sc->flags[0] = 1u;
  }
  const uint32_t c = sc->cell0 + lc;
  cell[g] = c;
  const uint32_t r = atomicAdd(&count[c], 1u);
  rank[g] = r;
  if (lc < gd.ncells && r >= gd.cap_cell) sc->flags[1] = 1u;  // count > cap
}

// The padding buckets' counts (after the counts are cleared).
template <class TF>
__global__ void k_pad_counts(const SortScene<TF>* __restrict__ scenes, uint32_t nscenes,
                             uint32_t* __restrict__ count) {
  for (uint32_t k = threadIdx.x; k < nscenes; k += blockDim.x)
    count[scenes[k].cell0 + scenes[k].g.ncells + 1] = scenes[k].pad;
}

__global__ void k_scatter_fused(const uint32_t* __restrict__ cell,
                                const uint32_t* __restrict__ rank,
                                const uint32_t* __restrict__ start, uint32_t n,
                                uint32_t* __restrict__ perm) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t c = cell[g];
  if (c != kNoCell) perm[start[c] + rank[g]] = g;
}

}  // namespace

namespace {
int scan_with_flags(al_engine* e, const uint32_t* count, uint32_t* start, uint32_t len,
                    uint32_t ncells, uint32_t cap, uint32_t* flags, cudaStream_t st) {
  const uint32_t ntiles = (len + kScanTile - 1) / kScanTile;
  uint32_t* sums = nullptr;
  ALB_TRY(e->buf("scan.sums", ntiles, &sums));
  k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(count, start, len, sums, ncells, cap, flags);
  k_scan_sums<<<1, 1024, 0, st>>>(sums, ntiles, start, len);
  if (ntiles > 1) k_scan_add<<<blocks_for(len, 256), 256, 0, st>>>(start, len, sums);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}
}  // namespace

template <class TF>
int grid_build(al_engine* e, const Cn<TF>& c, const GridDims& g, const TF* particle_x,
               uint32_t n, vec4<TF>* xs, uint32_t* flags, GridState& gs, cudaStream_t st) {
  gs.n = n;
  gs.ncells = g.ncells;
  gs.flags = flags;
  uint32_t* rank = nullptr;
  ALB_TRY(e->buf("grid.cell", n, &gs.cell));
  ALB_TRY(e->buf("grid.rank", n, &rank));
  ALB_TRY(e->buf("grid.perm", n, &gs.perm));
  ALB_TRY(e->buf("grid.inv", n, &gs.inv));
  ALB_TRY(e->buf("grid.count", size_t(g.ncells) + 1, &gs.count));
  ALB_TRY(e->buf("grid.start", size_t(g.ncells) + 2, &gs.cell_start));
  ALB_CUDA(cudaMemsetAsync(gs.count, 0, (size_t(g.ncells) + 1) * sizeof(uint32_t), st));
  if (n == 0) {
    ALB_CUDA(cudaMemsetAsync(gs.cell_start, 0, (size_t(g.ncells) + 2) * sizeof(uint32_t), st));
    return AL_OK;
  }
  k_hash<TF><<<blocks_for(n, kBlock), kBlock, 0, st>>>(particle_x, n, c.h, g, gs.cell, rank,
                                                       gs.count, flags);
  ALB_TRY(scan_with_flags(e, gs.count, gs.cell_start, g.ncells + 1, g.ncells, g.cap_cell, flags,
                          st));
  k_scatter<<<blocks_for(n, kBlock), kBlock, 0, st>>>(gs.cell, rank, gs.cell_start, n, g.ncells,
                                                      gs.perm);
  k_order_cells<<<blocks_for(g.ncells, kBlock), kBlock, 0, st>>>(gs.cell_start, g.ncells,
                                                                 gs.perm);
  k_order_crowded<<<crowded_blocks(g.ncells), kCrowdedThreads, 0, st>>>(gs.cell_start, g.ncells,
                                                                        gs.perm);
  k_gather_x<TF><<<blocks_for(n, kBlock), kBlock, 0, st>>>(particle_x, gs.perm, n, xs, gs.inv);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int grid_build_fused(al_engine* e, TF h, const uint32_t* blk_scene, const SortScene<TF>* scenes,
                     uint32_t nscenes, uint32_t narena, uint32_t ncells, GridState& gs,
                     cudaStream_t st) {
  gs.n = narena;
  gs.ncells = ncells;
  uint32_t* rank = nullptr;
  ALB_TRY(e->buf("grid.cell", narena, &gs.cell));
  ALB_TRY(e->buf("grid.rank", narena, &rank));
  ALB_TRY(e->buf("grid.perm", narena, &gs.perm));
  ALB_TRY(e->buf("grid.count", size_t(ncells) + 1, &gs.count));
  ALB_TRY(e->buf("grid.start", size_t(ncells) + 2, &gs.cell_start));
  ALB_CUDA(cudaMemsetAsync(gs.count, 0, (size_t(ncells) + 1) * sizeof(uint32_t), st));
  if (narena == 0) return AL_OK;
  k_pad_counts<TF><<<1, 256, 0, st>>>(scenes, nscenes, gs.count);
  k_hash_fused<TF><<<narena / kBlock, kBlock, 0, st>>>(h, blk_scene, scenes, nscenes, gs.cell,
                                                      rank, gs.count);
  // cell caps were checked by the hash: no cells to check in the scan
  ALB_TRY(scan_with_flags(e, gs.count, gs.cell_start, ncells + 1, 0u, 0u, nullptr, st));
  k_scatter_fused<<<blocks_for(narena, kBlock), kBlock, 0, st>>>(gs.cell, rank, gs.cell_start,
                                                                narena, gs.perm);
  k_order_cells<<<blocks_for(ncells, kBlock), kBlock, 0, st>>>(gs.cell_start, ncells, gs.perm);
  k_order_crowded<<<crowded_blocks(ncells), kCrowdedThreads, 0, st>>>(gs.cell_start, ncells,
                                                                      gs.perm);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

uint32_t grid_fused_kernels(uint32_t ncells) {
  return 7u + (grid_scan_tiles(ncells + 1) > 1 ? 1u : 0u);
}

uint32_t grid_scan_tiles(uint32_t len) { return (len + kScanTile - 1) / kScanTile; }

template <class TF>
int grid_sort_into(const Cn<TF>& c, const GridDims& g, const TF* particle_x, uint32_t n,
                   uint32_t* cell, uint32_t* perm, const GridSortScratch& sc, cudaStream_t st) {
  const uint32_t len = g.ncells + 1;
  ALB_CUDA(cudaMemsetAsync(sc.count, 0, size_t(len) * sizeof(uint32_t), st));
  ALB_CUDA(cudaMemsetAsync(sc.flags, 0, 4 * sizeof(uint32_t), st));
  if (n == 0) {
    ALB_CUDA(cudaMemsetAsync(sc.start, 0, (size_t(len) + 1) * sizeof(uint32_t), st));
    return AL_OK;
  }
  k_hash<TF><<<blocks_for(n, kBlock), kBlock, 0, st>>>(particle_x, n, c.h, g, cell, sc.rank,
                                                       sc.count, sc.flags);
  const uint32_t ntiles = grid_scan_tiles(len);
  k_scan_tiles<<<ntiles, kScanThreads, 0, st>>>(sc.count, sc.start, len, sc.sums, g.ncells,
                                                 g.cap_cell, sc.flags);
  k_scan_sums<<<1, 1024, 0, st>>>(sc.sums, ntiles, sc.start, len);
  if (ntiles > 1) k_scan_add<<<blocks_for(len, 256), 256, 0, st>>>(sc.start, len, sc.sums);
  k_scatter<<<blocks_for(n, kBlock), kBlock, 0, st>>>(cell, sc.rank, sc.start, n, g.ncells,
                                                      perm);
  k_order_cells<<<blocks_for(g.ncells, kBlock), kBlock, 0, st>>>(sc.start, g.ncells, perm);
  k_order_crowded<<<crowded_blocks(g.ncells), kCrowdedThreads, 0, st>>>(sc.start, g.ncells, perm);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template int grid_sort_into<float>(const Cn<float>&, const GridDims&, const float*, uint32_t,
                                   uint32_t*, uint32_t*, const GridSortScratch&, cudaStream_t);
template int grid_sort_into<double>(const Cn<double>&, const GridDims&, const double*, uint32_t,
                                    uint32_t*, uint32_t*, const GridSortScratch&, cudaStream_t);

template int grid_build_fused<float>(al_engine*, float, const uint32_t*,
                                     const SortScene<float>*, uint32_t, uint32_t, uint32_t,
                                     GridState&, cudaStream_t);
template int grid_build<float>(al_engine*, const Cn<float>&, const GridDims&, const float*,
                               uint32_t, vec4<float>*, uint32_t*, GridState&, cudaStream_t);
template int grid_build<double>(al_engine*, const Cn<double>&, const GridDims&, const double*,
                                uint32_t, vec4<double>*, uint32_t*, GridState&, cudaStream_t);

}  // namespace alb
