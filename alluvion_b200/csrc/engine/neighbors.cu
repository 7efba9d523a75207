// neighbors.cu -- neighbor-list build with fused density, and export to the
// reference layout.
#include "build_kernel.cuh"
#include "neighbors.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

template <class TF>
__global__ void k_export_neighbors(Cn<TF> c, uint32_t cap, uint32_t n,
                                   const uint32_t* __restrict__ perm,
                                   const uint32_t* __restrict__ inv,
                                   const vec4<TF>* __restrict__ xs,
                                   const uint32_t* __restrict__ nbr,
                                   const uint32_t* __restrict__ ncount,
                                   const TF* __restrict__ rho_sorted, TF* __restrict__ out_nbr,
                                   uint32_t* __restrict__ out_num, TF* __restrict__ out_rho) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t s = inv[i];
  const uint32_t cnt = ncount[s];
  out_num[i] = cnt;
  if (out_rho) out_rho[i] = rho_sorted[s];
  if (!out_nbr) return;
  const vec3<TF> xi = xyz(xs[s]);
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t t = nbr[size_t(k) * n + s];
    const uint32_t j = perm[t];
    const vec3<TF> xj = xyz(xs[t]);
    TF* e = out_nbr + (size_t(i) * cap + k) * 4;
    const vec3<TF> d = pdisp(c, xi, xj);  // wrapped in y on a periodic update
    e[0] = d.x;
    e[1] = d.y;
    e[2] = d.z;
    if constexpr (sizeof(TF) == 4) {
      e[3] = __uint_as_float(j);
    } else {
      e[3] = __longlong_as_double((long long)j);
    }
  }
}

}  // namespace

template <class TF, class BK>
int build_neighbors_density(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                            const vec4<TF>* xs, const BK& bk, uint32_t* nbr, uint32_t* ncount,
                            TF* rho, TF* alpha, TF* rho_rec, cudaStream_t st) {
  if (gs.n == 0) return AL_OK;
  const uint32_t blocks = blocks_for(gs.n, kBlock);
  // compile-time wrap flag: the non-periodic build carries no wrap branches
  if (alpha && c.wrap)
    k_build_neighbors<TF, BK, true, NoExtra<TF>, true><<<blocks, kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags,
        NoExtra<TF>{}, FusedBuild{});
  else if (alpha)
    k_build_neighbors<TF, BK, true, NoExtra<TF>, false><<<blocks, kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags,
        NoExtra<TF>{}, FusedBuild{});
  else if (c.wrap)
    k_build_neighbors<TF, BK, false, NoExtra<TF>, true><<<blocks, kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags,
        NoExtra<TF>{}, FusedBuild{});
  else
    k_build_neighbors<TF, BK, false, NoExtra<TF>, false><<<blocks, kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags,
        NoExtra<TF>{}, FusedBuild{});
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int export_neighbors(const Cn<TF>& c, const GridDims& g, const GridState& gs,
                     const vec4<TF>* xs,
                     const uint32_t* nbr, const uint32_t* ncount, const TF* rho_sorted,
                     TF* particle_neighbors, uint32_t* particle_num_neighbors,
                     TF* particle_density, cudaStream_t st) {
  if (gs.n == 0) return AL_OK;
  k_export_neighbors<TF><<<blocks_for(gs.n, kBlock), kBlock, 0, st>>>(
      c, g.cap_nbr, gs.n, gs.perm, gs.inv, xs, nbr, ncount, rho_sorted, particle_neighbors,
      particle_num_neighbors, particle_density);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

#define ALB_INST(TF, BK)                                                                  \
  template int build_neighbors_density<TF, BK<TF>>(                                       \
      const Cn<TF>&, const GridDims&, const GridState&, const vec4<TF>*, const BK<TF>&,    \
      uint32_t*, uint32_t*, TF*, TF*, TF*, cudaStream_t);
ALB_INST(float, RefBoundaryKernel)
ALB_INST(double, RefBoundaryKernel)
ALB_INST(float, SortedBoundaryKernel)
ALB_INST(double, SortedBoundaryKernel)
#undef ALB_INST
template int export_neighbors<float>(const Cn<float>&, const GridDims&, const GridState&,
                                     const vec4<float>*,
                                     const uint32_t*, const uint32_t*, const float*, float*,
                                     uint32_t*, float*, cudaStream_t);
template int export_neighbors<double>(const Cn<double>&, const GridDims&, const GridState&,
                                      const vec4<double>*,
                                      const uint32_t*, const uint32_t*, const double*, double*,
                                      uint32_t*, double*, cudaStream_t);

}  // namespace alb
