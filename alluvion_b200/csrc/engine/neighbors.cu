// neighbors.cu -- neighbor-list build with fused density, and export to the
// reference layout.
#include "neighbors.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

// Two phases per particle.  Phase 1 walks the 3x3 rows of z-contiguous
// cells around the particle's cell and appends every candidate closer than
// h to the list, in ascending sorted index; its accept branch is a store and
// an increment, so the warp pays little when its lanes accept different
// candidates (about 1 in 7 is accepted).  Phase 2 walks the compact list in
// the same order and evaluates W (and grad W for the DFSPH factor) only
// for neighbors, four list entries in flight at a time.  Both phases form
// d and |d|^2 with the same rounded operations, so phase 2 sees the
// distances phase 1 accepted.
template <class TF, class BK, bool FACTOR>
__global__ void __launch_bounds__(kBlock)
    k_build_neighbors(Cn<TF> c, GridDims g, const uint32_t* __restrict__ cell_start,
                      const vec4<TF>* __restrict__ xs, uint32_t n, BK bk,
                      uint32_t* __restrict__ nbr, uint32_t* __restrict__ ncount,
                      TF* __restrict__ rho, TF* __restrict__ alpha, TF* __restrict__ rho_rec,
                      uint32_t* __restrict__ flags) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const vec3<TF> xi = xyz(xs[s]);
  int ip[3];
  cell_coords(c.h, g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  const int z1 = min(ip[2] + 1, int(g.res[2]) - 1);
  uint32_t cnt = 0;
  // ---- phase 1: candidates -> list
  if (z0 <= z1) {
    for (int dx = -1; dx <= 1; ++dx) {
      const int cx = ip[0] + dx;
      if (cx < 0 || cx >= int(g.res[0])) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int cy = ip[1] + dy;
        if (cy < 0 || cy >= int(g.res[1])) continue;
        const uint32_t b = cell_start[cell_linear(g, cx, cy, z0)];
        const uint32_t e = cell_start[cell_linear(g, cx, cy, z1) + 1];
        for (uint32_t t = b; t < e; ++t) {
          const TF d2 = dist2_rn(xi, xyz(__ldg(xs + t)));
          if (d2 < c.h2 && t != s) {
            if (cnt < g.cap_nbr) nbr[size_t(cnt) * n + s] = t;
            ++cnt;
          }
        }
      }
    }
  }
  if (cnt > g.cap_nbr) {
    flags[2] = 1u;
    cnt = g.cap_nbr;
  }
  ncount[s] = cnt;
  // ---- phase 2: density (+ factor) over the list, in list order
  TF density = c.vol * c.w0;
  TF sum_grad = 0;
  vec3<TF> grad_i{0, 0, 0};
  constexpr uint32_t kB = 4;
  for (uint32_t k0 = 0; k0 < cnt; k0 += kB) {
    uint32_t t[kB];
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q)  // this thread's own stores: plain loads
      t[q] = k0 + q < cnt ? nbr[size_t(k0 + q) * n + s] : s;
    vec3<TF> xj[kB];
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q) xj[q] = xyz(__ldg(xs + t[q]));
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q) {
      if (k0 + q >= cnt) break;
      density += c.vol * W_r2(c, dist2_rn(xi, xj[q]));
      if (FACTOR) {
        const vec3<TF> d{sub_rn(xi.x, xj[q].x), sub_rn(xi.y, xj[q].y), sub_rn(xi.z, xj[q].z)};
        const vec3<TF> gpj = (-c.vol) * gradW(c, d);
        sum_grad += length_sqr(gpj);
        grad_i -= gpj;
      }
    }
  }
  density += bk.density_term(s);
  rho[s] = density * c.rho0;
  if (rho_rec) rho_rec[size_t(s) * kRecStride] = density * c.rho0;
  if (FACTOR) {
    grad_i += bk.grad_term(s);
    sum_grad += length_sqr(grad_i);
    alpha[s] = sum_grad > c.eps ? TF(-1) / sum_grad : TF(0);
  }
}

template <class TF>
__global__ void k_export_neighbors(uint32_t cap, uint32_t n, const uint32_t* __restrict__ perm,
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
    e[0] = sub_rn(xi.x, xj.x);
    e[1] = sub_rn(xi.y, xj.y);
    e[2] = sub_rn(xi.z, xj.z);
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
  if (alpha)
    k_build_neighbors<TF, BK, true><<<blocks_for(gs.n, kBlock), kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags);
  else
    k_build_neighbors<TF, BK, false><<<blocks_for(gs.n, kBlock), kBlock, 0, st>>>(
        c, g, gs.cell_start, xs, gs.n, bk, nbr, ncount, rho, alpha, rho_rec, gs.flags);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int export_neighbors(const GridDims& g, const GridState& gs, const vec4<TF>* xs,
                     const uint32_t* nbr, const uint32_t* ncount, const TF* rho_sorted,
                     TF* particle_neighbors, uint32_t* particle_num_neighbors,
                     TF* particle_density, cudaStream_t st) {
  if (gs.n == 0) return AL_OK;
  k_export_neighbors<TF><<<blocks_for(gs.n, kBlock), kBlock, 0, st>>>(
      g.cap_nbr, gs.n, gs.perm, gs.inv, xs, nbr, ncount, rho_sorted, particle_neighbors,
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
template int export_neighbors<float>(const GridDims&, const GridState&, const vec4<float>*,
                                     const uint32_t*, const uint32_t*, const float*, float*,
                                     uint32_t*, float*, cudaStream_t);
template int export_neighbors<double>(const GridDims&, const GridState&, const vec4<double>*,
                                      const uint32_t*, const uint32_t*, const double*, double*,
                                      uint32_t*, double*, cudaStream_t);

}  // namespace alb
