// pellet_relax.cu -- SolverPellet<TF>::step<wrap> (solver_pellet.hpp:57-119):
// the reference's relaxation that spreads boundary particles over a body.
// Each step sorts the particles into the grid, builds canonical neighbor
// lists of sorted slots with the pellet-branch density fused, then runs the
// cohesion / adhesion displacement, the DFSPH factor, one divergence
// iteration on the displacement with the max |dx|^2 reduced on the device
// (the last block forms the step's CFL fraction), and the boundary-avoiding
// move written back in original order.  One thread per particle in cell
// order.
#include <cfloat>
#include <cstring>

#include "body_geometry.cuh"
#include "boundary.cuh"
#include "engine.hpp"
#include "grid.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

template <class TF>
struct RelaxState {
  uint32_t n = 0, cap = 0;
  const vec4<TF>* xs = nullptr;  // sorted positions
  const uint32_t* perm = nullptr;
  uint32_t* nbr = nullptr;       // [cap][n] sorted slots
  uint32_t* cnt = nullptr;
  TF* rho = nullptr;             // sorted
  TF* factor = nullptr;          // sorted
  TF* dx = nullptr;              // sorted [n][3]
  unsigned long long* vmax = nullptr;  // max |dx|^2 as ordered bits
  uint32_t* ticket = nullptr;
  TF* cfl = nullptr;             // the step's CFL fraction
};

struct RelaxCoef {
  double cohesion, adhesion, cfl_factor, tolerance;
};

template <class TF>
__device__ __forceinline__ vec3<TF> lds(const TF* p, uint32_t s) {
  return vec3<TF>{p[3 * size_t(s)], p[3 * size_t(s) + 1], p[3 * size_t(s) + 2]};
}
template <class TF>
__device__ __forceinline__ void sts(TF* p, uint32_t s, vec3<TF> v) {
  p[3 * size_t(s)] = v.x;
  p[3 * size_t(s) + 1] = v.y;
  p[3 * size_t(s) + 2] = v.z;
}

// The body's signed distance (times sign) and outward normal at x, as the
// relaxation kernels read them: the distance grid (interpolate_and_derive,
// normal scaled by sign / |n|) for a mesh body, else the analytic distance
// minus the contact tolerance with the finite-difference normal of step
// 1e-3 (runner.hpp:2476-2479, 2509-2524, 4016-4018, 4045-4056).
template <class TF>
__device__ __forceinline__ bool body_distance(const BodyDev<TF>& b, TF tolerance, vec3<TF> x,
                                              TF& dist, vec3<TF>& normal) {
  if (b.shape == AL_SHAPE_MESH) {
    TF phi;
    vec3<TF> g;
    if (!interpolate_grid_gradient(b, b.dist, x, phi, g)) return false;
    dist = phi * b.sign;
    const TF nl2 = length_sqr(g);
    normal = (b.sign * (nl2 > TF(0) ? rsqrt_(nl2) : TF(0))) * g;
    return true;
  }
  dist = shape_sdf(b, x) * b.sign - tolerance;
  normal = shape_gradient(b, x, TF(1e-3)) * b.sign;
  return true;
}

// make_bead_pellet_neighbor_list without pellets and
// compute_density_with_pellets: rho = m (W(0) + sum_j W).
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_relax_lists(Cn<TF> c, GridDims g, const uint32_t* __restrict__ cell_start, RelaxState<TF> S,
                  uint32_t* flags) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const vec3<TF> xi = xyz(S.xs[s]);
  int ip[3];
  cell_coords(c.h, g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  const int z1 = min(ip[2] + 1, int(g.res[2]) - 1);
  uint32_t cnt = 0;
  TF wsum = 0;
  if (z0 <= z1) {
    for (int dx = -1; dx <= 1; ++dx) {
      const int cx = ip[0] + dx;
      if (cx < 0 || cx >= int(g.res[0])) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int cy = ip[1] + dy;
        if (c.wrap) {
          if (cy >= int(g.res[1]))
            cy -= int(g.res[1]);
          else if (cy < 0)
            cy += int(g.res[1]);
        }
        if (cy < 0 || cy >= int(g.res[1])) continue;
        const uint32_t b = cell_start[cell_linear(g, cx, cy, z0)];
        const uint32_t e = cell_start[cell_linear(g, cx, cy, z1) + 1];
        for (uint32_t t = b; t < e; ++t) {
          if (t == s) continue;
          const TF d2 = pdist2(c, xi, xyz(S.xs[t]));
          if (!(d2 < c.h2)) continue;
          if (cnt < S.cap) {
            S.nbr[size_t(cnt) * S.n + s] = t;
            wsum += W_r2(c, d2);
          }
          ++cnt;
        }
      }
    }
  }
  if (cnt > S.cap) {
    flags[2] = 1u;
    cnt = S.cap;
  }
  S.cnt[s] = cnt;
  S.rho[s] = (c.w0 + wsum) * c.mass;
}

// compute_cohesion_adhesion_displacement (runner.hpp:2453-2532).
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_relax_displacement(Cn<TF> c, BodyDev<TF> b, RelaxCoef k, RelaxState<TF> S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const vec3<TF> xi = xyz(S.xs[s]);
  const TF coh = TF(k.cohesion), adh = TF(k.adhesion);
  vec3<TF> dx{0, 0, 0};
  const uint32_t cnt = S.cnt[s];
  for (uint32_t q = 0; q < cnt; ++q) {
    const uint32_t t = S.nbr[size_t(q) * S.n + s];
    const vec3<TF> d = pdisp(c, xi, xyz(S.xs[t]));
    const TF w = W_r2(c, length_sqr(d));
    dx -= (coh * c.mass / S.rho[t] * (TF(1) - c.radius * TF(2) * rsqrt_(length_sqr(d))) * w) * d;
  }
  TF dist;
  vec3<TF> n;
  if (body_distance(b, TF(k.tolerance), xi, dist, n)) {
    const TF nn = length_sqr(n);
    if (b.shape == AL_SHAPE_MESH || nn >= TF(1e-7))
      dx -= (adh * c.mass / S.rho[s] * W_dist(c, dist)) * (dist * (rsqrt_(nn) * n));
  }
  sts(S.dx, s, dx);
}

// compute_dfsph_factor_with_pellets (runner.hpp:3156-3190) without pellets.
template <class TF>
__global__ void __launch_bounds__(kBlock) k_relax_factor(Cn<TF> c, RelaxState<TF> S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const vec3<TF> xi = xyz(S.xs[s]);
  TF sum = 0;
  vec3<TF> gi{0, 0, 0};
  const uint32_t cnt = S.cnt[s];
  for (uint32_t q = 0; q < cnt; ++q) {
    const uint32_t t = S.nbr[size_t(q) * S.n + s];
    const vec3<TF> gp = (-c.vol) * gradW(c, pdisp(c, xi, xyz(S.xs[t])));
    sum += length_sqr(gp);
    gi -= gp;
  }
  sum += length_sqr(gi);
  S.factor[s] = sum > c.eps ? TF(-1) / sum : TF(0);
}

// pellet_divergence_solve_iteration (runner.hpp:3365-3395) and the max of
// |dx|^2; the last block forms cfl = min(cfl_factor 0.4 2r / max|dx|, 1)
// (solver_pellet.hpp:100-103).
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_relax_divergence(Cn<TF> c, RelaxCoef k, RelaxState<TF> S, TF* dx_out) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  TF v2 = 0;
  if (s < S.n) {
    const vec3<TF> xi = xyz(S.xs[s]);
    const TF ki = (S.rho[s] / c.rho0 - TF(1)) * S.factor[s];
    vec3<TF> dx = lds(S.dx, s);
    const uint32_t cnt = S.cnt[s];
    for (uint32_t q = 0; q < cnt; ++q) {
      const uint32_t t = S.nbr[size_t(q) * S.n + s];
      const TF kj = (S.rho[t] / c.rho0 - TF(1)) * S.factor[t];
      const TF ks = ki + kj;
      if (fabs(ks) > c.eps) dx -= ks * ((-c.vol) * gradW(c, pdisp(c, xi, xyz(S.xs[t]))));
    }
    sts(dx_out, s, dx);
    v2 = length_sqr(dx);
  }
  __shared__ TF wmax[kBlock / 32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x == 0) {
    TF bm = wmax[0];
    for (int w = 1; w < kBlock / 32; ++w) bm = fmax(bm, wmax[w]);
    unsigned long long bits;
    if constexpr (sizeof(TF) == 4)
      bits = __float_as_uint(bm);
    else
      bits = (unsigned long long)__double_as_longlong(bm);
    atomicMax(S.vmax, bits);
    __threadfence();
    last = atomicAdd(S.ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const unsigned long long bits = atomicAdd(S.vmax, 0ull);
    TF m;
    if constexpr (sizeof(TF) == 4)
      m = __uint_as_float(uint32_t(bits));
    else
      m = __longlong_as_double((long long)bits);
    const TF f = TF(k.cfl_factor) * TF(0.4) * c.radius * TF(2) * (TF(1) / sqrt(m));
    *S.cfl = fmin(f, TF(1));
    *S.vmax = 0ull;
    *S.ticket = 0u;
  }
}

// move_and_avoid_boundary<wrap> (runner.hpp:4010-4066), written to the
// caller's arrays in original order.
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_relax_move(Cn<TF> c, BodyDev<TF> b, RelaxCoef k, RelaxState<TF> S, const TF* dx_sorted,
                 TF* __restrict__ x_ref, TF* __restrict__ dx_ref, TF* __restrict__ rho_ref) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const TF cfl = *S.cfl;
  const vec3<TF> d = lds(dx_sorted, s);
  vec3<TF> x = xyz(S.xs[s]) + d * cfl;
  TF dist;
  vec3<TF> n;
  if (body_distance(b, TF(k.tolerance), x, dist, n) && dist < c.radius)
    x += (c.radius - dist) * (rsqrt_(length_sqr(n)) * n);
  x.y = wrap_y(c, x.y);
  const uint32_t i = S.perm[s];
  sts(x_ref, i, x);
  if (dx_ref) sts(dx_ref, i, d);
  if (rho_ref) rho_ref[i] = S.rho[s];
}

template <class TF>
struct RelaxTypes;
template <>
struct RelaxTypes<float> {
  using cn = al_const_f32;
  using body = al_body_f32;
};
template <>
struct RelaxTypes<double> {
  using cn = al_const_f64;
  using body = al_body_f64;
};

template <class TF>
int relax(al_engine* e, const typename RelaxTypes<TF>::cn* cn, const al_consti* cni,
          const typename RelaxTypes<TF>::body* body, TF* x, uint32_t n,
          const al_pellet_relax_params* p, uint32_t steps, TF* dx_ref, TF* rho_ref,
          cudaStream_t st) {
  ALB_CHECK_ARG(e && cn && cni && body && p, "al_relax_pellets: null argument");
  ALB_CHECK_ARG(n == 0 || x, "al_relax_pellets: particle_x is null");
  ALB_CHECK_ARG(!p->wrap_y || p->wrap_length > 0, "al_relax_pellets: wrap_y needs a length");
  BodyDev<TF> b = to_body_dev<TF>(*body);
  if (b.shape == AL_SHAPE_MESH) {
    b.use_grid = 1;
    ALB_TRY(validate_body(b, true, false));
  } else {
    b.use_grid = 0;
    ALB_CHECK_ARG(b.shape <= AL_SHAPE_INFINITE_TUBE, "al_relax_pellets: unknown shape");
  }
  ALB_TRY(e->activate());
  if (n == 0 || steps == 0) return AL_OK;
  struct NsReset {
    al_engine* e;
    ~NsReset() { e->ns.clear(); }
  } reset{e};
  e->ns = "relax.";
  Cn<TF> c = to_cn<TF>(*cn);
  if (p->wrap_y) set_wrap(c, TF(p->wrap_length));
  const GridDims g = to_dims(*cni);
  const RelaxCoef k{p->cohesion, p->adhesion, p->cfl_factor, p->contact_tolerance};
  RelaxState<TF> S;
  S.n = n;
  S.cap = g.cap_nbr;
  vec4<TF>* xs = nullptr;
  uint32_t* flags = nullptr;
  TF* dx_new = nullptr;
  ALB_TRY(e->buf("sorted.x", n, &xs));
  ALB_TRY(e->buf("flags", 4, &flags));
  ALB_TRY(e->buf("nbr", size_t(n) * S.cap, &S.nbr));
  ALB_TRY(e->buf("cnt", n, &S.cnt));
  ALB_TRY(e->buf("rho", n, &S.rho));
  ALB_TRY(e->buf("factor", n, &S.factor));
  ALB_TRY(e->buf("dx", size_t(n) * 3, &S.dx));
  ALB_TRY(e->buf("dx_new", size_t(n) * 3, &dx_new));
  ALB_TRY(e->buf("vmax", 1, &S.vmax));
  ALB_TRY(e->buf("ticket", 1, &S.ticket));
  ALB_TRY(e->buf("cfl", 1, &S.cfl));
  S.xs = xs;
  ALB_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), st));
  ALB_CUDA(cudaMemsetAsync(S.vmax, 0, sizeof(unsigned long long), st));
  ALB_CUDA(cudaMemsetAsync(S.ticket, 0, sizeof(uint32_t), st));
  const uint32_t blocks = blocks_for(n, kBlock);
  for (uint32_t it = 0; it < steps; ++it) {
    const bool last = it + 1 == steps;
    GridState gs;
    ALB_LAUNCH(e, "relax_grid", kGridBuildKernels, st,
               ALB_TRY(grid_build<TF>(e, c, g, x, n, xs, flags, gs, st)));
    S.perm = gs.perm;
    ALB_LAUNCH(e, "relax_lists", 1, st,
               (k_relax_lists<TF><<<blocks, kBlock, 0, st>>>(c, g, gs.cell_start, S, flags)));
    ALB_LAUNCH(e, "relax_displacement", 1, st,
               (k_relax_displacement<TF><<<blocks, kBlock, 0, st>>>(c, b, k, S)));
    ALB_LAUNCH(e, "relax_factor", 1, st, (k_relax_factor<TF><<<blocks, kBlock, 0, st>>>(c, S)));
    ALB_LAUNCH(e, "relax_divergence", 1, st,
               (k_relax_divergence<TF><<<blocks, kBlock, 0, st>>>(c, k, S, dx_new)));
    ALB_LAUNCH(e, "relax_move", 1, st,
               (k_relax_move<TF><<<blocks, kBlock, 0, st>>>(c, b, k, S, dx_new, x,
                                                            last ? dx_ref : nullptr,
                                                            last ? rho_ref : nullptr)));
  }
  ALB_CUDA(cudaGetLastError());
  uint32_t hf[4];
  ALB_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  e->flush_stats();
  if (hf[0]) return AL_ERR_OUT_OF_GRID;
  if (hf[1]) return AL_ERR_CELL_OVERFLOW;
  if (hf[2]) return AL_ERR_NEIGHBOR_OVERFLOW;
  return AL_OK;
}

}  // namespace

}  // namespace alb

using namespace alb;

extern "C" {

int al_relax_pellets_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                         const al_body_f32* body, float* particle_x, uint32_t num_particles,
                         const al_pellet_relax_params* params, uint32_t steps,
                         float* particle_dx, float* particle_density, void* stream) {
  return relax<float>(engine, cn, cni, body, particle_x, num_particles, params, steps,
                      particle_dx, particle_density, static_cast<cudaStream_t>(stream));
}
int al_relax_pellets_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                         const al_body_f64* body, double* particle_x, uint32_t num_particles,
                         const al_pellet_relax_params* params, uint32_t steps,
                         double* particle_dx, double* particle_density, void* stream) {
  return relax<double>(engine, cn, cni, body, particle_x, num_particles, params, steps,
                       particle_dx, particle_density, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
