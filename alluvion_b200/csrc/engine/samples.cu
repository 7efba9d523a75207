// samples.cu -- fluid statistics at sample points and the reference's
// post-processing reductions, in float and double (Runner<float> and
// Runner<double>; the _f64 entries take the same arguments in double):
//   al_sample_fluid_f32      make_neighbor_list over sample_x
//                            (runner.hpp:1869-1911) followed by sample_fluid,
//                            sample_fluid_density, sample_position_density,
//                            compute_sample_velocity, compute_sample_vorticity
//                            (runner.hpp:4173-4323, 2100-2121)
//   al_density_mask_f32      compute_density_mask (runner.hpp:4359-4365)
//   al_boundary_mask_f32     compute_boundary_mask (runner.hpp:4367-4396)
//   al_distance_mask_multiple_f32
//                            compute_distance_mask_multiple (4272-4287)
//   al_histogram256_f32      quantize + histogram256[_with_mask] +
//                            merge_histogram256 (runner.hpp:4399-4536)
//   al_kl_divergence         calculate_kl_divergence (runner.hpp:4803-4815)
//
// Sampling: the particles, and the samples, are sorted into the engine's
// grid; threads take samples in cell order (a warp's samples read the same
// cells) and each walks the 3x3 rows of z-contiguous cells around its cell
// in canonical (cell, index) order and sums directly, so no sample neighbor
// list is stored.  As in the reference, whose neighbor kernel skips the candidate
// whose index equals the point's own (p_j != p_i, runner.hpp:1895),
// particle s is left out of sample s's sums.  With wrap_y the rows follow
// the reference's (dx, dy, dz) offset order, cells and displacements
// wrapped in y (make_neighbor_list<1>).  More than
// max_num_neighbors_per_particle neighbors raise the neighbor-overflow
// anomaly; the first ones in canonical order are summed.
//
// Histogram: one pass over v (HBM-bound, 4 B per value, 8 with a mask):
// 16-byte vector loads, per-warp shared-memory bins, one global atomicAdd
// per bin and block.  Integer counts make the result independent of the
// order of the atomics.
#include <cmath>

#include "body_geometry.cuh"
#include "boundary.cuh"
#include "engine.hpp"
#include "grid.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

template <class TF>
struct SampleDev {
  const TF* x;    // [S][3]
  uint32_t num;
  uint32_t qdim;
  const TF* rho;  // [N] particle density (original order)
  const TF* v;    // [N][3]
  const TF* q;    // [N][qdim]
  const TF* bnd;  // [nb][S][4] {x_b, V}
  const TF* bker; // [nb][S][4] {grad W V, W V}
  TF* density;    // [S]
  TF* pdensity;   // [S]
  TF* quantity;   // [S][qdim]
  TF* vel;        // [S][3]
  TF* vort;       // [S][3]
  uint32_t wrap;  // periodic in y
  TF wrap_length, wrap_min, wrap_max;
  uint32_t nbead; // points j < nbead are particles, the rest pellets
  uint32_t npel;  // pellets (0: volume-map bodies, if any)
  const TF* pv;   // [npel][3] pellet velocities
};

// wrap_y (runner.hpp:698-707) of a displacement's y component.
template <class TF>
__device__ __forceinline__ TF wrap_dy(const SampleDev<TF>& sd, TF dy) {
  if (dy >= sd.wrap_max) return sub_rn(dy, sd.wrap_length);
  if (dy < sd.wrap_min) return add_rn(dy, sd.wrap_length);
  return dy;
}

// Velocity of body b at the boundary point of sample s.
template <class TF>
__device__ __forceinline__ vec3<TF> body_velocity(const SampleDev<TF>& sd,
                                                  const RigidDev<TF>& r, uint32_t b,
                                                  uint32_t s) {
  const TF* bx = sd.bnd + (size_t(b) * sd.num + s) * 4;
  return cross(r.omega, vec3<TF>{bx[0], bx[1], bx[2]} - r.x) + r.v;
}

// Threads per block of the sampling kernel (one sample per thread; 256
// measured faster than the particle passes' 128 on the 1 M-sample case).
constexpr int kSampleBlock = 256;

// VORT = false: densities, quantity, velocity; VORT = true: vorticity
// (reads the samples' velocities written by the first pass).
template <class TF, bool VORT>
__global__ void __launch_bounds__(kSampleBlock)
    k_sample(Cn<TF> c, GridDims g, const uint32_t* __restrict__ cell_start,
             const vec4<TF>* __restrict__ xs, const uint32_t* __restrict__ perm,
             const vec4<TF>* __restrict__ sample_xs, const uint32_t* __restrict__ sample_perm,
             SampleDev<TF> sd, const RigidDev<TF>* __restrict__ rigid, uint32_t* flags) {
  using V3 = vec3<TF>;
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 >= sd.num) return;
  // samples in cell order: a warp's samples share cells
  const uint32_t s = __ldg(sample_perm + t0);
  const V3 xi = xyz(__ldg(sample_xs + t0));
  const V3 vi = VORT ? ld3(sd.vel, s) : V3{0, 0, 0};
  int ip[3];
  cell_coords(c.h, g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  const int z1 = min(ip[2] + 1, int(g.res[2]) - 1);
  const bool want_w = !VORT && (sd.density || sd.pdensity);
  TF dens = 0;
  TF qs[3] = {0, 0, 0};
  V3 vel{0, 0, 0}, vort{0, 0, 0};
  // pellet terms (the *_with_pellets kernels): sum W, V W v_p, V (v_p - v_s) x grad W
  TF wb = 0, wp = 0;
  V3 velp{0, 0, 0}, vortp{0, 0, 0};
  uint32_t cnt = 0, cntp = 0;
  if (z0 <= z1) {
    for (int dx = -1; dx <= 1; ++dx) {
      const int cx = ip[0] + dx;
      if (cx < 0 || cx >= int(g.res[0])) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int cy = ip[1] + dy;
        if (sd.wrap) {  // wrap_ipos_y: one period either way
          if (cy >= int(g.res[1]))
            cy -= int(g.res[1]);
          else if (cy < 0)
            cy += int(g.res[1]);
        }
        if (cy < 0 || cy >= int(g.res[1])) continue;
        const uint32_t b = cell_start[cell_linear(g, cx, cy, z0)];
        const uint32_t e = cell_start[cell_linear(g, cx, cy, z1) + 1];
        for (uint32_t t = b; t < e; ++t) {
          const uint32_t j = __ldg(perm + t);
          if (j == s) continue;  // the reference's p_j != p_i
          const V3 xj = xyz(__ldg(xs + t));
          V3 d{sub_rn(xi.x, xj.x), sub_rn(xi.y, xj.y), sub_rn(xi.z, xj.z)};
          if (sd.wrap) d.y = wrap_dy(sd, d.y);
          const TF d2 = add_rn(add_rn(mul_rn(d.x, d.x), mul_rn(d.y, d.y)), mul_rn(d.z, d.z));
          if (!(d2 < c.h2)) continue;
          if (j >= sd.nbead) {  // a pellet
            if (cntp++ >= g.cap_nbr) continue;
            const V3 vp = ld3(sd.pv, j - sd.nbead);
            if (!VORT) {
              const TF w = W_r2(c, d2);
              wp += w;
              if (sd.vel) velp += (c.vol * w) * vp;
            } else {
              vortp += c.vol * cross(vp - vi, gradW(c, d));
            }
            continue;
          }
          if (cnt++ >= g.cap_nbr) continue;
          if (!VORT) {
            const TF w = W_r2(c, d2);
            if (want_w) dens += c.vol * w;
            if (sd.npel) wb += w;
            if (sd.quantity || sd.vel) {
              const TF mrw = c.mass / __ldg(sd.rho + j) * w;
              for (uint32_t k = 0; k < sd.qdim; ++k) qs[k] += mrw * __ldg(sd.q + size_t(j) * sd.qdim + k);
              if (sd.vel) vel += mrw * ld3(sd.v, j);
            }
          } else {
            vort += (c.mass / __ldg(sd.rho + j)) * cross(ld3(sd.v, j) - vi, gradW(c, d));
          }
        }
      }
    }
  }
  if (cnt > g.cap_nbr || cntp > g.cap_nbr) flags[2] = 1u;
  // pellet sums after the particles' (the reference's list order)
  vel += velp;
  vort += vortp;
  // volume-map body terms (runner.hpp:2116-2118, 4228-4236, 4310-4321)
  TF bw = 0;
  for (uint32_t b = 0; b < (sd.npel ? 0u : g.nb); ++b) {
    const TF* bk = sd.bker + (size_t(b) * sd.num + s) * 4;
    if (!VORT) {
      bw += bk[3];
      if (sd.vel) vel += bk[3] * body_velocity(sd, rigid[b], b, s);
    } else {
      vort += cross(body_velocity(sd, rigid[b], b, s) - vi, V3{bk[0], bk[1], bk[2]});
    }
  }
  if (!VORT) {
    if (sd.density) sd.density[s] = dens * c.rho0;
    if (sd.pdensity)  // sample_position_density[_with_pellets]
      sd.pdensity[s] = sd.npel ? (wb + wp) * c.mass : (dens + bw) * c.rho0;
    if (sd.quantity)
      for (uint32_t k = 0; k < sd.qdim; ++k) sd.quantity[size_t(s) * sd.qdim + k] = qs[k];
    if (sd.vel) st3(sd.vel, s, vel);
  } else {
    st3(sd.vort, s, vort);
  }
}

template <class TF>
__global__ void k_density_mask(const TF* __restrict__ density, uint32_t n, uint32_t* mask) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) mask[i] = density[i] > TF(0);
}

// Mesh bodies use the distance grid, analytic shapes their distance
// function (the dispatch of launch_compute_boundary_mask).
template <class TF>
__global__ void k_boundary_mask(BodyDev<TF> b, RigidDev<TF> r, const TF* __restrict__ sx,
                                uint32_t n, TF threshold, TF* mask) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vec4<TF> qc{-r.q.x, -r.q.y, -r.q.z, r.q.w};
  const vec3<TF> local = rotate(ld3(sx, i) - r.x, qc);
  const TF d =
      (b.shape == AL_SHAPE_MESH ? interpolate_grid(b, b.dist, local) : shape_sdf(b, local)) *
      b.sign;
  mask[i] *= TF(d >= threshold);
}

template <class TF>
__global__ void k_distance_mask_multiple(const TF* __restrict__ gx, uint32_t n,
                                         const TF* __restrict__ buoy, uint32_t nbuoy, TF thr2,
                                         TF* mask) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vec3<TF> x = ld3(gx, i);
  for (uint32_t k = 0; k < nbuoy; ++k)
    mask[size_t(k) * n + i] = TF(length_sqr(ld3(buoy, k) - x) <= thr2);
}

constexpr int kHistBlock = 256;
constexpr int kHistWarps = kHistBlock / 32;

// quantize (runner.hpp:4516-4536): low byte of floor((v - v_min) * step_inverse)
// saturated to uint32.  In double the product reaches __float2uint_rd through
// the implicit conversion to float, as in quantize<double>.
__device__ __forceinline__ uint32_t quantize_byte(float v, float v_min, float step_inverse) {
  return __float2uint_rd(__fmul_rn(__fsub_rn(v, v_min), step_inverse)) & 0xFFu;
}
__device__ __forceinline__ uint32_t quantize_byte(double v, double v_min, double step_inverse) {
  return __float2uint_rd(__double2float_rn(__dmul_rn(__dsub_rn(v, v_min), step_inverse))) &
         0xFFu;
}

// 16-byte vectors of values: 4 floats or 2 doubles.
template <class TF>
struct Vec16;
template <>
struct Vec16<float> {
  using T = float4;
  static constexpr int kN = 4;
  __device__ static float at(const float4& a, int i) {
    return i == 0 ? a.x : i == 1 ? a.y : i == 2 ? a.z : a.w;
  }
};
template <>
struct Vec16<double> {
  using T = double2;
  static constexpr int kN = 2;
  __device__ static double at(const double2& a, int i) { return i == 0 ? a.x : a.y; }
};

// VEC: v (and mask) are 16-byte aligned; vector k covers values
// kN k .. kN k + kN - 1.
template <class TF, bool MASK, bool VEC>
__global__ void __launch_bounds__(kHistBlock)
    k_histogram256(const TF* __restrict__ v, const TF* __restrict__ mask, uint32_t n, TF v_min,
                   TF step_inverse, uint32_t* hist) {
  using VT = Vec16<TF>;
  __shared__ uint32_t bins[kHistWarps][256];
  for (int k = threadIdx.x; k < kHistWarps * 256; k += kHistBlock) (&bins[0][0])[k] = 0;
  __syncthreads();
  uint32_t* wb = bins[threadIdx.x >> 5];
  const size_t stride = size_t(gridDim.x) * kHistBlock;
  const size_t tid = size_t(blockIdx.x) * kHistBlock + threadIdx.x;
  auto add = [&](TF x, TF m) {
    if (!MASK || m == TF(1)) atomicAdd(wb + quantize_byte(x, v_min, step_inverse), 1u);
  };
  size_t head = 0;
  if (VEC) {
    const size_t nv = n / VT::kN;
    const typename VT::T* vv = reinterpret_cast<const typename VT::T*>(v);
    const typename VT::T* mv = reinterpret_cast<const typename VT::T*>(mask);
    for (size_t k = tid; k < nv; k += stride) {
      const typename VT::T a = __ldcs(vv + k);
      typename VT::T m{};
      if (MASK) m = __ldcs(mv + k);
#pragma unroll
      for (int e = 0; e < VT::kN; ++e) add(VT::at(a, e), MASK ? VT::at(m, e) : TF(1));
    }
    head = nv * VT::kN;
  }
  for (size_t i = head + tid; i < n; i += stride) add(v[i], MASK ? mask[i] : TF(1));
  __syncthreads();
  for (int b = threadIdx.x; b < 256; b += kHistBlock) {
    uint32_t sum = 0;
#pragma unroll
    for (int w = 0; w < kHistWarps; ++w) sum += bins[w][b];
    if (sum) atomicAdd(hist + b, sum);
  }
}

constexpr int kKlBlock = 256;

// Fixed-order reduction: thread t sums bins t, t + 256, ... in order, then
// a shared-memory tree.
__global__ void __launch_bounds__(kKlBlock)
    k_kl_divergence(const uint32_t* __restrict__ p, const uint32_t* __restrict__ q, double inv,
                    double ratio, double lower, uint32_t num_bins, double* out) {
  __shared__ double part[kKlBlock];
  double sum = 0;
  for (uint32_t b = threadIdx.x; b < num_bins; b += kKlBlock) {
    const uint32_t fp = p[b];
    if (fp == 0) continue;
    sum += double(fp) * inv * log(double(fp) / fmax(double(q[b]), lower) * ratio);
  }
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int s = kKlBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = part[0];
}

}  // namespace

}  // namespace alb

namespace alb {
namespace {

template <class TF>
struct SampleTypes;
template <>
struct SampleTypes<float> {
  using cn = al_const_f32;
  using rigid = al_rigid_f32;
  using req = al_sample_f32;
  using body = al_body_f32;
};
template <>
struct SampleTypes<double> {
  using cn = al_const_f64;
  using rigid = al_rigid_f64;
  using req = al_sample_f64;
  using body = al_body_f64;
};

template <class TF>
int sample_fluid(al_engine* engine, const typename SampleTypes<TF>::cn* cn, const al_consti* cni,
                 const TF* particle_x, uint32_t num_particles,
                 const typename SampleTypes<TF>::rigid* rigid,
                 const typename SampleTypes<TF>::req* req, void* stream) {
  ALB_CHECK_ARG(engine && cn && cni && req, "al_sample_fluid: null argument");
  ALB_CHECK_ARG(num_particles == 0 || particle_x, "al_sample_fluid: particle_x is null");
  ALB_CHECK_ARG(req->num_samples == 0 || req->sample_x, "al_sample_fluid: sample_x is null");
  ALB_CHECK_ARG(!req->sample_quantity ||
                    ((req->quantity_dim == 1 || req->quantity_dim == 3) && req->particle_quantity),
                "al_sample_fluid: quantity_dim must be 1 or 3 with particle_quantity set");
  const bool need_rho = req->sample_quantity || req->sample_v || req->sample_vorticity;
  ALB_CHECK_ARG(num_particles == 0 || !need_rho || req->particle_density,
                "al_sample_fluid: particle_density is null");
  ALB_CHECK_ARG(!(req->sample_v || req->sample_vorticity) || req->particle_v,
                "al_sample_fluid: velocities need particle_v");
  ALB_CHECK_ARG(!req->sample_vorticity || req->sample_v,
                "al_sample_fluid: vorticity needs sample_v");
  ALB_CHECK_ARG(cni->num_boundaries <= AL_MAX_BOUNDARIES, "al_sample_fluid: too many bodies");
  ALB_CHECK_ARG(!req->wrap_y || req->wrap_length > TF(0),
                "al_sample_fluid: wrap_y needs a positive wrap_length");
  const uint32_t npel = req->num_pellets;
  ALB_CHECK_ARG(npel == 0 || (req->pellet_x && (req->pellet_v || !(req->sample_v ||
                                                                  req->sample_vorticity))),
                "al_sample_fluid: pellet_x / pellet_v are null");
  ALB_CHECK_ARG(uint64_t(num_particles) + npel < (1ull << 31), "al_sample_fluid: too many points");
  const bool body_terms = npel == 0 && (req->sample_position_density || req->sample_v);
  ALB_CHECK_ARG(cni->num_boundaries == 0 || !body_terms || req->sample_boundary_kernel,
                "al_sample_fluid: sample_boundary_kernel is null");
  ALB_CHECK_ARG(cni->num_boundaries == 0 || npel || !req->sample_v ||
                    (req->sample_boundary && rigid),
                "al_sample_fluid: velocities need sample_boundary and rigid");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (req->num_samples == 0) return AL_OK;
  struct NsReset {
    al_engine* e;
    ~NsReset() { e->ns.clear(); }
  } reset{engine};
  const Cn<TF> c = to_cn<TF>(*cn);
  GridDims g = to_dims(*cni);
  // the samples' own cell order (their out-of-grid / crowded-cell flags are
  // not anomalies: the reference bins no samples)
  engine->ns = "sample.points.";
  vec4<TF>* sxs = nullptr;
  uint32_t* sflags = nullptr;
  ALB_TRY(engine->buf("sorted.x", req->num_samples, &sxs));
  ALB_TRY(engine->buf("flags", 4, &sflags));
  ALB_CUDA(cudaMemsetAsync(sflags, 0, 4 * sizeof(uint32_t), st));
  GridState ss;
  ALB_LAUNCH(engine, "sample_sort", kGridBuildKernels, st,
             ALB_TRY(grid_build<TF>(engine, c, g, req->sample_x, req->num_samples, sxs, sflags,
                                    ss, st)));
  engine->ns = "sample.";
  vec4<TF>* xs = nullptr;
  uint32_t* flags = nullptr;
  RigidDev<TF>* dr = nullptr;
  ALB_TRY(engine->buf("sorted.x", num_particles ? num_particles : 1, &xs));
  ALB_TRY(engine->buf("flags", 4, &flags));
  ALB_TRY(engine->buf("rigid", AL_MAX_BOUNDARIES, &dr));
  ALB_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), st));
  if (g.nb && req->sample_v && npel == 0) {
    RigidDev<TF> hr[AL_MAX_BOUNDARIES];
    for (uint32_t b = 0; b < g.nb; ++b) hr[b] = to_rigid_dev<TF>(rigid[b]);
    ALB_CUDA(cudaMemcpyAsync(dr, hr, sizeof(RigidDev<TF>) * g.nb, cudaMemcpyHostToDevice, st));
  }
  // with pellets, one grid over particles and pellets (pellets after the
  // particles, as the reference stores them)
  const TF* grid_x = particle_x;
  const uint32_t npts = num_particles + npel;
  if (npel) {
    TF* all = nullptr;
    ALB_TRY(engine->buf("all.x", size_t(npts) * 3, &all));
    if (num_particles)
      ALB_CUDA(cudaMemcpyAsync(all, particle_x, sizeof(TF) * 3 * num_particles,
                               cudaMemcpyDeviceToDevice, st));
    ALB_CUDA(cudaMemcpyAsync(all + size_t(num_particles) * 3, req->pellet_x,
                             sizeof(TF) * 3 * npel, cudaMemcpyDeviceToDevice, st));
    ALB_TRY(engine->buf("sorted.x", npts, &xs));
    grid_x = all;
  }
  GridState gs;
  ALB_LAUNCH(engine, "sample_grid", kGridBuildKernels, st,
             ALB_TRY(grid_build<TF>(engine, c, g, grid_x, npts, xs, flags, gs, st)));
  SampleDev<TF> sd{req->sample_x,
                   req->num_samples,
                   req->sample_quantity ? req->quantity_dim : 0u,
                   req->particle_density,
                   req->particle_v,
                   req->particle_quantity,
                   req->sample_boundary,
                   req->sample_boundary_kernel,
                   req->sample_density,
                   req->sample_position_density,
                   req->sample_quantity,
                   req->sample_v,
                   req->sample_vorticity,
                   req->wrap_y ? 1u : 0u,
                   TF(req->wrap_length),
                   TF(req->wrap_length) * TF(-0.5),
                   TF(req->wrap_length) * TF(0.5),
                   num_particles,
                   npel,
                   req->pellet_v};
  const uint32_t blocks = blocks_for(req->num_samples, kSampleBlock);
  GridDims g1 = g;
  if (!body_terms) g1.nb = 0;  // the first pass reads no body arrays
  ALB_LAUNCH(engine, "sample", 1, st,
             (k_sample<TF, false><<<blocks, kSampleBlock, 0, st>>>(c, g1, gs.cell_start, xs, gs.perm,
                                                             sxs, ss.perm, sd, dr, flags)));
  if (req->sample_vorticity)
    ALB_LAUNCH(engine, "sample_vorticity", 1, st,
               (k_sample<TF, true><<<blocks, kSampleBlock, 0, st>>>(c, g, gs.cell_start, xs, gs.perm,
                                                              sxs, ss.perm, sd, dr, flags)));
  ALB_CUDA(cudaGetLastError());
  uint32_t hf[4];
  ALB_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  if (hf[0]) return AL_ERR_OUT_OF_GRID;
  if (hf[1]) return AL_ERR_CELL_OVERFLOW;
  if (hf[2]) return AL_ERR_NEIGHBOR_OVERFLOW;
  return AL_OK;
}

template <class TF>
int density_mask(al_engine* engine, const TF* sample_density, uint32_t num_samples,
                 uint32_t* mask, void* stream) {
  ALB_CHECK_ARG(engine && (num_samples == 0 || (sample_density && mask)),
                "al_density_mask: null argument");
  ALB_TRY(engine->activate());
  if (num_samples == 0) return AL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ALB_LAUNCH(engine, "density_mask", 1, st,
             (k_density_mask<TF><<<blocks_for(num_samples, kBlock), kBlock, 0, st>>>(
                 sample_density, num_samples, mask)));
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int boundary_mask(al_engine* engine, const typename SampleTypes<TF>::body* body,
                  const typename SampleTypes<TF>::rigid* rigid, const TF* sample_x,
                  uint32_t num_samples, TF distance_threshold, TF* mask, void* stream) {
  ALB_CHECK_ARG(engine && body && rigid && (num_samples == 0 || (sample_x && mask)),
                "al_boundary_mask: null argument");
  const BodyDev<TF> b = to_body_dev<TF>(*body);
  ALB_TRY(validate_body(b, b.shape == AL_SHAPE_MESH, false));
  ALB_TRY(engine->activate());
  if (num_samples == 0) return AL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ALB_LAUNCH(engine, "boundary_mask", 1, st,
             (k_boundary_mask<TF><<<blocks_for(num_samples, kBlock), kBlock, 0, st>>>(
                 b, to_rigid_dev<TF>(*rigid), sample_x, num_samples, distance_threshold, mask)));
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int distance_mask_multiple(al_engine* engine, const TF* grid_x, uint32_t num_grid_points,
                           const TF* buoy_x, uint32_t num_buoys, TF distance_threshold, TF* mask,
                           void* stream) {
  ALB_CHECK_ARG(engine && (num_grid_points == 0 || num_buoys == 0 || (grid_x && buoy_x && mask)),
                "al_distance_mask_multiple: null argument");
  ALB_TRY(engine->activate());
  if (num_grid_points == 0 || num_buoys == 0) return AL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ALB_LAUNCH(engine, "distance_mask_multiple", 1, st,
             (k_distance_mask_multiple<TF><<<blocks_for(num_grid_points, kBlock), kBlock, 0, st>>>(
                 grid_x, num_grid_points, buoy_x, num_buoys,
                 distance_threshold * distance_threshold, mask)));
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int histogram256(al_engine* engine, const TF* v, const TF* mask, uint32_t n, TF v_min, TF v_max,
                 uint32_t* histogram, void* stream) {
  ALB_CHECK_ARG(engine && histogram && (n == 0 || v), "al_histogram256: null argument");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ALB_CUDA(cudaMemsetAsync(histogram, 0, 256 * sizeof(uint32_t), st));
  if (n == 0) return AL_OK;
  // launch_histogram256 (runner.hpp:5852-5853): the step in double, cast to TF
  const TF step_inverse =
      static_cast<TF>(256.0 / (static_cast<double>(v_max) - static_cast<double>(v_min)));
  const bool vec = (reinterpret_cast<uintptr_t>(v) & 15) == 0 &&
                   (!mask || (reinterpret_cast<uintptr_t>(mask) & 15) == 0);
  // enough resident blocks to cover the SMs, each thread about 16 values
  const uint32_t want = blocks_for((n + 15) / 16, kHistBlock);
  const uint32_t cap = uint32_t(engine->num_sms) * 8;
  const uint32_t grid = want < cap ? (want ? want : 1) : cap;
  ALB_LAUNCH(engine, "histogram256", 1, st, {
    if (mask) {
      if (vec)
        k_histogram256<TF, true, true><<<grid, kHistBlock, 0, st>>>(v, mask, n, v_min,
                                                                    step_inverse, histogram);
      else
        k_histogram256<TF, true, false><<<grid, kHistBlock, 0, st>>>(v, mask, n, v_min,
                                                                     step_inverse, histogram);
    } else {
      if (vec)
        k_histogram256<TF, false, true><<<grid, kHistBlock, 0, st>>>(v, nullptr, n, v_min,
                                                                     step_inverse, histogram);
      else
        k_histogram256<TF, false, false><<<grid, kHistBlock, 0, st>>>(v, nullptr, n, v_min,
                                                                      step_inverse, histogram);
    }
  });
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

}  // namespace
}  // namespace alb

using namespace alb;

extern "C" {

int al_sample_fluid_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                        const float* particle_x, uint32_t num_particles,
                        const al_rigid_f32* rigid, const al_sample_f32* req, void* stream) {
  return sample_fluid<float>(engine, cn, cni, particle_x, num_particles, rigid, req, stream);
}
int al_sample_fluid_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                        const double* particle_x, uint32_t num_particles,
                        const al_rigid_f64* rigid, const al_sample_f64* req, void* stream) {
  return sample_fluid<double>(engine, cn, cni, particle_x, num_particles, rigid, req, stream);
}

int al_density_mask_f32(al_engine* engine, const float* sample_density, uint32_t num_samples,
                        uint32_t* mask, void* stream) {
  return density_mask<float>(engine, sample_density, num_samples, mask, stream);
}
int al_density_mask_f64(al_engine* engine, const double* sample_density, uint32_t num_samples,
                        uint32_t* mask, void* stream) {
  return density_mask<double>(engine, sample_density, num_samples, mask, stream);
}

int al_boundary_mask_f32(al_engine* engine, const al_body_f32* body, const al_rigid_f32* rigid,
                         const float* sample_x, uint32_t num_samples, float distance_threshold,
                         float* mask, void* stream) {
  return boundary_mask<float>(engine, body, rigid, sample_x, num_samples, distance_threshold,
                              mask, stream);
}
int al_boundary_mask_f64(al_engine* engine, const al_body_f64* body, const al_rigid_f64* rigid,
                         const double* sample_x, uint32_t num_samples, double distance_threshold,
                         double* mask, void* stream) {
  return boundary_mask<double>(engine, body, rigid, sample_x, num_samples, distance_threshold,
                               mask, stream);
}

int al_distance_mask_multiple_f32(al_engine* engine, const float* grid_x,
                                  uint32_t num_grid_points, const float* buoy_x,
                                  uint32_t num_buoys, float distance_threshold, float* mask,
                                  void* stream) {
  return distance_mask_multiple<float>(engine, grid_x, num_grid_points, buoy_x, num_buoys,
                                       distance_threshold, mask, stream);
}
int al_distance_mask_multiple_f64(al_engine* engine, const double* grid_x,
                                  uint32_t num_grid_points, const double* buoy_x,
                                  uint32_t num_buoys, double distance_threshold, double* mask,
                                  void* stream) {
  return distance_mask_multiple<double>(engine, grid_x, num_grid_points, buoy_x, num_buoys,
                                        distance_threshold, mask, stream);
}

int al_histogram256_f32(al_engine* engine, const float* v, const float* mask, uint32_t n,
                        float v_min, float v_max, uint32_t* histogram, void* stream) {
  return histogram256<float>(engine, v, mask, n, v_min, v_max, histogram, stream);
}
int al_histogram256_f64(al_engine* engine, const double* v, const double* mask, uint32_t n,
                        double v_min, double v_max, uint32_t* histogram, void* stream) {
  return histogram256<double>(engine, v, mask, n, v_min, v_max, histogram, stream);
}

int al_kl_divergence(al_engine* engine, const uint32_t* histogram_p, const uint32_t* histogram_q,
                     uint32_t n_p, uint32_t n_q, double q_lower_bound, uint32_t num_bins,
                     double* result, void* stream) {
  ALB_CHECK_ARG(engine && result && (num_bins == 0 || (histogram_p && histogram_q)),
                "al_kl_divergence: null argument");
  ALB_CHECK_ARG(n_p > 0, "al_kl_divergence: n_p must be positive");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* dres = nullptr;
  ALB_TRY(engine->buf("kl.result", 1, &dres));
  ALB_LAUNCH(engine, "kl_divergence", 1, st,
             (k_kl_divergence<<<1, kKlBlock, 0, st>>>(histogram_p, histogram_q, 1.0 / n_p,
                                                      double(n_q) / n_p, q_lower_bound,
                                                      num_bins, dres)));
  ALB_CUDA(cudaGetLastError());
  ALB_CUDA(cudaMemcpyAsync(result, dres, sizeof(double), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  return AL_OK;
}

}  // extern "C"
