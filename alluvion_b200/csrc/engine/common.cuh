// common.cuh -- shared device-side types and SPH math of the B200 engine.
//
// Kernels are templated on the real type TF (float / double), like the
// reference's Runner<TF> (include/alluvion/runner.hpp).  Arithmetic that
// decides discrete outcomes (cell index, neighbor membership) uses
// explicitly rounded intrinsics so that it is reproducible bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "alluvion_b200.h"

namespace alb {

constexpr uint32_t kNoCell = 0xffffffffu;
constexpr int kBlock = 128;  // threads per block of the particle passes (64..512 measured: 128 best)
// Largest block of the passes whose shape the launch-shape table can set
// (their __launch_bounds__ and block-sized shared arrays).
constexpr int kMaxBlock = 256;

// ------------------------------------------------------------- vectors
template <class TF>
struct vec3 {
  TF x, y, z;
};
template <class TF>
struct alignas(sizeof(TF) * 4) vec4 {
  TF x, y, z, w;
};

template <class TF>
__host__ __device__ __forceinline__ vec3<TF> make3(TF x, TF y, TF z) {
  return vec3<TF>{x, y, z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> xyz(const vec4<TF>& a) {
  return vec3<TF>{a.x, a.y, a.z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> operator+(vec3<TF> a, vec3<TF> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> operator-(vec3<TF> a, vec3<TF> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> operator-(vec3<TF> a) {
  return {-a.x, -a.y, -a.z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> operator*(TF s, vec3<TF> a) {
  return {s * a.x, s * a.y, s * a.z};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> operator*(vec3<TF> a, TF s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF>& operator+=(vec3<TF>& a, vec3<TF> b) {
  a = a + b;
  return a;
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF>& operator-=(vec3<TF>& a, vec3<TF> b) {
  a = a - b;
  return a;
}
template <class TF>
__host__ __device__ __forceinline__ TF dot(vec3<TF> a, vec3<TF> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class TF>
__host__ __device__ __forceinline__ TF length_sqr(vec3<TF> a) {
  return a.x * a.x + a.y * a.y + a.z * a.z;
}
template <class TF>
__host__ __device__ __forceinline__ vec3<TF> cross(vec3<TF> a, vec3<TF> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <class TF>
__host__ __device__ __forceinline__ constexpr TF max_value();
template <>
__host__ __device__ __forceinline__ constexpr float max_value<float>() {
  return 3.40282346638528859811704183484516925e+38f;
}
template <>
__host__ __device__ __forceinline__ constexpr double max_value<double>() {
  return 1.79769313486231570814527423731704357e+308;
}

__device__ __forceinline__ float rsqrt_(float v) { return rsqrtf(v); }
__device__ __forceinline__ double rsqrt_(double v) { return rsqrt(v); }

// Exactly rounded primitives for the discrete decisions.
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }

// |a - b|^2 evaluated as ((dx*dx + dy*dy) + dz*dz) with every operation
// rounded on its own: the order length_sqr(x_i - x_j) has in the reference
// (runner.hpp:1893-1895), without contraction into FMAs.
template <class TF>
__device__ __forceinline__ TF dist2_rn(vec3<TF> a, vec3<TF> b) {
  TF dx = sub_rn(a.x, b.x), dy = sub_rn(a.y, b.y), dz = sub_rn(a.z, b.z);
  return add_rn(add_rn(mul_rn(dx, dx), mul_rn(dy, dy)), mul_rn(dz, dz));
}

// ------------------------------------------------------------ loads/stores
template <class TF>
__device__ __forceinline__ vec3<TF> ld3(const TF* p, size_t i) {
  return vec3<TF>{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
template <class TF>
__device__ __forceinline__ void st3(TF* p, size_t i, vec3<TF> v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
template <class TF>
__device__ __forceinline__ vec4<TF> ld4(const vec4<TF>* p, size_t i) {
  return p[i];
}
template <class TF>
__device__ __forceinline__ vec4<TF> ldg4(const vec4<TF>* p, size_t i) {
  return __ldg(reinterpret_cast<const vec4<TF>*>(p) + i);
}

}  // namespace alb

// __ldg overloads for the engine's aligned vector types.
__device__ __forceinline__ alb::vec4<float> __ldg(const alb::vec4<float>* p) {
  float4 v = __ldg(reinterpret_cast<const float4*>(p));
  return alb::vec4<float>{v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ alb::vec4<double> __ldg(const alb::vec4<double>* p) {
  const double2* q = reinterpret_cast<const double2*>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return alb::vec4<double>{a.x, a.y, b.x, b.y};
}

namespace alb {

// ------------------------------------------------------------- constants
// Device copy of the caller's Const<TF> subset; passed by value to kernels.
template <class TF>
struct Cn {
  TF h, h2, k, l, w0, radius, vol, mass, rho0, visc, bvisc, eps;
  vec3<TF> g;
  TF inv_h, inv_h2;  // 1 / h and 1 / h^2, rounded once on the host
  // periodic in y (the solvers' step<1>): Const::wrap_length and its
  // half-range bounds (constants.hpp:130-136); wrap = 0 otherwise
  TF wrap_len = 0, wrap_min = 0, wrap_max = 0;
  int wrap = 0;
};

// Sets the periodic-y fields as Const::set_wrap_length does.
template <class TF>
inline void set_wrap(Cn<TF>& c, TF length) {
  c.wrap = 1;
  c.wrap_len = length;
  c.wrap_min = length * TF(-0.5);
  c.wrap_max = length * TF(0.5);
}

// wrap_y (runner.hpp:698-707) of a displacement's or position's y.
template <class TF>
__device__ __forceinline__ TF wrap_y(const Cn<TF>& c, TF y) {
  if (!c.wrap) return y;
  if (y >= c.wrap_max) return sub_rn(y, c.wrap_len);
  if (y < c.wrap_min) return add_rn(y, c.wrap_len);
  return y;
}

// x_i - x_j with each difference rounded on its own, y wrapped when the
// step is periodic: the displacement make_neighbor_list<wrap> stores
// (runner.hpp:1893-1894).
template <class TF>
__device__ __forceinline__ vec3<TF> pdisp(const Cn<TF>& c, vec3<TF> a, vec3<TF> b) {
  return vec3<TF>{sub_rn(a.x, b.x), wrap_y(c, sub_rn(a.y, b.y)), sub_rn(a.z, b.z)};
}
// |pdisp|^2 as ((dx*dx + dy*dy) + dz*dz), every operation rounded.
template <class TF>
__device__ __forceinline__ TF pdist2(const Cn<TF>& c, vec3<TF> a, vec3<TF> b) {
  const vec3<TF> d = pdisp(c, a, b);
  return add_rn(add_rn(mul_rn(d.x, d.x), mul_rn(d.y, d.y)), mul_rn(d.z, d.z));
}


template <class TF, class C>
inline Cn<TF> to_cn(const C& c) {
  Cn<TF> o;
  o.h = c.kernel_radius;
  o.h2 = c.kernel_radius_sqr;
  o.k = c.cubic_kernel_k;
  o.l = c.cubic_kernel_l;
  o.w0 = c.cubic_kernel_zero;
  o.radius = c.particle_radius;
  o.vol = c.particle_vol;
  o.mass = c.particle_mass;
  o.rho0 = c.density0;
  o.visc = c.viscosity;
  o.bvisc = c.boundary_viscosity;
  o.eps = c.dfsph_factor_epsilon;
  o.g = vec3<TF>{c.gravity[0], c.gravity[1], c.gravity[2]};
  o.inv_h = TF(1) / o.h;
  o.inv_h2 = TF(1) / o.h2;
  return o;
}

struct GridDims {
  uint32_t res[3];
  int32_t off[3];
  uint32_t cap_cell, cap_nbr, nb;
  uint32_t ncells;
};

inline GridDims to_dims(const al_consti& g) {
  GridDims d;
  for (int k = 0; k < 3; ++k) {
    d.res[k] = g.grid_res[k];
    d.off[k] = g.grid_offset[k];
  }
  d.cap_cell = g.max_num_particles_per_cell;
  d.cap_nbr = g.max_num_neighbors_per_particle;
  d.nb = g.num_boundaries;
  d.ncells = g.grid_res[0] * g.grid_res[1] * g.grid_res[2];
  return d;
}

// ------------------------------------------------------------ SPH kernels
// Cubic spline of a distance (dist_cubic_kernel, runner.hpp:596-606).
template <class TF>
__device__ __forceinline__ TF W_dist(const Cn<TF>& c, TF r) {
  TF q = fabs(r) / c.h;
  TF conj = TF(1) - q;
  TF s = 0;
  if (q <= TF(0.5))
    s = (TF(6) * q - TF(6)) * q * q + TF(1);
  else if (q <= TF(1))
    s = TF(2) * conj * conj * conj;
  return s * c.k;
}

// Cubic spline of a squared distance (d2_cubic_kernel, runner.hpp:608-619).
// float: q from the hardware reciprocal square root and 1/h, no IEEE
// division or square-root sequence (the reference is built with
// --use_fast_math, whose division and sqrt are approximate as well).
__device__ __forceinline__ float W_r2(const Cn<float>& c, float r2) {
  const float q2 = r2 * c.inv_h2;
  const float q = r2 > 0.f ? r2 * rsqrtf(r2) * c.inv_h : 0.f;
  const float conj = 1.f - q;
  float s = 0.f;
  if (q <= 0.5f)
    s = (6.f * q - 6.f) * q2 + 1.f;
  else if (q <= 1.f)
    s = 2.f * conj * conj * conj;
  return s * c.k;
}
template <class TF>
__device__ __forceinline__ TF W_r2(const Cn<TF>& c, TF r2) {
  TF q2 = r2 / c.h2;
  TF q = sqrt(r2) / c.h;
  TF conj = TF(1) - q;
  TF s = 0;
  if (q <= TF(0.5))
    s = (TF(6) * q - TF(6)) * q2 + TF(1);
  else if (q <= TF(1))
    s = TF(2) * conj * conj * conj;
  return s * c.k;
}

// Kernel gradient of a displacement (displacement_cubic_kernel_grad,
// runner.hpp:628-638).  float: one hardware reciprocal square root gives
// both |d| and 1/|d|.
__device__ __forceinline__ vec3<float> gradW(const Cn<float>& c, vec3<float> d) {
  const float rl2 = length_sqr(d);
  const float inv_rl = rl2 > 0.f ? rsqrtf(rl2) : 0.f;
  const float rl = rl2 * inv_rl;
  const float q = rl * c.inv_h;
  const float s = q <= 0.5f ? (q * 3.f - 2.f) * c.inv_h
                            : (q <= 1.f ? (1.f - q) * (q - 1.f) * inv_rl : 0.f);
  return (c.l * s) * d;
}
template <class TF>
__device__ __forceinline__ vec3<TF> gradW(const Cn<TF>& c, vec3<TF> d) {
  TF rl2 = length_sqr(d);
  TF rl = sqrt(rl2);
  TF q = rl / c.h;
  TF s = q <= TF(0.5) ? (q * TF(3) - TF(2)) / c.h
                      : (q <= TF(1) ? (TF(1) - q) * (q - TF(1)) / rl : TF(0));
  return (c.l * s) * d;
}

// Cell coordinates floor(x / h) - grid_offset (get_ipos, runner.hpp:1827-1831)
// with IEEE division.
template <class TF>
__device__ __forceinline__ void cell_coords(TF h, const GridDims& g, vec3<TF> x, int p[3]) {
  p[0] = int(floor(div_rn(x.x, h))) - g.off[0];
  p[1] = int(floor(div_rn(x.y, h))) - g.off[1];
  p[2] = int(floor(div_rn(x.z, h))) - g.off[2];
}
__device__ __forceinline__ bool in_grid(const GridDims& g, const int p[3]) {
  return p[0] >= 0 && p[0] < int(g.res[0]) && p[1] >= 0 && p[1] < int(g.res[1]) && p[2] >= 0 &&
         p[2] < int(g.res[2]);
}
__device__ __forceinline__ uint32_t cell_linear(const GridDims& g, int x, int y, int z) {
  return (uint32_t(x) * g.res[1] + uint32_t(y)) * g.res[2] + uint32_t(z);
}

// ------------------------------------------------------------ reductions
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic block sum in double: warp trees, then warp 0 sums the warp
// partials in warp order.  All threads of the block must call it.
__device__ __forceinline__ double block_sum_double(double v) {
  __shared__ double part[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) part[warp] = v;
  __syncthreads();
  double s = 0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    s = lane < nw ? part[lane] : 0.0;
    s = warp_sum(s);
  }
  __syncthreads();
  return s;  // valid in thread 0
}

}  // namespace alb
