// body_geometry.cuh -- device geometry of rigid bodies shared by the
// boundary sampling and the contact detection: quaternion rotation,
// analytic signed distances and gradients, and evaluation of the 32-node
// cubic Lagrange element on a body's grid.  Internal linkage: every
// translation unit that includes it compiles its own copy.
#pragma once

#include "boundary.cuh"

namespace alb {
namespace {

// ------------------------------------------------------------- geometry
__host__ __device__ __forceinline__ bool shape_is_y_invariant(uint32_t shape) {
  return shape == AL_SHAPE_INFINITE_CYLINDER || shape == AL_SHAPE_INFINITE_TUBE;
}

template <class TF>
__device__ __forceinline__ vec3<TF> rotate(vec3<TF> v, vec4<TF> q) {
  vec3<TF> r;
  r.x = (TF(1) - TF(2) * (q.y * q.y + q.z * q.z)) * v.x + TF(2) * (q.x * q.y - q.z * q.w) * v.y +
        TF(2) * (q.x * q.z + q.y * q.w) * v.z;
  r.y = TF(2) * (q.x * q.y + q.z * q.w) * v.x + (TF(1) - TF(2) * (q.x * q.x + q.z * q.z)) * v.y +
        TF(2) * (q.y * q.z - q.x * q.w) * v.z;
  r.z = TF(2) * (q.x * q.z - q.y * q.w) * v.x + TF(2) * (q.y * q.z + q.x * q.w) * v.y +
        (TF(1) - TF(2) * (q.x * q.x + q.y * q.y)) * v.z;
  return r;
}

template <class TF>
__device__ __forceinline__ TF box_sdf(vec3<TF> x, TF hx, TF hy, TF hz, TF outset) {
  vec3<TF> d{fabs(x.x) - hx, fabs(x.y) - hy, fabs(x.z) - hz};
  vec3<TF> cl{fmax(d.x, TF(0)), fmax(d.y, TF(0)), fmax(d.z, TF(0))};
  return sqrt(length_sqr(cl)) + fmin(fmax(d.x, fmax(d.y, d.z)), TF(0)) - outset;
}

// Analytic signed distances (dg/box_distance.hpp:23-30,
// dg/sphere_distance.hpp:18-20, dg/box_shell_distance.hpp:36-47,
// dg/cylinder_distance.hpp:28-35, dg/capsule_distance.hpp:24-27,
// dg/infinite_cylinder_distance.hpp:20-22, dg/infinite_tube_distance.hpp:32-36)
// and the torus |(|x_xz| - R, y)| - r.
template <class TF>
__device__ __forceinline__ TF shape_sdf(const BodyDev<TF>& b, vec3<TF> x) {
  switch (b.shape) {
    case AL_SHAPE_CYLINDER: {
      const TF d0 = sqrt(x.x * x.x + x.z * x.z) - b.p[0];
      const TF d1 = fabs(x.y + b.p[2]) - b.p[1] * TF(0.5);
      const TF c0 = fmax(d0, TF(0)), c1 = fmax(d1, TF(0));
      return fmin(fmax(d0, d1), TF(0)) + sqrt(c0 * c0 + c1 * c1);
    }
    case AL_SHAPE_CAPSULE: {
      const TF hh = b.p[1] * TF(0.5);
      const vec3<TF> m{x.x, x.y - fmax(-hh, fmin(x.y, hh)), x.z};
      return sqrt(length_sqr(m)) - b.p[0];
    }
    case AL_SHAPE_INFINITE_CYLINDER:
      return sqrt(x.x * x.x + x.z * x.z) - b.p[0];
    case AL_SHAPE_INFINITE_TUBE: {
      const TF rd = sqrt(x.x * x.x + x.z * x.z);
      return fmax(b.p[0] - rd, rd - b.p[1]);
    }
    case AL_SHAPE_BOX:
      return box_sdf(x, b.p[0], b.p[1], b.p[2], b.p[3]);
    case AL_SHAPE_SPHERE:
      return sqrt(length_sqr(x)) - b.p[0];
    case AL_SHAPE_BOX_SHELL: {
      TF inner = box_sdf(x, b.p[0], b.p[1], b.p[2], b.p[6]);
      TF outer = box_sdf(x, b.p[3], b.p[4], b.p[5], b.p[6]);
      return fmax(outer, -inner);
    }
    default: {
      TF rho = sqrt(x.x * x.x + x.z * x.z) - b.p[0];
      return sqrt(rho * rho + x.y * x.y) - b.p[1];
    }
  }
}

// Un-normalised outward direction: the position for a sphere
// (sphere_distance.hpp:21), the radial direction for the y-invariant shapes,
// central differences with step h/256 otherwise (box_distance.hpp:28-38).
template <class TF>
__device__ __forceinline__ vec3<TF> shape_gradient(const BodyDev<TF>& b, vec3<TF> x, TF h) {
  if (b.shape == AL_SHAPE_SPHERE) return x;
  // the y-invariant shapes return the radial direction
  // (dg/infinite_cylinder_distance.hpp:23-25, dg/infinite_tube_distance.hpp:37-43)
  if (b.shape == AL_SHAPE_INFINITE_CYLINDER) return vec3<TF>{x.x, TF(0), x.z};
  if (b.shape == AL_SHAPE_INFINITE_TUBE) {
    const TF s = (x.x * x.x + x.z * x.z) * TF(4) > (b.p[0] + b.p[1]) * (b.p[0] + b.p[1])
                     ? TF(1)
                     : TF(-1);
    return vec3<TF>{s * x.x, TF(0), s * x.z};
  }
  const TF s = h * TF(0.00390625);
  return vec3<TF>{shape_sdf(b, vec3<TF>{x.x + s, x.y, x.z}) - shape_sdf(b, vec3<TF>{x.x - s, x.y, x.z}),
                  shape_sdf(b, vec3<TF>{x.x, x.y + s, x.z}) - shape_sdf(b, vec3<TF>{x.x, x.y - s, x.z}),
                  shape_sdf(b, vec3<TF>{x.x, x.y, x.z + s}) - shape_sdf(b, vec3<TF>{x.x, x.y, x.z - s})};
}

// resolve (runner.hpp:1180-1195): cell of x and reference coordinates.
template <class TF>
__device__ __forceinline__ bool resolve(const BodyDev<TF>& b, vec3<TF> x, int ip[3],
                                        vec3<TF>& xi) {
  if (!(x.x >= b.dmin.x && x.y >= b.dmin.y && x.z >= b.dmin.z && b.dmax.x >= x.x &&
        b.dmax.y >= x.y && b.dmax.z >= x.z))
    return false;
  const vec3<TF> inv{TF(1) / b.cs.x, TF(1) / b.cs.y, TF(1) / b.cs.z};
  ip[0] = min(int((x.x - b.dmin.x) * inv.x), int(b.res[0]) - 1);
  ip[1] = min(int((x.y - b.dmin.y) * inv.y), int(b.res[1]) - 1);
  ip[2] = min(int((x.z - b.dmin.z) * inv.z), int(b.res[2]) - 1);
  const vec3<TF> lo{b.dmin.x + b.cs.x * TF(ip[0]), b.dmin.y + b.cs.y * TF(ip[1]),
                    b.dmin.z + b.cs.z * TF(ip[2])};
  xi = vec3<TF>{TF(2) * (x.x - lo.x) * inv.x - TF(1), TF(2) * (x.y - lo.y) * inv.y - TF(1),
                TF(2) * (x.z - lo.z) * inv.z - TF(1)};
  return true;
}

// Linear index of the j-th node of cell ip (get_cells, runner.hpp:1197-1257):
// 8 vertices, then per x-, y-, z-edge family four edges of two third-point
// nodes.
__device__ __forceinline__ uint32_t lagrange_node(const uint32_t r[3], uint32_t x, uint32_t y,
                                                  uint32_t z, int j) {
  const uint32_t nx = r[0], ny = r[1], nz = r[2];
  if (j < 8)
    return (nx + 1) * (ny + 1) * (z + ((j >> 2) & 1)) + (nx + 1) * (y + ((j >> 1) & 1)) + x +
           (j & 1);
  uint32_t base = (nx + 1) * (ny + 1) * (nz + 1);
  if (j < 16) {
    const int e = j - 8;
    return base + 2 * (nx * (ny + 1) * (z + ((e >> 1) & 1)) + nx * (y + ((e >> 2) & 1)) + x) +
           (e & 1);
  }
  base += 2 * nx * (ny + 1) * (nz + 1);
  if (j < 24) {
    const int e = j - 16;
    return base + 2 * (ny * (nz + 1) * (x + ((e >> 1) & 1)) + ny * (z + ((e >> 2) & 1)) + y) +
           (e & 1);
  }
  base += 2 * (nx + 1) * ny * (nz + 1);
  const int e = j - 24;
  return base + 2 * (nz * (nx + 1) * (y + ((e >> 1) & 1)) + nz * (x + ((e >> 2) & 1)) + z) +
         (e & 1);
}

// Shape function j of the 32-node element at reference point p and,
// if GRAD, its derivatives (the element of get_shape_function_and_gradient,
// runner.hpp:1354-1584):
//   corner: (1/64)(1+sx x)(1+sy y)(1+sz z)(9|p|^2 - 19)
//   edge:   (9/64)(1-t^2)(1+3 s t)(1+s1 u)(1+s2 w)
template <class TF, bool GRAD>
__device__ __forceinline__ void shape_j(int j, vec3<TF> p, TF r2, TF& N, vec3<TF>& dN) {
  const TF c64 = TF(1) / TF(64), e64 = TF(9) / TF(64);
  if (j < 8) {
    const TF sx = (j & 1) ? TF(1) : TF(-1), sy = (j & 2) ? TF(1) : TF(-1),
             sz = (j & 4) ? TF(1) : TF(-1);
    const TF ax = TF(1) + sx * p.x, ay = TF(1) + sy * p.y, az = TF(1) + sz * p.z;
    const TF f = TF(9) * r2 - TF(19);
    N = c64 * ax * ay * az * f;
    if (GRAD) {
      dN.x = c64 * ay * az * (sx * f + TF(18) * p.x * ax);
      dN.y = c64 * ax * az * (sy * f + TF(18) * p.y * ay);
      dN.z = c64 * ax * ay * (sz * f + TF(18) * p.z * az);
    }
    return;
  }
  // family: axis of the edge, and the axes selected by bits 1 and 2
  int axis, a1, a2, e;
  if (j < 16) {
    e = j - 8;
    axis = 0;
    a1 = 2;
    a2 = 1;
  } else if (j < 24) {
    e = j - 16;
    axis = 1;
    a1 = 0;
    a2 = 2;
  } else {
    e = j - 24;
    axis = 2;
    a1 = 1;
    a2 = 0;
  }
  const TF u[3] = {p.x, p.y, p.z};
  const TF s = (e & 1) ? TF(1) : TF(-1), s1 = (e & 2) ? TF(1) : TF(-1),
           s2 = (e & 4) ? TF(1) : TF(-1);
  const TF t = u[axis], A = TF(1) + s1 * u[a1], B = TF(1) + s2 * u[a2];
  const TF g = (TF(1) - t * t) * (TF(1) + TF(3) * s * t);
  N = e64 * g * A * B;
  if (GRAD) {
    const TF dg = TF(3) * s * (TF(1) - t * t) - TF(2) * t * (TF(1) + TF(3) * s * t);
    TF d[3];
    d[axis] = e64 * dg * A * B;
    d[a1] = e64 * g * s1 * B;
    d[a2] = e64 * g * A * s2;
    dN = vec3<TF>{d[0], d[1], d[2]};
  }
}

// Interpolated value of `nodes` at x (interpolate_distance_without_
// intermediates, runner.hpp:1596-1614): +max outside the domain.
template <class TF>
__device__ __forceinline__ TF interpolate_grid(const BodyDev<TF>& b, const TF* __restrict__ nodes,
                                               vec3<TF> x) {
  int ip[3];
  vec3<TF> xi;
  if (!resolve(b, x, ip, xi)) return max_value<TF>();
  const TF r2 = xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
  TF phi = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    TF N;
    vec3<TF> dN;
    shape_j<TF, false>(j, xi, r2, N, dN);
    phi += __ldg(nodes + lagrange_node(b.res, ip[0], ip[1], ip[2], j)) * N;
  }
  return phi;
}

// Interpolated value of `nodes` at x and its gradient scaled by 2 / cell
// size (interpolate_and_derive, runner.hpp:1773-1791); false outside the
// domain.
template <class TF>
__device__ __forceinline__ bool interpolate_grid_gradient(const BodyDev<TF>& b,
                                                          const TF* __restrict__ nodes,
                                                          vec3<TF> x, TF& phi, vec3<TF>& grad) {
  int ip[3];
  vec3<TF> xi;
  if (!resolve(b, x, ip, xi)) return false;
  const TF r2 = xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
  phi = 0;
  grad = vec3<TF>{0, 0, 0};
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    TF N;
    vec3<TF> dN;
    shape_j<TF, true>(j, xi, r2, N, dN);
    const TF v = __ldg(nodes + lagrange_node(b.res, ip[0], ip[1], ip[2], j));
    phi += v * N;
    grad.x += v * dN.x;
    grad.y += v * dN.y;
    grad.z += v * dN.z;
  }
  grad.x *= TF(2) / b.cs.x;
  grad.y *= TF(2) / b.cs.y;
  grad.z *= TF(2) / b.cs.z;
  return true;
}

// index_to_node_position (runner.hpp:1131-1178).
template <class TF>
__device__ __forceinline__ vec3<TF> node_position(const BodyDev<TF>& b, uint32_t l) {
  const uint32_t nx = b.res[0], ny = b.res[1], nz = b.res[2];
  const uint32_t nv = (nx + 1) * (ny + 1) * (nz + 1);
  const uint32_t nex = nx * (ny + 1) * (nz + 1);
  const uint32_t ney = (nx + 1) * ny * (nz + 1);
  auto at = [&](uint32_t a, uint32_t bb, uint32_t cc) {
    return vec3<TF>{b.dmin.x + b.cs.x * TF(a), b.dmin.y + b.cs.y * TF(bb),
                    b.dmin.z + b.cs.z * TF(cc)};
  };
  if (l < nv) {
    const uint32_t t = l % ((ny + 1) * (nx + 1));
    return at(t % (nx + 1), t / (nx + 1), l / ((ny + 1) * (nx + 1)));
  }
  if (l < nv + 2 * nex) {
    l -= nv;
    const uint32_t e = l / 2, t = e % ((ny + 1) * nx);
    vec3<TF> p = at(t % nx, t / nx, e / ((ny + 1) * nx));
    p.x += (TF(1) + TF(l % 2)) / TF(3) * b.cs.x;
    return p;
  }
  if (l < nv + 2 * (nex + ney)) {
    l -= nv + 2 * nex;
    const uint32_t e = l / 2, t = e % ((nz + 1) * ny);
    vec3<TF> p = at(e / ((nz + 1) * ny), t % ny, t / ny);
    p.y += (TF(1) + TF(l % 2)) / TF(3) * b.cs.y;
    return p;
  }
  l -= nv + 2 * (nex + ney);
  const uint32_t e = l / 2, t = e % ((nx + 1) * nz);
  vec3<TF> p = at(t / nz, e / ((nx + 1) * nz), t % nz);
  p.z += (TF(1) + TF(l % 2)) / TF(3) * b.cs.z;
  return p;
}

}  // namespace
}  // namespace alb
