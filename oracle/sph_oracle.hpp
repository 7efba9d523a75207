// sph_oracle.hpp -- CPU ORACLE (test infrastructure, not product code).
//
// A C++17 + OpenMP restatement of kennychufk/alluvion's SPH fluid-step path,
// templated on the real type (float / double).  Only tests/, the smoke check
// and bench.py's CPU-baseline leg may load it; the engine never calls it.
//
// Every routine cites the reference file:line it restates.  Paths are
// relative to the reference project root; "runner.hpp" means
// include/alluvion/runner.hpp.
//
// Deliberate, documented differences from the reference:
//  * cell index uses IEEE x / h (the reference builds with --use_fast_math,
//    whose division is not reproducible); the engine uses the same rule.
//  * buckets are unbounded and ordered canonically by (cell, index) instead
//    of atomicAdd order (runner.hpp:1853); neighbor lists follow that order.
//  * rigid force / torque totals and the solvers' convergence means are
//    accumulated in double (the reference sums FP32 with thrust).
//  * contacts (pile.hpp:826-979) are out of scope and not applied.
// Arithmetic that decides neighbor membership is written with explicit
// operation order; this file must be compiled with -ffp-contract=off.
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <map>
#include <array>

#include "alluvion_b200.h"

namespace oracle {

// ------------------------------------------------------------------ vectors
template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
struct V4 {
  T x, y, z, w;
};
template <class T>
inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T>
inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T>
inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T>
inline V3<T>& operator+=(V3<T>& a, V3<T> b) { a = a + b; return a; }
template <class T>
inline V3<T>& operator-=(V3<T>& a, V3<T> b) { a = a - b; return a; }
template <class T>
inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
inline T length_sqr(V3<T> a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
template <class T>
inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
inline T inv_sqrt(T v) { return T(1) / std::sqrt(v); }
template <class T>
inline V3<T> normalized(V3<T> a) { return inv_sqrt(dot(a, a)) * a; }

// Quaternion {x, y, z, w}.  Rotation matrix as runner.hpp:141-154.
template <class T>
inline V3<T> rotate(V3<T> v, V4<T> q) {
  V3<T> r;
  r.x = (1 - 2 * (q.y * q.y + q.z * q.z)) * v.x + 2 * (q.x * q.y - q.z * q.w) * v.y +
        2 * (q.x * q.z + q.y * q.w) * v.z;
  r.y = 2 * (q.x * q.y + q.z * q.w) * v.x + (1 - 2 * (q.x * q.x + q.z * q.z)) * v.y +
        2 * (q.y * q.z - q.x * q.w) * v.z;
  r.z = 2 * (q.x * q.z - q.y * q.w) * v.x + 2 * (q.y * q.z + q.x * q.w) * v.y +
        (1 - 2 * (q.x * q.x + q.y * q.y)) * v.z;
  return r;
}
template <class T>
inline V4<T> conjugate(V4<T> q) { return {-q.x, -q.y, -q.z, q.w}; }

// ---------------------------------------------------------- parameter view
template <class TF>
struct Cn {
  TF h, h2, k, l, w0, radius, vol, mass, rho0, visc, bvisc, eps;
  V3<TF> g;
};
template <class TF, class C>
inline Cn<TF> make_cn(const C& c) {
  return Cn<TF>{c.kernel_radius, c.kernel_radius_sqr, c.cubic_kernel_k, c.cubic_kernel_l,
                c.cubic_kernel_zero, c.particle_radius, c.particle_vol, c.particle_mass,
                c.density0, c.viscosity, c.boundary_viscosity, c.dfsph_factor_epsilon,
                V3<TF>{c.gravity[0], c.gravity[1], c.gravity[2]}};
}

// ------------------------------------------------------------ SPH kernels
// Cubic spline W(r) of a distance (dist_cubic_kernel, runner.hpp:596-606).
template <class TF>
inline TF W_dist(const Cn<TF>& c, TF r) {
  TF q = std::fabs(r) / c.h;
  TF conj = 1 - q;
  TF s = 0;
  if (q <= TF(0.5))
    s = (6 * q - 6) * q * q + 1;
  else if (q <= 1)
    s = 2 * conj * conj * conj;
  return s * c.k;
}
// W of a squared distance (d2_cubic_kernel, runner.hpp:608-619).
template <class TF>
inline TF W_r2(const Cn<TF>& c, TF r2) {
  TF q2 = r2 / c.h2;
  TF q = std::sqrt(r2) / c.h;
  TF conj = 1 - q;
  TF s = 0;
  if (q <= TF(0.5))
    s = (6 * q - 6) * q2 + 1;
  else if (q <= 1)
    s = 2 * conj * conj * conj;
  return s * c.k;
}
// Gradient of W for a displacement (displacement_cubic_kernel_grad,
// runner.hpp:628-638).
template <class TF>
inline V3<TF> gradW(const Cn<TF>& c, V3<TF> d) {
  TF rl2 = length_sqr(d);
  TF rl = std::sqrt(rl2);
  TF q = rl / c.h;
  TF s = q <= TF(0.5) ? (q * 3 - 2) / c.h : (q <= 1 ? (1 - q) * (q - 1) / rl : TF(0));
  return (c.l * s) * d;
}

// ------------------------------------------------------------------- grid
constexpr uint32_t kNoCell = 0xffffffffu;

// Cell of a position (get_ipos / within_grid, runner.hpp:1827-1838) with
// IEEE division.  Returns kNoCell outside the grid.
template <class TF>
inline void cell_coords(const Cn<TF>& c, const al_consti& g, V3<TF> x, int out[3]) {
  out[0] = int(std::floor(x.x / c.h)) - g.grid_offset[0];
  out[1] = int(std::floor(x.y / c.h)) - g.grid_offset[1];
  out[2] = int(std::floor(x.z / c.h)) - g.grid_offset[2];
}
inline bool in_grid(const al_consti& g, const int p[3]) {
  return p[0] >= 0 && p[0] < int(g.grid_res[0]) && p[1] >= 0 && p[1] < int(g.grid_res[1]) &&
         p[2] >= 0 && p[2] < int(g.grid_res[2]);
}
inline uint32_t cell_linear(const al_consti& g, const int p[3]) {
  return (uint32_t(p[0]) * g.grid_res[1] + uint32_t(p[1])) * g.grid_res[2] + uint32_t(p[2]);
}

struct GridSort {
  std::vector<uint32_t> cell;        // per original particle
  std::vector<uint32_t> sorted;      // sorted slot -> original index
  std::vector<uint32_t> cell_start;  // ncells + 1
  bool out_of_grid = false;
  bool cell_overflow = false;
};

// Canonical replacement of update_particle_grid (runner.hpp:1840-1867):
// stable counting sort by cell; out-of-grid particles go last.
template <class TF>
GridSort grid_sort(const Cn<TF>& c, const al_consti& g, const V3<TF>* x, uint32_t n) {
  GridSort s;
  const uint32_t ncells = g.grid_res[0] * g.grid_res[1] * g.grid_res[2];
  s.cell.resize(n);
  s.cell_start.assign(size_t(ncells) + 1, 0);
  std::vector<uint32_t> count(ncells, 0);
  for (uint32_t i = 0; i < n; ++i) {
    int p[3];
    cell_coords(c, g, x[i], p);
    if (in_grid(g, p)) {
      s.cell[i] = cell_linear(g, p);
      ++count[s.cell[i]];
    } else {
      s.cell[i] = kNoCell;
      s.out_of_grid = true;
    }
  }
  uint32_t run = 0;
  for (uint32_t k = 0; k < ncells; ++k) {
    s.cell_start[k] = run;
    run += count[k];
    if (count[k] > g.max_num_particles_per_cell) s.cell_overflow = true;
  }
  s.cell_start[ncells] = run;
  s.sorted.resize(n);
  std::vector<uint32_t> cursor(s.cell_start.begin(), s.cell_start.end() - 1);
  uint32_t tail = run;
  for (uint32_t i = 0; i < n; ++i) {
    if (s.cell[i] == kNoCell)
      s.sorted[tail++] = i;
    else
      s.sorted[cursor[s.cell[i]]++] = i;
  }
  return s;
}

// wrap_y (runner.hpp:698-707) with the half-range bounds of
// Const::set_wrap_length (constants.hpp:130-136).
template <class TF>
inline TF wrap_coord(bool wrap, TF len, TF y) {
  if (!wrap) return y;
  if (y >= len * TF(0.5)) return y - len;
  if (y < len * TF(-0.5)) return y + len;
  return y;
}

// Squared distance with a fixed operation order ((dx*dx + dy*dy) + dz*dz),
// the order length_sqr uses in the reference.
template <class TF>
inline TF dist2(V3<TF> a, V3<TF> b) {
  TF dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  return (dx * dx + dy * dy) + dz * dz;
}

struct NeighborList {
  uint32_t cap = 0;
  std::vector<uint32_t> count;  // min(found, cap)
  std::vector<uint32_t> index;  // [n][cap] original indices, canonical order
  bool overflow = false;
};

// make_neighbor_list<0> (runner.hpp:1869-1911): scan the 27 cells in
// ascending cell order, keep j != i with |x_i - x_j|^2 < h^2.  The reference
// clamps at cap with slot cap-1 overwritten; here the first cap canonical
// entries are kept and `overflow` is raised.
template <class TF>
NeighborList neighbor_list(const Cn<TF>& c, const al_consti& g, const V3<TF>* x, uint32_t n,
                           const GridSort& s, bool wrap = false, TF wrap_len = 0) {
  NeighborList nl;
  nl.cap = g.max_num_neighbors_per_particle;
  nl.count.assign(n, 0);
  nl.index.assign(size_t(n) * nl.cap, 0);
  bool overflow = false;
#pragma omp parallel for schedule(static) reduction(|| : overflow)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    uint32_t i = uint32_t(ii);
    int p[3];
    cell_coords(c, g, x[i], p);
    uint32_t found = 0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          int q[3] = {p[0] + dx, p[1] + dy, p[2] + dz};
          if (wrap) {  // wrap_ipos_y (runner.hpp:689-697)
            if (q[1] >= int(g.grid_res[1]))
              q[1] -= int(g.grid_res[1]);
            else if (q[1] < 0)
              q[1] += int(g.grid_res[1]);
          }
          if (!in_grid(g, q)) continue;
          uint32_t cell = cell_linear(g, q);
          for (uint32_t t = s.cell_start[cell]; t < s.cell_start[cell + 1]; ++t) {
            uint32_t j = s.sorted[t];
            if (j == i) continue;
            V3<TF> d = x[i] - x[j];
            d.y = wrap_coord(wrap, wrap_len, d.y);
            if ((d.x * d.x + d.y * d.y) + d.z * d.z < c.h2) {
              if (found < nl.cap) nl.index[size_t(i) * nl.cap + found] = j;
              ++found;
            }
          }
        }
    if (found > nl.cap) overflow = true;
    nl.count[i] = std::min(found, nl.cap);
  }
  nl.overflow = overflow;
  return nl;
}

// -------------------------------------------- cubic Lagrange grid (32 nodes)
struct GridShape {
  uint32_t res[3];
};

// Node position of linear node index l (index_to_node_position,
// runner.hpp:1131-1178): vertices first (x fastest), then the two
// third-point nodes of every x-, y- and z-edge.
template <class TF>
V3<TF> node_position(V3<TF> dmin, const uint32_t r[3], V3<TF> cs, uint32_t l) {
  const uint32_t nx = r[0], ny = r[1], nz = r[2];
  const uint32_t nv = (nx + 1) * (ny + 1) * (nz + 1);
  const uint32_t nex = nx * (ny + 1) * (nz + 1);
  const uint32_t ney = (nx + 1) * ny * (nz + 1);
  auto at = [&](uint32_t a, uint32_t b, uint32_t cc) {
    return V3<TF>{dmin.x + cs.x * TF(a), dmin.y + cs.y * TF(b), dmin.z + cs.z * TF(cc)};
  };
  if (l < nv) {
    uint32_t t = l % ((ny + 1) * (nx + 1));
    return at(t % (nx + 1), t / (nx + 1), l / ((ny + 1) * (nx + 1)));
  }
  if (l < nv + 2 * nex) {
    l -= nv;
    uint32_t e = l / 2, t = e % ((ny + 1) * nx);
    V3<TF> p = at(t % nx, t / nx, e / ((ny + 1) * nx));
    p.x += (TF(1) + TF(l % 2)) / TF(3) * cs.x;
    return p;
  }
  if (l < nv + 2 * (nex + ney)) {
    l -= nv + 2 * nex;
    uint32_t e = l / 2, t = e % ((nz + 1) * ny);
    V3<TF> p = at(e / ((nz + 1) * ny), t % ny, t / ny);
    p.y += (TF(1) + TF(l % 2)) / TF(3) * cs.y;
    return p;
  }
  l -= nv + 2 * (nex + ney);
  uint32_t e = l / 2, t = e % ((nx + 1) * nz);
  V3<TF> p = at(t / nz, e / ((nx + 1) * nz), t % nz);
  p.z += (TF(1) + TF(l % 2)) / TF(3) * cs.z;
  return p;
}

inline uint32_t num_grid_nodes(const uint32_t r[3]) {
  const uint32_t nx = r[0], ny = r[1], nz = r[2];
  return (nx + 1) * (ny + 1) * (nz + 1) +
         2 * (nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz);
}

// Cell lookup (resolve, runner.hpp:1180-1195).  Returns false outside.
template <class TF>
bool resolve(V3<TF> dmin, V3<TF> dmax, const uint32_t r[3], V3<TF> cs, V3<TF> x, int ip[3],
             V3<TF>& xi) {
  V3<TF> inv{TF(1) / cs.x, TF(1) / cs.y, TF(1) / cs.z};
  if (!(x.x >= dmin.x && x.y >= dmin.y && x.z >= dmin.z && dmax.x >= x.x && dmax.y >= x.y &&
        dmax.z >= x.z))
    return false;
  ip[0] = std::min(int((x.x - dmin.x) * inv.x), int(r[0]) - 1);
  ip[1] = std::min(int((x.y - dmin.y) * inv.y), int(r[1]) - 1);
  ip[2] = std::min(int((x.z - dmin.z) * inv.z), int(r[2]) - 1);
  V3<TF> lo{dmin.x + cs.x * TF(ip[0]), dmin.y + cs.y * TF(ip[1]), dmin.z + cs.z * TF(ip[2])};
  xi = {2 * (x.x - lo.x) * inv.x - 1, 2 * (x.y - lo.y) * inv.y - 1, 2 * (x.z - lo.z) * inv.z - 1};
  return true;
}

// The 32 node indices of a cell (get_cells, runner.hpp:1197-1257): 8 corner
// vertices, then for the x-, y- and z-edge families four edges of two
// third-point nodes each.
inline void cell_nodes(const uint32_t r[3], const int ip[3], uint32_t out[32]) {
  const uint32_t nx = r[0], ny = r[1], nz = r[2];
  const uint32_t x = ip[0], y = ip[1], z = ip[2];
  for (uint32_t j = 0; j < 8; ++j) {
    uint32_t a = x + (j & 1), b = y + ((j >> 1) & 1), cc = z + ((j >> 2) & 1);
    out[j] = (nx + 1) * (ny + 1) * cc + (nx + 1) * b + a;
  }
  uint32_t base = (nx + 1) * (ny + 1) * (nz + 1);
  // x-edges: pair (e>>1)&1 -> z offset, (e>>2)&1 -> y offset
  for (uint32_t e = 0; e < 8; e += 2) {
    uint32_t oz = (e >> 1) & 1, oy = (e >> 2) & 1;
    uint32_t k = base + 2 * (nx * (ny + 1) * (z + oz) + nx * (y + oy) + x);
    out[8 + e] = k;
    out[9 + e] = k + 1;
  }
  base += 2 * (nx * (ny + 1) * (nz + 1));
  // y-edges: (e>>1)&1 -> x offset, (e>>2)&1 -> z offset
  for (uint32_t e = 0; e < 8; e += 2) {
    uint32_t ox = (e >> 1) & 1, oz = (e >> 2) & 1;
    uint32_t k = base + 2 * (ny * (nz + 1) * (x + ox) + ny * (z + oz) + y);
    out[16 + e] = k;
    out[17 + e] = k + 1;
  }
  base += 2 * ((nx + 1) * ny * (nz + 1));
  // z-edges: (e>>1)&1 -> y offset, (e>>2)&1 -> x offset
  for (uint32_t e = 0; e < 8; e += 2) {
    uint32_t oy = (e >> 1) & 1, ox = (e >> 2) & 1;
    uint32_t k = base + 2 * (nz * (nx + 1) * (y + oy) + nz * (x + ox) + z);
    out[24 + e] = k;
    out[25 + e] = k + 1;
  }
}

// Shape functions of the 32-node cubic serendipity-type element and their
// derivatives (the element of get_shape_function[_and_gradient],
// runner.hpp:1259-1584):
//   corner (sx,sy,sz):  (1/64)(1+sx x)(1+sy y)(1+sz z)(9(x^2+y^2+z^2) - 19)
//   x-edge (s,sy,sz):   (9/64)(1-x^2)(1+3 s x)(1+sy y)(1+sz z)   (likewise y, z)
// Node order matches cell_nodes().  Derivatives by the product rule.
template <class TF>
void shape_functions(V3<TF> p, TF N[32], TF* dN0, TF* dN1, TF* dN2) {
  const TF x = p.x, y = p.y, z = p.z;
  const TF r2 = x * x + y * y + z * z;
  const TF c64 = TF(1) / TF(64), e64 = TF(9) / TF(64);
  for (int j = 0; j < 8; ++j) {
    TF sx = (j & 1) ? 1 : -1, sy = (j & 2) ? 1 : -1, sz = (j & 4) ? 1 : -1;
    TF ax = 1 + sx * x, ay = 1 + sy * y, az = 1 + sz * z, f = 9 * r2 - 19;
    N[j] = c64 * ax * ay * az * f;
    if (dN0) {
      dN0[j] = c64 * ay * az * (sx * f + 18 * x * ax);
      dN1[j] = c64 * ax * az * (sy * f + 18 * y * ay);
      dN2[j] = c64 * ax * ay * (sz * f + 18 * z * az);
    }
  }
  // axis a is the edge direction; (b, c) the perpendicular directions whose
  // offsets are selected by bits 1 and 2 of the node's index within the
  // family (see cell_nodes).
  auto edge_family = [&](int first, int axis, int bit1_axis, int bit2_axis) {
    TF u[3] = {x, y, z};
    for (int e = 0; e < 8; ++e) {
      TF s = (e & 1) ? 1 : -1;
      TF s1 = (e & 2) ? 1 : -1;
      TF s2 = (e & 4) ? 1 : -1;
      TF t = u[axis], a = 1 + s1 * u[bit1_axis], b = 1 + s2 * u[bit2_axis];
      TF g = (1 - t * t) * (1 + 3 * s * t);
      TF dg = 3 * s * (1 - t * t) - 2 * t * (1 + 3 * s * t);
      N[first + e] = e64 * g * a * b;
      if (dN0) {
        TF d[3];
        d[axis] = e64 * dg * a * b;
        d[bit1_axis] = e64 * g * s1 * b;
        d[bit2_axis] = e64 * g * a * s2;
        dN0[first + e] = d[0];
        dN1[first + e] = d[1];
        dN2[first + e] = d[2];
      }
    }
  };
  edge_family(8, 0, 2, 1);   // x-edges: bit1 -> z, bit2 -> y
  edge_family(16, 1, 0, 2);  // y-edges: bit1 -> x, bit2 -> z
  edge_family(24, 2, 1, 0);  // z-edges: bit1 -> y, bit2 -> x
}

// The values N of shape_functions() without derivatives, bit for bit (the
// same rounded operations in the same order; sign factors +-1 multiply
// exactly), with the per-axis factors formed once.  Used by the volume-map
// integration, which evaluates 27,000 samples per node.
template <class TF>
inline void shape_values(V3<TF> p, TF N[32]) {
  const TF u[3] = {p.x, p.y, p.z};
  const TF r2 = p.x * p.x + p.y * p.y + p.z * p.z;
  const TF c64 = TF(1) / TF(64), e64 = TF(9) / TF(64);
  const TF f = 9 * r2 - 19;
  TF m[3], q[3], g[3][2];
  for (int k = 0; k < 3; ++k) {
    m[k] = 1 - u[k];  // 1 + (-1) u
    q[k] = 1 + u[k];
    const TF tt = 1 - u[k] * u[k];
    const TF t3 = 3 * u[k];
    g[k][0] = tt * (1 - t3);  // s = -1: 1 + (-3) t
    g[k][1] = tt * (1 + t3);
  }
  for (int j = 0; j < 8; ++j) {
    const TF ax = (j & 1) ? q[0] : m[0], ay = (j & 2) ? q[1] : m[1], az = (j & 4) ? q[2] : m[2];
    N[j] = c64 * ax * ay * az * f;
  }
  const int fam[3][3] = {{0, 2, 1}, {1, 0, 2}, {2, 1, 0}};  // axis, bit1 axis, bit2 axis
  for (int fi = 0; fi < 3; ++fi) {
    const int axis = fam[fi][0], b1 = fam[fi][1], b2 = fam[fi][2];
    for (int e = 0; e < 8; ++e) {
      const TF gg = g[axis][e & 1];
      const TF a = (e & 2) ? q[b1] : m[b1];
      const TF b = (e & 4) ? q[b2] : m[b2];
      N[8 + 8 * fi + e] = e64 * gg * a * b;
    }
  }
}

// Interpolated value (interpolate, runner.hpp:1586-1594) and, optionally,
// gradient scaled by 2 / cell size (interpolate_and_derive,
// runner.hpp:1773-1791).  Returns FLT/DBL max outside the domain
// (interpolate_distance_without_intermediates, runner.hpp:1596-1614).
template <class TF>
struct LagrangeGrid {
  V3<TF> dmin, dmax, cs;
  uint32_t res[3];
  const TF* nodes;
  TF value(V3<TF> x) const {
    // resolve() with the reciprocal cell sizes formed once (same bits)
    const V3<TF> inv{TF(1) / cs.x, TF(1) / cs.y, TF(1) / cs.z};
    if (!(x.x >= dmin.x && x.y >= dmin.y && x.z >= dmin.z && dmax.x >= x.x && dmax.y >= x.y &&
          dmax.z >= x.z))
      return std::numeric_limits<TF>::max();
    int ip[3];
    ip[0] = std::min(int((x.x - dmin.x) * inv.x), int(res[0]) - 1);
    ip[1] = std::min(int((x.y - dmin.y) * inv.y), int(res[1]) - 1);
    ip[2] = std::min(int((x.z - dmin.z) * inv.z), int(res[2]) - 1);
    const V3<TF> lo{dmin.x + cs.x * TF(ip[0]), dmin.y + cs.y * TF(ip[1]),
                    dmin.z + cs.z * TF(ip[2])};
    const V3<TF> xi{2 * (x.x - lo.x) * inv.x - 1, 2 * (x.y - lo.y) * inv.y - 1,
                    2 * (x.z - lo.z) * inv.z - 1};
    TF N[32];
    shape_values(xi, N);
    if (!cache || ip[0] != cache->ip[0] || ip[1] != cache->ip[1] || ip[2] != cache->ip[2]) {
      uint32_t cells[32];
      cell_nodes(res, ip, cells);
      Cache local;
      Cache& c = cache ? *cache : local;
      for (int j = 0; j < 32; ++j) c.v[j] = nodes[cells[j]];
      for (int k = 0; k < 3; ++k) c.ip[k] = ip[k];
      TF phi = 0;
      for (int j = 0; j < 32; ++j) phi += c.v[j] * N[j];
      return phi;
    }
    TF phi = 0;
    for (int j = 0; j < 32; ++j) phi += cache->v[j] * N[j];
    return phi;
  }
  // The node values of the last cell value() visited (consecutive samples of
  // one volume-map node mostly fall into the same cell).
  struct Cache {
    int ip[3] = {-1, -1, -1};
    TF v[32];
  };
  mutable Cache* cache = nullptr;
};

// ------------------------------------------------------- analytic distances
// dg/box_distance.hpp:23-39, dg/sphere_distance.hpp:18-21,
// dg/box_shell_distance.hpp:36-59, the cylinder, capsule, infinite cylinder
// and infinite tube below.  The torus (tube radius r around a circle of
// radius R in the x-z plane) has no reference counterpart.
template <class TF>
struct Shape {
  uint32_t kind;
  TF p[8];
  TF sdf(V3<TF> x) const {
    switch (kind) {
      case AL_SHAPE_BOX: {
        V3<TF> d{std::fabs(x.x) - p[0], std::fabs(x.y) - p[1], std::fabs(x.z) - p[2]};
        V3<TF> cl{std::max(d.x, TF(0)), std::max(d.y, TF(0)), std::max(d.z, TF(0))};
        return std::sqrt(dot(cl, cl)) + std::min(std::max(d.x, std::max(d.y, d.z)), TF(0)) - p[3];
      }
      case AL_SHAPE_SPHERE:
        return std::sqrt(dot(x, x)) - p[0];
      case AL_SHAPE_BOX_SHELL: {
        auto box = [&](TF hx, TF hy, TF hz) {
          V3<TF> d{std::fabs(x.x) - hx, std::fabs(x.y) - hy, std::fabs(x.z) - hz};
          V3<TF> cl{std::max(d.x, TF(0)), std::max(d.y, TF(0)), std::max(d.z, TF(0))};
          return std::sqrt(dot(cl, cl)) + std::min(std::max(d.x, std::max(d.y, d.z)), TF(0)) -
                 p[6];
        };
        TF inner = box(p[0], p[1], p[2]);
        TF outer = box(p[3], p[4], p[5]);
        return std::max(outer, -inner);
      }
      case AL_SHAPE_TORUS: {
        TF rho = std::sqrt(x.x * x.x + x.z * x.z) - p[0];
        return std::sqrt(rho * rho + x.y * x.y) - p[1];
      }
      case AL_SHAPE_CYLINDER: {  // dg/cylinder_distance.hpp:28-35
        const TF d0 = std::sqrt(x.x * x.x + x.z * x.z) - p[0];
        const TF d1 = std::fabs(x.y + p[2]) - p[1] * TF(0.5);
        const TF c0 = std::max(d0, TF(0)), c1 = std::max(d1, TF(0));
        return std::min(std::max(d0, d1), TF(0)) + std::sqrt(c0 * c0 + c1 * c1);
      }
      case AL_SHAPE_CAPSULE: {  // dg/capsule_distance.hpp:24-27
        const TF hh = p[1] * TF(0.5);
        const V3<TF> m{x.x, x.y - std::max(-hh, std::min(x.y, hh)), x.z};
        return std::sqrt(dot(m, m)) - p[0];
      }
      case AL_SHAPE_INFINITE_CYLINDER:  // dg/infinite_cylinder_distance.hpp:20-22
        return std::sqrt(x.x * x.x + x.z * x.z) - p[0];
      case AL_SHAPE_INFINITE_TUBE: {  // dg/infinite_tube_distance.hpp:32-36
        const TF rd = std::sqrt(x.x * x.x + x.z * x.z);
        return std::max(p[0] - rd, rd - p[1]);
      }
      default:
        return std::numeric_limits<TF>::max();
    }
  }
  // Un-normalised outward direction.  Sphere: the position itself
  // (sphere_distance.hpp:21); others: central differences with step
  // h * 2^-8 (box_distance.hpp:28-38).
  V3<TF> gradient(V3<TF> x, TF h) const {
    if (kind == AL_SHAPE_SPHERE) return x;
    // radial direction of the y-invariant shapes
    // (dg/infinite_cylinder_distance.hpp:23-25, dg/infinite_tube_distance.hpp:37-43)
    if (kind == AL_SHAPE_INFINITE_CYLINDER) return V3<TF>{x.x, 0, x.z};
    if (kind == AL_SHAPE_INFINITE_TUBE) {
      const TF s = (x.x * x.x + x.z * x.z) * 4 > (p[0] + p[1]) * (p[0] + p[1]) ? TF(1) : TF(-1);
      return V3<TF>{s * x.x, 0, s * x.z};
    }
    const TF step = h * TF(0.00390625);
    return V3<TF>{sdf(x + V3<TF>{step, 0, 0}) - sdf(x - V3<TF>{step, 0, 0}),
                  sdf(x + V3<TF>{0, step, 0}) - sdf(x - V3<TF>{0, step, 0}),
                  sdf(x + V3<TF>{0, 0, step}) - sdf(x - V3<TF>{0, 0, step})};
  }
};

// -------------------------------------------------------- Peirce quadrature
// Peirce's product rule on the ball (dg/peirce_quadrature.hpp:10-13,
// 484-510) for m = 14: 60 equally spaced azimuths theta_i = 2 pi (i+1)/60,
// 30 Gauss-Legendre nodes in cos(phi) with weights b_j, and 15 radial
// nodes r_k = sqrt(s_k) with s_k the Gauss-Jacobi(0, 1/2) nodes mapped to
// [0,1] and weights c_k = w_k / 2^(5/2), so that sum c_k f(r_k) integrates
// r^2 f(r) over [0,1].  Computed here from those definitions in long double.
constexpr int kNumTheta = 60, kNumPhi = 30, kNumR = 15;

struct PeirceTables {
  double cosphi[kNumPhi], sinphi[kNumPhi], b[kNumPhi], r[kNumR], c[kNumR];
};

namespace detail {
// Jacobi polynomial P_n^(a,b)(t) and its derivative by the three-term
// recurrence (Abramowitz & Stegun 22.7.1, 22.8.1).
inline void jacobi(int n, long double a, long double b, long double t, long double& p,
                   long double& dp) {
  auto value = [&](int m, long double aa, long double bb) {
    long double p0 = 1, p1 = (aa + 1) + (aa + bb + 2) * (t - 1) / 2;
    if (m == 0) return p0;
    for (int k = 2; k <= m; ++k) {
      long double s = 2 * k + aa + bb;
      long double a1 = 2 * k * (k + aa + bb) * (s - 2);
      long double a2 = (s - 1) * (aa * aa - bb * bb);
      long double a3 = (s - 2) * (s - 1) * s;
      long double a4 = 2 * (k + aa - 1) * (k + bb - 1) * s;
      long double p2 = ((a2 + a3 * t) * p1 - a4 * p0) / a1;
      p0 = p1;
      p1 = p2;
    }
    return p1;
  };
  p = value(n, a, b);
  dp = n == 0 ? 0 : (n + a + b + 1) / 2 * value(n - 1, a + 1, b + 1);
}
// Roots of P_n^(a,b) on (-1,1): sign-change bracketing then Newton.
inline std::vector<long double> jacobi_roots(int n, long double a, long double b) {
  std::vector<long double> roots;
  const int kScan = 200000;
  long double prev_t = -1, prev_p, dp;
  jacobi(n, a, b, prev_t, prev_p, dp);
  for (int s = 1; s <= kScan; ++s) {
    long double t = -1 + 2.0L * s / kScan, p;
    jacobi(n, a, b, t, p, dp);
    if ((p < 0) != (prev_p < 0)) {
      long double lo = prev_t, hi = t, plo = prev_p;
      for (int it = 0; it < 200; ++it) {
        long double mid = (lo + hi) / 2, pm;
        jacobi(n, a, b, mid, pm, dp);
        if ((pm < 0) == (plo < 0)) {
          lo = mid;
          plo = pm;
        } else {
          hi = mid;
        }
      }
      long double x = (lo + hi) / 2;
      for (int it = 0; it < 5; ++it) {
        long double px;
        jacobi(n, a, b, x, px, dp);
        if (dp != 0) x -= px / dp;
      }
      roots.push_back(x);
    }
    prev_t = t;
    prev_p = p;
  }
  return roots;
}
}  // namespace detail

inline PeirceTables peirce_tables() {
  PeirceTables t{};
  // Gauss-Legendre (Jacobi a = b = 0): w = 2 / ((1 - x^2) P'(x)^2).
  auto xs = detail::jacobi_roots(kNumPhi, 0, 0);
  for (int j = 0; j < kNumPhi; ++j) {
    long double p, dp;
    detail::jacobi(kNumPhi, 0, 0, xs[j], p, dp);
    t.cosphi[j] = double(xs[j]);
    t.sinphi[j] = double(std::sqrt(1 - xs[j] * xs[j]));
    t.b[j] = double(2 / ((1 - xs[j] * xs[j]) * dp * dp));
  }
  // Gauss-Jacobi (a = 0, b = 1/2): w = 2^(a+b+1) G(n+a+1)G(n+b+1) /
  // (G(n+a+b+1) n!) / ((1 - t^2) P'(t)^2); the Gamma ratio is 1 for a = 0.
  auto ts = detail::jacobi_roots(kNumR, 0, 0.5L);
  for (int k = 0; k < kNumR; ++k) {
    long double p, dp;
    detail::jacobi(kNumR, 0, 0.5L, ts[k], p, dp);
    long double w = std::pow(2.0L, 1.5L) / ((1 - ts[k] * ts[k]) * dp * dp);
    t.r[k] = double(std::sqrt((1 + ts[k]) / 2));
    t.c[k] = double(w / std::pow(2.0L, 2.5L));
  }
  return t;
}

// Volume-map node value (update_volume_field, runner.hpp:1616-1694):
//   V(x) = h^3 sum_ijk w_ijk * ext(sign * phi(x + h r_k u_ij)),
//   ext(d) = 1 for d <= 0, W(d) / W(0) otherwise.
// The per-sample arithmetic follows the reference in TF; the sum is
// accumulated in double (the reference's host check, tests/field_gen.cu:35-46,
// accumulates in double as PeirceQuadrature::integrate does).
template <class TF, class Phi>
TF volume_at(const Cn<TF>& c, const PeirceTables& pt, V3<TF> x, TF sign, Phi phi) {
  const TF pi = TF(3.14159265358979323846264338327950288L);
  double sum = 0;
  for (int i = 0; i < kNumTheta; ++i) {
    TF theta = 2 * pi * TF(i + 1) / TF(kNumTheta);
    TF ct = std::cos(theta), st = std::sin(theta);
    for (int j = 0; j < kNumPhi; ++j) {
      V3<TF> u{TF(pt.sinphi[j]) * ct, TF(pt.sinphi[j]) * st, TF(pt.cosphi[j])};
      for (int k = 0; k < kNumR; ++k) {
        TF w = 2 * pi * TF(pt.b[j]) * TF(pt.c[k]) / TF(kNumTheta);
        TF d = phi(x + (c.h * TF(pt.r[k])) * u) * sign;
        TF ext = d <= 0 ? TF(1) : W_dist(c, d) / c.w0;
        sum += double(w) * double(ext);
      }
    }
  }
  return TF(sum * double(c.h2) * double(c.h));
}

// A volume map whose node values are computed on first use, each by the
// same volume_at() as the eager build (so every value read is the one the
// eager build writes, bit for bit).  A step reads the map only at the 32
// nodes of the Lagrange cells that hold particles; building the whole map
// on the host (1.9 M nodes x 27,000 samples at 64^3) would take far longer
// than the steps it serves.  For analytic distances (exact, 1-Lipschitz
// SDFs) two node classes need no sampling: a node at least 2h (plus
// rounding slack) outside the body has every sample point at d > h, where
// W = 0, so its value is exactly 0; a node at least h inside has every
// sample at d <= 0, so its value is the all-ones sum, computed once with
// the same loop.  Concurrent first uses of one node compute the same bits.
template <class TF>
struct LazyVolume {
  Cn<TF> c;
  PeirceTables pt;
  V3<TF> dmin, dmax, cs;
  uint32_t res[3];
  uint32_t num_nodes;
  uint32_t use_grid;
  TF sign;
  Shape<TF> sdf;
  const TF* dist_nodes;
  TF* values;
  std::vector<std::atomic<uint8_t>> done;
  std::atomic<uint64_t> sampled{0}, skipped{0};
  TF full = 0;

  LazyVolume(const Cn<TF>& c_, V3<TF> dmin_, V3<TF> dmax_, V3<TF> cs_, const uint32_t r[3],
             uint32_t use_grid_, TF sign_, const Shape<TF>& sdf_, const TF* dist, TF* out)
      : c(c_), pt(peirce_tables()), dmin(dmin_), dmax(dmax_), cs(cs_),
        num_nodes(num_grid_nodes(r)), use_grid(use_grid_), sign(sign_), sdf(sdf_),
        dist_nodes(dist), values(out), done(num_grid_nodes(r)) {
    for (int k = 0; k < 3; ++k) res[k] = r[k];
    for (auto& d : done) d.store(0, std::memory_order_relaxed);
    const TF big = std::numeric_limits<TF>::max() / TF(4);
    full = volume_at(c, pt, V3<TF>{0, 0, 0}, sign, [&](V3<TF>) { return -sign * big; });
  }
  // Value of node l; `skip` tells whether a shortcut gave it.
  TF compute(uint32_t l, bool& skip) {
    const V3<TF> x = node_position(dmin, res, cs, l);
    skip = false;
    if (use_grid) {
      LagrangeGrid<TF> grid{dmin, dmax, cs, {res[0], res[1], res[2]}, dist_nodes};
      typename LagrangeGrid<TF>::Cache cache;
      grid.cache = &cache;
      return volume_at(c, pt, x, sign, [&](V3<TF> p) { return grid.value(p); });
    }
    const TF d0 = sdf.sdf(x) * sign;
    const TF mag = std::max(std::fabs(x.x), std::max(std::fabs(x.y), std::fabs(x.z))) + c.h;
    const TF slack = TF(1e-3) * c.h + TF(64) * std::numeric_limits<TF>::epsilon() * mag;
    skip = true;
    if (d0 >= TF(2) * c.h + slack) return TF(0);
    if (d0 <= -(c.h + slack)) return full;
    skip = false;
    return volume_at(c, pt, x, sign, [&](V3<TF> p) { return sdf.sdf(p); });
  }
  TF get(uint32_t l) {
    if (done[l].load(std::memory_order_acquire)) return values[l];
    bool skip;
    const TF v = compute(l, skip);
    __atomic_store(&values[l], &v, __ATOMIC_RELAXED);
    uint8_t expected = 0;
    if (done[l].compare_exchange_strong(expected, 1, std::memory_order_acq_rel))
      (skip ? skipped : sampled).fetch_add(1, std::memory_order_relaxed);
    return v;
  }
};

// ------------------------------------------------------------------ bodies
template <class TF>
struct Body {
  uint32_t shape, use_grid;
  TF sign;
  V3<TF> dmin, dmax, cs;
  uint32_t res[3];
  uint32_t num_nodes;
  const TF* dist_nodes;
  const TF* vol_nodes;
  LazyVolume<TF>* lazy_vol = nullptr;  // when set, vol_nodes fill on first use
  Shape<TF> sdf;
  TF max_distance, mass;
  V3<TF> inertia;
  // kinematics (pile.hpp:103-110)
  V3<TF> x, v, omega;
  V4<TF> q;
  TF vol(uint32_t l) const { return lazy_vol ? lazy_vol->get(l) : vol_nodes[l]; }
};

// Boundary sample of one particle against one body:
// compute_volume_and_boundary_x (runner.hpp:1696-1734, distance grid) and
// compute_volume_and_boundary_x_analytic<0> (runner.hpp:1736-1771), then
// compute_particle_boundary[_analytic] (runner.hpp:1982-2025).
template <class TF>
void boundary_sample(const Cn<TF>& c, const Body<TF>& b, V3<TF> x, V4<TF>& bnd, V4<TF>& bk) {
  V3<TF> local = rotate(x - b.x, conjugate(b.q));
  // compute_volume_and_boundary_x_analytic<1> (runner.hpp:1744-1746)
  if (b.shape == AL_SHAPE_INFINITE_CYLINDER || b.shape == AL_SHAPE_INFINITE_TUBE) local.y = 0;
  V3<TF> bx = x, xi_bxj{0, 0, 0};
  TF d = 0, vol = 0;
  int ip[3];
  V3<TF> xi;
  bool inside = resolve(b.dmin, b.dmax, b.res, b.cs, local, ip, xi);
  TF N[32], d0[32], d1[32], d2[32];
  uint32_t cells[32];
  if (b.use_grid) {
    if (inside) {
      shape_functions<TF>(xi, N, d0, d1, d2);
      cell_nodes(b.res, ip, cells);
      TF phi = 0;
      V3<TF> grad{0, 0, 0};
      for (int j = 0; j < 32; ++j) {
        TF v = b.dist_nodes[cells[j]];
        phi += v * N[j];
        grad.x += v * d0[j];
        grad.y += v * d1[j];
        grad.z += v * d2[j];
      }
      grad.x *= TF(2) / b.cs.x;
      grad.y *= TF(2) / b.cs.y;
      grad.z *= TF(2) / b.cs.z;
      d = phi * b.sign;
      V3<TF> nrm = rotate(grad * b.sign, b.q);
      TF nl2 = length_sqr(nrm);
      nrm = (nl2 > 0 ? inv_sqrt(nl2) : TF(0)) * nrm;
      xi_bxj = d * nrm;
      bx = x - xi_bxj;
      for (int j = 0; j < 32; ++j) vol += b.vol(cells[j]) * N[j];
    }
  } else {
    d = b.sdf.sdf(local) * b.sign;
    V3<TF> nrm = rotate(b.sdf.gradient(local, c.h) * b.sign, b.q);
    TF nl2 = length_sqr(nrm);
    nrm = (nl2 > 0 ? inv_sqrt(nl2) : TF(0)) * nrm;
    xi_bxj = d * nrm;
    bx = x - xi_bxj;
    if (inside) {
      shape_functions<TF>(xi, N, nullptr, nullptr, nullptr);
      cell_nodes(b.res, ip, cells);
      for (int j = 0; j < 32; ++j) vol += b.vol(cells[j]) * N[j];
    }
  }
  V3<TF> kg = gradW(c, xi_bxj);
  bnd = {bx.x, bx.y, bx.z, vol};
  bk = {vol * kg.x, vol * kg.y, vol * kg.z, vol * W_dist(c, d)};
}

// ------------------------------------------------------------- fluid state
template <class TF>
struct Fluid {
  uint32_t n = 0, nb = 0;
  // periodic in y (step<1>): Const::wrap_length, 0 when not periodic
  bool wrap = false;
  TF wrap_len = 0;
  std::vector<V3<TF>> x, v, a;
  std::vector<TF> density, factor, kappa, kappa_v, density_adv;
  std::vector<TF> pressure, last_pressure, aii, density_err;
  std::vector<V3<TF>> dii, dij_pj, pressure_accel;
  std::vector<V4<TF>> bnd, bk;          // [nb][n]
  std::vector<V3<TF>> force, torque;    // [nb][n] per-particle rigid force
  NeighborList nl;
  GridSort gs;
  void resize(uint32_t n_, uint32_t nb_) {
    n = n_;
    nb = nb_;
    a.assign(n, {0, 0, 0});
    density.assign(n, 0);
    factor.assign(n, 0);
    density_adv.assign(n, 0);
    if (kappa.size() != n) kappa.assign(n, 0);
    if (kappa_v.size() != n) kappa_v.assign(n, 0);
    if (pressure.size() != n) pressure.assign(n, 0);
    last_pressure.assign(n, 0);
    aii.assign(n, 0);
    density_err.assign(n, 0);
    dii.assign(n, {0, 0, 0});
    dij_pj.assign(n, {0, 0, 0});
    pressure_accel.assign(n, {0, 0, 0});
    bnd.assign(size_t(nb) * n, {0, 0, 0, 0});
    bk.assign(size_t(nb) * n, {0, 0, 0, 0});
    force.assign(size_t(nb) * n, {0, 0, 0});
    torque.assign(size_t(nb) * n, {0, 0, 0});
  }
};

// compute_all_boundaries (solver.hpp:170-185).
template <class TF>
void compute_boundaries(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, Fluid<TF>& f) {
  for (uint32_t b = 0; b < f.nb; ++b) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(f.n); ++i)
      boundary_sample(c, bodies[b], f.x[i], f.bnd[size_t(b) * f.n + i], f.bk[size_t(b) * f.n + i]);
  }
}

// compute_density (runner.hpp:2052-2072).
template <class TF>
void compute_density(const Cn<TF>& c, Fluid<TF>& f) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(f.n); ++ii) {
    uint32_t i = uint32_t(ii);
    TF rho = c.vol * c.w0;
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      rho += c.vol * W_r2(c, length_sqr(xv(f, i, j)));
    }
    for (uint32_t b = 0; b < f.nb; ++b) rho += f.bk[size_t(b) * f.n + i].w;
    f.density[i] = rho * c.rho0;
  }
}

// update_particle_neighbors<0> (solver.hpp:225-260): grid, list, density.
template <class TF>
void update_particle_neighbors(const Cn<TF>& c, const al_consti& g, Fluid<TF>& f) {
  f.gs = grid_sort(c, g, f.x.data(), f.n);
  f.nl = neighbor_list(c, g, f.x.data(), f.n, f.gs, f.wrap, f.wrap_len);
  compute_density(c, f);
}

// x_i - x_j, y wrapped on a periodic step (make_neighbor_list<1>,
// runner.hpp:1893-1894).
template <class TF>
inline V3<TF> xv(const Fluid<TF>& f, uint32_t i, uint32_t j) {
  V3<TF> d = f.x[i] - f.x[j];
  d.y = wrap_coord(f.wrap, f.wrap_len, d.y);
  return d;
}
template <class TF>
inline V3<TF> body_velocity(const Body<TF>& b, V3<TF> at) {
  return cross(b.omega, at - b.x) + b.v;
}

// compute_dfsph_factor (runner.hpp:3123-3154).
template <class TF>
void compute_dfsph_factor(const Cn<TF>& c, Fluid<TF>& f) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(f.n); ++ii) {
    uint32_t i = uint32_t(ii);
    TF sum = 0;
    V3<TF> gi{0, 0, 0};
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      V3<TF> gj = (-c.vol) * gradW(c, xv(f, i, j));
      sum += length_sqr(gj);
      gi -= gj;
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      gi += V3<TF>{k4.x, k4.y, k4.z};
    }
    sum += length_sqr(gi);
    f.factor[i] = sum > c.eps ? -1 / sum : TF(0);
  }
}

// compute_density_change (runner.hpp:3192-3228).
template <class TF>
TF density_change(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, const Fluid<TF>& f,
                  uint32_t i) {
  TF adv = 0;
  V3<TF> vi = f.v[i];
  for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
    uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
    adv += c.vol * dot(vi - f.v[j], gradW(c, xv(f, i, j)));
  }
  for (uint32_t b = 0; b < f.nb; ++b) {
    const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
    const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
    V3<TF> vj = body_velocity(bodies[b], V3<TF>{bn.x, bn.y, bn.z});
    adv += dot(vi - vj, V3<TF>{k4.x, k4.y, k4.z});
  }
  adv = std::max(adv, TF(0));
  if (f.nl.count[i] < 20) adv = 0;
  return adv;
}

// compute_density_adv (runner.hpp:3493-3523).
template <class TF>
TF density_adv(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, const Fluid<TF>& f,
               uint32_t i, TF dt) {
  TF delta = 0;
  V3<TF> vi = f.v[i];
  for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
    uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
    delta += c.vol * dot(vi - f.v[j], gradW(c, xv(f, i, j)));
  }
  for (uint32_t b = 0; b < f.nb; ++b) {
    const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
    const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
    V3<TF> vj = body_velocity(bodies[b], V3<TF>{bn.x, bn.y, bn.z});
    delta += dot(vi - vj, V3<TF>{k4.x, k4.y, k4.z});
  }
  return std::max(f.density[i] / c.rho0 + dt * delta, TF(1));
}

// Shared body of the kappa-driven velocity updates
// (warm_start_divergence_solve_1 runner.hpp:3251-3295,
//  divergence_solve_iteration :3316-3363, warm_start_pressure_solve1
//  :3451-3491, pressure_solve_iteration :3543-3588).  `kappa_of(j)` returns
// the neighbor's coefficient; the pair term is dv += sgn * dt * (k_i + k_j)
// * V * gradW with sgn = -1 for the divergence forms (written there as
// dv -= dt * k_sum * (-V gradW)) and +1 for the pressure forms.
template <class TF, class KappaOf>
void kappa_velocity_update(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, Fluid<TF>& f,
                           uint32_t i, TF ki, KappaOf kappa_of, TF dt, bool divergence_form,
                           V3<TF>& dv) {
  dv = {0, 0, 0};
  for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
    uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
    TF ksum = ki + kappa_of(j);
    if (std::fabs(ksum) > c.eps) {
      if (divergence_form) {
        V3<TF> gpj = (-c.vol) * gradW(c, xv(f, i, j));
        dv -= (dt * ksum) * gpj;
      } else {
        dv += (dt * ksum * c.vol) * gradW(c, xv(f, i, j));
      }
    }
  }
  if (std::fabs(ki) > c.eps) {
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      V3<TF> a = ki * (-V3<TF>{k4.x, k4.y, k4.z});
      V3<TF> force = c.mass * a;
      dv -= dt * a;
      f.force[size_t(b) * f.n + i] += force;
      f.torque[size_t(b) * f.n + i] += cross(V3<TF>{bn.x, bn.y, bn.z} - bodies[b].x, force);
    }
  }
}

// Orthonormal tangents of a unit normal (get_orthogonal_vectors,
// runner.hpp:119-131).
template <class TF>
void tangents(V3<TF> n, V3<TF>& t1, V3<TF>& t2) {
  V3<TF> v{1, 0, 0};
  if (std::fabs(dot(v, n)) > TF(0.999)) v = {0, 1, 0};
  t1 = cross(n, v);
  t2 = cross(n, t1);
  t1 = normalized(t1);
  t2 = normalized(t2);
}

// clear_acceleration + compute_viscosity (runner.hpp:1974-1980, 2150-2249).
template <class TF>
void compute_viscosity(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, Fluid<TF>& f) {
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(f.n); ++ii) {
    uint32_t i = uint32_t(ii);
    V3<TF> vi = f.v[i], xi = f.x[i], da{0, 0, 0};
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      V3<TF> d = xv(f, i, j);
      da += (c.visc * c.mass / f.density[j] * dot(d, gradW(c, d)) /
             (length_sqr(d) + TF(0.01) * c.h2)) *
            (vi - f.v[j]);
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
      V3<TF> bxj{bn.x, bn.y, bn.z};
      const Body<TF>& body = bodies[b];
      V3<TF> nrm = bxj - xi;
      TF nl2 = length_sqr(nrm);
      if (!(nl2 > 0)) continue;
      nrm = inv_sqrt(nl2) * nrm;
      V3<TF> t1, t2;
      tangents(nrm, t1, t2);
      TF dist = c.h - std::sqrt(nl2);
      V3<TF> pts[4] = {bxj - t1 * dist, bxj + t1 * dist, bxj - t2 * dist, bxj + t2 * dist};
      TF vol = TF(0.25) * bn.w;
      V3<TF> fsum{0, 0, 0}, tsum{0, 0, 0};
      V3<TF> acc[4];
      for (int s = 0; s < 4; ++s) {
        V3<TF> xix = xi - pts[s];
        V3<TF> vb = body_velocity(body, pts[s]);
        acc[s] = (c.bvisc * vol * dot(xix, gradW(c, xix)) / (length_sqr(xix) + TF(0.01) * c.h2)) *
                 (vi - vb);
      }
      da += acc[0] + acc[1] + acc[2] + acc[3];
      for (int s = 0; s < 4; ++s) {
        V3<TF> fs = (-c.mass) * acc[s];
        fsum += fs;
        tsum += cross(pts[s] - body.x, fs);
      }
      f.force[size_t(b) * f.n + i] += fsum;
      f.torque[size_t(b) * f.n + i] += tsum;
    }
    f.a[i] = c.g + da;
  }
}

// --------------------------------------------------------------- solvers
struct SolverParams {
  double density_change_tolerance = 1e-3, density_error_tolerance = 1e-3;
  uint32_t min_density_solve = 2, max_density_solve = 100;
  uint32_t min_divergence_solve = 1, max_divergence_solve = 100;
  double cfl = 0.4, max_dt = 2e-4, min_dt = 0;
  bool enable_divergence_solve = true, enable_density_solve = true;
};

struct StepReport {
  uint32_t num_divergence_solve = 0, num_density_solve = 0;
  double mean_density_change = 0, mean_density_error = 0;
  double particle_max_v2 = 0, pile_max_v2 = 0, max_v2 = 0, cfl_dt = 0, utilized_cfl = 0;
  double dt = 0;
  uint32_t grid_anomaly[3] = {0, 0, 0};
};

// Pile::calculate_cfl_v2 (pile.hpp:816-825).
template <class TF>
double pile_max_v2(const std::vector<Body<TF>>& bodies) {
  double m = -std::numeric_limits<TF>::max();
  for (const Body<TF>& b : bodies) {
    V3<TF> w = cross(b.omega, V3<TF>{b.max_distance, 0, 0}) + b.v;
    m = std::max(m, double(length_sqr(w)));
  }
  return m;
}

// Solver::update_dt (solver.hpp:153-169) with calculate_cfl_v2
// (runner.hpp:2533-2541).
template <class TF>
void update_dt(const Cn<TF>& c, const std::vector<Body<TF>>& bodies, Fluid<TF>& f,
               const SolverParams& sp, TF& dt, StepReport& rep) {
  TF pmax = -std::numeric_limits<TF>::max();
  for (uint32_t i = 0; i < f.n; ++i) pmax = std::max(pmax, length_sqr(f.v[i] + f.a[i] * dt));
  rep.particle_max_v2 = pmax;
  rep.pile_max_v2 = bodies.empty() ? -std::numeric_limits<TF>::max() : TF(pile_max_v2(bodies));
  TF max_v2 = std::max(TF(rep.particle_max_v2), TF(rep.pile_max_v2));
  rep.max_v2 = max_v2;
  TF max_v = std::sqrt(max_v2);
  TF length_scale = c.radius * 2;
  TF cfl_dt = TF(sp.cfl) * length_scale / max_v;
  rep.cfl_dt = cfl_dt;
  dt = std::max(std::min(cfl_dt, TF(sp.max_dt)), TF(sp.min_dt));
  rep.utilized_cfl = dt * max_v / length_scale;
}

// Per-body totals of the per-particle rigid force/torque entries
// (solver_df.hpp:346-353), accumulated in double.
template <class TF>
void rigid_totals(const Fluid<TF>& f, std::vector<V3<double>>& F, std::vector<V3<double>>& T) {
  F.assign(f.nb, {0, 0, 0});
  T.assign(f.nb, {0, 0, 0});
  for (uint32_t b = 0; b < f.nb; ++b)
    for (uint32_t i = 0; i < f.n; ++i) {
      const V3<TF>& fi = f.force[size_t(b) * f.n + i];
      const V3<TF>& ti = f.torque[size_t(b) * f.n + i];
      F[b] += V3<double>{fi.x, fi.y, fi.z};
      T[b] += V3<double>{ti.x, ti.y, ti.z};
    }
}

// Pile::integrate_kinematics (pile.hpp:794-815) with calculate_dq and
// calculate_angular_acceleration (runner.hpp:202-251).
template <class TF>
void integrate_kinematics(std::vector<Body<TF>>& bodies, const std::vector<V3<double>>& F,
                          const std::vector<V3<double>>& T, V3<TF> gravity, TF dt) {
  for (size_t i = 0; i < bodies.size(); ++i) {
    Body<TF>& b = bodies[i];
    auto dq = [](V3<TF> w, V4<TF> q) {
      return V4<TF>{TF(0.5) * (w.x * q.w + w.y * q.z - w.z * q.y),
                    TF(0.5) * (-w.x * q.z + w.y * q.w + w.z * q.x),
                    TF(0.5) * (w.x * q.y - w.y * q.x + w.z * q.w),
                    TF(0.5) * (-w.x * q.x - w.y * q.y - w.z * q.z)};
    };
    auto advance_q = [&](void) {
      V4<TF> d = dq(b.omega, b.q);
      V4<TF> q{b.q.x + dt * d.x, b.q.y + dt * d.y, b.q.z + dt * d.z, b.q.w + dt * d.w};
      TF inv = inv_sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
      b.q = {q.x * inv, q.y * inv, q.z * inv, q.w * inv};
    };
    if (b.mass == 0) {
      b.x += b.v * dt;
      advance_q();
      continue;
    }
    V3<TF> force{TF(F[i].x), TF(F[i].y), TF(F[i].z)};
    V3<TF> torque{TF(T[i].x), TF(T[i].y), TF(T[i].z)};
    b.v += (1 / b.mass) * force * dt;
    // world-frame inverse inertia R diag(1/I) R^T applied to the torque
    V4<TF> q = b.q;
    V3<TF> ii{1 / b.inertia.x, 1 / b.inertia.y, 1 / b.inertia.z};
    TF m[3][3] = {{1 - 2 * (q.y * q.y + q.z * q.z), 2 * (q.x * q.y - q.z * q.w),
                   2 * (q.x * q.z + q.y * q.w)},
                  {2 * (q.x * q.y + q.z * q.w), 1 - 2 * (q.x * q.x + q.z * q.z),
                   2 * (q.y * q.z - q.x * q.w)},
                  {2 * (q.x * q.z - q.y * q.w), 2 * (q.y * q.z + q.x * q.w),
                   1 - 2 * (q.x * q.x + q.y * q.y)}};
    TF tq[3] = {torque.x, torque.y, torque.z}, alpha[3];
    for (int r = 0; r < 3; ++r) {
      TF s = 0;
      for (int k = 0; k < 3; ++k) {
        TF cong = ii.x * m[r][0] * m[k][0] + ii.y * m[r][1] * m[k][1] + ii.z * m[r][2] * m[k][2];
        s += tq[k] * cong;
      }
      alpha[r] = s;
    }
    b.omega += V3<TF>{alpha[0], alpha[1], alpha[2]} * dt;
    advance_q();
    V3<TF> dx = (gravity * dt + b.v) * dt;
    b.x += dx;
    b.v = (1 / dt) * dx;
  }
}

// SolverDf<TF>::step<0> (solver_df.hpp:74-359) without contacts.
template <class TF>
StepReport df_step(const Cn<TF>& c, const al_consti& g, std::vector<Body<TF>>& bodies, Fluid<TF>& f,
                   const SolverParams& sp, TF& dt, V3<TF> pile_gravity, bool integrate_bodies,
                   std::vector<V3<double>>* F_out = nullptr,
                   std::vector<V3<double>>* T_out = nullptr) {
  StepReport rep;
  const uint32_t n = f.n;
  std::fill(f.force.begin(), f.force.end(), V3<TF>{0, 0, 0});
  std::fill(f.torque.begin(), f.torque.end(), V3<TF>{0, 0, 0});
  compute_boundaries(c, bodies, f);
  update_particle_neighbors(c, g, f);
  rep.grid_anomaly[0] = f.gs.out_of_grid;
  rep.grid_anomaly[1] = f.gs.cell_overflow;
  rep.grid_anomaly[2] = f.nl.overflow;
  compute_dfsph_factor(c, f);
  if (sp.enable_divergence_solve) {
    // warm_start_divergence_solve_0 (runner.hpp:3230-3249)
    std::vector<TF> adv0(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) adv0[i] = density_change(c, bodies, f, uint32_t(i));
    for (uint32_t i = 0; i < n; ++i)
      f.kappa_v[i] = adv0[i] > 0 ? TF(0.5) * std::max(f.kappa_v[i], TF(-0.5)) / dt : TF(0);
    // warm_start_divergence_solve_1
    std::vector<V3<TF>> dv(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i)
      kappa_velocity_update(c, bodies, f, uint32_t(i), f.kappa_v[i],
                            [&](uint32_t j) { return f.kappa_v[j]; }, dt, true, dv[i]);
    for (uint32_t i = 0; i < n; ++i) f.v[i] += dv[i];
    // compute_velocity_of_density_change (runner.hpp:3297-3314)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
      f.density_adv[i] = density_change(c, bodies, f, uint32_t(i));
      f.factor[i] *= 1 / dt;
    }
    double mean = std::numeric_limits<double>::max();
    uint32_t it = 0;
    std::vector<TF> ki(n);
    while ((mean > sp.density_change_tolerance / double(dt) || it < sp.min_divergence_solve) &&
           it < sp.max_divergence_solve) {
      // divergence_solve_iteration (runner.hpp:3316-3363)
      for (uint32_t i = 0; i < n; ++i) ki[i] = f.density_adv[i] * f.factor[i];
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < int64_t(n); ++i)
        kappa_velocity_update(c, bodies, f, uint32_t(i), ki[i],
                              [&](uint32_t j) { return ki[j]; }, dt, true, dv[i]);
      for (uint32_t i = 0; i < n; ++i) {
        f.kappa_v[i] += ki[i];
        f.v[i] += dv[i];
      }
      // compute_divergence_solve_density_error (runner.hpp:3396-3410)
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < int64_t(n); ++i)
        f.density_adv[i] = density_change(c, bodies, f, uint32_t(i));
      double s = 0;
      for (uint32_t i = 0; i < n; ++i) s += double(f.density_adv[i]);
      mean = s / double(n);
      ++it;
    }
    rep.num_divergence_solve = it;
    rep.mean_density_change = mean;
    // divergence_solve_finish (runner.hpp:3412-3420)
    for (uint32_t i = 0; i < n; ++i) {
      f.factor[i] *= dt;
      f.kappa_v[i] *= dt;
    }
  }
  compute_viscosity(c, bodies, f);
  update_dt(c, bodies, f, sp, dt, rep);
  rep.dt = dt;
  // integrate_non_pressure_acceleration (runner.hpp:3422-3428)
  for (uint32_t i = 0; i < n; ++i) f.v[i] += dt * f.a[i];
  if (sp.enable_density_solve) {
    // warm_start_pressure_solve0 (runner.hpp:3430-3449)
    std::vector<TF> adv0(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) adv0[i] = density_adv(c, bodies, f, uint32_t(i), dt);
    for (uint32_t i = 0; i < n; ++i)
      f.kappa[i] = adv0[i] > TF(1.0)
                       ? TF(0.5) * std::max(f.kappa[i], TF(-0.00025)) / (dt * dt)
                       : TF(0);
    // warm_start_pressure_solve1
    std::vector<V3<TF>> dv(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i)
      kappa_velocity_update(c, bodies, f, uint32_t(i), f.kappa[i],
                            [&](uint32_t j) { return f.kappa[j]; }, dt, false, dv[i]);
    for (uint32_t i = 0; i < n; ++i) f.v[i] += dv[i];
    // compute_rho_adv (runner.hpp:3525-3541)
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i) {
      f.density_adv[i] = density_adv(c, bodies, f, uint32_t(i), dt);
      f.factor[i] *= 1 / (dt * dt);
    }
    double mean = std::numeric_limits<double>::max();
    uint32_t it = 0;
    std::vector<TF> ki(n);
    while ((mean > sp.density_error_tolerance || it < sp.min_density_solve) &&
           it < sp.max_density_solve) {
      // pressure_solve_iteration (runner.hpp:3543-3588)
      for (uint32_t i = 0; i < n; ++i) ki[i] = (f.density_adv[i] - 1) * f.factor[i];
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < int64_t(n); ++i)
        kappa_velocity_update(c, bodies, f, uint32_t(i), ki[i],
                              [&](uint32_t j) { return ki[j]; }, dt, false, dv[i]);
      for (uint32_t i = 0; i < n; ++i) {
        f.kappa[i] += ki[i];
        f.v[i] += dv[i];
      }
      // compute_pressure_solve_density_error (runner.hpp:3590-3604); the
      // mean is formed as sum(rho_adv - 1) / N in double
      // (solver_df.hpp:323-325 forms sum / N - 1 in TF).
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < int64_t(n); ++i)
        f.density_adv[i] = density_adv(c, bodies, f, uint32_t(i), dt);
      double s = 0;
      for (uint32_t i = 0; i < n; ++i) s += double(f.density_adv[i]) - 1.0;
      mean = s / double(n);
      ++it;
    }
    rep.num_density_solve = it;
    rep.mean_density_error = mean;
    // pressure_solve_finish (runner.hpp:3606-3611)
    for (uint32_t i = 0; i < n; ++i) f.kappa[i] *= dt * dt;
  }
  // integrate_velocity<0> (runner.hpp:3613-3623)
  for (uint32_t i = 0; i < n; ++i) {  // integrate_velocity<wrap>
    f.x[i] += dt * f.v[i];
    f.x[i].y = wrap_coord(f.wrap, f.wrap_len, f.x[i].y);
  }
  std::vector<V3<double>> F, T;
  rigid_totals(f, F, T);
  if (F_out) *F_out = F;
  if (T_out) *T_out = T;
  if (integrate_bodies) integrate_kinematics(bodies, F, T, pile_gravity, dt);
  return rep;
}

// compute_pressure_accels (runner.hpp:2774-2817), kinematic_integration<0>
// (runner.hpp:2873-2887), the per-body totals and Pile::integrate_kinematics:
// the common tail of SolverIi::step and SolverI::step.
template <class TF>
void pressure_accels_and_integrate(const Cn<TF>& c, std::vector<Body<TF>>& bodies, Fluid<TF>& f,
                                   TF dt, std::vector<V3<double>>* F_out,
                                   std::vector<V3<double>>* T_out, V3<TF> pile_gravity,
                                   bool integrate_bodies) {
  const uint32_t n = f.n;
  const TF rho0 = c.rho0;
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    uint32_t i = uint32_t(ii);
    TF rho = f.density[i], dpi = f.pressure[i] / (rho * rho);
    V3<TF> ai{0, 0, 0};
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      TF rj = f.density[j], dpj = f.pressure[j] / (rj * rj);
      ai -= (c.mass * (dpi + dpj)) * gradW(c, xv(f, i, j));
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      V3<TF> a = (rho0 * dpi) * V3<TF>{k4.x, k4.y, k4.z};
      V3<TF> force = c.mass * a;
      ai -= a;
      f.force[size_t(b) * f.n + i] += force;
      f.torque[size_t(b) * f.n + i] += cross(V3<TF>{bn.x, bn.y, bn.z} - bodies[b].x, force);
    }
    f.pressure_accel[i] = rho0 * ai;
  }
  // kinematic_integration<wrap> (runner.hpp:2873-2887)
  for (uint32_t i = 0; i < n; ++i) {
    V3<TF> v = f.v[i] + f.pressure_accel[i] * dt;
    f.x[i] += v * dt;
    f.x[i].y = wrap_coord(f.wrap, f.wrap_len, f.x[i].y);
    f.v[i] = v;
  }
  std::vector<V3<double>> F, T;
  rigid_totals(f, F, T);
  if (F_out) *F_out = F;
  if (T_out) *T_out = T;
  if (integrate_bodies) integrate_kinematics(bodies, F, T, pile_gravity, dt);
}

// SolverIi<TF>::step<0> (solver_ii.hpp:76-243) without contacts.
template <class TF>
StepReport ii_step(const Cn<TF>& c, const al_consti& g, std::vector<Body<TF>>& bodies, Fluid<TF>& f,
                   const SolverParams& sp, TF& dt, V3<TF> pile_gravity, bool integrate_bodies,
                   std::vector<V3<double>>* F_out = nullptr,
                   std::vector<V3<double>>* T_out = nullptr) {
  StepReport rep;
  const uint32_t n = f.n;
  std::fill(f.force.begin(), f.force.end(), V3<TF>{0, 0, 0});
  std::fill(f.torque.begin(), f.torque.end(), V3<TF>{0, 0, 0});
  compute_boundaries(c, bodies, f);
  update_particle_neighbors(c, g, f);
  rep.grid_anomaly[0] = f.gs.out_of_grid;
  rep.grid_anomaly[1] = f.gs.cell_overflow;
  rep.grid_anomaly[2] = f.nl.overflow;
  compute_viscosity(c, bodies, f);
  update_dt(c, bodies, f, sp, dt, rep);
  rep.dt = dt;
  const TF V = c.vol, rho0 = c.rho0;
  // predict_advection0 (runner.hpp:2609-2639)
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    uint32_t i = uint32_t(ii);
    f.v[i] += dt * f.a[i];
    f.last_pressure[i] = f.pressure[i] * TF(0.5);
    TF rho = f.density[i], rho2 = rho * rho;
    V3<TF> dii{0, 0, 0};
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      dii -= (V / rho2) * gradW(c, xv(f, i, j));
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      dii -= V3<TF>{k4.x / rho2, k4.y / rho2, k4.z / rho2};
    }
    f.dii[i] = dii * rho0;
  }
  // predict_advection1 (runner.hpp:2640-2690)
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    uint32_t i = uint32_t(ii);
    V3<TF> vi = f.v[i], dii = f.dii[i];
    TF rho = f.density[i], rho2 = rho * rho, inv_rho2 = 1 / rho2, dpi = V * inv_rho2;
    TF adv = rho / rho0, aii = 0;
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      V3<TF> gw = gradW(c, xv(f, i, j));
      V3<TF> dji = (dpi * rho0) * gw;
      adv += dt * V * dot(vi - f.v[j], gw);
      aii += V * dot(dii - dji, gw);
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      V3<TF> gw{k4.x, k4.y, k4.z};
      V3<TF> vj = body_velocity(bodies[b], V3<TF>{bn.x, bn.y, bn.z});
      V3<TF> dji = (inv_rho2 * rho0) * gw;
      adv += dt * dot(vi - vj, gw);
      aii += dot(dii - dji, gw);
    }
    f.density_adv[i] = adv;
    f.aii[i] = aii * rho0;
  }
  double mean = std::numeric_limits<double>::max();
  uint32_t it = 0;
  while ((mean > sp.density_error_tolerance || it < sp.min_density_solve) &&
         it < sp.max_density_solve) {
    // pressure_solve_iteration0 (runner.hpp:2691-2715)
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(n); ++ii) {
      uint32_t i = uint32_t(ii);
      V3<TF> s{0, 0, 0};
      for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
        uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
        TF rj = f.density[j], rj2 = rj * rj;
        s -= (V / rj2 * f.last_pressure[j]) * gradW(c, xv(f, i, j));
      }
      f.dij_pj[i] = s * rho0;
    }
    // pressure_solve_iteration1 (runner.hpp:2716-2772)
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(n); ++ii) {
      uint32_t i = uint32_t(ii);
      TF lp = f.last_pressure[i];
      V3<TF> dij_pj = f.dij_pj[i];
      TF rho = f.density[i], rho2 = rho * rho, dpi = V / rho2;
      TF bterm = 1 - f.density_adv[i], dt2 = dt * dt, aii = f.aii[i], denom = aii * dt2;
      const TF omega = TF(2) / 3;
      TF p = 0, sum = 0;
      for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
        uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
        V3<TF> gw = gradW(c, xv(f, i, j));
        V3<TF> dji = (dpi * rho0) * gw;
        V3<TF> dji_pi = dji * lp;
        sum += V * dot(dij_pj - f.dii[j] * f.last_pressure[j] - (f.dij_pj[j] - dji_pi), gw);
      }
      for (uint32_t b = 0; b < f.nb; ++b) {
        const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
        sum += dot(dij_pj, V3<TF>{k4.x, k4.y, k4.z});
      }
      sum *= rho0;
      if (std::fabs(denom) > TF(1.0e-9))
        p = std::max((1 - omega) * lp + omega / denom * (bterm - dt2 * sum), TF(0));
      f.density_err[i] = p == 0 ? TF(0) : (denom * p + sum * dt2 - bterm);
      f.pressure[i] = p;
    }
    for (uint32_t i = 0; i < n; ++i) f.last_pressure[i] = f.pressure[i];
    double s = 0;
    for (uint32_t i = 0; i < n; ++i) s += double(f.density_err[i]);
    mean = s / double(n);
    ++it;
  }
  rep.num_density_solve = it;
  rep.mean_density_error = mean;
  pressure_accels_and_integrate(c, bodies, f, dt, F_out, T_out, pile_gravity, integrate_bodies);
  return rep;
}

// SolverI<TF>::step<0> (solver_i.hpp:79-327), the implicit SPH solver
// with volume-map boundaries, without contacts:
//   advect_and_init_pressure (runner.hpp:2889-2900)
//   calculate_isph_diagonal_adv_density (runner.hpp:2901-2954)
//   isph_solve_iteration (runner.hpp:3006-3053): damped Jacobi, weight 2/3,
//     on the last pressures, then last <- pressure and the mean density
//     error (solver_i.hpp:243-276)
//   then the tail shared with SolverIi.
template <class TF>
StepReport i_step(const Cn<TF>& c, const al_consti& g, std::vector<Body<TF>>& bodies, Fluid<TF>& f,
                  const SolverParams& sp, TF& dt, V3<TF> pile_gravity, bool integrate_bodies,
                  std::vector<V3<double>>* F_out = nullptr,
                  std::vector<V3<double>>* T_out = nullptr) {
  StepReport rep;
  const uint32_t n = f.n;
  std::fill(f.force.begin(), f.force.end(), V3<TF>{0, 0, 0});
  std::fill(f.torque.begin(), f.torque.end(), V3<TF>{0, 0, 0});
  compute_boundaries(c, bodies, f);
  update_particle_neighbors(c, g, f);
  rep.grid_anomaly[0] = f.gs.out_of_grid;
  rep.grid_anomaly[1] = f.gs.cell_overflow;
  rep.grid_anomaly[2] = f.nl.overflow;
  compute_viscosity(c, bodies, f);
  update_dt(c, bodies, f, sp, dt, rep);
  rep.dt = dt;
  const TF V = c.vol, rho0 = c.rho0, eps = TF(0.01) * c.h2;
  for (uint32_t i = 0; i < n; ++i) {
    f.v[i] += dt * f.a[i];
    f.last_pressure[i] = f.pressure[i] * TF(0.5);
  }
  // diag (times rho0) into aii, density_adv
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    const uint32_t i = uint32_t(ii);
    const V3<TF> vi = f.v[i];
    const TF rho = f.density[i];
    TF adv = rho / rho0, diag = 0;
    for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
      const uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
      const V3<TF> d = xv(f, i, j);
      const TF rj = f.density[j];
      const V3<TF> gw = gradW(c, d);
      adv += dt * V * dot(vi - f.v[j], gw);
      diag += V * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gw);
    }
    for (uint32_t b = 0; b < f.nb; ++b) {
      const V4<TF>& bn = f.bnd[size_t(b) * f.n + i];
      const V4<TF>& k4 = f.bk[size_t(b) * f.n + i];
      const V3<TF> gwv{k4.x, k4.y, k4.z};
      const V3<TF> xib = f.x[i] - V3<TF>{bn.x, bn.y, bn.z};
      const V3<TF> vj = body_velocity(bodies[b], V3<TF>{bn.x, bn.y, bn.z});
      adv += dt * dot(vi - vj, gwv);
      diag += (rho + rho0) / (rho * rho0) / (length_sqr(xib) + eps) * dot(xib, gwv);
    }
    f.aii[i] = diag * rho0;
    f.density_adv[i] = adv;
  }
  double mean = std::numeric_limits<double>::max();
  uint32_t it = 0;
  while ((mean > sp.density_error_tolerance || it < sp.min_density_solve) &&
         it < sp.max_density_solve) {
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(n); ++ii) {
      const uint32_t i = uint32_t(ii);
      const TF lp = f.last_pressure[i], rho = f.density[i], diag = f.aii[i];
      const TF bterm = 1 - f.density_adv[i], dt2 = dt * dt, denom = diag * dt2;
      const TF w = TF(2) / 3;
      TF p = 0, off = 0;
      for (uint32_t k = 0; k < f.nl.count[i]; ++k) {
        const uint32_t j = f.nl.index[size_t(i) * f.nl.cap + k];
        const V3<TF> d = xv(f, i, j);
        const TF rj = f.density[j];
        off -= V * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gradW(c, d)) *
               f.last_pressure[j];
      }
      off *= rho0;
      if (std::fabs(denom) > TF(1.0e-9))
        p = std::max((1 - w) * lp + w * (bterm / denom - off / diag), TF(0));
      f.density_err[i] = p == 0 ? TF(0) : (denom * p + off * dt2 - bterm);
      f.pressure[i] = p;
    }
    for (uint32_t i = 0; i < n; ++i) f.last_pressure[i] = f.pressure[i];
    double sum = 0;
    for (uint32_t i = 0; i < n; ++i) sum += double(f.density_err[i]);
    mean = sum / double(n);
    ++it;
  }
  rep.num_density_solve = it;
  rep.mean_density_error = mean;
  pressure_accels_and_integrate(c, bodies, f, dt, F_out, T_out, pile_gravity, integrate_bodies);
  return rep;
}

// ------------------------------------------------- pellet boundary model
// SolverI<TF>::step<0> (solver_i.hpp:79-327) on the pellet branch
// (VolumeMethod::pellets), without contacts.  Pellets are boundary particles
// given in their body's frame; points 0..n-1 are the fluid particles
// ("beads"), n..n+P-1 the pellets.
template <class TF>
struct PelletSet {
  std::vector<V3<TF>> local;   // body frame
  std::vector<uint32_t> body;  // body of each pellet
};

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Golub and Van Loan, Matrix Computations, sec. 8.5), six sweeps: a ends
// diagonal, the columns of q are the eigenvectors.
template <class TF>
void jacobi_eigen3(TF a[3][3], TF q[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) q[r][k] = r == k ? TF(1) : TF(0);
  for (int sweep = 0; sweep < 6; ++sweep) {
    for (int pr = 0; pr < 3; ++pr) {
      const int p = pr == 2 ? 1 : 0;
      const int r = pr == 0 ? 1 : 2;
      const TF apr = a[p][r];
      if (apr == TF(0)) continue;
      const TF theta = (a[r][r] - a[p][p]) / (TF(2) * apr);
      const TF t = (theta >= TF(0) ? TF(1) : TF(-1)) /
                   (std::fabs(theta) + std::sqrt(theta * theta + TF(1)));
      const TF cs = TF(1) / std::sqrt(t * t + TF(1));
      const TF sn = t * cs;
      a[p][p] -= t * apr;
      a[r][r] += t * apr;
      a[p][r] = a[r][p] = TF(0);
      const int k = 3 - p - r;
      const TF akp = a[k][p], akr = a[k][r];
      a[k][p] = a[p][k] = cs * akp - sn * akr;
      a[k][r] = a[r][k] = sn * akp + cs * akr;
      for (int row = 0; row < 3; ++row) {
        const TF qp = q[row][p], qr = q[row][r];
        q[row][p] = cs * qp - sn * qr;
        q[row][r] = sn * qp + cs * qr;
      }
    }
  }
}

// extrapolate_pressure_to_pellet (runner.hpp:2543-2607) for point i from
// its bead list: Shepard average plus the linear MLS term through the
// pseudo-inverse of the weighted second moment (eigenvalues of magnitude
// <= 1e-2 dropped), clamped at 0; 0 without bead neighbors (the
// reference's 0/0 becomes 0 through fmax).
template <class TF>
TF extrapolate_pellet(const Cn<TF>& c, const std::vector<V3<TF>>& X, const std::vector<TF>& pr,
                      const uint32_t* list, uint32_t cnt, V3<TF> xi, bool wrap = false,
                      TF wrap_len = 0) {
  // W of the list's (wrapped) x_ij; the centre from absolute positions, as
  // the reference computes it
  auto w2 = [&](uint32_t j) {
    V3<TF> d = xi - X[j];
    d.y = wrap_coord(wrap, wrap_len, d.y);
    return length_sqr(d);
  };
  TF wsum = 0;
  V3<TF> center{0, 0, 0};
  for (uint32_t k = 0; k < cnt; ++k) {
    const TF w = W_r2(c, w2(list[k])) * c.vol;
    wsum += w;
    center += w * X[list[k]];
  }
  if (!(wsum > 0)) return 0;
  center = (TF(1) / wsum) * center;
  TF alpha = 0;
  V3<TF> psum{0, 0, 0};
  TF m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = list[k];
    const V3<TF> xt = X[j] - center;
    const TF w = W_r2(c, w2(j)) * c.vol;
    const TF wp = w * pr[j];
    alpha += wp;
    psum += wp * xt;
    m[0][0] += w * xt.x * xt.x;
    m[1][1] += w * xt.y * xt.y;
    m[2][2] += w * xt.z * xt.z;
    m[0][1] += w * (xt.x * xt.y);
    m[0][2] += w * (xt.x * xt.z);
    m[1][2] += w * (xt.y * xt.z);
  }
  m[1][0] = m[0][1];
  m[2][0] = m[0][2];
  m[2][1] = m[1][2];
  alpha /= wsum;
  TF q[3][3];
  jacobi_eigen3(m, q);
  V3<TF> plane{0, 0, 0};
  for (int e = 0; e < 3; ++e) {
    const TF lam = m[e][e];
    if (!(std::fabs(lam) > TF(1e-2))) continue;
    const V3<TF> qe{q[0][e], q[1][e], q[2][e]};
    plane += (dot(qe, psum) / lam) * qe;
  }
  return std::max(alpha + dot(plane, xi - center), TF(0));
}

template <class TF>
StepReport i_step_pellets(const Cn<TF>& c, const al_consti& g, std::vector<Body<TF>>& bodies,
                          Fluid<TF>& f, const PelletSet<TF>& pel, const SolverParams& sp, TF& dt,
                          V3<TF> pile_gravity, bool integrate_bodies,
                          std::vector<V3<double>>* F_out, std::vector<V3<double>>* T_out,
                          std::vector<V3<TF>>* pellet_x, std::vector<TF>* pellet_p) {
  StepReport rep;
  const uint32_t n = f.n, np = uint32_t(pel.local.size()), total = n + np;
  const TF eps = TF(0.01) * c.h2;
  std::fill(f.force.begin(), f.force.end(), V3<TF>{0, 0, 0});
  std::fill(f.torque.begin(), f.torque.end(), V3<TF>{0, 0, 0});
  // transform_pellets (runner.hpp:4070-4082)
  std::vector<V3<TF>> X(f.x), Vv(f.v);
  X.resize(total);
  Vv.resize(total);
  for (uint32_t p = 0; p < np; ++p) {
    const Body<TF>& b = bodies[pel.body[p]];
    const V3<TF> rl = rotate(pel.local[p], b.q);
    X[n + p] = rl + b.x;
    Vv[n + p] = cross(b.omega, rl) + b.v;
  }
  // one grid, bead / pellet lists (make_bead_pellet_neighbor_list,
  // runner.hpp:1912-1966) for every point
  const GridSort s = grid_sort(c, g, X.data(), total);
  rep.grid_anomaly[0] = s.out_of_grid;
  rep.grid_anomaly[1] = s.cell_overflow;
  // x_i - x_j of the lists, y wrapped on a periodic step
  auto D = [&](uint32_t i, uint32_t j) {
    V3<TF> d = X[i] - X[j];
    d.y = wrap_coord(f.wrap, f.wrap_len, d.y);
    return d;
  };
  const uint32_t cap = g.max_num_neighbors_per_particle;
  std::vector<uint32_t> bl(size_t(total) * cap), pl(size_t(total) * cap), bc(total), pc(total);
  bool overflow = false;
#pragma omp parallel for schedule(static) reduction(|| : overflow)
  for (int64_t ii = 0; ii < int64_t(total); ++ii) {
    const uint32_t i = uint32_t(ii);
    int p[3];
    cell_coords(c, g, X[i], p);
    uint32_t nbd = 0, npl = 0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          int q[3] = {p[0] + dx, p[1] + dy, p[2] + dz};
          if (f.wrap) {  // make_bead_pellet_neighbor_list<1>
            if (q[1] >= int(g.grid_res[1]))
              q[1] -= int(g.grid_res[1]);
            else if (q[1] < 0)
              q[1] += int(g.grid_res[1]);
          }
          if (!in_grid(g, q)) continue;
          const uint32_t cell = cell_linear(g, q);
          for (uint32_t t = s.cell_start[cell]; t < s.cell_start[cell + 1]; ++t) {
            const uint32_t j = s.sorted[t];
            if (j == i || !(length_sqr(D(i, j)) < c.h2)) continue;
            if (j < n) {
              if (nbd < cap) bl[size_t(i) * cap + nbd] = j;
              ++nbd;
            } else {
              if (npl < cap) pl[size_t(i) * cap + npl] = j;
              ++npl;
            }
          }
        }
    if (nbd > cap || npl > cap) overflow = true;
    bc[i] = std::min(nbd, cap);
    pc[i] = std::min(npl, cap);
  }
  rep.grid_anomaly[2] = overflow;
  auto B = [&](uint32_t i, uint32_t k) { return bl[size_t(i) * cap + k]; };
  auto Pn = [&](uint32_t i, uint32_t k) { return pl[size_t(i) * cap + k]; };
  // compute_density_with_pellets (runner.hpp:2074-2098)
  for (uint32_t i = 0; i < n; ++i) {
    TF d = c.w0;
    for (uint32_t k = 0; k < bc[i]; ++k) d += W_r2(c, length_sqr(D(i, B(i, k))));
    for (uint32_t k = 0; k < pc[i]; ++k) d += W_r2(c, length_sqr(D(i, Pn(i, k))));
    f.density[i] = d * c.mass;
  }
  // clear_acceleration + compute_viscosity_with_pellets (runner.hpp:2251-2299)
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    const uint32_t i = uint32_t(ii);
    V3<TF> da{0, 0, 0};
    for (uint32_t k = 0; k < bc[i]; ++k) {
      const uint32_t j = B(i, k);
      const V3<TF> d = D(i, j);
      da += (c.visc * c.mass / f.density[j] * dot(d, gradW(c, d)) / (length_sqr(d) + eps)) *
            (Vv[i] - Vv[j]);
    }
    for (uint32_t k = 0; k < pc[i]; ++k) {
      const uint32_t j = Pn(i, k);
      const V3<TF> d = D(i, j);
      const V3<TF> a =
          (c.vol * c.bvisc * dot(d, gradW(c, d)) / (length_sqr(d) + eps)) * (Vv[i] - Vv[j]);
      da += a;
      const uint32_t b = pel.body[j - n];
      const V3<TF> force = (-c.mass) * a;
      f.force[size_t(b) * n + i] += force;
      f.torque[size_t(b) * n + i] += cross((X[i] - d) - bodies[b].x, force);  // pellet_x
    }
    f.a[i] = c.g + da;
  }
  update_dt(c, bodies, f, sp, dt, rep);
  rep.dt = dt;
  // advect_and_init_pressure
  std::vector<TF> P(total, 0), L(total, 0);
  for (uint32_t i = 0; i < n; ++i) {
    f.v[i] += dt * f.a[i];
    Vv[i] = f.v[i];
    P[i] = f.pressure[i];
    L[i] = f.pressure[i] * TF(0.5);
  }
  // calculate_isph_diagonal_adv_density_with_pellets (runner.hpp:2955-3004)
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    const uint32_t i = uint32_t(ii);
    const TF rho = f.density[i];
    TF adv = rho / c.rho0, diag = 0;
    for (uint32_t k = 0; k < bc[i]; ++k) {
      const uint32_t j = B(i, k);
      const V3<TF> d = D(i, j);
      const TF rj = f.density[j];
      const V3<TF> gw = gradW(c, d);
      adv += dt * c.vol * dot(Vv[i] - Vv[j], gw);
      diag += c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gw);
    }
    for (uint32_t k = 0; k < pc[i]; ++k) {
      const uint32_t j = Pn(i, k);
      const V3<TF> d = D(i, j);
      const V3<TF> gwv = c.vol * gradW(c, d);
      adv += dt * dot(Vv[i] - Vv[j], gwv);
      diag += (rho + c.rho0) / (rho * c.rho0) / (length_sqr(d) + eps) * dot(d, gwv);
    }
    f.aii[i] = diag * c.rho0;
    f.density_adv[i] = adv;
  }
  auto extrapolate = [&](std::vector<TF>& pr) {
#pragma omp parallel for schedule(static)
    for (int64_t pp = 0; pp < int64_t(np); ++pp) {
      const uint32_t i = n + uint32_t(pp);
      pr[i] = extrapolate_pellet(c, X, pr, &bl[size_t(i) * cap], bc[i], X[i], f.wrap, f.wrap_len);
    }
  };
  double mean = std::numeric_limits<double>::max();
  uint32_t it = 0;
  while ((mean > sp.density_error_tolerance || it < sp.min_density_solve) &&
         it < sp.max_density_solve) {
    extrapolate(L);
    // isph_solve_iteration_with_pellets (runner.hpp:3055-3121)
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < int64_t(n); ++ii) {
      const uint32_t i = uint32_t(ii);
      const TF rho = f.density[i], diag = f.aii[i];
      const TF bterm = 1 - f.density_adv[i], dt2 = dt * dt, denom = diag * dt2;
      const TF w = TF(2) / 3;
      TF off = 0, pv = 0;
      for (uint32_t k = 0; k < bc[i]; ++k) {
        const uint32_t j = B(i, k);
        const V3<TF> d = D(i, j);
        const TF rj = f.density[j];
        off -= c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gradW(c, d)) *
               L[j];
      }
      for (uint32_t k = 0; k < pc[i]; ++k) {
        const uint32_t j = Pn(i, k);
        const V3<TF> d = D(i, j);
        off -= c.vol * (rho + c.rho0) / (rho * c.rho0) / (length_sqr(d) + eps) *
               dot(d, gradW(c, d)) * L[j];
      }
      off *= c.rho0;
      if (std::fabs(denom) > TF(1.0e-9))
        pv = std::max((1 - w) * L[i] + w * (bterm / denom - off / diag), TF(0));
      f.density_err[i] = pv == 0 ? TF(0) : (denom * pv + off * dt2 - bterm);
      P[i] = pv;
    }
    for (uint32_t i = 0; i < n; ++i) L[i] = P[i];
    double sum = 0;
    for (uint32_t i = 0; i < n; ++i) sum += double(f.density_err[i]);
    mean = sum / double(n);
    ++it;
  }
  rep.num_density_solve = it;
  rep.mean_density_error = mean;
  extrapolate(P);
  // compute_pressure_accels_with_pellets (runner.hpp:2819-2871) and
  // kinematic_integration<0>
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < int64_t(n); ++ii) {
    const uint32_t i = uint32_t(ii);
    const TF rho = f.density[i], dpi = P[i] / (rho * rho);
    V3<TF> ai{0, 0, 0};
    for (uint32_t k = 0; k < bc[i]; ++k) {
      const uint32_t j = B(i, k);
      const TF rj = f.density[j], dpj = P[j] / (rj * rj);
      ai -= (c.mass * (dpi + dpj)) * gradW(c, D(i, j));
    }
    for (uint32_t k = 0; k < pc[i]; ++k) {
      const uint32_t j = Pn(i, k);
      const TF dpj = P[j] / (c.rho0 * c.rho0);
      const V3<TF> d = D(i, j);
      const V3<TF> a = (c.mass * (dpi + dpj)) * gradW(c, d);
      const V3<TF> force = c.mass * a;
      ai -= a;
      const uint32_t b = pel.body[j - n];
      f.force[size_t(b) * n + i] += force;
      f.torque[size_t(b) * n + i] += cross((X[i] - d) - bodies[b].x, force);
    }
    f.pressure_accel[i] = c.rho0 * ai;
  }
  for (uint32_t i = 0; i < n; ++i) {
    const V3<TF> v = f.v[i] + f.pressure_accel[i] * dt;
    f.x[i] += v * dt;
    f.x[i].y = wrap_coord(f.wrap, f.wrap_len, f.x[i].y);
    f.v[i] = v;
    f.pressure[i] = P[i];
  }
  if (pellet_x) pellet_x->assign(X.begin() + n, X.end());
  if (pellet_p) pellet_p->assign(P.begin() + n, P.end());
  std::vector<V3<double>> F, T;
  rigid_totals(f, F, T);
  if (F_out) *F_out = F;
  if (T_out) *T_out = T;
  if (integrate_bodies) integrate_kinematics(bodies, F, T, pile_gravity, dt);
  return rep;
}

// ----------------------------------------------------- pellet relaxation
// SolverPellet<TF>::step<wrap> (solver_pellet.hpp:57-119): the body is
// evaluated in its own frame at the particle positions.
struct RelaxParams {
  double cohesion = 4, adhesion = 2, cfl_factor = 0.25, tolerance = 0;
  bool wrap = false;
  double wrap_length = 0;
};

// interpolate_and_derive (runner.hpp:1773-1791): value and gradient scaled
// by 2 / cell size; false outside the domain.
template <class TF>
bool grid_value_gradient(const Body<TF>& b, V3<TF> x, TF& phi, V3<TF>& grad) {
  int ip[3];
  V3<TF> xi;
  if (!resolve(b.dmin, b.dmax, b.res, b.cs, x, ip, xi)) return false;
  TF N[32], d0[32], d1[32], d2[32];
  uint32_t cells[32];
  shape_functions<TF>(xi, N, d0, d1, d2);
  cell_nodes(b.res, ip, cells);
  phi = 0;
  grad = {0, 0, 0};
  for (int j = 0; j < 32; ++j) {
    const TF v = b.dist_nodes[cells[j]];
    phi += v * N[j];
    grad.x += v * d0[j];
    grad.y += v * d1[j];
    grad.z += v * d2[j];
  }
  grad.x *= TF(2) / b.cs.x;
  grad.y *= TF(2) / b.cs.y;
  grad.z *= TF(2) / b.cs.z;
  return true;
}

// The body's distance (times sign) and normal as the relaxation kernels read
// them: the grid for a mesh body (normal scaled by sign / |n|), else the
// analytic distance minus the tolerance with the step-1e-3 normal.
template <class TF>
bool relax_body_distance(const Body<TF>& b, TF tolerance, V3<TF> x, TF& dist, V3<TF>& n) {
  if (b.shape == AL_SHAPE_MESH) {
    TF phi;
    V3<TF> g;
    if (!grid_value_gradient(b, x, phi, g)) return false;
    dist = phi * b.sign;
    const TF nl2 = length_sqr(g);
    n = (b.sign * (nl2 > 0 ? inv_sqrt(nl2) : TF(0))) * g;
    return true;
  }
  dist = b.sdf.sdf(x) * b.sign - tolerance;
  n = b.sdf.gradient(x, TF(1e-3)) * b.sign;
  return true;
}

template <class TF>
bool relax_pellets(const Cn<TF>& c, const al_consti& g, const Body<TF>& b,
                   std::vector<V3<TF>>& x, const RelaxParams& p, uint32_t steps,
                   std::vector<V3<TF>>* dx_out, std::vector<TF>* rho_out) {
  const uint32_t n = uint32_t(x.size());
  const TF len = TF(p.wrap_length), tol = TF(p.tolerance);
  const TF coh = TF(p.cohesion), adh = TF(p.adhesion);
  bool overflow = false;
  std::vector<TF> rho(n), factor(n);
  std::vector<V3<TF>> dx(n);
  for (uint32_t step = 0; step < steps; ++step) {
    const GridSort s = grid_sort(c, g, x.data(), n);
    const NeighborList nl = neighbor_list(c, g, x.data(), n, s, p.wrap, len);
    overflow = overflow || nl.overflow;
    auto disp = [&](uint32_t i, uint32_t j) {
      V3<TF> d = x[i] - x[j];
      d.y = wrap_coord(p.wrap, len, d.y);
      return d;
    };
    // compute_density_with_pellets without pellets
    for (uint32_t i = 0; i < n; ++i) {
      TF d = c.w0;
      for (uint32_t k = 0; k < nl.count[i]; ++k)
        d += W_r2(c, length_sqr(disp(i, nl.index[size_t(i) * nl.cap + k])));
      rho[i] = d * c.mass;
    }
    // compute_cohesion_adhesion_displacement (runner.hpp:2453-2532)
    for (uint32_t i = 0; i < n; ++i) {
      V3<TF> v{0, 0, 0};
      for (uint32_t k = 0; k < nl.count[i]; ++k) {
        const uint32_t j = nl.index[size_t(i) * nl.cap + k];
        const V3<TF> d = disp(i, j);
        const TF w = W_r2(c, length_sqr(d));
        v -= (coh * c.mass / rho[j] * (TF(1) - c.radius * TF(2) * inv_sqrt(length_sqr(d))) * w) *
             d;
      }
      TF dist;
      V3<TF> nrm;
      if (relax_body_distance(b, tol, x[i], dist, nrm)) {
        const TF nn = length_sqr(nrm);
        if (b.shape == AL_SHAPE_MESH || nn >= TF(1e-7))
          v -= (adh * c.mass / rho[i] * W_dist(c, dist)) * (dist * (inv_sqrt(nn) * nrm));
      }
      dx[i] = v;
    }
    // compute_dfsph_factor_with_pellets (runner.hpp:3156-3190)
    for (uint32_t i = 0; i < n; ++i) {
      TF sum = 0;
      V3<TF> gi{0, 0, 0};
      for (uint32_t k = 0; k < nl.count[i]; ++k) {
        const V3<TF> gp = (-c.vol) * gradW(c, disp(i, nl.index[size_t(i) * nl.cap + k]));
        sum += length_sqr(gp);
        gi -= gp;
      }
      sum += length_sqr(gi);
      factor[i] = sum > c.eps ? TF(-1) / sum : TF(0);
    }
    // pellet_divergence_solve_iteration (runner.hpp:3365-3395) and the CFL
    TF vmax = 0;
    std::vector<V3<TF>> dn(n);
    for (uint32_t i = 0; i < n; ++i) {
      const TF ki = (rho[i] / c.rho0 - TF(1)) * factor[i];
      V3<TF> v = dx[i];
      for (uint32_t k = 0; k < nl.count[i]; ++k) {
        const uint32_t j = nl.index[size_t(i) * nl.cap + k];
        const TF ks = ki + (rho[j] / c.rho0 - TF(1)) * factor[j];
        if (std::fabs(ks) > c.eps) v -= ks * ((-c.vol) * gradW(c, disp(i, j)));
      }
      dn[i] = v;
      vmax = std::max(vmax, length_sqr(v));
    }
    const TF cfl = std::min(TF(p.cfl_factor) * TF(0.4) * c.radius * TF(2) * (TF(1) / std::sqrt(vmax)),
                            TF(1));
    // move_and_avoid_boundary<wrap> (runner.hpp:4010-4066)
    for (uint32_t i = 0; i < n; ++i) {
      V3<TF> xi = x[i] + dn[i] * cfl;
      TF dist;
      V3<TF> nrm;
      if (relax_body_distance(b, tol, xi, dist, nrm) && dist < c.radius)
        xi += (c.radius - dist) * (inv_sqrt(length_sqr(nrm)) * nrm);
      xi.y = wrap_coord(p.wrap, len, xi.y);
      x[i] = xi;
    }
    if (step + 1 == steps) {
      if (dx_out) *dx_out = dn;
      if (rho_out) *rho_out = rho;
    }
  }
  return overflow;
}

// ---------------------------------------------------------------- contacts
// Rigid-rigid contacts: Contact (contact.hpp:8-25), collision_test
// (runner.hpp:3833-4010; analytic distance for analytic bodies, the
// distance grid through collision_find_dist_normal, runner.hpp:1793-1822,
// for grid bodies), Pile::find_contacts (pile.hpp:886-900, volume-map
// branch) and Pile::solve_contacts (pile.hpp:906-979).  The reference
// appends contacts with an atomic counter, so its order (and the
// sequential-impulse result) is not reproducible; here contacts are listed
// in (i, j, vertex) order, the order of its loops.
template <class TF>
struct Contact {
  uint32_t i, j;
  V3<TF> cp_i, cp_j, n, t;
  V3<TF> iiwi_diag, iiwi_off, iiwj_diag, iiwj_off;
  TF friction, nkninv, pmax, goalu, impulse_sum;
};

// calculate_congruent_matrix (runner.hpp:178-199): R diag(v) R^T.
template <class TF>
void congruent_matrix(V3<TF> v, V4<TF> q, V3<TF>& diag, V3<TF>& off) {
  TF m00 = 1 - 2 * (q.y * q.y + q.z * q.z), m01 = 2 * (q.x * q.y - q.z * q.w),
     m02 = 2 * (q.x * q.z + q.y * q.w);
  TF m10 = 2 * (q.x * q.y + q.z * q.w), m11 = 1 - 2 * (q.x * q.x + q.z * q.z),
     m12 = 2 * (q.y * q.z - q.x * q.w);
  TF m20 = 2 * (q.x * q.z - q.y * q.w), m21 = 2 * (q.y * q.z + q.x * q.w),
     m22 = 1 - 2 * (q.x * q.x + q.y * q.y);
  diag = {v.x * m00 * m00 + v.y * m01 * m01 + v.z * m02 * m02,
          v.x * m10 * m10 + v.y * m11 * m11 + v.z * m12 * m12,
          v.x * m20 * m20 + v.y * m21 * m21 + v.z * m22 * m22};
  off = {v.x * m00 * m10 + v.y * m01 * m11 + v.z * m02 * m12,
         v.x * m00 * m20 + v.y * m01 * m21 + v.z * m02 * m22,
         v.x * m10 * m20 + v.y * m11 * m21 + v.z * m12 * m22};
}

// apply_congruent (runner.hpp:253-262).
template <class TF>
V3<TF> apply_congruent(V3<TF> v, V3<TF> d, V3<TF> o) {
  return {v.x * d.x + v.y * o.x + v.z * o.y, v.x * o.x + v.y * d.y + v.z * o.z,
          v.x * o.y + v.y * o.z + v.z * d.z};
}

// calculate_congruent_k (runner.hpp:264-288).
template <class TF>
void congruent_k(V3<TF> r, TF mass, V3<TF> d, V3<TF> o, V3<TF>& kd, V3<TF>& ko) {
  kd = {0, 0, 0};
  ko = {0, 0, 0};
  if (mass == 0) return;
  TF im = 1 / mass;
  kd.x = r.z * r.z * d.y - r.y * r.z * o.z * 2 + r.y * r.y * d.z + im;
  kd.y = r.z * r.z * d.x - r.x * r.z * o.y * 2 + r.x * r.x * d.z + im;
  kd.z = r.y * r.y * d.x - r.x * r.y * o.x * 2 + r.x * r.x * d.y + im;
  ko.x = -r.z * r.z * o.x + r.x * r.z * o.z + r.y * r.z * o.y - r.x * r.y * d.z;
  ko.y = r.y * r.z * o.x - r.x * r.z * d.y - r.y * r.y * o.y + r.x * r.y * o.z;
  ko.z = -(r.y * r.z * d.x) + r.x * r.z * o.x + r.x * r.y * o.y - r.x * r.x * o.z;
}

template <class TF>
V3<TF> operator/(V3<TF> a, TF s) {
  return {a.x / s, a.y / s, a.z / s};
}

// One vertex of body i against body j; returns true and fills `ct` on contact.
template <class TF>
bool contact_test(const Body<TF>& bi, const Body<TF>& bj, uint32_t i, uint32_t j, V3<TF> vertex,
                  TF tol, TF restitution, TF friction, Contact<TF>& ct) {
  ct.cp_i = rotate(vertex, bi.q) + bi.x;
  const V3<TF> local = rotate(ct.cp_i - bj.x, conjugate(bj.q));
  TF dist;
  V3<TF> n{0, 0, 0};
  if (bj.use_grid) {
    dist = bj.sign;  // outside the map: only the existence of a collision is known
    V3<TF> nt{0, 1, 0};
    int ip[3];
    V3<TF> xi;
    if (resolve(bj.dmin, bj.dmax, bj.res, bj.cs, local, ip, xi)) {
      TF N[32], d0[32], d1[32], d2[32];
      uint32_t cells[32];
      shape_functions<TF>(xi, N, d0, d1, d2);
      cell_nodes(bj.res, ip, cells);
      TF phi = 0;
      V3<TF> g{0, 0, 0};
      for (int k = 0; k < 32; ++k) {
        const TF c = bj.dist_nodes[cells[k]];
        phi += c * N[k];
        g.x += c * d0[k];
        g.y += c * d1[k];
        g.z += c * d2[k];
      }
      g.x *= TF(2) / bj.cs.x;
      g.y *= TF(2) / bj.cs.y;
      g.z *= TF(2) / bj.cs.z;
      dist = bj.sign * phi - tol;
      nt = g * bj.sign;
    }
    if (dist < 0) n = normalized(nt);
  } else {
    dist = bj.sdf.sdf(local) * bj.sign - tol;
    n = normalized(bj.sdf.gradient(local, TF(1e-3)) * bj.sign);
  }
  if (!(dist < 0)) return false;
  const V3<TF> cp = local - dist * n;
  ct.i = i;
  ct.j = j;
  ct.cp_j = rotate(cp, bj.q) + bj.x;
  ct.n = rotate(n, bj.q);
  ct.friction = friction;
  const V3<TF> ri = ct.cp_i - bi.x, rj = ct.cp_j - bj.x;
  const V3<TF> ui = bi.v + cross(bi.omega, ri), uj = bj.v + cross(bj.omega, rj);
  const V3<TF> urel = ui - uj;
  const TF urn = dot(ct.n, urel);
  ct.t = urel - urn * ct.n;
  if (length_sqr(ct.t) > TF(1e-6)) ct.t = normalized(ct.t);
  congruent_matrix(V3<TF>{1 / bi.inertia.x, 1 / bi.inertia.y, 1 / bi.inertia.z}, bi.q,
                   ct.iiwi_diag, ct.iiwi_off);
  congruent_matrix(V3<TF>{1 / bj.inertia.x, 1 / bj.inertia.y, 1 / bj.inertia.z}, bj.q,
                   ct.iiwj_diag, ct.iiwj_off);
  V3<TF> kid, kio, kjd, kjo;
  congruent_k(ri, bi.mass, ct.iiwi_diag, ct.iiwi_off, kid, kio);
  congruent_k(rj, bj.mass, ct.iiwj_diag, ct.iiwj_off, kjd, kjo);
  const V3<TF> kd = kid + kjd, ko = kio + kjo;
  ct.nkninv = 1 / dot(ct.n, apply_congruent(ct.n, kd, ko));
  ct.pmax = 1 / dot(ct.t, apply_congruent(ct.t, kd, ko)) * dot(urel, ct.t);
  ct.goalu = urn < 0 ? -restitution * urn : TF(0);
  ct.impulse_sum = 0;
  return true;
}

// Pile::find_contacts over every ordered pair (i, j), i != j, not both
// kinematic; restitution r_i r_j, friction f_i + f_j.
template <class TF>
void find_contacts(const std::vector<Body<TF>>& bodies, const std::vector<const TF*>& vertices,
                   const std::vector<uint32_t>& num_vertices, const std::vector<TF>& restitution,
                   const std::vector<TF>& friction, TF tol, std::vector<Contact<TF>>& out) {
  out.clear();
  const uint32_t nb = uint32_t(bodies.size());
  for (uint32_t i = 0; i < nb; ++i)
    for (uint32_t j = 0; j < nb; ++j) {
      if (i == j || (bodies[i].mass == 0 && bodies[j].mass == 0)) continue;
      for (uint32_t v = 0; v < num_vertices[i]; ++v) {
        Contact<TF> ct;
        const TF* p = vertices[i] + 3 * size_t(v);
        if (contact_test(bodies[i], bodies[j], i, j, V3<TF>{p[0], p[1], p[2]}, tol,
                         restitution[i] * restitution[j], friction[i] + friction[j], ct))
          out.push_back(ct);
      }
    }
}

// Pile::solve_contacts: five sequential-impulse sweeps in contact order.
template <class TF>
void solve_contacts(std::vector<Body<TF>>& bodies, std::vector<Contact<TF>>& contacts) {
  for (int sweep = 0; sweep < 5; ++sweep)
    for (Contact<TF>& c : contacts) {
      Body<TF>& bi = bodies[c.i];
      Body<TF>& bj = bodies[c.j];
      const TF depth = dot(c.n, c.cp_i - c.cp_j);
      const V3<TF> ri = c.cp_i - bi.x, rj = c.cp_j - bj.x;
      const V3<TF> ui = bi.v + cross(bi.omega, ri), uj = bj.v + cross(bj.omega, rj);
      const V3<TF> urel = ui - uj;
      const TF urn = dot(c.n, urel);
      TF corr = c.nkninv * (c.goalu - urn);
      if (corr < -c.impulse_sum) corr = -c.impulse_sum;
      if (depth < 0) corr -= c.nkninv * depth;  // stiffness 1
      V3<TF> p = corr * c.n;
      c.impulse_sum += corr;
      const TF pn = dot(p, c.n);
      if (c.friction * pn > c.pmax)
        p -= c.pmax * c.t;
      else if (c.friction * pn < -c.pmax)
        p += c.pmax * c.t;
      else
        p -= c.friction * pn * c.t;
      if (bi.mass != 0) {
        bi.v += p / bi.mass;
        bi.omega += apply_congruent(cross(ri, p), c.iiwi_diag, c.iiwi_off);
      }
      if (bj.mass != 0) {
        bj.v += -p / bj.mass;
        bj.omega += apply_congruent(cross(rj, -p), c.iiwj_diag, c.iiwj_off);
      }
    }
}

// ------------------------------------------------------------ mesh distance
// MeshDistance::signedDistance (dg/mesh_distance.hpp:186-223) by brute
// force: exact point-triangle distance with the closest point's region
// (Ericson, Real-Time Collision Detection, sec. 5.1.5), first nearest face,
// sign from the angle-weighted pseudonormals of the nearest feature
// (dg/mesh_distance.hpp:80-104, 228-266), minus the offset.
template <class TF>
struct TriMesh {
  std::vector<V3<TF>> v;
  std::vector<std::array<uint32_t, 3>> f;
  std::vector<V3<TF>> fn, vn, en;  // en: [face][3] (halfedge k: vertex k -> k + 1)
};

template <class TF>
TriMesh<TF> make_mesh(const TF* verts, uint32_t nv, const uint32_t* faces, uint32_t nf) {
  TriMesh<TF> m;
  for (uint32_t i = 0; i < nv; ++i) m.v.push_back({verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]});
  for (uint32_t i = 0; i < nf; ++i) m.f.push_back({faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]});
  std::vector<V3<double>> fn(nf), vn(nv, V3<double>{0, 0, 0});
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> edge_face;
  auto d3 = [&](uint32_t i) { return V3<double>{double(m.v[i].x), double(m.v[i].y), double(m.v[i].z)}; };
  for (uint32_t i = 0; i < nf; ++i) {
    const auto& t = m.f[i];
    const V3<double> x0 = d3(t[0]), x1 = d3(t[1]), x2 = d3(t[2]);
    fn[i] = normalized(cross(x1 - x0, x2 - x0));
    const V3<double> e1 = normalized(x1 - x0), e2 = normalized(x2 - x1), e3 = normalized(x0 - x2);
    auto ang = [](V3<double> a, V3<double> c) {
      double d = -dot(a, c);
      return std::acos(d < -1 ? -1 : (d > 1 ? 1 : d));
    };
    const double alpha[3] = {ang(e1, e3), ang(e2, e1), ang(e3, e2)};
    for (int k = 0; k < 3; ++k) vn[t[k]] += alpha[k] * fn[i];
    for (int k = 0; k < 3; ++k) edge_face[{t[k], t[(k + 1) % 3]}] = i;
  }
  auto cvt = [](V3<double> a) { return V3<TF>{TF(a.x), TF(a.y), TF(a.z)}; };
  for (uint32_t i = 0; i < nf; ++i) {
    m.fn.push_back(cvt(fn[i]));
    for (int k = 0; k < 3; ++k) {
      auto it = edge_face.find({m.f[i][(k + 1) % 3], m.f[i][k]});
      m.en.push_back(cvt(it != edge_face.end() ? fn[i] + fn[it->second] : fn[i]));
    }
  }
  for (uint32_t i = 0; i < nv; ++i) m.vn.push_back(cvt(vn[i]));
  return m;
}

// Closest point of triangle (a, b, c) to p; region 0-2 vertex, 3 edge ab,
// 4 edge bc, 5 edge ca, 6 face.
template <class TF>
V3<TF> closest_on_triangle(V3<TF> p, V3<TF> a, V3<TF> b, V3<TF> c, int& region) {
  const V3<TF> ab = b - a, ac = c - a, ap = p - a;
  const TF d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) { region = 0; return a; }
  const V3<TF> bp = p - b;
  const TF d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) { region = 1; return b; }
  const TF vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) { region = 3; return a + (d1 / (d1 - d3)) * ab; }
  const V3<TF> cp = p - c;
  const TF d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) { region = 2; return c; }
  const TF vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) { region = 5; return a + (d2 / (d2 - d6)) * ac; }
  const TF va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    region = 4;
    return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
  }
  region = 6;
  const TF denom = TF(1) / (va + vb + vc);
  return a + (vb * denom) * ab + (vc * denom) * ac;
}

template <class TF>
TF mesh_signed_distance(const TriMesh<TF>& m, V3<TF> p, TF offset) {
  TF best = std::numeric_limits<TF>::max();
  uint32_t bf = 0;
  int br = 6;
  V3<TF> bq{0, 0, 0};
  for (uint32_t i = 0; i < m.f.size(); ++i) {
    int r;
    const V3<TF> q = closest_on_triangle(p, m.v[m.f[i][0]], m.v[m.f[i][1]], m.v[m.f[i][2]], r);
    const TF d2 = length_sqr(p - q);
    if (d2 < best) {
      best = d2;
      bf = i;
      br = r;
      bq = q;
    }
  }
  const V3<TF> n = br < 3 ? m.vn[m.f[bf][br]] : (br < 6 ? m.en[3 * bf + (br - 3)] : m.fn[bf]);
  TF dist = std::sqrt(best);
  if (dot(p - bq, n) < 0) dist = -dist;
  return dist - offset;
}

// ------------------------------------------------------------- sampling
// Fluid quantities at sample points.  The sample neighbor list is
// make_neighbor_list<0> (runner.hpp:1869-1911) over sample_x: the 27 cells
// around the sample's cell, candidates j != s (the kernel compares the
// particle index with the sample index) with |x_s - x_j|^2 < h^2, the first
// cap of them in canonical order.  Then:
//   sample_fluid             (runner.hpp:4173-4191)  sum m / rho_j W q_j
//   sample_fluid_density     (runner.hpp:4193-4209)  rho0 sum V W
//   sample_position_density  (runner.hpp:2100-2121)  rho0 (sum V W + sum_b (W V)_b)
//   compute_sample_velocity  (runner.hpp:4211-4240)  sum m / rho_j W v_j + sum_b v_b (W V)_b
//   compute_sample_vorticity (runner.hpp:4289-4323)  sum m / rho_j (v_j - v_s) x grad W
//                                                    + sum_b (v_b - v_s) x (grad W V)_b
// with v_b = omega_b x (x_b - x_body) + v_body the body's velocity at the
// boundary point.  Boundary terms run over every body of `bodies`.
template <class TF>
struct SampleRequest {
  const V3<TF>* sx = nullptr;
  uint32_t num = 0;
  const TF* rho = nullptr;
  const V3<TF>* v = nullptr;
  const TF* q = nullptr;
  uint32_t qdim = 0;
  const V4<TF>* bnd = nullptr;  // [nb][S]
  const V4<TF>* bk = nullptr;   // [nb][S]
  TF* density = nullptr;
  TF* position_density = nullptr;
  TF* quantity = nullptr;
  V3<TF>* vel = nullptr;
  V3<TF>* vort = nullptr;
  // make_neighbor_list<1>: cells wrap in y (wrap_ipos_y, runner.hpp:689-697)
  // and displacements wrap into [-L/2, L/2) (wrap_y, runner.hpp:698-707)
  bool wrap = false;
  TF wrap_length = 0;
  // pellet boundary model (*_with_pellets, runner.hpp:2122-2147,
  // 4242-4275, 4325-4357): pellets join the grid after the particles
  const V3<TF>* pel_x = nullptr;
  const V3<TF>* pel_v = nullptr;
  uint32_t npel = 0;
};

template <class TF>
bool sample_fluid(const Cn<TF>& c, const al_consti& g, const V3<TF>* px_in, uint32_t n,
                  const std::vector<Body<TF>>& bodies, const SampleRequest<TF>& r) {
  std::vector<V3<TF>> all(px_in, px_in + n);
  for (uint32_t k = 0; k < r.npel; ++k) all.push_back(r.pel_x[k]);
  const V3<TF>* px = all.data();
  const GridSort s = grid_sort(c, g, px, n + r.npel);
  const uint32_t cap = g.max_num_neighbors_per_particle;
  const uint32_t nb = uint32_t(bodies.size());
  bool overflow = false;
#pragma omp parallel for schedule(static) reduction(|| : overflow)
  for (int64_t ii = 0; ii < int64_t(r.num); ++ii) {
    const uint32_t i = uint32_t(ii);
    const V3<TF> xi = r.sx[i];
    int p[3];
    cell_coords(c, g, xi, p);
    std::vector<uint32_t> nbr, pnbr;
    std::vector<V3<TF>> disp, pdisp;  // x_s - x_j, wrapped
    const TF wmin = r.wrap_length * TF(-0.5), wmax = r.wrap_length * TF(0.5);
    uint32_t found = 0, pfound = 0;
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          int q[3] = {p[0] + dx, p[1] + dy, p[2] + dz};
          if (r.wrap) {
            if (q[1] >= int(g.grid_res[1]))
              q[1] -= int(g.grid_res[1]);
            else if (q[1] < 0)
              q[1] += int(g.grid_res[1]);
          }
          if (!in_grid(g, q)) continue;
          const uint32_t cell = cell_linear(g, q);
          for (uint32_t t = s.cell_start[cell]; t < s.cell_start[cell + 1]; ++t) {
            const uint32_t j = s.sorted[t];
            if (j == i) continue;
            V3<TF> d = xi - px[j];
            if (r.wrap) {
              if (d.y >= wmax)
                d.y -= r.wrap_length;
              else if (d.y < wmin)
                d.y += r.wrap_length;
            }
            if (!((d.x * d.x + d.y * d.y) + d.z * d.z < c.h2)) continue;
            if (j >= n) {
              if (pfound < cap) {
                pnbr.push_back(j - n);
                pdisp.push_back(d);
              }
              ++pfound;
              continue;
            }
            if (found < cap) {
              nbr.push_back(j);
              disp.push_back(d);
            }
            ++found;
          }
        }
    if (found > cap || pfound > cap) overflow = true;
    TF dens = 0, qs[3] = {0, 0, 0}, wb = 0, wp = 0;
    V3<TF> vel{0, 0, 0};
    for (size_t k = 0; k < nbr.size(); ++k) {
      const uint32_t j = nbr[k];
      const V3<TF> d = disp[k];
      const TF w = W_r2(c, (d.x * d.x + d.y * d.y) + d.z * d.z);
      dens += c.vol * w;
      wb += w;
      if (r.quantity) {
        const TF mr = c.mass / r.rho[j];
        for (uint32_t k = 0; k < r.qdim; ++k) qs[k] += mr * w * r.q[size_t(j) * r.qdim + k];
      }
      if (r.vel) vel += (c.mass / r.rho[j] * w) * r.v[j];
    }
    for (size_t k = 0; k < pnbr.size(); ++k) {
      const V3<TF> d = pdisp[k];
      const TF w = W_r2(c, (d.x * d.x + d.y * d.y) + d.z * d.z);
      wp += w;
      if (r.vel) vel += (c.vol * w) * r.pel_v[pnbr[k]];
    }
    TF bw = 0;
    for (uint32_t b = 0; r.npel == 0 && r.bk && b < nb; ++b) {
      const V4<TF> bx = r.bnd ? r.bnd[size_t(b) * r.num + i] : V4<TF>{0, 0, 0, 0};
      const V4<TF> bk = r.bk[size_t(b) * r.num + i];
      bw += bk.w;
      if (r.vel) {
        const V3<TF> vb =
            cross(bodies[b].omega, V3<TF>{bx.x, bx.y, bx.z} - bodies[b].x) + bodies[b].v;
        vel += bk.w * vb;
      }
    }
    if (r.density) r.density[i] = dens * c.rho0;
    if (r.position_density)
      r.position_density[i] = r.npel ? (wb + wp) * c.mass : (dens + bw) * c.rho0;
    if (r.quantity)
      for (uint32_t k = 0; k < r.qdim; ++k) r.quantity[size_t(i) * r.qdim + k] = qs[k];
    if (r.vel) r.vel[i] = vel;
    if (r.vort) {
      V3<TF> w{0, 0, 0};
      for (size_t k = 0; k < nbr.size(); ++k)
        w += (c.mass / r.rho[nbr[k]]) * cross(r.v[nbr[k]] - vel, gradW(c, disp[k]));
      for (size_t k = 0; k < pnbr.size(); ++k)
        w += c.vol * cross(r.pel_v[pnbr[k]] - vel, gradW(c, pdisp[k]));
      for (uint32_t b = 0; r.npel == 0 && b < nb; ++b) {
        const V4<TF> bx = r.bnd[size_t(b) * r.num + i];
        const V4<TF> bk = r.bk[size_t(b) * r.num + i];
        const V3<TF> vb =
            cross(bodies[b].omega, V3<TF>{bx.x, bx.y, bx.z} - bodies[b].x) + bodies[b].v;
        w += cross(vb - vel, V3<TF>{bk.x, bk.y, bk.z});
      }
      r.vort[i] = w;
    }
  }
  return overflow;
}

// compute_boundary_mask (runner.hpp:4367-4396): mask *= (sign d >= threshold)
// with d the distance grid's interpolation for a mesh body, the analytic
// distance otherwise, at the sample in the body's frame.
template <class TF>
void boundary_mask(const Body<TF>& b, const V3<TF>* sx, uint32_t n, TF threshold, TF* mask) {
  const LagrangeGrid<TF> grid{b.dmin, b.dmax, b.cs, {b.res[0], b.res[1], b.res[2]}, b.dist_nodes};
  for (uint32_t i = 0; i < n; ++i) {
    const V3<TF> local = rotate(sx[i] - b.x, conjugate(b.q));
    const TF d = (b.shape == AL_SHAPE_MESH ? grid.value(local) : b.sdf.sdf(local)) * b.sign;
    mask[i] *= TF(d >= threshold);
  }
}

// quantize (runner.hpp:4516-4536) of one value: floor((v - v_min) *
// step_inverse) saturated to [0, 2^32 - 1] (NaN -> 0) as __float2uint_rd
// does, low byte kept.
inline uint32_t quantize_byte(float v, float v_min, float step_inverse) {
  const float d = v - v_min;
  const float t = d * step_inverse;
  if (!(t > 0.0f)) return 0;
  if (t >= 4294967296.0f) return 0xFFu;
  return uint32_t(std::floor(t)) & 0xFFu;
}

// quantize<double>: (v - v_min) * step_inverse is formed in double and
// reaches __float2uint_rd through the implicit conversion to float (round to
// nearest), then the same saturation.
inline uint32_t quantize_byte(double v, double v_min, double step_inverse) {
  const double d = v - v_min;
  const float t = float(d * step_inverse);
  if (!(t > 0.0f)) return 0;
  if (t >= 4294967296.0f) return 0xFFu;
  return uint32_t(std::floor(t)) & 0xFFu;
}

// launch_histogram256[_with_mask] (runner.hpp:5849-5889, kernels
// runner.hpp:4399-4514): counts of quantized bytes over v[0, n), where
// mask[i] == 1 when a mask is given.  step_inverse is
// TF(256 / (double(v_max) - double(v_min))).
template <class TF>
void histogram256(const TF* v, const TF* mask, uint32_t n, TF v_min, TF v_max,
                  uint32_t hist[256]) {
  const TF step_inverse = TF(256.0 / (double(v_max) - double(v_min)));
  for (int b = 0; b < 256; ++b) hist[b] = 0;
  for (uint32_t i = 0; i < n; ++i)
    if (!mask || mask[i] == TF(1)) ++hist[quantize_byte(v[i], v_min, step_inverse)];
}

// calculate_kl_divergence (runner.hpp:4803-4815 with KLDivergence,
// runner.hpp:746-762): sum over bins with p > 0 of
// p / n_p * log(p / max(q, q_lower_bound) * n_q / n_p), in double.
inline double kl_divergence(const uint32_t* p, const uint32_t* q, uint32_t n_p, uint32_t n_q,
                            double q_lower_bound, uint32_t num_bins) {
  const double inv = 1.0 / n_p, ratio = double(n_q) / n_p;
  double sum = 0;
  for (uint32_t b = 0; b < num_bins; ++b) {
    if (p[b] == 0) continue;
    sum += p[b] * inv * std::log(p[b] / std::max(double(q[b]), q_lower_bound) * ratio);
  }
  return sum;
}

}  // namespace oracle
