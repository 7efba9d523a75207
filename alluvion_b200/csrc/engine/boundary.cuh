// boundary.cuh -- rigid-boundary terms from volume maps and signed distance
// fields on cubic Lagrange grids.
//
// Replaces compute_particle_boundary (runner.hpp:2004-2025, distance grid),
// compute_particle_boundary_analytic<0> (runner.hpp:1982-2002, analytic SDF)
// and update_volume_field (runner.hpp:1616-1694) with the Lagrange helpers
// they use (runner.hpp:1131-1257, 1259-1614, 1696-1791).
//
// The 32-node element is evaluated node by node and fused with the node
// gathers, so no shape-function arrays are held per thread.  Results are
// kept sparse: per sorted particle a bitmask of the bodies whose
// interpolated volume is non-zero, and {x_b, V}, {grad W V, W V} only for
// those (particle, body) pairs.  Every term of the solver passes vanishes
// exactly for V == 0, so the sparse form changes no sum.
#pragma once

#include "common.cuh"
#include "engine.hpp"

namespace alb {

template <class TF>
struct BodyDev {
  uint32_t shape, use_grid;
  TF sign;
  TF p[8];
  vec3<TF> dmin, dmax, cs;
  uint32_t res[3];
  uint32_t num_nodes;
  const TF* dist;
  const TF* vol;
  TF max_distance, mass;
  vec3<TF> inertia;
};

template <class TF>
struct RigidDev {
  vec3<TF> x, v, omega;
  vec4<TF> q;
};

template <class TF, class B>
BodyDev<TF> to_body_dev(const B& b) {
  BodyDev<TF> o;
  o.shape = b.shape;
  o.use_grid = b.use_distance_grid;
  o.sign = b.sign;
  for (int k = 0; k < 8; ++k) o.p[k] = b.shape_params[k];
  o.dmin = vec3<TF>{b.domain_min[0], b.domain_min[1], b.domain_min[2]};
  o.dmax = vec3<TF>{b.domain_max[0], b.domain_max[1], b.domain_max[2]};
  o.cs = vec3<TF>{b.cell_size[0], b.cell_size[1], b.cell_size[2]};
  for (int k = 0; k < 3; ++k) o.res[k] = b.resolution[k];
  o.num_nodes = b.num_nodes;
  o.dist = b.distance_nodes;
  o.vol = b.volume_nodes;
  o.max_distance = b.max_distance;
  o.mass = b.mass;
  o.inertia = vec3<TF>{b.inertia[0], b.inertia[1], b.inertia[2]};
  return o;
}

template <class TF, class R>
RigidDev<TF> to_rigid_dev(const R& r) {
  RigidDev<TF> o;
  o.x = vec3<TF>{r.x[0], r.x[1], r.x[2]};
  o.v = vec3<TF>{r.v[0], r.v[1], r.v[2]};
  o.omega = vec3<TF>{r.omega[0], r.omega[1], r.omega[2]};
  o.q = vec4<TF>{r.q[0], r.q[1], r.q[2], r.q[3]};
  return o;
}

template <class TF>
inline int validate_body(const BodyDev<TF>& b, bool need_dist, bool need_vol) {
  ALB_CHECK_ARG(b.shape <= AL_SHAPE_INFINITE_TUBE, "body: unknown shape");
  ALB_CHECK_ARG(b.shape != AL_SHAPE_MESH || b.use_grid,
                "body: a mesh body needs its distance grid (use_distance_grid = 1)");
  ALB_CHECK_ARG(!(b.shape == AL_SHAPE_INFINITE_CYLINDER || b.shape == AL_SHAPE_INFINITE_TUBE) ||
                    !b.use_grid,
                "body: y-invariant shapes are sampled analytically (use_distance_grid = 0)");
  ALB_CHECK_ARG(b.res[0] > 0 && b.res[1] > 0 && b.res[2] > 0, "body: zero resolution");
  uint64_t nx = b.res[0], ny = b.res[1], nz = b.res[2];
  uint64_t nn = (nx + 1) * (ny + 1) * (nz + 1) +
                2 * (nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz);
  ALB_CHECK_ARG(nn == b.num_nodes, "body: num_nodes does not match resolution");
  ALB_CHECK_ARG(nn < (1ull << 31), "body: grid too large");
  ALB_CHECK_ARG(!need_dist || !b.use_grid || b.dist != nullptr, "body: distance_nodes is null");
  ALB_CHECK_ARG(!need_vol || b.vol != nullptr, "body: volume_nodes is null");
  return AL_OK;
}

// Sparse boundary state in sorted order.
template <class TF>
struct BoundaryState {
  uint32_t nb = 0;
  uint32_t* mask = nullptr;  // [n] bit b set: V_b != 0
  vec4<TF>* bx = nullptr;    // [nb][n] {x_b, V}
  vec4<TF>* bk = nullptr;    // [nb][n] {grad W * V, W * V}
  uint32_t* active = nullptr;  // optional counter += number of set mask bits
  uint32_t stride = 0;         // row stride of bx / bk (0: n)
};

// Samples every body for every sorted particle (positions xs).  When
// ref_boundary / ref_kernel are non-null, also writes the dense reference
// layout [nb][N][4] in original order (perm: sorted -> original).
template <class TF>
int sample_boundaries(const Cn<TF>& c, const BodyDev<TF>* bodies_dev, const RigidDev<TF>* rigid_dev,
                      uint32_t nb, const vec4<TF>* xs, const uint32_t* perm, uint32_t n,
                      const BoundaryState<TF>& bs, TF* ref_boundary, TF* ref_kernel,
                      cudaStream_t st);

// One scene of a fused batch for sample_boundaries_fused: its bodies, rigid
// state, the batch's permutation (sorted arena slot -> arena slot s0 + i of
// the scene's particle i), optional reference-layout outputs ([nb][n][4],
// original order), active-pair counter and arena range [s0, s0 + n).
template <class TF>
struct BoundaryScene {
  const BodyDev<TF>* bodies;
  const RigidDev<TF>* rigid;
  const uint32_t* perm;
  TF* ref_b;
  TF* ref_k;
  uint32_t* active;
  uint32_t nb, s0, n, pad;
};

// sample_boundaries for every scene of a fused batch in one launch over the
// arena (kBlock-thread blocks; blk_scene[block] = the block's scene, or
// nscenes past every scene): mask / bx / bk over the arena, rows `stride`
// apart.
template <class TF>
int sample_boundaries_fused(const Cn<TF>& c, const vec4<TF>* xs, uint32_t stride,
                            const uint32_t* blk_scene, const BoundaryScene<TF>* scenes,
                            uint32_t nscenes, uint32_t nblocks, uint32_t* mask, vec4<TF>* bx,
                            vec4<TF>* bk, cudaStream_t st);

// Volume-map nodes of one body (update_volume_field).  Distance from the
// body's grid when use_grid, else from its analytic SDF.
template <class TF>
int build_volume_field(const Cn<TF>& c, const BodyDev<TF>& b, TF* out, cudaStream_t st);

// Distance nodes sampled from the analytic SDF at the node positions.
template <class TF>
int build_distance_grid(const BodyDev<TF>& b, TF* out, cudaStream_t st);

// Node positions (index_to_node_position), [num_nodes][3].
template <class TF>
int node_positions(const BodyDev<TF>& b, TF* out, cudaStream_t st);

// Uploads the Peirce tables (computed on the host) to constant memory.
int upload_peirce_tables(cudaStream_t st);

}  // namespace alb
