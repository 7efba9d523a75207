// mesh.cu -- signed distance of a closed triangle mesh at the nodes of a
// body's cubic Lagrange grid, on the device: the distance grid Pile builds
// on the host for MeshDistance bodies (construct_distance_grid,
// pile.hpp:79-94, with MeshDistance::signedDistance,
// dg/mesh_distance.hpp:186-223).
//
// Distance: exact point-triangle distance with the closest point's Voronoi
// region (vertex, edge or face) classified as in Ericson, Real-Time
// Collision Detection, sec. 5.1.5; every node tests every face (faces are
// staged through shared memory, so each load is a broadcast) and keeps the
// first nearest one.  Sign: angle-weighted pseudonormals (Baerentzen and
// Aanaes) of the nearest feature, as MeshDistance does: face normal, the
// sum of the two faces' normals at an edge, the incident-angle-weighted sum
// at a vertex; negative where (x - closest) . n < 0.  The reference finds
// the nearest face through a bounding-sphere hierarchy; at exact ties the
// two may pick different faces, whose pseudonormals agree in sign for a
// closed 2-manifold.
#include <array>
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include "body_geometry.cuh"
#include "boundary.cuh"
#include "engine.hpp"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

constexpr int kMeshBlock = 256;

using V3 = vec3<float>;

__device__ __forceinline__ V3 ld(const float* p, uint32_t i) {
  return V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}

// Closest point of triangle (a, b, c) to p and its region: 0-2 vertex
// a/b/c, 3 edge ab, 4 edge bc, 5 edge ca, 6 face.
__device__ __forceinline__ V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c, int& region) {
  const V3 ab = b - a, ac = c - a, ap = p - a;
  const float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) {
    region = 0;
    return a;
  }
  const V3 bp = p - b;
  const float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.f && d4 <= d3) {
    region = 1;
    return b;
  }
  const float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
    region = 3;
    return a + (d1 / (d1 - d3)) * ab;
  }
  const V3 cp = p - c;
  const float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.f && d5 <= d6) {
    region = 2;
    return c;
  }
  const float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
    region = 5;
    return a + (d2 / (d2 - d6)) * ac;
  }
  const float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
    region = 4;
    return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
  }
  region = 6;
  const float denom = 1.f / (va + vb + vc);
  return a + (vb * denom) * ab + (vc * denom) * ac;
}

// out[l] = signed distance of node l (minus offset).
__global__ void __launch_bounds__(kMeshBlock)
    k_mesh_distance(BodyDev<float> b, const float* __restrict__ verts,
                    const uint32_t* __restrict__ faces, const float* __restrict__ fnormal,
                    const float* __restrict__ vnormal, const float* __restrict__ enormal,
                    uint32_t nf, float offset, float* __restrict__ out) {
  __shared__ float tri[kMeshBlock][9];
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = l < b.num_nodes;
  const V3 p = active ? node_position(b, l) : V3{0, 0, 0};
  float best = 3.4e38f;
  uint32_t best_f = 0;
  int best_r = 6;
  V3 best_q{0, 0, 0};
  for (uint32_t f0 = 0; f0 < nf; f0 += kMeshBlock) {
    const uint32_t f = f0 + threadIdx.x;
    if (f < nf) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const V3 v = ld(verts, faces[3 * f + k]);
        tri[threadIdx.x][3 * k] = v.x;
        tri[threadIdx.x][3 * k + 1] = v.y;
        tri[threadIdx.x][3 * k + 2] = v.z;
      }
    }
    __syncthreads();
    const uint32_t cnt = nf - f0 < kMeshBlock ? nf - f0 : kMeshBlock;
    for (uint32_t k = 0; k < cnt; ++k) {
      const float* t = tri[k];
      int region;
      const V3 q = closest_on_triangle(p, V3{t[0], t[1], t[2]}, V3{t[3], t[4], t[5]},
                                       V3{t[6], t[7], t[8]}, region);
      const float d2 = length_sqr(p - q);
      if (d2 < best) {
        best = d2;
        best_f = f0 + k;
        best_r = region;
        best_q = q;
      }
    }
    __syncthreads();
  }
  if (!active) return;
  V3 n;
  if (best_r < 3)
    n = ld(vnormal, faces[3 * best_f + best_r]);
  else if (best_r < 6)
    n = ld(enormal, 3 * best_f + (best_r - 3));
  else
    n = ld(fnormal, best_f);
  float dist = sqrtf(best);
  if (dot(p - best_q, n) < 0.f) dist = -dist;
  out[l] = dist - offset;
}

}  // namespace

}  // namespace alb

using namespace alb;

extern "C" {

int al_build_mesh_distance_grid_f32(al_engine* engine, const al_body_f32* body,
                                    const float* vertices, uint32_t num_vertices,
                                    const uint32_t* faces, uint32_t num_faces, float offset,
                                    float* nodes, void* stream) {
  ALB_CHECK_ARG(engine && body && nodes, "al_build_mesh_distance_grid_f32: null argument");
  ALB_CHECK_ARG(num_faces > 0 && num_vertices >= 3 && vertices && faces,
                "al_build_mesh_distance_grid_f32: empty mesh");
  BodyDev<float> b = to_body_dev<float>(*body);
  b.use_grid = 1;
  ALB_TRY(validate_body(b, false, false));
  for (uint64_t k = 0; k < uint64_t(num_faces) * 3; ++k)
    ALB_CHECK_ARG(faces[k] < num_vertices, "al_build_mesh_distance_grid_f32: face index out of range");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // pseudonormals in double on the host (MeshDistance's precomputed normals,
  // dg/mesh_distance.hpp:80-104, 247-266)
  auto vtx = [&](uint32_t i) {
    return std::array<double, 3>{vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]};
  };
  auto sub = [](std::array<double, 3> a, std::array<double, 3> c) {
    return std::array<double, 3>{a[0] - c[0], a[1] - c[1], a[2] - c[2]};
  };
  auto crs = [](std::array<double, 3> a, std::array<double, 3> c) {
    return std::array<double, 3>{a[1] * c[2] - a[2] * c[1], a[2] * c[0] - a[0] * c[2],
                                 a[0] * c[1] - a[1] * c[0]};
  };
  auto unit = [](std::array<double, 3> a) {
    const double l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    return l > 0 ? std::array<double, 3>{a[0] / l, a[1] / l, a[2] / l} : a;
  };
  auto dt = [](std::array<double, 3> a, std::array<double, 3> c) {
    return a[0] * c[0] + a[1] * c[1] + a[2] * c[2];
  };
  std::vector<std::array<double, 3>> fn(num_faces), vn(num_vertices, {0, 0, 0});
  std::map<std::pair<uint32_t, uint32_t>, uint32_t> edge_face;  // directed edge -> face
  for (uint32_t f = 0; f < num_faces; ++f) {
    const uint32_t* t = faces + 3 * f;
    const auto x0 = vtx(t[0]), x1 = vtx(t[1]), x2 = vtx(t[2]);
    fn[f] = unit(crs(sub(x1, x0), sub(x2, x0)));
    const auto e1 = unit(sub(x1, x0)), e2 = unit(sub(x2, x1)), e3 = unit(sub(x0, x2));
    auto ang = [&](std::array<double, 3> a, std::array<double, 3> c) {
      double d = -dt(a, c);
      d = d < -1 ? -1 : (d > 1 ? 1 : d);
      return std::acos(d);
    };
    const double alpha[3] = {ang(e1, e3), ang(e2, e1), ang(e3, e2)};
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) vn[t[k]][c] += alpha[k] * fn[f][c];
    for (int k = 0; k < 3; ++k) edge_face[{t[k], t[(k + 1) % 3]}] = f;
  }
  std::vector<float> hf(3 * size_t(num_faces)), hv(3 * size_t(num_vertices)),
      he(9 * size_t(num_faces));
  for (uint32_t f = 0; f < num_faces; ++f) {
    const uint32_t* t = faces + 3 * f;
    for (int c = 0; c < 3; ++c) hf[3 * f + c] = float(fn[f][c]);
    for (int k = 0; k < 3; ++k) {  // halfedge k: vertex k -> vertex k + 1
      auto it = edge_face.find({t[(k + 1) % 3], t[k]});
      for (int c = 0; c < 3; ++c)
        he[9 * f + 3 * k + c] =
            float(fn[f][c] + (it != edge_face.end() ? fn[it->second][c] : 0.0));
    }
  }
  for (uint32_t v = 0; v < num_vertices; ++v)
    for (int c = 0; c < 3; ++c) hv[3 * v + c] = float(vn[v][c]);
  float *dverts = nullptr, *dfn = nullptr, *dvn = nullptr, *den = nullptr;
  uint32_t* dfaces = nullptr;
  ALB_TRY(engine->buf("mesh.vertices", 3 * size_t(num_vertices), &dverts));
  ALB_TRY(engine->buf("mesh.faces", 3 * size_t(num_faces), &dfaces));
  ALB_TRY(engine->buf("mesh.fn", hf.size(), &dfn));
  ALB_TRY(engine->buf("mesh.vn", hv.size(), &dvn));
  ALB_TRY(engine->buf("mesh.en", he.size(), &den));
  ALB_CUDA(cudaMemcpyAsync(dverts, vertices, sizeof(float) * 3 * num_vertices,
                           cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dfaces, faces, sizeof(uint32_t) * 3 * num_faces,
                           cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dfn, hf.data(), sizeof(float) * hf.size(), cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dvn, hv.data(), sizeof(float) * hv.size(), cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(den, he.data(), sizeof(float) * he.size(), cudaMemcpyHostToDevice, st));
  ALB_LAUNCH(engine, "mesh_distance", 1, st,
             (k_mesh_distance<<<blocks_for(b.num_nodes, kMeshBlock), kMeshBlock, 0, st>>>(
                 b, dverts, dfaces, dfn, dvn, den, num_faces, offset, nodes)));
  ALB_CUDA(cudaGetLastError());
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  return AL_OK;
}

}  // extern "C"
