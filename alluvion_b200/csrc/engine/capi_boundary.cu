// capi_boundary.cu -- extern "C" entry points for boundary sampling, volume
// maps, distance grids and node positions.
#include <vector>

#include "boundary.cuh"

using namespace alb;

namespace {

template <class TF>
__global__ void k_pack_positions(const TF* __restrict__ x, uint32_t n, vec4<TF>* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const vec3<TF> p = ld3(x, i);
  out[i] = vec4<TF>{p.x, p.y, p.z, TF(0)};
}

template <class TF, class C, class B, class R>
int boundary_impl(al_engine* e, const C* cn, uint32_t nb, const B* bodies, const R* rigid,
                  const TF* x, uint32_t n, TF* ref_b, TF* ref_k, cudaStream_t st) {
  ALB_CHECK_ARG(e && cn && x && ref_b && ref_k, "al_compute_particle_boundary: null argument");
  ALB_CHECK_ARG(nb <= AL_MAX_BOUNDARIES, "al_compute_particle_boundary: too many boundaries");
  ALB_CHECK_ARG(nb == 0 || (bodies && rigid), "al_compute_particle_boundary: bodies are null");
  ALB_TRY(e->activate());
  if (nb == 0 || n == 0) return AL_OK;
  const Cn<TF> c = to_cn<TF>(*cn);
  std::vector<BodyDev<TF>> hb(nb);
  std::vector<RigidDev<TF>> hr(nb);
  for (uint32_t b = 0; b < nb; ++b) {
    hb[b] = to_body_dev<TF>(bodies[b]);
    ALB_TRY(validate_body(hb[b], true, true));
    hr[b] = to_rigid_dev<TF>(rigid[b]);
  }
  BodyDev<TF>* db = nullptr;
  RigidDev<TF>* dr = nullptr;
  vec4<TF>* xs = nullptr;
  ALB_TRY(e->buf("sample.bodies", nb, &db));
  ALB_TRY(e->buf("sample.rigid", nb, &dr));
  ALB_TRY(e->buf("sample.x", n, &xs));
  ALB_CUDA(cudaMemcpyAsync(db, hb.data(), sizeof(BodyDev<TF>) * nb, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dr, hr.data(), sizeof(RigidDev<TF>) * nb, cudaMemcpyHostToDevice, st));
  k_pack_positions<TF><<<(n + 255) / 256, 256, 0, st>>>(x, n, xs);
  BoundaryState<TF> bs;  // dense reference output only
  ALB_TRY(sample_boundaries<TF>(c, db, dr, nb, xs, nullptr, n, bs, ref_b, ref_k, st));
  ALB_CUDA(cudaStreamSynchronize(st));  // host staging vectors go out of scope
  return AL_OK;
}

template <class TF, class C, class B>
int volume_impl(al_engine* e, const C* cn, const B* body, TF* out, cudaStream_t st) {
  ALB_CHECK_ARG(e && cn && body && out, "al_build_volume_field: null argument");
  ALB_TRY(e->activate());
  const BodyDev<TF> b = to_body_dev<TF>(*body);
  ALB_TRY(validate_body(b, true, false));
  return build_volume_field<TF>(to_cn<TF>(*cn), b, out, st);
}

template <class TF, class B>
int distance_impl(al_engine* e, const B* body, TF* out, cudaStream_t st) {
  ALB_CHECK_ARG(e && body && out, "al_build_distance_grid: null argument");
  ALB_CHECK_ARG(body->shape != AL_SHAPE_MESH,
                "al_build_distance_grid: mesh bodies use al_build_mesh_distance_grid_f32");
  ALB_TRY(e->activate());
  const BodyDev<TF> b = to_body_dev<TF>(*body);
  ALB_TRY(validate_body(b, false, false));
  return build_distance_grid<TF>(b, out, st);
}

template <class TF, class B>
int positions_impl(al_engine* e, const B* body, TF* out, cudaStream_t st) {
  ALB_CHECK_ARG(e && body && out, "al_node_positions: null argument");
  ALB_TRY(e->activate());
  const BodyDev<TF> b = to_body_dev<TF>(*body);
  ALB_TRY(validate_body(b, false, false));
  return node_positions<TF>(b, out, st);
}

}  // namespace

extern "C" {

int al_compute_particle_boundary_f32(al_engine* engine, const al_const_f32* cn,
                                     uint32_t num_boundaries, const al_body_f32* bodies,
                                     const al_rigid_f32* rigid, const float* particle_x,
                                     uint32_t num_particles, float* particle_boundary,
                                     float* particle_boundary_kernel, void* stream) {
  return boundary_impl<float>(engine, cn, num_boundaries, bodies, rigid, particle_x,
                              num_particles, particle_boundary, particle_boundary_kernel,
                              static_cast<cudaStream_t>(stream));
}
int al_compute_particle_boundary_f64(al_engine* engine, const al_const_f64* cn,
                                     uint32_t num_boundaries, const al_body_f64* bodies,
                                     const al_rigid_f64* rigid, const double* particle_x,
                                     uint32_t num_particles, double* particle_boundary,
                                     double* particle_boundary_kernel, void* stream) {
  return boundary_impl<double>(engine, cn, num_boundaries, bodies, rigid, particle_x,
                               num_particles, particle_boundary, particle_boundary_kernel,
                               static_cast<cudaStream_t>(stream));
}
int al_build_volume_field_f32(al_engine* engine, const al_const_f32* cn, const al_body_f32* body,
                              float* volume_nodes, void* stream) {
  return volume_impl<float>(engine, cn, body, volume_nodes, static_cast<cudaStream_t>(stream));
}
int al_build_volume_field_f64(al_engine* engine, const al_const_f64* cn, const al_body_f64* body,
                              double* volume_nodes, void* stream) {
  return volume_impl<double>(engine, cn, body, volume_nodes, static_cast<cudaStream_t>(stream));
}
int al_build_distance_grid_f32(al_engine* engine, const al_body_f32* body, float* distance_nodes,
                               void* stream) {
  return distance_impl<float>(engine, body, distance_nodes, static_cast<cudaStream_t>(stream));
}
int al_build_distance_grid_f64(al_engine* engine, const al_body_f64* body,
                               double* distance_nodes, void* stream) {
  return distance_impl<double>(engine, body, distance_nodes, static_cast<cudaStream_t>(stream));
}
int al_node_positions_f32(al_engine* engine, const al_body_f32* body, float* positions,
                          void* stream) {
  return positions_impl<float>(engine, body, positions, static_cast<cudaStream_t>(stream));
}
int al_node_positions_f64(al_engine* engine, const al_body_f64* body, double* positions,
                          void* stream) {
  return positions_impl<double>(engine, body, positions, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
