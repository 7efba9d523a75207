// contacts.cu -- rigid-rigid contacts on the device: Pile::find_contacts
// (pile.hpp:886-900, volume-map branch) with collision_test
// (runner.hpp:3833-4010) and Pile::solve_contacts (pile.hpp:906-979).
//
// Detection runs in one block over the flattened (pair, vertex) items in
// chunks of the block size; a block-wide exclusive scan of the hit flags
// places every contact at its rank in (i, j, vertex) order, so the list is
// deterministic (the reference appends with an atomic counter).  The
// sequential-impulse solve is inherently ordered: one thread applies the
// five sweeps to the rigid state in device memory.
#include <vector>

#include "body_geometry.cuh"
#include "boundary.cuh"
#include "engine.hpp"

namespace alb {

namespace {

constexpr int kContactBlock = 1024;

struct PairDev {
  uint32_t i, j;
  uint32_t first;  // first item of this pair in the flattened item space
  uint32_t count;  // vertices of body i
  float restitution, friction;
};

using V3 = vec3<float>;

__device__ __forceinline__ void put3(float* d, V3 v) {
  d[0] = v.x;
  d[1] = v.y;
  d[2] = v.z;
}
__device__ __forceinline__ V3 get3(const float* d) { return V3{d[0], d[1], d[2]}; }

// calculate_congruent_matrix (runner.hpp:178-199): R diag(v) R^T.
__device__ void congruent_matrix(V3 v, vec4<float> q, V3& diag, V3& off) {
  const float m00 = 1 - 2 * (q.y * q.y + q.z * q.z), m01 = 2 * (q.x * q.y - q.z * q.w),
              m02 = 2 * (q.x * q.z + q.y * q.w);
  const float m10 = 2 * (q.x * q.y + q.z * q.w), m11 = 1 - 2 * (q.x * q.x + q.z * q.z),
              m12 = 2 * (q.y * q.z - q.x * q.w);
  const float m20 = 2 * (q.x * q.z - q.y * q.w), m21 = 2 * (q.y * q.z + q.x * q.w),
              m22 = 1 - 2 * (q.x * q.x + q.y * q.y);
  diag = V3{v.x * m00 * m00 + v.y * m01 * m01 + v.z * m02 * m02,
            v.x * m10 * m10 + v.y * m11 * m11 + v.z * m12 * m12,
            v.x * m20 * m20 + v.y * m21 * m21 + v.z * m22 * m22};
  off = V3{v.x * m00 * m10 + v.y * m01 * m11 + v.z * m02 * m12,
           v.x * m00 * m20 + v.y * m01 * m21 + v.z * m02 * m22,
           v.x * m10 * m20 + v.y * m11 * m21 + v.z * m12 * m22};
}

// apply_congruent (runner.hpp:253-262).
__device__ __forceinline__ V3 apply_congruent(V3 v, V3 d, V3 o) {
  return V3{v.x * d.x + v.y * o.x + v.z * o.y, v.x * o.x + v.y * d.y + v.z * o.z,
            v.x * o.y + v.y * o.z + v.z * d.z};
}

// calculate_congruent_k (runner.hpp:264-288).
__device__ void congruent_k(V3 r, float mass, V3 d, V3 o, V3& kd, V3& ko) {
  kd = V3{0, 0, 0};
  ko = V3{0, 0, 0};
  if (mass == 0.f) return;
  const float im = 1 / mass;
  kd.x = r.z * r.z * d.y - r.y * r.z * o.z * 2 + r.y * r.y * d.z + im;
  kd.y = r.z * r.z * d.x - r.x * r.z * o.y * 2 + r.x * r.x * d.z + im;
  kd.z = r.y * r.y * d.x - r.x * r.y * o.x * 2 + r.x * r.x * d.y + im;
  ko.x = -r.z * r.z * o.x + r.x * r.z * o.z + r.y * r.z * o.y - r.x * r.y * d.z;
  ko.y = r.y * r.z * o.x - r.x * r.z * d.y - r.y * r.y * o.y + r.x * r.y * o.z;
  ko.z = -(r.y * r.z * d.x) + r.x * r.z * o.x + r.x * r.y * o.y - r.x * r.x * o.z;
}

__device__ __forceinline__ V3 unit(V3 v) { return (1.f / sqrtf(length_sqr(v))) * v; }

// collision_test for one vertex of body i against body j
// (runner.hpp:3833-4010 with collision_find_dist_normal, 1793-1822).
__device__ bool contact_test(const BodyDev<float>& bi, const RigidDev<float>& ri_,
                             const BodyDev<float>& bj, const RigidDev<float>& rj_, uint32_t i,
                             uint32_t j, V3 vertex, float tol, float restitution,
                             float friction, al_contact_f32& ct) {
  const V3 cp_i = rotate(vertex, ri_.q) + ri_.x;
  const vec4<float> qcj{-rj_.q.x, -rj_.q.y, -rj_.q.z, rj_.q.w};
  const V3 local = rotate(cp_i - rj_.x, qcj);
  float dist;
  V3 n{0, 0, 0};
  if (bj.use_grid) {
    dist = bj.sign;  // outside the map: only the existence of a collision is known
    V3 nt{0, 1, 0};
    int ip[3];
    V3 xi;
    if (resolve(bj, local, ip, xi)) {
      const float r2 = xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
      float phi = 0;
      V3 g{0, 0, 0};
#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        float N;
        V3 dN;
        shape_j<float, true>(k, xi, r2, N, dN);
        const float c = bj.dist[lagrange_node(bj.res, ip[0], ip[1], ip[2], k)];
        phi += c * N;
        g.x += c * dN.x;
        g.y += c * dN.y;
        g.z += c * dN.z;
      }
      g.x *= 2.f / bj.cs.x;
      g.y *= 2.f / bj.cs.y;
      g.z *= 2.f / bj.cs.z;
      dist = bj.sign * phi - tol;
      nt = g * bj.sign;
    }
    if (dist < 0) n = unit(nt);
  } else {
    dist = shape_sdf(bj, local) * bj.sign - tol;
    n = unit(shape_gradient(bj, local, 1e-3f) * bj.sign);
  }
  if (!(dist < 0)) return false;
  const V3 cp = local - dist * n;
  ct.i = i;
  ct.j = j;
  const V3 cp_j = rotate(cp, rj_.q) + rj_.x;
  const V3 nw = rotate(n, rj_.q);
  put3(ct.cp_i, cp_i);
  put3(ct.cp_j, cp_j);
  put3(ct.n, nw);
  ct.friction = friction;
  const V3 r_i = cp_i - ri_.x, r_j = cp_j - rj_.x;
  const V3 u_i = ri_.v + cross(ri_.omega, r_i), u_j = rj_.v + cross(rj_.omega, r_j);
  const V3 urel = u_i - u_j;
  const float urn = dot(nw, urel);
  V3 t = urel - urn * nw;
  if (length_sqr(t) > 1e-6f) t = unit(t);
  put3(ct.t, t);
  V3 iid, iio, ijd, ijo;
  congruent_matrix(V3{1 / bi.inertia.x, 1 / bi.inertia.y, 1 / bi.inertia.z}, ri_.q, iid, iio);
  congruent_matrix(V3{1 / bj.inertia.x, 1 / bj.inertia.y, 1 / bj.inertia.z}, rj_.q, ijd, ijo);
  put3(ct.iiwi_diag, iid);
  put3(ct.iiwi_off_diag, iio);
  put3(ct.iiwj_diag, ijd);
  put3(ct.iiwj_off_diag, ijo);
  V3 kid, kio, kjd, kjo;
  congruent_k(r_i, bi.mass, iid, iio, kid, kio);
  congruent_k(r_j, bj.mass, ijd, ijo, kjd, kjo);
  const V3 kd = kid + kjd, ko = kio + kjo;
  ct.nkninv = 1 / dot(nw, apply_congruent(nw, kd, ko));
  ct.pmax = 1 / dot(t, apply_congruent(t, kd, ko)) * dot(urel, t);
  ct.goalu = urn < 0 ? -restitution * urn : 0.f;
  ct.impulse_sum = 0;
  return true;
}

__global__ void __launch_bounds__(kContactBlock)
    k_find_contacts(const BodyDev<float>* __restrict__ bodies,
                    const RigidDev<float>* __restrict__ rigid,
                    const float* const* __restrict__ vertices, const PairDev* __restrict__ pairs,
                    uint32_t num_pairs, uint32_t total, float tol, uint32_t max_contacts,
                    al_contact_f32* __restrict__ out, uint32_t* __restrict__ found) {
  __shared__ uint32_t warp_count[kContactBlock / 32];
  __shared__ uint32_t base;
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) base = 0;
  __syncthreads();
  for (uint32_t chunk = 0; chunk < total; chunk += kContactBlock) {
    const uint32_t item = chunk + tid;
    bool hit = false;
    al_contact_f32 ct;
    if (item < total) {
      uint32_t lo = 0, hi = num_pairs;  // last pair with first <= item
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (pairs[mid].first <= item) lo = mid; else hi = mid;
      }
      const PairDev p = pairs[lo];
      const uint32_t v = item - p.first;
      const float* vp = vertices[p.i] + 3 * size_t(v);
      hit = contact_test(bodies[p.i], rigid[p.i], bodies[p.j], rigid[p.j], p.i, p.j,
                         V3{vp[0], vp[1], vp[2]}, tol, p.restitution, p.friction, ct);
    }
    // block-wide exclusive scan of the hits: rank in (i, j, vertex) order
    const uint32_t ballot = __ballot_sync(0xffffffffu, hit);
    const uint32_t in_warp = __popc(ballot & ((1u << lane) - 1u));
    if (lane == 0) warp_count[warp] = __popc(ballot);
    __syncthreads();
    uint32_t before = 0, chunk_total = 0;
    for (uint32_t w = 0; w < kContactBlock / 32; ++w) {
      if (w < warp) before += warp_count[w];
      chunk_total += warp_count[w];
    }
    const uint32_t rank = base + before + in_warp;
    if (hit && rank < max_contacts) out[rank] = ct;
    __syncthreads();
    if (tid == 0) base += chunk_total;
    __syncthreads();
  }
  if (tid == 0) *found = base;
}

// Pile::solve_contacts (pile.hpp:906-979): five sweeps in contact order.
__global__ void k_solve_contacts(const BodyDev<float>* __restrict__ bodies,
                                 RigidDev<float>* __restrict__ rigid,
                                 al_contact_f32* __restrict__ contacts, uint32_t num) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int sweep = 0; sweep < 5; ++sweep)
    for (uint32_t k = 0; k < num; ++k) {
      al_contact_f32& c = contacts[k];
      RigidDev<float>& bi = rigid[c.i];
      RigidDev<float>& bj = rigid[c.j];
      const float mi = bodies[c.i].mass, mj = bodies[c.j].mass;
      const V3 n = get3(c.n), t = get3(c.t), cpi = get3(c.cp_i), cpj = get3(c.cp_j);
      const float depth = dot(n, cpi - cpj);
      const V3 r_i = cpi - bi.x, r_j = cpj - bj.x;
      const V3 u_i = bi.v + cross(bi.omega, r_i), u_j = bj.v + cross(bj.omega, r_j);
      const V3 urel = u_i - u_j;
      const float urn = dot(n, urel);
      float corr = c.nkninv * (c.goalu - urn);
      if (corr < -c.impulse_sum) corr = -c.impulse_sum;
      if (depth < 0) corr -= c.nkninv * depth;  // stiffness 1
      V3 p = corr * n;
      c.impulse_sum += corr;
      const float pn = dot(p, n);
      if (c.friction * pn > c.pmax)
        p = p - c.pmax * t;
      else if (c.friction * pn < -c.pmax)
        p = p + c.pmax * t;
      else
        p = p - (c.friction * pn) * t;
      if (mi != 0.f) {
        bi.v = bi.v + (1.f / mi) * p;
        bi.omega = bi.omega + apply_congruent(cross(r_i, p), get3(c.iiwi_diag),
                                              get3(c.iiwi_off_diag));
      }
      if (mj != 0.f) {
        bj.v = bj.v - (1.f / mj) * p;
        bj.omega = bj.omega + apply_congruent(cross(r_j, -1.f * p), get3(c.iiwj_diag),
                                              get3(c.iiwj_off_diag));
      }
    }
}

}  // namespace

}  // namespace alb

using namespace alb;

extern "C" {

int al_find_contacts_f32(al_engine* engine, const al_body_f32* bodies, const al_rigid_f32* rigid,
                         const al_contact_body_f32* cb, uint32_t nb, float tol,
                         uint32_t max_contacts, al_contact_f32* contacts, uint32_t* num_found,
                         void* stream) {
  ALB_CHECK_ARG(engine && num_found && (nb == 0 || (bodies && rigid && cb)),
                "al_find_contacts_f32: null argument");
  ALB_CHECK_ARG(nb <= AL_MAX_BOUNDARIES, "al_find_contacts_f32: too many bodies");
  ALB_CHECK_ARG(max_contacts == 0 || contacts, "al_find_contacts_f32: contacts is null");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  *num_found = 0;
  std::vector<BodyDev<float>> hb(nb);
  std::vector<RigidDev<float>> hr(nb);
  std::vector<const float*> hv(nb);
  for (uint32_t b = 0; b < nb; ++b) {
    hb[b] = to_body_dev<float>(bodies[b]);
    ALB_TRY(validate_body(hb[b], true, false));
    hr[b] = to_rigid_dev<float>(rigid[b]);
    ALB_CHECK_ARG(cb[b].num_vertices == 0 || cb[b].vertices,
                  "al_find_contacts_f32: vertices are null");
    hv[b] = cb[b].vertices;
  }
  std::vector<PairDev> pairs;
  uint64_t total = 0;
  for (uint32_t i = 0; i < nb; ++i)
    for (uint32_t j = 0; j < nb; ++j) {
      if (i == j || (bodies[i].mass == 0 && bodies[j].mass == 0)) continue;
      if (cb[i].num_vertices == 0) continue;
      pairs.push_back(PairDev{i, j, uint32_t(total), cb[i].num_vertices,
                              cb[i].restitution * cb[j].restitution,
                              cb[i].friction + cb[j].friction});
      total += cb[i].num_vertices;
    }
  ALB_CHECK_ARG(total < (1ull << 31), "al_find_contacts_f32: too many collision vertices");
  if (pairs.empty()) return AL_OK;
  BodyDev<float>* db = nullptr;
  RigidDev<float>* dr = nullptr;
  const float** dv = nullptr;
  PairDev* dp = nullptr;
  uint32_t* dfound = nullptr;
  ALB_TRY(engine->buf("contact.bodies", nb, &db));
  ALB_TRY(engine->buf("contact.rigid", nb, &dr));
  ALB_TRY(engine->buf("contact.vertices", nb, &dv));
  ALB_TRY(engine->buf("contact.pairs", pairs.size(), &dp));
  ALB_TRY(engine->buf("contact.found", 1, &dfound));
  ALB_CUDA(cudaMemcpyAsync(db, hb.data(), sizeof(BodyDev<float>) * nb, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dr, hr.data(), sizeof(RigidDev<float>) * nb, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dv, hv.data(), sizeof(float*) * nb, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dp, pairs.data(), sizeof(PairDev) * pairs.size(),
                           cudaMemcpyHostToDevice, st));
  ALB_LAUNCH(engine, "find_contacts", 1, st,
             (k_find_contacts<<<1, kContactBlock, 0, st>>>(db, dr, dv, dp, uint32_t(pairs.size()),
                                                            uint32_t(total), tol, max_contacts,
                                                            contacts, dfound)));
  ALB_CUDA(cudaGetLastError());
  ALB_CUDA(cudaMemcpyAsync(num_found, dfound, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  return AL_OK;
}

int al_solve_contacts_f32(al_engine* engine, const al_body_f32* bodies, al_rigid_f32* rigid,
                          uint32_t nb, al_contact_f32* contacts, uint32_t num_contacts,
                          void* stream) {
  ALB_CHECK_ARG(engine && (nb == 0 || (bodies && rigid)), "al_solve_contacts_f32: null argument");
  ALB_CHECK_ARG(nb <= AL_MAX_BOUNDARIES, "al_solve_contacts_f32: too many bodies");
  ALB_CHECK_ARG(num_contacts == 0 || contacts, "al_solve_contacts_f32: contacts is null");
  if (num_contacts == 0 || nb == 0) return AL_OK;
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::vector<BodyDev<float>> hb(nb);
  std::vector<RigidDev<float>> hr(nb);
  for (uint32_t b = 0; b < nb; ++b) {
    hb[b] = to_body_dev<float>(bodies[b]);
    hr[b] = to_rigid_dev<float>(rigid[b]);
  }
  BodyDev<float>* db = nullptr;
  RigidDev<float>* dr = nullptr;
  ALB_TRY(engine->buf("contact.bodies", nb, &db));
  ALB_TRY(engine->buf("contact.rigid", nb, &dr));
  ALB_CUDA(cudaMemcpyAsync(db, hb.data(), sizeof(BodyDev<float>) * nb, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(dr, hr.data(), sizeof(RigidDev<float>) * nb, cudaMemcpyHostToDevice, st));
  ALB_LAUNCH(engine, "solve_contacts", 1, st,
             (k_solve_contacts<<<1, 1, 0, st>>>(db, dr, contacts, num_contacts)));
  ALB_CUDA(cudaGetLastError());
  ALB_CUDA(cudaMemcpyAsync(hr.data(), dr, sizeof(RigidDev<float>) * nb, cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  for (uint32_t b = 0; b < nb; ++b) {
    rigid[b].v[0] = hr[b].v.x;
    rigid[b].v[1] = hr[b].v.y;
    rigid[b].v[2] = hr[b].v.z;
    rigid[b].omega[0] = hr[b].omega.x;
    rigid[b].omega[1] = hr[b].omega.y;
    rigid[b].omega[2] = hr[b].omega.z;
  }
  return AL_OK;
}

}  // extern "C"
