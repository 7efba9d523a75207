// boundary.cu -- Lagrange-grid / analytic boundary sampling, volume maps,
// distance grids.
#include <cmath>

#include "boundary.cuh"
#include "body_geometry.cuh"
#include "peirce_tables.h"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

// Quadrature tables in constant memory: per azimuth i cos/sin(theta_i), per
// polar node j sin/cos(phi_j), per (j, k) the weight 2 pi b_j c_k / 60, per
// k the radius.
template <class T>
struct PeirceTab {
  T ct[peirce::kNumTheta], st[peirce::kNumTheta];
  T sp[peirce::kNumPhi], cp[peirce::kNumPhi];
  T w[peirce::kNumPhi * peirce::kNumR];
  T r[peirce::kNumR];
};
using PeirceDev = PeirceTab<float>;
using PeirceDevD = PeirceTab<double>;
__constant__ PeirceDev c_peirce_f;
__constant__ PeirceDevD c_peirce_d;

template <class TF>
struct PeirceSel;
template <>
struct PeirceSel<float> {
  __device__ static const PeirceDev& get() { return c_peirce_f; }
};
template <>
struct PeirceSel<double> {
  __device__ static const PeirceDevD& get() { return c_peirce_d; }
};

// Boundary sample of one particle against one body
// (compute_volume_and_boundary_x[_analytic], runner.hpp:1696-1771, and the
// writes of compute_particle_boundary[_analytic], runner.hpp:1982-2025).
template <class TF>
__device__ __forceinline__ void sample_body(const Cn<TF>& c, const BodyDev<TF>& b,
                                            const RigidDev<TF>& r, vec3<TF> x, vec4<TF>& bnd,
                                            vec4<TF>& bk) {
  const vec4<TF> qc{-r.q.x, -r.q.y, -r.q.z, r.q.w};
  vec3<TF> local = rotate(x - r.x, qc);
  // compute_volume_and_boundary_x_analytic<1> for the y-invariant shapes
  // (runner.hpp:1744-1746)
  if (shape_is_y_invariant(b.shape)) local.y = TF(0);
  vec3<TF> bx = x, xi_bxj{0, 0, 0};
  TF d = 0, vol = 0;
  int ip[3];
  vec3<TF> xi;
  const bool inside = resolve(b, local, ip, xi);
  if (b.use_grid) {
    if (inside) {
      const TF r2 = xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
      TF phi = 0;
      vec3<TF> grad{0, 0, 0};
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        TF N;
        vec3<TF> dN;
        shape_j<TF, true>(j, xi, r2, N, dN);
        const uint32_t node = lagrange_node(b.res, ip[0], ip[1], ip[2], j);
        const TF dv = __ldg(b.dist + node);
        phi += dv * N;
        grad.x += dv * dN.x;
        grad.y += dv * dN.y;
        grad.z += dv * dN.z;
        vol += __ldg(b.vol + node) * N;
      }
      grad.x *= TF(2) / b.cs.x;
      grad.y *= TF(2) / b.cs.y;
      grad.z *= TF(2) / b.cs.z;
      d = phi * b.sign;
      vec3<TF> nrm = rotate(grad * b.sign, r.q);
      const TF nl2 = length_sqr(nrm);
      nrm = (nl2 > TF(0) ? rsqrt_(nl2) : TF(0)) * nrm;
      xi_bxj = d * nrm;
      bx = x - xi_bxj;
    }
  } else {
    d = shape_sdf(b, local) * b.sign;
    vec3<TF> nrm = rotate(shape_gradient(b, local, c.h) * b.sign, r.q);
    const TF nl2 = length_sqr(nrm);
    nrm = (nl2 > TF(0) ? rsqrt_(nl2) : TF(0)) * nrm;
    xi_bxj = d * nrm;
    bx = x - xi_bxj;
    if (inside) {
      const TF r2 = xi.x * xi.x + xi.y * xi.y + xi.z * xi.z;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        TF N;
        vec3<TF> dN;
        shape_j<TF, false>(j, xi, r2, N, dN);
        vol += __ldg(b.vol + lagrange_node(b.res, ip[0], ip[1], ip[2], j)) * N;
      }
    }
  }
  const vec3<TF> kg = gradW(c, xi_bxj);
  bnd = vec4<TF>{bx.x, bx.y, bx.z, vol};
  bk = vec4<TF>{vol * kg.x, vol * kg.y, vol * kg.z, vol * W_dist(c, d)};
}

// Samples every body for the particle at slot s (position xs[s]; mask,
// bx, bk at s, rows `stride` apart) and, when ref_b / ref_k are set, writes
// the dense reference layout at its original index i (rows of n_ref).
template <class TF>
__device__ __forceinline__ void sample_particle(
    const Cn<TF>& c, const BodyDev<TF>* __restrict__ bodies, const RigidDev<TF>* __restrict__ rigid,
    uint32_t nb, const vec4<TF>* __restrict__ xs, uint32_t s, uint32_t i, uint32_t n_ref,
    uint32_t stride, uint32_t* __restrict__ mask, vec4<TF>* __restrict__ bx,
    vec4<TF>* __restrict__ bk, TF* __restrict__ ref_b, TF* __restrict__ ref_k,
    uint32_t* __restrict__ active) {
  const vec3<TF> x = xyz(xs[s]);
  uint32_t m = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    vec4<TF> bnd, kk;
    sample_body(c, bodies[b], rigid[b], x, bnd, kk);
    if (bnd.w != TF(0)) {
      m |= 1u << b;
      if (bx) {
        bx[size_t(b) * stride + s] = bnd;
        bk[size_t(b) * stride + s] = kk;
      }
    }
    if (ref_b) {
      TF* o = ref_b + (size_t(b) * n_ref + i) * 4;
      o[0] = bnd.x;
      o[1] = bnd.y;
      o[2] = bnd.z;
      o[3] = bnd.w;
      TF* k = ref_k + (size_t(b) * n_ref + i) * 4;
      k[0] = kk.x;
      k[1] = kk.y;
      k[2] = kk.z;
      k[3] = kk.w;
    }
  }
  if (mask) mask[s] = m;
  if (active) {
    // warp-aggregated count of active (particle, body) pairs
    const unsigned live = __activemask();
    const unsigned tot = __reduce_add_sync(live, unsigned(__popc(m)));
    if ((threadIdx.x & 31) == unsigned(__ffs(live) - 1) && tot) atomicAdd(active, tot);
  }
}

template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_sample_boundaries(Cn<TF> c, const BodyDev<TF>* __restrict__ bodies,
                        const RigidDev<TF>* __restrict__ rigid, uint32_t nb,
                        const vec4<TF>* __restrict__ xs, const uint32_t* __restrict__ perm,
                        uint32_t n, uint32_t stride, uint32_t* __restrict__ mask,
                        vec4<TF>* __restrict__ bx, vec4<TF>* __restrict__ bk,
                        TF* __restrict__ ref_b, TF* __restrict__ ref_k,
                        uint32_t* __restrict__ active) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  sample_particle(c, bodies, rigid, nb, xs, s, perm ? perm[s] : s, n, stride, mask, bx, bk,
                  ref_b, ref_k, active);
}

// Every scene of a fused batch in one launch: block -> scene, the scene's
// particle at arena slot s0 + s.
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_sample_boundaries_fused(Cn<TF> c, const vec4<TF>* __restrict__ xs, uint32_t stride,
                              const uint32_t* __restrict__ blk_scene,
                              const BoundaryScene<TF>* __restrict__ scenes, uint32_t nscenes,
                              uint32_t* __restrict__ mask, vec4<TF>* __restrict__ bx,
                              vec4<TF>* __restrict__ bk) {
  const uint32_t k = __ldg(blk_scene + blockIdx.x);
  if (k >= nscenes) return;
  const BoundaryScene<TF>& sc = scenes[k];
  const uint32_t sl = blockIdx.x * blockDim.x + threadIdx.x - sc.s0;
  if (sl >= sc.n) return;
  const uint32_t s = sc.s0 + sl;
  sample_particle(c, sc.bodies, sc.rigid, sc.nb, xs, s, sc.perm ? sc.perm[s] - sc.s0 : sl, sc.n,
                  stride, mask, bx, bk, sc.ref_b, sc.ref_k, sc.active);
}

template <class TF>
__global__ void k_node_positions(BodyDev<TF> b, TF* __restrict__ out) {
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= b.num_nodes) return;
  st3(out, l, node_position(b, l));
}

template <class TF>
__global__ void k_distance_grid(BodyDev<TF> b, TF* __restrict__ out) {
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= b.num_nodes) return;
  out[l] = shape_sdf(b, node_position(b, l));
}

// update_volume_field: one warp per node; lanes stride over the 27,000
// (theta, phi, r) samples and accumulate in double; the warp sum is the
// node's integral times h^3.
template <class TF>
__global__ void __launch_bounds__(256)
    k_volume_field(Cn<TF> c, BodyDev<TF> b, TF* __restrict__ out) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= b.num_nodes) return;
  const auto& pt = PeirceSel<TF>::get();
  const vec3<TF> x = node_position(b, warp);
  constexpr int kDirs = peirce::kNumTheta * peirce::kNumPhi;
  double sum = 0;
  for (int f = lane; f < kDirs * peirce::kNumR; f += 32) {
    const int k = f % peirce::kNumR;
    const int dir = f / peirce::kNumR;  // dir = i * kNumPhi + j
    const int j = dir % peirce::kNumPhi;
    const int i = dir / peirce::kNumPhi;
    const TF rr = c.h * pt.r[k];
    const TF ux = pt.sp[j] * pt.ct[i], uy = pt.sp[j] * pt.st[i], uz = pt.cp[j];
    const vec3<TF> p{x.x + rr * ux, x.y + rr * uy, x.z + rr * uz};
    const TF dist = b.use_grid ? interpolate_grid(b, b.dist, p) : shape_sdf(b, p);
    const TF dm = dist * b.sign;
    const TF ext = dm <= TF(0) ? TF(1) : W_dist(c, dm) / c.w0;
    sum += double(pt.w[j * peirce::kNumR + k]) * double(ext);
  }
  sum = warp_sum(sum);
  if (lane == 0) out[warp] = TF(sum * double(c.h2) * double(c.h));
}

}  // namespace

int upload_peirce_tables(cudaStream_t st) {
  static PeirceDev tf;
  static PeirceDevD td;
  const double pi = 3.14159265358979323846264338327950288;
  for (int i = 0; i < peirce::kNumTheta; ++i) {
    const double theta = 2 * pi * (i + 1) / peirce::kNumTheta;
    td.ct[i] = std::cos(theta);
    td.st[i] = std::sin(theta);
    tf.ct[i] = float(td.ct[i]);
    tf.st[i] = float(td.st[i]);
  }
  for (int j = 0; j < peirce::kNumPhi; ++j) {
    td.sp[j] = peirce::k_sinphi[j];
    td.cp[j] = peirce::k_cosphi[j];
    tf.sp[j] = float(td.sp[j]);
    tf.cp[j] = float(td.cp[j]);
  }
  for (int j = 0; j < peirce::kNumPhi; ++j)
    for (int k = 0; k < peirce::kNumR; ++k) {
      td.w[j * peirce::kNumR + k] =
          2 * pi * peirce::k_b[j] * peirce::k_c[k] / peirce::kNumTheta;
      tf.w[j * peirce::kNumR + k] = float(td.w[j * peirce::kNumR + k]);
    }
  for (int k = 0; k < peirce::kNumR; ++k) {
    td.r[k] = peirce::k_r[k];
    tf.r[k] = float(td.r[k]);
  }
  ALB_CUDA(cudaMemcpyToSymbolAsync(c_peirce_f, &tf, sizeof(tf), 0, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyToSymbolAsync(c_peirce_d, &td, sizeof(td), 0, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  return AL_OK;
}

template <class TF>
int sample_boundaries(const Cn<TF>& c, const BodyDev<TF>* bodies_dev, const RigidDev<TF>* rigid_dev,
                      uint32_t nb, const vec4<TF>* xs, const uint32_t* perm, uint32_t n,
                      const BoundaryState<TF>& bs, TF* ref_boundary, TF* ref_kernel,
                      cudaStream_t st) {
  if (n == 0) return AL_OK;
  k_sample_boundaries<TF><<<blocks_for(n, kBlock), kBlock, 0, st>>>(
      c, bodies_dev, rigid_dev, nb, xs, perm, n, bs.stride ? bs.stride : n, bs.mask, bs.bx, bs.bk,
      ref_boundary, ref_kernel, bs.active);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int sample_boundaries_fused(const Cn<TF>& c, const vec4<TF>* xs, uint32_t stride,
                            const uint32_t* blk_scene, const BoundaryScene<TF>* scenes,
                            uint32_t nscenes, uint32_t nblocks, uint32_t* mask, vec4<TF>* bx,
                            vec4<TF>* bk, cudaStream_t st) {
  if (nblocks == 0) return AL_OK;
  k_sample_boundaries_fused<TF><<<nblocks, kBlock, 0, st>>>(c, xs, stride, blk_scene, scenes,
                                                            nscenes, mask, bx, bk);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int build_volume_field(const Cn<TF>& c, const BodyDev<TF>& b, TF* out, cudaStream_t st) {
  const uint64_t threads = uint64_t(b.num_nodes) * 32;
  k_volume_field<TF><<<uint32_t((threads + 255) / 256), 256, 0, st>>>(c, b, out);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int build_distance_grid(const BodyDev<TF>& b, TF* out, cudaStream_t st) {
  k_distance_grid<TF><<<blocks_for(b.num_nodes, 256), 256, 0, st>>>(b, out);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int node_positions(const BodyDev<TF>& b, TF* out, cudaStream_t st) {
  k_node_positions<TF><<<blocks_for(b.num_nodes, 256), 256, 0, st>>>(b, out);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

#define ALB_INST(TF)                                                                          \
  template int sample_boundaries<TF>(const Cn<TF>&, const BodyDev<TF>*, const RigidDev<TF>*,  \
                                     uint32_t, const vec4<TF>*, const uint32_t*, uint32_t,     \
                                     const BoundaryState<TF>&, TF*, TF*, cudaStream_t);        \
  template int sample_boundaries_fused<TF>(const Cn<TF>&, const vec4<TF>*, uint32_t,            \
                                           const uint32_t*, const BoundaryScene<TF>*, uint32_t, \
                                           uint32_t, uint32_t*, vec4<TF>*, vec4<TF>*,           \
                                           cudaStream_t);                                       \
  template int build_volume_field<TF>(const Cn<TF>&, const BodyDev<TF>&, TF*, cudaStream_t); \
  template int build_distance_grid<TF>(const BodyDev<TF>&, TF*, cudaStream_t);               \
  template int node_positions<TF>(const BodyDev<TF>&, TF*, cudaStream_t);
ALB_INST(float)
ALB_INST(double)
#undef ALB_INST

}  // namespace alb
