// step_shared.cuh -- device pieces every solver step uses: the step's
// control-block initialisation, deterministic grid reductions, the loop
// decision of the pressure / divergence solves, Solver::update_dt and the
// rigid-body totals + Pile::integrate_kinematics.  Internal linkage: each
// translation unit that includes it compiles its own copy.
#pragma once

#include <cfloat>

#include "solver.cuh"

namespace alb {

namespace {

template <class TF>
__device__ __forceinline__ vec3<TF> body_velocity(const RigidDev<TF>& r, vec3<TF> at) {
  return cross(r.omega, at - r.x) + r.v;
}

// Deterministic double sum over `nblk` blocks (block `blk` of them): every
// block writes its block sum to red[blk]; the last block to finish (ticket)
// sums the partials in block order.  Returns true in the last block, with
// the total in thread 0.
__device__ __forceinline__ bool grid_sum_last(double value, double* red, uint32_t* ticket,
                                              double* total, uint32_t blk, uint32_t nblk) {
  __shared__ bool last;
  const double bsum = block_sum_double(value);
  if (threadIdx.x == 0) {
    red[blk] = bsum;
    __threadfence();
    last = atomicAdd(ticket, 1u) == nblk - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s = 0;
  for (uint32_t k = threadIdx.x; k < nblk; k += blockDim.x) s += __ldcg(red + k);
  s = block_sum_double(s);
  if (threadIdx.x == 0) {
    *total = s;
    *ticket = 0;
  }
  return true;
}
// The same over the whole grid.
__device__ __forceinline__ bool grid_sum_last(double value, double* red, uint32_t* ticket,
                                              double* total) {
  return grid_sum_last(value, red, ticket, total, blockIdx.x, gridDim.x);
}

// The step's control-block initialisation; thread 0 of the calling block.
template <class TF>
__device__ __forceinline__ void step_init(const StepState<TF>& S) {
  Ctrl<TF>& C = *S.ctrl;
  if (threadIdx.x == 0) {
    C.ticket = 0;
    C.vmax_bits = 0;
    C.warm_ran = 0;
    C.it = 0;
    C.keep_going = 0;
    C.mean = 0;
    al_step_report& r = C.rep;
    r.num_divergence_solve = 0;
    r.num_density_solve = 0;
    r.mean_density_change = DBL_MAX;
    r.mean_density_error = DBL_MAX;
    r.num_active_boundary_pairs = 0;
    for (int k = 0; k < AL_MAX_BOUNDARIES; ++k)
      for (int j = 0; j < 3; ++j) r.force[k][j] = r.torque[k][j] = 0;
    // Pile::calculate_cfl_v2 (pile.hpp:816-825)
    TF m = -max_value<TF>();
    for (uint32_t b = 0; b < S.nb; ++b) {
      const RigidDev<TF>& rg = S.rigid[b];
      const vec3<TF> w =
          cross(rg.omega, vec3<TF>{S.bodies[b].max_distance, TF(0), TF(0)}) + rg.v;
      m = fmax(m, length_sqr(w));
    }
    r.pile_max_v2 = double(m);
  }
}

template <class TF>
__global__ void k_step_init(StepState<TF> S) {
  step_init(S);
}

// ------------------------------------------------------------ loop control
template <class TF>
__global__ void k_loop_begin(StepState<TF> S, int density_solve,
                             cudaGraphConditionalHandle handle, int use_handle) {
  Ctrl<TF>& C = *S.ctrl;
  C.it = 0;
  C.ticket = 0;
  const uint32_t mx = density_solve ? C.max_den : C.max_div;
  C.keep_going = mx > 0;
  if (use_handle) cudaGraphSetConditional(handle, C.keep_going);
}

// Loop decision of solver_df.hpp:131-133 / 296-298 and solver_ii.hpp:181-183.
template <class TF>
__device__ __forceinline__ void finish_iteration(Ctrl<TF>& C, double total, uint32_t n,
                                                 int which, cudaGraphConditionalHandle handle,
                                                 int use_handle) {
  C.mean = total / double(n);
  C.it += 1;
  bool go;
  if (which == 0) {
    go = (C.mean > C.tol_div / double(C.dt) || C.it < C.min_div) && C.it < C.max_div;
    C.rep.num_divergence_solve = C.it;
    C.rep.mean_density_change = C.mean;
  } else {
    go = (C.mean > C.tol_den || C.it < C.min_den) && C.it < C.max_den;
    C.rep.num_density_solve = C.it;
    C.rep.mean_density_error = C.mean;
  }
  C.keep_going = go;
  if (use_handle) cudaGraphSetConditional(handle, go);
}

// Solver::update_dt (solver.hpp:153-169) given the particles' max
// |v + a dt|^2 (calculate_cfl_v2, runner.hpp:2533-2541) and the pile's in
// the report.
template <class TF>
__device__ __forceinline__ void apply_update_dt(Ctrl<TF>& C, TF pmax) {
  const TF pile = TF(C.rep.pile_max_v2);
  const TF max_v2 = fmax(pmax, pile);
  const TF max_v = sqrt(max_v2);
  const TF cfl_dt = C.cfl * C.length_scale / max_v;
  const TF ndt = fmax(fmin(cfl_dt, C.max_dt), C.min_dt);
  C.rep.particle_max_v2 = double(pmax);
  C.rep.max_v2 = double(max_v2);
  C.rep.cfl_dt = double(cfl_dt);
  C.rep.utilized_cfl = double(ndt * max_v / C.length_scale);
  C.rep.dt = double(ndt);
  C.dt = ndt;
}

// First stage of the per-body rigid totals for large grids: block (c, b)
// sums body b's slots of the c-th contiguous chunk of the [grid][nb][6]
// slots, in a fixed order, into slot c of `part` (same layout, gridDim.x
// slots).  Deterministic: the chunking depends on `grid` only.
constexpr uint32_t kRigidChunks = 128;

// Chunk c of body b (one block).
__device__ __forceinline__ void rigid_partial(const double* __restrict__ ft, uint32_t grid,
                                              uint32_t nb, double* __restrict__ part, uint32_t b,
                                              uint32_t c) {
  const uint32_t len = (grid + kRigidChunks - 1) / kRigidChunks;
  const uint32_t lo = c * len, hi = min(lo + len, grid);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t g = lo + threadIdx.x; g < hi; g += blockDim.x) {
    const double* slot = ft + (size_t(g) * nb + b) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] += slot[k];
  }
  double tot[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) tot[k] = block_sum_double(acc[k]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) part[(size_t(c) * nb + b) * 6 + k] = tot[k];
  }
}

__global__ void k_rigid_partial(const double* __restrict__ ft, uint32_t grid, uint32_t nb,
                                double* __restrict__ part) {
  rigid_partial(ft, grid, nb, part, blockIdx.y, blockIdx.x);
}

// Per-body totals of the rigid slots (solver_df.hpp:346-353) in double and
// Pile::integrate_kinematics (pile.hpp:794-815) of body b (one block), over
// `nslots` slots of `slots` ([nslots][nb][6]).
template <class TF>
__device__ __forceinline__ void rigid_finish(const StepState<TF>& S,
                                             const double* __restrict__ slots, uint32_t nslots,
                                             uint32_t b) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t g = threadIdx.x; g < nslots; g += blockDim.x) {
    const double* slot = slots + (size_t(g) * S.nb + b) * 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] += slot[k];
  }
  double tot[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) tot[k] = block_sum_double(acc[k]);
  if (threadIdx.x != 0) return;
  Ctrl<TF>& C = *S.ctrl;
  for (int k = 0; k < 3; ++k) {
    C.rep.force[b][k] = tot[k];
    C.rep.torque[b][k] = tot[3 + k];
  }
  if (!C.integrate_rigids) return;
  const TF dt = C.dt;
  const BodyDev<TF>& body = S.bodies[b];
  RigidDev<TF> r = S.rigid[b];
  auto advance_q = [&]() {
    const vec3<TF> w = r.omega;
    const vec4<TF> q = r.q;
    const vec4<TF> dq{TF(0.5) * (w.x * q.w + w.y * q.z - w.z * q.y),
                      TF(0.5) * (-w.x * q.z + w.y * q.w + w.z * q.x),
                      TF(0.5) * (w.x * q.y - w.y * q.x + w.z * q.w),
                      TF(0.5) * (-w.x * q.x - w.y * q.y - w.z * q.z)};
    vec4<TF> nq{q.x + dt * dq.x, q.y + dt * dq.y, q.z + dt * dq.z, q.w + dt * dq.w};
    const TF inv = rsqrt_(nq.x * nq.x + nq.y * nq.y + nq.z * nq.z + nq.w * nq.w);
    r.q = vec4<TF>{nq.x * inv, nq.y * inv, nq.z * inv, nq.w * inv};
  };
  if (body.mass == TF(0)) {
    r.x += r.v * dt;
    advance_q();
  } else {
    const vec3<TF> force{TF(tot[0]), TF(tot[1]), TF(tot[2])};
    const vec3<TF> torque{TF(tot[3]), TF(tot[4]), TF(tot[5])};
    r.v += (TF(1) / body.mass) * force * dt;
    // calculate_angular_acceleration (runner.hpp:202-239)
    const vec4<TF> q = r.q;
    const vec3<TF> ii{TF(1) / body.inertia.x, TF(1) / body.inertia.y, TF(1) / body.inertia.z};
    const TF m[3][3] = {{TF(1) - TF(2) * (q.y * q.y + q.z * q.z), TF(2) * (q.x * q.y - q.z * q.w),
                         TF(2) * (q.x * q.z + q.y * q.w)},
                        {TF(2) * (q.x * q.y + q.z * q.w), TF(1) - TF(2) * (q.x * q.x + q.z * q.z),
                         TF(2) * (q.y * q.z - q.x * q.w)},
                        {TF(2) * (q.x * q.z - q.y * q.w), TF(2) * (q.y * q.z + q.x * q.w),
                         TF(1) - TF(2) * (q.x * q.x + q.y * q.y)}};
    const TF tqa[3] = {torque.x, torque.y, torque.z};
    TF alpha[3];
    for (int row = 0; row < 3; ++row) {
      TF sacc = 0;
      for (int k = 0; k < 3; ++k) {
        const TF cong = ii.x * m[row][0] * m[k][0] + ii.y * m[row][1] * m[k][1] +
                        ii.z * m[row][2] * m[k][2];
        sacc += tqa[k] * cong;
      }
      alpha[row] = sacc;
    }
    r.omega += vec3<TF>{alpha[0], alpha[1], alpha[2]} * dt;
    advance_q();
    const vec3<TF> g{C.pile_gravity[0], C.pile_gravity[1], C.pile_gravity[2]};
    const vec3<TF> dx = (g * dt + r.v) * dt;
    r.x += dx;
    r.v = (TF(1) / dt) * dx;
  }
  S.rigid[b] = r;
}

// One block per body.
template <class TF>
__global__ void k_rigid_finish(StepState<TF> S, const double* __restrict__ slots,
                               uint32_t nslots) {
  rigid_finish(S, slots, nslots, blockIdx.x);
}

// Host read of the loop flag of an eagerly launched solve.
template <class TF>
int read_keep_going(const StepState<TF>& S, uint32_t* pinned, cudaStream_t st, bool* go) {
  ALB_CUDA(cudaMemcpyAsync(pinned, &S.ctrl->keep_going, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                           st));
  ALB_CUDA(cudaStreamSynchronize(st));
  *go = *pinned != 0;
  return AL_OK;
}

}  // namespace

}  // namespace alb
