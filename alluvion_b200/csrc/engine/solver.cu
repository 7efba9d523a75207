// solver.cu -- DFSPH, IISPH and implicit SPH step kernels and their orchestration.
#include <cfloat>
#include <cstring>
#include <vector>

#include "build_kernel.cuh"
#include "neighbors.cuh"
#include "solver.cuh"
#include "step_shared.cuh"
#include "warmnet.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

template <class TF>
__device__ __forceinline__ vec3<TF> ldx(const vec4<TF>* p, uint32_t i) {
  return xyz(__ldg(p + i));
}

// Record halves of particle s (see StepState::rec).
template <class TF>
__device__ __forceinline__ vec4<TF>& RX(const StepState<TF>& S, uint32_t s) {
  return S.rec[2 * size_t(s)];
}
template <class TF>
__device__ __forceinline__ vec4<TF>& RV(const StepState<TF>& S, uint32_t s) {
  return S.rec[2 * size_t(s) + 1];
}
// Neighbor loads of the two halves through the read-only path.
template <class TF>
__device__ __forceinline__ vec4<TF> gX(const StepState<TF>& S, uint32_t t) {
  return __ldg(S.rec + 2 * size_t(t));
}
template <class TF>
__device__ __forceinline__ vec4<TF> gV(const StepState<TF>& S, uint32_t t) {
  return __ldg(S.rec + 2 * size_t(t) + 1);
}

// Both halves of record t through the read-only path with 256-bit loads
// (sm_100): one load instruction per float record, two per double record,
// instead of one per 16 bytes.  Records start on 32-byte (float) and
// 64-byte (double) boundaries: the buffer is cudaMalloc-aligned and a
// record is 2 x vec4.
__device__ __forceinline__ void gXV(const StepState<float>& S, uint32_t t, vec4<float>& x,
                                    vec4<float>& v) {
  const vec4<float>* p = S.rec + 2 * size_t(t);
  asm volatile("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(v.x), "=f"(v.y), "=f"(v.z),
                 "=f"(v.w)
               : "l"(p));
}
__device__ __forceinline__ void gXV(const StepState<double>& S, uint32_t t, vec4<double>& x,
                                    vec4<double>& v) {
  const vec4<double>* p = S.rec + 2 * size_t(t);
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(x.x), "=d"(x.y), "=d"(x.z), "=d"(x.w)
               : "l"(p));
  asm volatile("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
               : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(v.w)
               : "l"(p + 1));
}

// Adds the block's contributions (f, t) for body b to the block's rigid
// force/torque slot: warp trees, then warp partials in warp order.  All
// threads of the block call it.  Deterministic.
template <class TF>
__device__ __forceinline__ void block_add_ft(const StepState<TF>& S, uint32_t bid, uint32_t b,
                                             vec3<TF> f, vec3<TF> t) {
  __shared__ double part[6][kMaxBlock / 32];
  double v[6] = {double(f.x), double(f.y), double(f.z), double(t.x), double(t.y), double(t.z)};
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) part[k][warp] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) s += part[threadIdx.x][w];
    S.ft[(size_t(bid) * S.nb + b) * 6 + threadIdx.x] += s;
  }
  __syncthreads();
}
template <class TF>
__device__ __forceinline__ void block_add_ft(const StepState<TF>& S, uint32_t b, vec3<TF> f,
                                             vec3<TF> t) {
  block_add_ft(S, blockIdx.x, b, f, t);
}

// Pair passes run `tpp` threads per particle (1, 2, 4 or 8, chosen per
// step from the particle count): lane `sub` of a particle's group walks
// neighbors sub, sub + tpp, ...; the group combines its partial sums with
// warp shuffles (fixed order, deterministic) and lane 0 applies the boundary
// terms and writes the results.  With batched gathers (for_each_neighbor)
// and 128-thread blocks one thread per particle keeps enough gathers in
// flight once the particles alone fill the GPU (measured on the 1 M-particle
// dam break: 1.93 ms per step at 1 thread, 1.98 at 2, 2.33 at 4); smaller
// scenes split each particle's neighbors over more lanes until about
// kPairThreads threads run (the 32,768-particle dam break: 0.29 / 0.255 /
// 0.268 ms per step at 8 / 4 / 2 threads per particle).
constexpr uint64_t kPairThreads = uint64_t(1) << 17;

inline uint32_t pair_tpp(uint32_t n) {
  uint32_t tpp = 1;
  while (tpp < 8 && uint64_t(n) * tpp < kPairThreads) tpp <<= 1;
  return tpp;
}

// Threads per block and per particle of one pass launch.
struct LaunchShape {
  uint32_t block, tpp;
};

// The pass groups whose launch shape the table sets: `pair` groups walk
// neighbor lists and take threads per particle too.
struct TunableGroup {
  const char* name;
  bool pair;
};
constexpr TunableGroup kTunable[] = {
    {"neighbors", false},    {"div_warm1", true},     {"div_rho_adv", true},
    {"div_iter", true},      {"div_residual", true},  {"viscosity", true},
    {"press_warm0", true},   {"press_warm1", true},   {"press_rho_adv", true},
    {"press_iter", true},    {"press_residual", true}, {"ii_predict0", true},
    {"ii_predict1", true},   {"ii_iter0", true},      {"ii_iter1", true},
    {"i_diag", true},        {"i_iter", true},        {"finish", true}};
constexpr uint32_t kNumTunable = sizeof(kTunable) / sizeof(kTunable[0]);

struct Lane {
  uint32_t s, sub, tpp;
  bool act;
  __device__ __forceinline__ bool lead() const { return act && sub == 0; }
};

// A pass block's place in its scene: the scene, the block's index among
// the scene's blocks, their count, the end of the scene's particle range and
// its particle count.  A one-scene launch is all one scene.
struct BlockSpan {
  uint32_t k, bid, nblk, end, n;
};

// With BT (a pass launched over every scene of a fused batch) narrows S to
// the block's scene: its control block and reduction partials.  False for
// a block past every scene.
template <bool BT, class TF>
__device__ __forceinline__ bool block_scene(StepState<TF>& S, BlockSpan& B) {
  if constexpr (BT) {
    const uint32_t k = __ldg(S.blk_scene + blockIdx.x);
    if (k >= S.nscenes) return false;
    const FusedScene<TF>& f = S.fused[k];
    S.ctrl = f.ctrl;
    S.red = f.red;
    B = BlockSpan{k, blockIdx.x - f.blk0, f.nblk, f.s0 + f.n, f.n};
  } else {
    B = BlockSpan{0, blockIdx.x, gridDim.x, S.n, S.n};
  }
  return true;
}

// The rest of the narrowing of block_scene: the scene's bodies, rigid state
// and rigid slots (loaded where a pass reaches its boundary terms).
template <bool BT, class TF>
__device__ __forceinline__ void scene_bodies(StepState<TF>& S, const BlockSpan& B) {
  if constexpr (BT) {
    const FusedScene<TF>& f = S.fused[B.k];
    S.bodies = f.bodies;
    S.rigid = f.rigid;
    S.ft = f.ft;
    S.nb = f.nb;
  }
}

template <class TF>
__device__ __forceinline__ Lane pair_lane(const StepState<TF>& S, const BlockSpan& B) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t shift = __ffs(S.tpp) - 1;
  Lane l;
  l.tpp = S.tpp;
  l.s = g >> shift;
  l.sub = g & (S.tpp - 1);
  l.act = l.s < B.end;
  return l;
}
template <class TF>
__device__ __forceinline__ Lane pair_lane(const StepState<TF>& S) {
  return pair_lane(S, BlockSpan{0, blockIdx.x, gridDim.x, S.n, S.n});
}

inline uint32_t pair_blocks(uint32_t n, uint32_t tpp, uint32_t block = kBlock) {
  return uint32_t((uint64_t(n) * tpp + block - 1) / block);
}

// Sum over the particle's lane group (every lane of the warp calls it; the
// group's lanes are consecutive and tpp divides 32).
template <class T>
__device__ __forceinline__ T group_sum(T v, const Lane& L) {
  for (uint32_t o = L.tpp >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <class TF>
__device__ __forceinline__ vec3<TF> group_sum(vec3<TF> v, const Lane& L) {
  return vec3<TF>{group_sum(v.x, L), group_sum(v.y, L), group_sum(v.z, L)};
}

template <class TF>
__device__ __forceinline__ uint32_t nbr_at(const StepState<TF>& S, uint32_t k, uint32_t s) {
  return __ldcs(S.nbr + size_t(k) * S.ls + s);
}

// Visits the lane's neighbors k = sub, sub + tpp, ... < cnt in batches of
// B: the batch's list entries are loaded first, then all their records,
// then `f(t, x_j, v_j)` runs for each in list order.  At one thread per
// particle that is the order of a plain loop over the list, so sums are
// bit-identical to one; with tpp > 1 each lane sums every tpp-th neighbor
// and group_sum combines the partial sums, a different (fixed) order whose
// float results differ in the last bits.  Batching keeps B dependent
// index -> record chains in flight per lane; it pays in the passes with
// much arithmetic per neighbor (measured on the 1M-particle dam break at
// one thread per particle: B = 8 for k_kappa (1.922 vs 1.928 ms per step at
// 4, 1.946 at 2), 4 for viscosity, 2 for the velocity-divergence passes,
// which have little arithmetic per neighbor).  `v_j` is loaded only when
// V.
template <int B, bool V, class TF, class F>
__device__ __forceinline__ void for_each_neighbor(const StepState<TF>& S, const Lane& L,
                                                  uint32_t cnt, F&& f) {
  for (uint32_t k0 = L.sub; k0 < cnt; k0 += B * L.tpp) {
    uint32_t t[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      const uint32_t k = k0 + b * L.tpp;
      t[b] = k < cnt ? nbr_at(S, k, L.s) : L.s;  // own slot: a valid address
    }
    vec4<TF> xj[B], vj[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
      if (V) {
        gXV(S, t[b], xj[b], vj[b]);
      } else {
        xj[b] = gX(S, t[b]);
        vj[b] = vec4<TF>{0, 0, 0, 0};
      }
    }
#pragma unroll
    for (int b = 0; b < B; ++b)
      if (k0 + b * L.tpp < cnt) f(t[b], xj[b], vj[b]);
  }
}

// Sum over neighbors of V (v_i - v_j) . grad W_ij plus the boundary terms
// (v_i - v_b) . (grad W V)_b: the shared body of compute_density_change
// (runner.hpp:3192-3228) and compute_density_adv (runner.hpp:3493-3523).
// Every lane of the group calls it and receives the full sum.
template <class TF>
__device__ __forceinline__ TF velocity_divergence(const Cn<TF>& c, const StepState<TF>& S,
                                                  const Lane& L, vec3<TF> xi, vec3<TF> vi,
                                                  uint32_t cnt) {
  TF acc = 0;
  for_each_neighbor<2, true>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const vec3<TF> d = pdisp(c, xi, xyz(xj));
    acc += c.vol * dot(vi - xyz(vj), gradW(c, d));
  });
  acc = group_sum(acc, L);
  if (L.act) {
    for (uint32_t m = S.mask[L.s]; m; m &= m - 1) {
      const uint32_t b = __ffs(m) - 1;
      const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
      const vec4<TF> kg = S.bk[size_t(b) * S.ls + L.s];
      const vec3<TF> vj = body_velocity(S.rigid[b], xyz(bn));
      acc += dot(vi - vj, xyz(kg));
    }
  }
  return acc;
}

template <class TF>
__device__ __forceinline__ TF density_change(const Cn<TF>& c, const StepState<TF>& S,
                                             const Lane& L) {
  const uint32_t cnt = L.act ? S.ncount[L.s] : 0u;
  const vec3<TF> xi = L.act ? xyz(RX(S, L.s)) : vec3<TF>{0, 0, 0};
  const vec3<TF> vi = L.act ? xyz(RV(S, L.s)) : vec3<TF>{0, 0, 0};
  TF adv = velocity_divergence(c, S, L, xi, vi, cnt);
  adv = fmax(adv, TF(0));
  if (cnt < 20) adv = 0;
  return adv;
}

template <class TF>
__device__ __forceinline__ TF density_adv(const Cn<TF>& c, const StepState<TF>& S, const Lane& L,
                                          TF dt) {
  const uint32_t cnt = L.act ? S.ncount[L.s] : 0u;
  const vec3<TF> xi = L.act ? xyz(RX(S, L.s)) : vec3<TF>{0, 0, 0};
  const vec3<TF> vi = L.act ? xyz(RV(S, L.s)) : vec3<TF>{0, 0, 0};
  const TF delta = velocity_divergence(c, S, L, xi, vi, cnt);
  const TF rho = L.act ? S.rho[L.s] : c.rho0;
  return fmax(rho / c.rho0 + dt * delta, TF(1));
}

// ------------------------------------------------------------- kernels
// With BT every scene of a fused batch in one launch: the block's scene's
// buffers (S.io; S.perm holds arena slots s0 + i), the sorted positions
// gathered here too.
template <class TF, bool DF, bool BT = false>
__global__ void k_gather_state(StepState<TF> S, const TF* __restrict__ v_ref,
                               const TF* __restrict__ k_ref, const TF* __restrict__ kv_ref) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  BlockSpan B;
  if (!block_scene<BT>(S, B) || s >= B.end) return;
  uint32_t i;
  if constexpr (BT) {
    const FusedIo<TF>& io = S.io[B.k];
    i = S.perm[s] - (B.end - B.n);
    v_ref = io.v_in;
    k_ref = io.kappa_in;
    kv_ref = io.kappa_v_in;
    const vec3<TF> p = ld3(io.x_in, i);
    S.x[s] = vec4<TF>{p.x, p.y, p.z, TF(0)};
  } else {
    i = S.perm[s];
  }
  const vec3<TF> v = ld3(v_ref, i);
  RX(S, s) = vec4<TF>{S.x[s].x, S.x[s].y, S.x[s].z, TF(0)};
  RV(S, s) = vec4<TF>{v.x, v.y, v.z, TF(0)};  // rho follows from the build
  S.kappa[s] = k_ref ? k_ref[i] : TF(0);
  if (DF) S.kappa_v[s] = kv_ref ? kv_ref[i] : TF(0);
}

// warm_start_divergence_solve_0 (runner.hpp:3230-3249), fused into the
// neighbor build: the build's phase 2 sums the velocity divergence
// sum_j V (v_i - v_j) . grad W_ij over the list; finish() adds the boundary
// terms (compute_density_change, runner.hpp:3192-3228) and applies the
// warm start.  The result also becomes the payload read by k_kappa.
//
// With `feat` / `feat_out` set it also writes the learned warm start's 12
// features (the list and units are those of al_warm_net in the C header) in
// sorted / original particle order.
template <class TF>
struct WarmDivergence {
  static constexpr bool kOn = true;
  StepState<TF> S;
  float* feat = nullptr;      // [n][12] sorted order
  float* feat_out = nullptr;  // [n][12] original order
  TF two_r = 0, vol = 0;
  // learned warm start gate (warm_gate_update): nonzero when this step skips
  // the network
  const uint32_t* floor = nullptr;
  // a build over every scene of a fused batch: scene k's dt and rigid state
  __device__ __forceinline__ void narrow(uint32_t k) {
    S.ctrl = S.fused[k].ctrl;
    S.rigid = S.fused[k].rigid;
  }
  __device__ __forceinline__ vec3<TF> self_v(uint32_t s) const { return xyz(RV(S, s)); }
  // neighbor t's position and velocity in one load of its 32-byte record
  // (the record's position is the sorted position the scan used)
  __device__ __forceinline__ void xv(const vec4<TF>*, uint32_t t, vec3<TF>& x, vec3<TF>& v) const {
    vec4<TF> x4, v4;
    gXV(S, t, x4, v4);
    x = xyz(x4);
    v = xyz(v4);
  }
  __device__ __forceinline__ void finish(uint32_t s, const BuildOut<TF>& o) const {
    TF acc = o.div, bvol = 0, bden = 0;
    for (uint32_t m = S.mask[s]; m; m &= m - 1) {
      const uint32_t b = __ffs(m) - 1;
      const vec4<TF> bn = S.bx[size_t(b) * S.ls + s];
      const vec4<TF> kg = S.bk[size_t(b) * S.ls + s];
      acc += dot(o.vi - body_velocity(S.rigid[b], xyz(bn)), xyz(kg));
      bvol += bn.w;
      bden += kg.w;
    }
    TF adv = fmax(acc, TF(0));
    if (o.cnt < 20) adv = 0;
    const TF dt = S.ctrl->dt;
    const TF kv = S.kappa_v[s];
    const TF w = adv > TF(0) ? TF(0.5) * fmax(kv, TF(-0.5)) / dt : TF(0);
    S.kappa_v[s] = w;
    RX(S, s).w = w;
    const bool learned = feat && !(floor && *floor);
    if (learned || feat_out) {
      const TF speed = sqrt(length_sqr(o.vi));
      const float f[AL_WARM_NUM_FEATURES] = {
          float(o.density - TF(1)), float(adv * dt), float(TF(o.cnt) / TF(32)),
          float(kv / dt), float(S.kappa[s] / (dt * dt)), float(bvol / vol),
          float(speed), float(speed * dt / two_r), float(o.alpha), float(bden),
          float(sqrt(o.grad_norm2) * two_r), float(dt)};
      if (learned) {
#pragma unroll
        for (int k = 0; k < AL_WARM_NUM_FEATURES; ++k)
          feat[size_t(s) * AL_WARM_NUM_FEATURES + k] = f[k];
      }
      if (feat_out) {
        const uint32_t i = S.perm[s];
#pragma unroll
        for (int k = 0; k < AL_WARM_NUM_FEATURES; ++k)
          feat_out[size_t(i) * AL_WARM_NUM_FEATURES + k] = f[k];
      }
    }
  }
};

// The learned warm start's per-scene gate, kept in four device words:
//   [0] 1 when the next step skips the network (plain warm starts)
//   [1] steps since the network last ran
//   [2] solver iterations (divergence + density) of the last step that ran it
//   [3] solver iterations of the last step that did not
// A fresh scene starts at zero (the first step runs the network).  After
// each step (k_df_finish): the network runs next only if this step's solves
// went beyond their minimum iteration counts (at the minimum no warm start
// can save an iteration) and its last outcome was no worse than the plain
// start's last outcome, or it has not run for 64 steps (a new try).  So a
// network that predicts poorly for a scene costs at most one step in 64.
template <class TF>
__device__ __forceinline__ void warm_gate_update(const Ctrl<TF>& C, uint32_t* w) {
  const bool used = w[0] == 0u;
  const uint32_t tot = C.rep.num_divergence_solve + C.rep.num_density_solve;
  if (used)
    w[2] = tot;
  else
    w[3] = tot;
  w[1] = used ? 0u : w[1] + 1u;
  const bool at_floor =
      C.rep.num_divergence_solve <= C.min_div && C.rep.num_density_solve <= C.min_den;
  const bool net_ok = w[2] <= w[3] || w[1] >= 64u;
  w[0] = (!at_floor && net_ok) ? 0u : 1u;
}

// Learned divergence warm start: kappa_v = predicted kappa_v where the
// reference's gate holds (rho_dot > 0, i.e. feature 1 > 0), else 0.  When
// the floor gate is set the build's plain warm start stays.
template <class TF>
__global__ void k_apply_warm_div(StepState<TF> S, const float* __restrict__ feat,
                                 const float* __restrict__ pred,
                                 const uint32_t* __restrict__ floor) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n || *floor) return;
  const TF w = feat[size_t(s) * AL_WARM_NUM_FEATURES + 1] > 0.f ? TF(pred[2 * size_t(s)]) : TF(0);
  S.kappa_v[s] = w;
  RX(S, s).w = w;
}

enum KappaMode { kDivWarm = 0, kDivIter = 1, kPressWarm = 2, kPressIter = 3 };

// The kappa-driven velocity updates: warm_start_divergence_solve_1
// (runner.hpp:3251-3295), divergence_solve_iteration (:3316-3363),
// warm_start_pressure_solve1 (:3451-3491), pressure_solve_iteration
// (:3543-3588).  Boundary reaction forces go to the per-block rigid slots.
// The float kernel is held at 56 registers (9 resident 128-thread blocks
// per SM; with 256-thread launch bounds the compiler took 58, and the
// 256-register allocation granule then allows only 8); double needs more.
template <class TF, int MODE, bool WR = false, bool BT = false>
__global__ void __maxnreg__(sizeof(TF) == 4 ? 56 : 128) k_kappa(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  constexpr bool kDiv = MODE == kDivWarm || MODE == kDivIter;
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  // a scene of a fused batch whose solve has converged sits out the
  // remaining iterations of the others
  if (BT && (MODE == kDivIter || MODE == kPressIter) && !S.ctrl->keep_going) return;
  const Lane L = pair_lane(S, B);
  const TF dt = S.ctrl->dt;
  TF ki = 0;
  vec3<TF> dv{0, 0, 0};
  uint32_t cnt = 0;
  vec3<TF> xi{0, 0, 0};
  if (L.act) {
    const vec4<TF> r = RX(S, L.s);
    ki = r.w;
    xi = xyz(r);
    cnt = S.ncount[L.s];
  }
  for_each_neighbor<8, false>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>&) {
    const TF ksum = ki + xj.w;
    if (fabs(ksum) > c.eps) {
      const vec3<TF> gw = gradW(c, pdisp(c, xi, xyz(xj)));
      if (kDiv) {
        const vec3<TF> gpj = (-c.vol) * gw;
        dv -= (dt * ksum) * gpj;
      } else {
        dv += (dt * ksum * c.vol) * gw;
      }
    }
  });
  dv = group_sum(dv, L);
  scene_bodies<BT>(S, B);
  const uint32_t m = (L.lead() && fabs(ki) > c.eps) ? S.mask[L.s] : 0u;
  for (uint32_t b = 0; b < S.nb; ++b) {
    const bool mine = (m >> b) & 1u;
    if (!__syncthreads_or(mine)) continue;
    vec3<TF> f{0, 0, 0}, tq{0, 0, 0};
    if (mine) {
      const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
      const vec4<TF> kg = S.bk[size_t(b) * S.ls + L.s];
      const vec3<TF> a = ki * (-xyz(kg));
      f = c.mass * a;
      dv -= dt * a;
      tq = cross(xyz(bn) - S.rigid[b].x, f);
    }
    block_add_ft(S, B.bid, b, f, tq);
  }
  if (L.lead()) {
    if (MODE == kDivIter) S.kappa_v[L.s] += ki;
    if (MODE == kPressIter) S.kappa[L.s] += ki;
    const vec4<TF> v = RV(S, L.s);
    RV(S, L.s) = vec4<TF>{v.x + dv.x, v.y + dv.y, v.z + dv.z, v.w};
  }
}

// compute_velocity_of_density_change (runner.hpp:3297-3314); also forms
// k = rho_adv * alpha for the first divergence iteration.
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock) k_df_rho_adv_init(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  scene_bodies<BT>(S, B);
  const Lane L = pair_lane(S, B);
  const TF adv = density_change(c, S, L);
  if (!L.lead()) return;
  const TF dt = S.ctrl->dt;
  const TF alpha = S.alpha[L.s] * (TF(1) / dt);
  S.rho_adv[L.s] = adv;
  S.alpha[L.s] = alpha;
  RX(S, L.s).w = adv * alpha;
}

// compute_divergence_solve_density_error (runner.hpp:3396-3410) with the
// mean of solver_df.hpp:160-161 reduced in double on the device.
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_df_residual(Cn<TF> c, StepState<TF> S, cudaGraphConditionalHandle handle, int use_handle) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  if (BT && !S.ctrl->keep_going) return;
  scene_bodies<BT>(S, B);
  const Lane L = pair_lane(S, B);
  const TF adv = density_change(c, S, L);
  double val = 0;
  if (L.lead()) {
    S.rho_adv[L.s] = adv;
    RX(S, L.s).w = adv * S.alpha[L.s];
    val = double(adv);
  }
  double total;
  if (grid_sum_last(val, S.red, &S.ctrl->ticket, &total, B.bid, B.nblk) && threadIdx.x == 0)
    finish_iteration(*S.ctrl, total, B.n, 0, handle, use_handle);
}

// clear_acceleration + compute_viscosity (runner.hpp:1974-1980, 2150-2249),
// divergence_solve_finish (runner.hpp:3412-3420) when `finish_div`, and
// calculate_cfl_v2 (runner.hpp:2533-2541) reduced to the global max; the
// last block applies Solver::update_dt (solver.hpp:153-169).
//
// The float kernel is held at 64 registers (8 resident 128-thread blocks per
// SM): a fused batch's scene lookups would otherwise take it to 76.
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock, sizeof(TF) == 4 ? 4 : 1)
    k_viscosity(Cn<TF> c, StepState<TF> S, int finish_div) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  const Lane L = pair_lane(S, B);
  const TF dt = S.ctrl->dt;
  vec3<TF> xi{0, 0, 0}, vi{0, 0, 0}, da{0, 0, 0};
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    vi = xyz(RV(S, L.s));
    cnt = S.ncount[L.s];
  }
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const vec3<TF> d = pdisp(c, xi, xyz(xj));  // vj = {v, rho}
    da += (c.visc * c.mass / vj.w * dot(d, gradW(c, d)) /
           (length_sqr(d) + TF(0.01) * c.h2)) *
          (vi - xyz(vj));
  });
  da = group_sum(da, L);
  scene_bodies<BT>(S, B);
  const uint32_t m = L.lead() ? S.mask[L.s] : 0u;
  for (uint32_t b = 0; b < S.nb; ++b) {
    const bool mine = (m >> b) & 1u;
    if (!__syncthreads_or(mine)) continue;
    vec3<TF> fsum{0, 0, 0}, tsum{0, 0, 0};
    if (mine) {
      const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
      const vec3<TF> bxj = xyz(bn);
      const RigidDev<TF> rg = S.rigid[b];
      vec3<TF> nrm = bxj - xi;
      const TF nl2 = length_sqr(nrm);
      if (nl2 > TF(0)) {
        nrm = rsqrt_(nl2) * nrm;
        // get_orthogonal_vectors (runner.hpp:119-131)
        vec3<TF> ref{TF(1), TF(0), TF(0)};
        if (fabs(dot(ref, nrm)) > TF(0.999)) ref = vec3<TF>{TF(0), TF(1), TF(0)};
        vec3<TF> t1 = cross(nrm, ref);
        vec3<TF> t2 = cross(nrm, t1);
        t1 = rsqrt_(dot(t1, t1)) * t1;
        t2 = rsqrt_(dot(t2, t2)) * t2;
        const TF dist = c.h - sqrt(nl2);
        const vec3<TF> pts[4] = {bxj - t1 * dist, bxj + t1 * dist, bxj - t2 * dist,
                                 bxj + t2 * dist};
        const TF vol = TF(0.25) * bn.w;
        vec3<TF> acc[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const vec3<TF> xix = xi - pts[q];
          const vec3<TF> vb = body_velocity(rg, pts[q]);
          acc[q] = (c.bvisc * vol * dot(xix, gradW(c, xix)) /
                    (length_sqr(xix) + TF(0.01) * c.h2)) *
                   (vi - vb);
        }
        da += acc[0] + acc[1] + acc[2] + acc[3];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const vec3<TF> fq = (-c.mass) * acc[q];
          fsum += fq;
          tsum += cross(pts[q] - rg.x, fq);
        }
      }
    }
    block_add_ft(S, B.bid, b, fsum, tsum);
  }
  TF v2 = 0;
  if (L.lead()) {
    const vec3<TF> a = c.g + da;
    S.a[L.s] = vec4<TF>{a.x, a.y, a.z, TF(0)};
    if (finish_div) {
      S.alpha[L.s] *= dt;
      S.kappa_v[L.s] *= dt;
    }
    v2 = length_sqr(vi + a * dt);
  }
  // block max, then one ordered-bits atomicMax per block
  __shared__ TF wmax[kMaxBlock / 32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x == 0) {
    TF bm = wmax[0];
    for (int w = 1; w < int(blockDim.x >> 5); ++w) bm = fmax(bm, wmax[w]);
    unsigned long long bits;
    if constexpr (sizeof(TF) == 4)
      bits = __float_as_uint(bm);
    else
      bits = (unsigned long long)__double_as_longlong(bm);
    atomicMax(&S.ctrl->vmax_bits, bits);
    __threadfence();
    last = atomicAdd(&S.ctrl->ticket, 1u) == B.nblk - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    Ctrl<TF>& C = *S.ctrl;
    __threadfence();
    const unsigned long long bits = atomicAdd(&C.vmax_bits, 0ull);
    TF pmax;
    if constexpr (sizeof(TF) == 4)
      pmax = __uint_as_float(uint32_t(bits));
    else
      pmax = __longlong_as_double((long long)bits);
    apply_update_dt(C, pmax);
    C.ticket = 0;
  }
}

// integrate_non_pressure_acceleration (runner.hpp:3422-3428).
template <class TF, bool BT = false>
__global__ void k_integrate_np(StepState<TF> S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  BlockSpan B;
  if (!block_scene<BT>(S, B) || s >= B.end) return;
  const TF dt = S.ctrl->dt;
  const vec4<TF> a = S.a[s];
  const vec4<TF> v = RV(S, s);
  RV(S, s) = vec4<TF>{v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z, v.w};
}

// warm_start_pressure_solve0 (runner.hpp:3430-3449).
// With `pred` (learned warm start) the predicted kappa replaces the
// previous-step value under the same gate (rho_adv > 1), unless the floor
// gate is set.
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_p_warm0(Cn<TF> c, StepState<TF> S, const float* __restrict__ pred,
              const uint32_t* __restrict__ floor) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  scene_bodies<BT>(S, B);
  const Lane L = pair_lane(S, B);
  const TF dt = S.ctrl->dt;
  const TF adv = density_adv(c, S, L, dt);
  if (!L.lead()) return;
  const TF kp = S.kappa[L.s];
  const bool learned = pred && !(floor && *floor);
  const TF warm = learned ? TF(pred[2 * size_t(L.s) + 1])
                       : TF(0.5) * fmax(kp, TF(-0.00025)) / (dt * dt);
  const TF w = adv > TF(1) ? warm : TF(0);
  S.kappa[L.s] = w;
  RX(S, L.s).w = w;
}

// compute_rho_adv (runner.hpp:3525-3541); also k for the first iteration.
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock) k_p_rho_adv_init(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  scene_bodies<BT>(S, B);
  const Lane L = pair_lane(S, B);
  const TF dt = S.ctrl->dt;
  const TF adv = density_adv(c, S, L, dt);
  if (!L.lead()) return;
  const TF alpha = S.alpha[L.s] * (TF(1) / (dt * dt));
  S.rho_adv[L.s] = adv;
  S.alpha[L.s] = alpha;
  RX(S, L.s).w = (adv - TF(1)) * alpha;
}

// compute_pressure_solve_density_error (runner.hpp:3590-3604); the mean is
// sum(rho_adv - 1) / N in double (solver_df.hpp:323-325 forms sum/N - 1).
template <class TF, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_p_residual(Cn<TF> c, StepState<TF> S, cudaGraphConditionalHandle handle, int use_handle) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  BlockSpan B;
  if (!block_scene<BT>(S, B)) return;
  if (BT && !S.ctrl->keep_going) return;
  scene_bodies<BT>(S, B);
  const Lane L = pair_lane(S, B);
  const TF adv = density_adv(c, S, L, S.ctrl->dt);
  double val = 0;
  if (L.lead()) {
    S.rho_adv[L.s] = adv;
    RX(S, L.s).w = (adv - TF(1)) * S.alpha[L.s];
    val = double(adv) - 1.0;
  }
  double total;
  if (grid_sum_last(val, S.red, &S.ctrl->ticket, &total, B.bid, B.nblk) && threadIdx.x == 0)
    finish_iteration(*S.ctrl, total, B.n, 1, handle, use_handle);
}

// pressure_solve_finish + integrate_velocity<0> (runner.hpp:3606-3623),
// written straight back to the caller's buffers in original order.
// With BT every scene of a fused batch in one launch, into each scene's own
// buffers (S.io; S.perm holds arena slots s0 + i).
template <class TF, bool WR = false, bool BT = false>
__global__ void k_df_finish(Cn<TF> c, StepState<TF> S, int density_solve, TF* __restrict__ x_ref,
                            TF* __restrict__ v_ref, TF* __restrict__ a_ref,
                            TF* __restrict__ rho_ref, TF* __restrict__ alpha_ref,
                            TF* __restrict__ kappa_ref, TF* __restrict__ kappa_v_ref,
                            TF* __restrict__ rho_adv_ref, uint32_t* __restrict__ warm_floor) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (warm_floor && s == 0) warm_gate_update(*S.ctrl, warm_floor);
  BlockSpan B;
  if (!block_scene<BT>(S, B) || s >= B.end) return;
  uint32_t i;
  if constexpr (BT) {
    const FusedIo<TF>& io = S.io[B.k];
    i = S.perm[s] - (B.end - B.n);
    x_ref = io.x_out;
    v_ref = io.v_out;
    a_ref = io.a_out;
    rho_ref = io.rho_out;
    alpha_ref = io.alpha_out;
    kappa_ref = io.kappa_out;
    kappa_v_ref = io.kappa_v_out;
    rho_adv_ref = io.rho_adv_out;
  } else {
    i = S.perm[s];
  }
  const TF dt = S.ctrl->dt;
  const vec3<TF> v = xyz(RV(S, s));
  const vec3<TF> x = xyz(RX(S, s));
  vec3<TF> xn = x + dt * v;
  xn.y = wrap_y(c, xn.y);  // integrate_velocity<1> (runner.hpp:3619-3620)
  st3(x_ref, i, xn);
  st3(v_ref, i, v);
  if (a_ref) st3(a_ref, i, xyz(S.a[s]));
  if (rho_ref) rho_ref[i] = S.rho[s];
  if (alpha_ref) alpha_ref[i] = S.alpha[s];
  TF kp = S.kappa[s];
  if (density_solve) kp *= dt * dt;
  if (kappa_ref) kappa_ref[i] = kp;
  if (kappa_v_ref) kappa_v_ref[i] = S.kappa_v[s];
  if (rho_adv_ref) rho_adv_ref[i] = S.rho_adv[s];
}

// ------------------------------------------------------------------ IISPH
// predict_advection0 (runner.hpp:2609-2639).  kappa holds the pressure,
// kappa_v the last pressure.
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock) k_ii_predict0(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  vec3<TF> xi{0, 0, 0};
  TF rho2 = 1;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    const TF rho = S.rho[L.s];
    rho2 = rho * rho;
    cnt = S.ncount[L.s];
  }
  vec3<TF> dii{0, 0, 0};
  for_each_neighbor<4, false>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>&) {
    dii -= (c.vol / rho2) * gradW(c, pdisp(c, xi, xyz(xj)));
  });
  dii = group_sum(dii, L);
  if (!L.lead()) return;
  const TF dt = S.ctrl->dt;
  const vec4<TF> a = S.a[L.s];
  const vec4<TF> v = RV(S, L.s);
  RV(S, L.s) = vec4<TF>{v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z, v.w};
  const TF lp = S.kappa[L.s] * TF(0.5);
  S.kappa_v[L.s] = lp;
  RX(S, L.s).w = lp;  // pressure read by the first iteration
  for (uint32_t m = S.mask[L.s]; m; m &= m - 1) {
    const uint32_t b = __ffs(m) - 1;
    const vec4<TF> kg = S.bk[size_t(b) * S.ls + L.s];
    dii -= vec3<TF>{kg.x / rho2, kg.y / rho2, kg.z / rho2};
  }
  dii = dii * c.rho0;
  S.dii[L.s] = vec4<TF>{dii.x, dii.y, dii.z, TF(0)};
}

// predict_advection1 (runner.hpp:2640-2690).  aii goes to kk.
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock) k_ii_predict1(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  const TF dt = S.ctrl->dt;
  vec3<TF> xi{0, 0, 0}, vi{0, 0, 0}, dii{0, 0, 0};
  TF rho = c.rho0;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    vi = xyz(RV(S, L.s));
    dii = xyz(S.dii[L.s]);
    rho = S.rho[L.s];
    cnt = S.ncount[L.s];
  }
  const TF rho2 = rho * rho, inv_rho2 = TF(1) / rho2, dpi = c.vol * inv_rho2;
  TF adv = 0, aii = 0;
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const vec3<TF> gw = gradW(c, pdisp(c, xi, xyz(xj)));
    const vec3<TF> dji = (dpi * c.rho0) * gw;
    adv += dt * c.vol * dot(vi - xyz(vj), gw);
    aii += c.vol * dot(dii - dji, gw);
  });
  adv = group_sum(adv, L);
  aii = group_sum(aii, L);
  if (!L.lead()) return;
  adv += rho / c.rho0;
  for (uint32_t m = S.mask[L.s]; m; m &= m - 1) {
    const uint32_t b = __ffs(m) - 1;
    const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
    const vec3<TF> gw = xyz(S.bk[size_t(b) * S.ls + L.s]);
    const vec3<TF> vj = body_velocity(S.rigid[b], xyz(bn));
    const vec3<TF> dji = (inv_rho2 * c.rho0) * gw;
    adv += dt * dot(vi - vj, gw);
    aii += dot(dii - dji, gw);
  }
  S.rho_adv[L.s] = adv;
  S.kk[L.s] = aii * c.rho0;
}

// pressure_solve_iteration0 (runner.hpp:2691-2715).  On iterations after
// the first, also performs the reference's last_pressure <- pressure copy
// (solver_ii.hpp:204) for the own particle; this kernel reads the
// neighbors' pressure (equal to their last pressure after that copy).
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock) k_ii_iter0(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  const bool first = S.ctrl->it == 0;
  vec3<TF> xi{0, 0, 0};
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    cnt = S.ncount[L.s];
  }
  // the payload holds the last pressure on the first iteration
  // (k_ii_predict0) and the pressure afterwards (k_ii_iter1)
  vec3<TF> acc{0, 0, 0};
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const TF rj = vj.w, rj2 = rj * rj;
    acc -= (c.vol / rj2 * xj.w) * gradW(c, pdisp(c, xi, xyz(xj)));
  });
  acc = group_sum(acc, L);
  if (!L.lead()) return;
  if (!first) S.kappa_v[L.s] = S.kappa[L.s];
  acc = acc * c.rho0;
  S.dij_pj[L.s] = vec4<TF>{acc.x, acc.y, acc.z, TF(0)};
}

// pressure_solve_iteration1 (runner.hpp:2716-2772) and the mean of
// solver_ii.hpp:205-206 (double, on the device).
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_ii_iter1(Cn<TF> c, StepState<TF> S, cudaGraphConditionalHandle handle, int use_handle) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  const TF dt = S.ctrl->dt;
  vec3<TF> xi{0, 0, 0}, dij_pj{0, 0, 0};
  TF lp = 0, rho = c.rho0;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    lp = S.kappa_v[L.s];
    dij_pj = xyz(S.dij_pj[L.s]);
    rho = S.rho[L.s];
    cnt = S.ncount[L.s];
  }
  const TF rho2 = rho * rho, dpi = c.vol / rho2;
  TF sum = 0;
  for_each_neighbor<4, false>(S, L, cnt, [&](uint32_t t, const vec4<TF>& xj, const vec4<TF>&) {
    const vec3<TF> gw = gradW(c, pdisp(c, xi, xyz(xj)));
    const vec3<TF> dji = (dpi * c.rho0) * gw;
    const vec3<TF> dji_pi = dji * lp;
    sum += c.vol *
           dot(dij_pj - ldx(S.dii, t) * __ldg(S.kappa_v + t) - (ldx(S.dij_pj, t) - dji_pi), gw);
  });
  sum = group_sum(sum, L);
  double val = 0;
  if (L.lead()) {
    for (uint32_t m = S.mask[L.s]; m; m &= m - 1) {
      const uint32_t b = __ffs(m) - 1;
      sum += dot(dij_pj, xyz(S.bk[size_t(b) * S.ls + L.s]));
    }
    sum *= c.rho0;
    const TF bterm = TF(1) - S.rho_adv[L.s];
    const TF dt2 = dt * dt;
    const TF denom = S.kk[L.s] * dt2;
    const TF omega = TF(2) / TF(3);
    TF p = 0;
    if (fabs(denom) > TF(1.0e-9))
      p = fmax((TF(1) - omega) * lp + omega / denom * (bterm - dt2 * sum), TF(0));
    const TF err = p == TF(0) ? TF(0) : (denom * p + sum * dt2 - bterm);
    S.err[L.s] = err;
    S.kappa[L.s] = p;
    RX(S, L.s).w = p;  // pressure read by the next iteration
    val = double(err);
  }
  double total;
  if (grid_sum_last(val, S.red, &S.ctrl->ticket, &total) && threadIdx.x == 0)
    finish_iteration(*S.ctrl, total, S.n, 1, handle, use_handle);
}

// compute_pressure_accels (runner.hpp:2774-2817) + kinematic_integration<0>
// (runner.hpp:2873-2887), written back in original order.
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_ii_accel_finish(Cn<TF> c, StepState<TF> S, TF* __restrict__ x_ref, TF* __restrict__ v_ref,
                      TF* __restrict__ a_ref, TF* __restrict__ rho_ref, TF* __restrict__ p_ref,
                      TF* __restrict__ rho_adv_ref) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  vec3<TF> ai{0, 0, 0}, xi{0, 0, 0};
  TF dpi = 0;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    const TF rho = S.rho[L.s];
    dpi = S.kappa[L.s] / (rho * rho);
    cnt = S.ncount[L.s];
  }
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const TF rj = vj.w;
    const TF dpj = __ldg(S.kappa + t) / (rj * rj);
    ai -= (c.mass * (dpi + dpj)) * gradW(c, pdisp(c, xi, xyz(xj)));
  });
  ai = group_sum(ai, L);
  const uint32_t m = L.lead() ? S.mask[L.s] : 0u;
  for (uint32_t b = 0; b < S.nb; ++b) {
    const bool mine = (m >> b) & 1u;
    if (!__syncthreads_or(mine)) continue;
    vec3<TF> f{0, 0, 0}, tq{0, 0, 0};
    if (mine) {
      const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
      const vec3<TF> a = (c.rho0 * dpi) * xyz(S.bk[size_t(b) * S.ls + L.s]);
      f = c.mass * a;
      ai -= a;
      tq = cross(xyz(bn) - S.rigid[b].x, f);
    }
    block_add_ft(S, b, f, tq);
  }
  if (!L.lead()) return;
  const TF dt = S.ctrl->dt;
  const vec3<TF> ap = c.rho0 * ai;
  const vec3<TF> v = xyz(RV(S, L.s)) + ap * dt;
  const uint32_t i = S.perm[L.s];
  vec3<TF> xn = xi + v * dt;
  xn.y = wrap_y(c, xn.y);  // kinematic_integration<1> (runner.hpp:2881-2884)
  st3(x_ref, i, xn);
  st3(v_ref, i, v);
  if (a_ref) st3(a_ref, i, xyz(S.a[L.s]));
  if (rho_ref) rho_ref[i] = S.rho[L.s];
  if (p_ref) p_ref[i] = S.kappa[L.s];
  if (rho_adv_ref) rho_adv_ref[i] = S.rho_adv[L.s];
}

// ---------------------------------------------------- implicit SPH (SolverI)
// advect_and_init_pressure (runner.hpp:2889-2900): v += dt a, last pressure
// (kappa_v) = pressure / 2.
template <class TF>
__global__ void __launch_bounds__(kMaxBlock) k_i_advect(StepState<TF> S) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S.n) return;
  const TF dt = S.ctrl->dt;
  const vec4<TF> a = S.a[s];
  const vec4<TF> v = RV(S, s);
  RV(S, s) = vec4<TF>{v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z, v.w};
  S.kappa_v[s] = S.kappa[s] * TF(0.5);
}

// calculate_isph_diagonal_adv_density (runner.hpp:2901-2954): the Jacobi
// diagonal (times rho0) into kk, the advected density into rho_adv.
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock) k_i_diag(Cn<TF> c, StepState<TF> S) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  const TF dt = S.ctrl->dt;
  vec3<TF> xi{0, 0, 0}, vi{0, 0, 0};
  TF rho = c.rho0;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    vi = xyz(RV(S, L.s));
    rho = S.rho[L.s];
    cnt = S.ncount[L.s];
  }
  const TF eps = TF(0.01) * c.h2;
  TF adv = 0, diag = 0;
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const vec3<TF> d = pdisp(c, xi, xyz(xj));  // vj = {v, rho}
    const vec3<TF> gw = gradW(c, d);
    const TF rj = vj.w;
    adv += dt * c.vol * dot(vi - xyz(vj), gw);
    diag += c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gw);
  });
  adv = group_sum(adv, L);
  diag = group_sum(diag, L);
  if (!L.lead()) return;
  adv += rho / c.rho0;
  for (uint32_t m = S.mask[L.s]; m; m &= m - 1) {
    const uint32_t b = __ffs(m) - 1;
    const vec4<TF> bn = S.bx[size_t(b) * S.ls + L.s];
    const vec3<TF> gwv = xyz(S.bk[size_t(b) * S.ls + L.s]);
    const vec3<TF> xib = xi - xyz(bn);
    adv += dt * dot(vi - body_velocity(S.rigid[b], xyz(bn)), gwv);
    diag += (rho + c.rho0) / (rho * c.rho0) / (length_sqr(xib) + eps) * dot(xib, gwv);
  }
  S.kk[L.s] = diag * c.rho0;
  S.rho_adv[L.s] = adv;
}

// isph_solve_iteration (runner.hpp:3006-3053): damped Jacobi (weight 2/3)
// on the neighbors' last pressures, and the mean density error of
// solver_i.hpp:272-274 (double, on the device).  The reference copies
// pressure into last_pressure after each iteration; here the two arrays
// swap roles by iteration parity: iteration k reads kappa_v and writes
// kappa when k is even, the reverse when odd.
template <class TF, bool WR = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_i_iter(Cn<TF> c, StepState<TF> S, cudaGraphConditionalHandle handle, int use_handle) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  const Lane L = pair_lane(S);
  const TF dt = S.ctrl->dt;
  const bool odd = (S.ctrl->it & 1u) != 0;
  const TF* __restrict__ last = odd ? S.kappa : S.kappa_v;
  TF* __restrict__ next = odd ? S.kappa_v : S.kappa;
  vec3<TF> xi{0, 0, 0};
  TF rho = c.rho0, lp = 0;
  uint32_t cnt = 0;
  if (L.act) {
    xi = xyz(RX(S, L.s));
    rho = S.rho[L.s];
    lp = last[L.s];
    cnt = S.ncount[L.s];
  }
  const TF eps = TF(0.01) * c.h2;
  TF off = 0;
  for_each_neighbor<4, true>(S, L, cnt, [&](uint32_t t, const vec4<TF>& xj, const vec4<TF>& vj) {
    const vec3<TF> d = pdisp(c, xi, xyz(xj));
    const TF rj = vj.w;
    off -= c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gradW(c, d)) *
           __ldg(last + t);
  });
  off = group_sum(off, L);
  double val = 0;
  if (L.lead()) {
    off *= c.rho0;
    const TF diag = S.kk[L.s];
    const TF bterm = TF(1) - S.rho_adv[L.s];
    const TF dt2 = dt * dt;
    const TF denom = diag * dt2;
    const TF w = TF(2) / TF(3);
    TF p = 0;
    if (fabs(denom) > TF(1.0e-9))
      p = fmax((TF(1) - w) * lp + w * (bterm / denom - off / diag), TF(0));
    const TF err = p == TF(0) ? TF(0) : (denom * p + off * dt2 - bterm);
    S.err[L.s] = err;
    next[L.s] = p;
    val = double(err);
  }
  double total;
  if (grid_sum_last(val, S.red, &S.ctrl->ticket, &total) && threadIdx.x == 0)
    finish_iteration(*S.ctrl, total, S.n, 1, handle, use_handle);
}

// After an even, non-zero number of iterations the final pressure sits in
// kappa_v: move it to kappa, where the acceleration pass reads it.
template <class TF>
__global__ void k_i_final(StepState<TF> S) {
  const uint32_t it = S.ctrl->it;
  if (it == 0 || (it & 1u)) return;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S.n; s += gridDim.x * blockDim.x)
    S.kappa[s] = S.kappa_v[s];
}

// ------------------------------------------------------------ host side
template <class TF>
struct FluidT;
template <>
struct FluidT<float> {
  using type = al_fluid_f32;
  using body = al_body_f32;
  using rigid = al_rigid_f32;
  using cn = al_const_f32;
};
template <>
struct FluidT<double> {
  using type = al_fluid_f64;
  using body = al_body_f64;
  using rigid = al_rigid_f64;
  using cn = al_const_f64;
};

template <class TF>
int check_step_args(const typename FluidT<TF>::type* f, const al_consti* cni,
                    const typename FluidT<TF>::body* bodies, const void* rigid,
                    const al_solver_params* sp, const TF* dt) {
  ALB_CHECK_ARG(f && cni && sp && dt, "step: null argument");
  ALB_CHECK_ARG(f->num_particles == 0 || (f->particle_x && f->particle_v),
                "step: particle_x / particle_v are null");
  ALB_CHECK_ARG(cni->num_boundaries == 0 || (bodies && rigid), "step: bodies / rigid are null");
  ALB_CHECK_ARG(cni->num_boundaries <= AL_MAX_BOUNDARIES, "step: too many boundaries");
  ALB_CHECK_ARG(cni->grid_res[0] > 0 && cni->grid_res[1] > 0 && cni->grid_res[2] > 0,
                "step: grid_res must be positive");
  ALB_CHECK_ARG(uint64_t(cni->grid_res[0]) * cni->grid_res[1] * cni->grid_res[2] < (1ull << 31),
                "step: grid has too many cells");
  ALB_CHECK_ARG(cni->max_num_neighbors_per_particle > 0, "step: neighbor capacity is 0");
  ALB_CHECK_ARG(*dt > TF(0), "step: dt must be positive");
  return AL_OK;
}

// Reads the loop flag (eager mode: one small readback per iteration).
// Pinned host staging of one step: control block, body descriptors, rigid
// state, the eager loop flag and the grid anomaly flags.  Every section
// starts on a 64-byte boundary (RigidDev<double> holds 32-byte-aligned
// vectors).  A captured graph copies from and to these addresses.
template <class TF>
struct Staging {
  Ctrl<TF>* hc = nullptr;
  BodyDev<TF>* hb = nullptr;
  RigidDev<TF>* hr = nullptr;
  uint32_t* hflag = nullptr;
  uint32_t* hf = nullptr;  // [4]
};

// Layout of one staging slot: control block at 0, bodies at `bodies`, rigid
// state at `rigid`, the eager loop flag at `flag`, the anomaly flags at
// flag + 64; `bytes` in all.
template <class TF>
struct StagingLayout {
  static constexpr size_t up64(size_t b) { return (b + 63) & ~size_t(63); }
  static constexpr size_t bodies = up64(sizeof(Ctrl<TF>));
  static constexpr size_t rigid = bodies + up64(sizeof(BodyDev<TF>) * AL_MAX_BOUNDARIES);
  static constexpr size_t flag = rigid + up64(sizeof(RigidDev<TF>) * AL_MAX_BOUNDARIES);
  static constexpr size_t bytes = flag + 128;
};

// Staging of slot `slot` out of `nslots` equal slots (batched steps give
// every scene its own slot).
template <class TF>
int staging(al_engine* e, Staging<TF>* out, uint32_t slot = 0, uint32_t nslots = 1) {
  using L = StagingLayout<TF>;
  const size_t off_b = L::bodies, off_r = L::rigid, off_f = L::flag, slot_bytes = L::bytes;
  void* pinned = nullptr;
  ALB_TRY(e->host_pinned(slot_bytes * nslots, &pinned));
  // cudaMallocHost: page aligned; slots are multiples of 64 bytes
  char* base = static_cast<char*>(pinned) + slot_bytes * slot;
  out->hc = reinterpret_cast<Ctrl<TF>*>(base);
  out->hb = reinterpret_cast<BodyDev<TF>*>(base + off_b);
  out->hr = reinterpret_cast<RigidDev<TF>*>(base + off_r);
  out->hflag = reinterpret_cast<uint32_t*>(base + off_f);
  out->hf = reinterpret_cast<uint32_t*>(base + off_f + 64);
  return AL_OK;
}

// Everything one step launches, resolved on the host.
template <class TF>
struct StepPlan {
  bool iisph = false, div = false, den = false;
  bool isph = false;  // implicit SPH (SolverI); iisph is set too (pressure state)
  Cn<TF> c;
  GridDims g;
  const typename FluidT<TF>::type* f = nullptr;
  StepState<TF> S;
  uint32_t* flags = nullptr;
  BodyDev<TF>* bodies_dev = nullptr;
  Staging<TF> io;
  // learned warm start (float DFSPH steps): features in sorted order and
  // the network's predictions; features_out in original order
  bool learned = false;
  WarmNetDev net{};
  float* warm_feat = nullptr;
  float* warm_feat_out = nullptr;
  float* warm_pred = nullptr;
  // the learned warm start's gate words (warm_gate_update); zero for a fresh
  // scene
  uint32_t* warm_floor = nullptr;
  // launch shapes: particle-count bucket and context of the shape table
  uint32_t bucket = 0, ctx = 0;
  // first-stage partials of the rigid totals ([kRigidChunks][nb][6])
  double* ftp = nullptr;
  // Shape of pass group `group` (defaults: 128-thread blocks; pair passes
  // pair_tpp(n) threads per particle, other passes one).
  LaunchShape shape(const al_engine* e, const char* group, bool pair) const {
    LaunchShape sh{uint32_t(kBlock), pair ? pair_tpp(S.n) : 1u};
    auto it = e->shapes.find(std::make_tuple(std::string(group), bucket, ctx));
    if (it != e->shapes.end()) {
      if (it->second.first) sh.block = it->second.first;
      if (pair && it->second.second) sh.tpp = it->second.second;
    }
    return sh;
  }
};

// Adds a device-driven WHILE loop at the current end of the capture on
// `st`: `begin(h)` launches the kernel that sets the first condition,
// `body(stream, h, 1)` launches one iteration whose last kernel sets the
// next.  The body is captured on the engine's second stream into the
// conditional node's own graph.
template <class Begin, class Body>
int capture_while(al_engine* e, cudaStream_t st, Begin&& begin, Body&& body) {
  cudaStreamCaptureStatus status;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  ALB_CUDA(cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphConditionalHandle h;
  ALB_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault));
  ALB_TRY(begin(h));
  ALB_CUDA(cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  ALB_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &np));
  ALB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  cudaStream_t bs = e->body_stream;
  ALB_CUDA(cudaStreamBeginCaptureToGraph(bs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  const int rc = body(bs, h, 1);
  cudaGraph_t captured = nullptr;
  const cudaError_t end = cudaStreamEndCapture(bs, &captured);
  ALB_TRY(rc);
  ALB_CUDA(end);
  return AL_OK;
}

// Adds a device-decided IF node at the current end of the capture on `st`:
// `begin(h)` launches the kernel that sets the condition, `body(stream)`
// launches the conditional work, captured on the engine's second stream into
// the node's own graph.  When the condition is 0 nothing in the body runs.
template <class Begin, class Body>
int capture_if(al_engine* e, cudaStream_t st, Begin&& begin, Body&& body) {
  cudaStreamCaptureStatus status;
  cudaGraph_t graph = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  ALB_CUDA(cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphConditionalHandle h;
  ALB_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, cudaGraphCondAssignDefault));
  ALB_TRY(begin(h));
  ALB_CUDA(cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps));
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeIf;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  ALB_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &np));
  ALB_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  cudaStream_t bs = e->body_stream;
  ALB_CUDA(cudaStreamBeginCaptureToGraph(bs, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal));
  const int rc = body(bs);
  cudaGraph_t captured = nullptr;
  const cudaError_t end = cudaStreamEndCapture(bs, &captured);
  ALB_TRY(rc);
  ALB_CUDA(end);
  return AL_OK;
}

// Condition of the learned warm start's IF node: run the network unless the
// gate (warm_gate_update) says this step skips it.  Also recorded in the
// control block (the host counts the node's launches from it).
template <class TF>
__global__ void k_warm_if(cudaGraphConditionalHandle h, const uint32_t* __restrict__ gate,
                          Ctrl<TF>* C) {
  const uint32_t run = gate[0] == 0u ? 1u : 0u;
  C->warm_ran = run;
  cudaGraphSetConditional(h, run);
}

// Kernels inside the learned warm start's IF node (inference, application).
constexpr uint32_t kWarmIfLaunches = 2;

// Enqueues one whole step on `st`: staging uploads, grid, boundaries,
// neighbors, the solves, write-back and the report readback.  With
// `capture` the solver loops become conditional WHILE nodes (and `loops`
// counts them); otherwise the host reads the loop flag every iteration.
template <class TF>
int enqueue_step(al_engine* e, StepPlan<TF>& P, cudaStream_t st, bool capture, int* loops) {
  StepState<TF>& S = P.S;
  const Cn<TF>& c = P.c;
  const auto* f = P.f;
  const uint32_t n = S.n, nb = S.nb;
  const bool iisph = P.iisph, div = P.div, den = P.den;
  const bool wr = c.wrap != 0;  // periodic-y instantiations of the pair passes
  ALB_CUDA(cudaMemcpyAsync(S.ctrl, P.io.hc, sizeof(Ctrl<TF>), cudaMemcpyHostToDevice, st));
  if (nb) {
    ALB_CUDA(cudaMemcpyAsync(P.bodies_dev, P.io.hb, sizeof(BodyDev<TF>) * nb,
                             cudaMemcpyHostToDevice, st));
    ALB_CUDA(cudaMemcpyAsync(S.rigid, P.io.hr, sizeof(RigidDev<TF>) * nb, cudaMemcpyHostToDevice,
                             st));
  }
  ALB_CUDA(cudaMemsetAsync(P.flags, 0, 4 * sizeof(uint32_t), st));
  ALB_CUDA(cudaMemsetAsync(S.ft, 0, size_t(S.grid) * (nb ? nb : 1) * 6 * sizeof(double), st));
  ALB_LAUNCH(e, "step_init", 1, st, k_step_init<TF><<<1, 32, 0, st>>>(S));
  // ---- grid, boundaries, neighbors, density (+ DFSPH factor)
  GridState gs;
  ALB_LAUNCH(e, "grid_sort", kGridBuildKernels, st,
             ALB_TRY(grid_build<TF>(e, c, P.g, f->particle_x, n, S.x, P.flags, gs, st)));
  S.perm = gs.perm;
  const uint32_t blocks = blocks_for(n, kBlock);
  // grid, block and lane state of pair pass group `g` (launch-shape table)
  auto pair_shape = [&](const char* g, uint32_t& grid, uint32_t& block) {
    const LaunchShape sh = P.shape(e, g, true);
    StepState<TF> Sg = S;
    Sg.tpp = sh.tpp;
    grid = pair_blocks(n, sh.tpp, sh.block);
    block = sh.block;
    return Sg;
  };
  if (n > 0) {
    const TF* kref = iisph ? f->particle_pressure : f->particle_kappa;
    if (iisph)
      ALB_LAUNCH(e, "gather_state", 1, st,
                 k_gather_state<TF, false><<<blocks, kBlock, 0, st>>>(S, f->particle_v, kref,
                                                                      nullptr));
    else
      ALB_LAUNCH(e, "gather_state", 1, st,
                 k_gather_state<TF, true><<<blocks, kBlock, 0, st>>>(S, f->particle_v, kref,
                                                                     f->particle_kappa_v));
  }
  BoundaryState<TF> bs{nb, S.mask, S.bx, S.bk, &S.ctrl->rep.num_active_boundary_pairs, S.ls};
  if (nb)
    ALB_LAUNCH(e, "boundary", 1, st,
               ALB_TRY(sample_boundaries<TF>(c, P.bodies_dev, S.rigid, nb, S.x, gs.perm, n, bs,
                                             f->particle_boundary, f->particle_boundary_kernel,
                                             st)));
  else if (n)
    ALB_CUDA(cudaMemsetAsync(S.mask, 0, size_t(n) * sizeof(uint32_t), st));
  SortedBoundaryKernel<TF> sbk{S.mask, S.bk, S.ls};
  TF* rho_rec = reinterpret_cast<TF*>(S.rec) + 7;  // rec[2s + 1].w
  if (div && n > 0) {
    WarmDivergence<TF> wd{S, P.warm_feat, P.warm_feat_out, c.radius * TF(2), c.vol,
                          P.warm_floor};
    const uint32_t nbb = P.shape(e, "neighbors", false).block;
    ALB_LAUNCH(e, "neighbors", 1, st,
               (wr ? k_build_neighbors<TF, SortedBoundaryKernel<TF>, true, WarmDivergence<TF>, true>
                         <<<blocks_for(n, nbb), nbb, 0, st>>>(
                             c, P.g, gs.cell_start, S.x, n, S.ls, sbk, S.nbr, S.ncount, S.rho,
                             S.alpha, rho_rec, gs.flags, wd, FusedBuild{})
                   : k_build_neighbors<TF, SortedBoundaryKernel<TF>, true, WarmDivergence<TF>, false>
                         <<<blocks_for(n, nbb), nbb, 0, st>>>(
                             c, P.g, gs.cell_start, S.x, n, S.ls, sbk, S.nbr, S.ncount, S.rho,
                             S.alpha, rho_rec, gs.flags, wd, FusedBuild{})));
    if (P.learned) {
      // inference and its application; in a captured step they sit in an IF
      // node, so a step whose gate is closed launches neither
      auto infer = [&](cudaStream_t s) -> int {
        ALB_LAUNCH(e, "warm_net", 1, s,
                   ALB_TRY(warm_forward(e, P.net, P.warm_feat, n, P.warm_pred, P.flags + 3, s,
                                        P.warm_floor)));
        ALB_LAUNCH(e, "warm_apply", 1, s,
                   (k_apply_warm_div<TF><<<blocks_for(n, kBlock), kBlock, 0, s>>>(
                       S, P.warm_feat, P.warm_pred, P.warm_floor)));
        return AL_OK;
      };
      if (capture)
        ALB_TRY(capture_if(
            e, st,
            [&](cudaGraphConditionalHandle h) -> int {
              ALB_LAUNCH(e, "warm_gate", 1, st,
                         (k_warm_if<TF><<<1, 1, 0, st>>>(h, P.warm_floor, S.ctrl)));
              return AL_OK;
            },
            infer));
      else
        ALB_TRY(infer(st));
    }
  } else
    ALB_LAUNCH(e, "neighbors", 1, st,
               ALB_TRY(build_neighbors_density<TF>(c, P.g, gs, S.x, sbk, S.nbr, S.ncount, S.rho,
                                                   iisph ? nullptr : S.alpha, rho_rec, st)));
  // One solver loop: kernel `k_loop_begin` sets the first condition, `body`
  // launches one iteration on the given stream.
  auto solve = [&](int density_solve, uint32_t max_iter, auto&& body) -> int {
    if (capture) {
      ++*loops;
      return capture_while(
          e, st,
          [&](cudaGraphConditionalHandle h) -> int {
            ALB_LAUNCH(e, "loop_begin", 1, st,
                       k_loop_begin<TF><<<1, 1, 0, st>>>(S, density_solve, h, 1));
            return AL_OK;
          },
          body);
    }
    ALB_LAUNCH(e, "loop_begin", 1, st, k_loop_begin<TF><<<1, 1, 0, st>>>(S, density_solve, 0, 0));
    bool go = max_iter > 0;
    while (go) {
      ALB_TRY(body(st, cudaGraphConditionalHandle(0), 0));
      ALB_TRY(read_keep_going(S, P.io.hflag, st, &go));
    }
    return AL_OK;
  };
  if (n > 0) {
    if (div) {
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("div_warm1", pg_, pb_);
        ALB_LAUNCH(e, "div_warm1", 1, st,
                   (wr ? k_kappa<TF, kDivWarm, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_kappa<TF, kDivWarm, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
      }
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("div_rho_adv", pg_, pb_);
        ALB_LAUNCH(e, "div_rho_adv", 1, st,
                   (wr ? k_df_rho_adv_init<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_df_rho_adv_init<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
      }
      ALB_TRY(solve(0, P.io.hc->max_div,
                    [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
                      {
                        uint32_t pg_, pb_;
                        const StepState<TF> Sg_ = pair_shape("div_iter", pg_, pb_);
                        ALB_LAUNCH(e, "div_iter", 1, s,
                                   (wr ? k_kappa<TF, kDivIter, true><<<pg_, pb_, 0, s>>>(c, Sg_) : k_kappa<TF, kDivIter, false><<<pg_, pb_, 0, s>>>(c, Sg_)));
                      }
                      {
                        uint32_t pg_, pb_;
                        const StepState<TF> Sg_ = pair_shape("div_residual", pg_, pb_);
                        ALB_LAUNCH(e, "div_residual", 1, s,
                                   (wr ? k_df_residual<TF, true><<<pg_, pb_, 0, s>>>(c, Sg_, h, use) : k_df_residual<TF, false><<<pg_, pb_, 0, s>>>(c, Sg_, h, use)));
                      }
                      return AL_OK;
                    }));
    }
    {
      uint32_t pg_, pb_;
      const StepState<TF> Sg_ = pair_shape("viscosity", pg_, pb_);
      ALB_LAUNCH(e, "viscosity", 1, st,
                 (wr ? k_viscosity<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_, div ? 1 : 0) : k_viscosity<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_, div ? 1 : 0)));
    }
    if (!iisph) {
      ALB_LAUNCH(e, "integrate_np", 1, st, k_integrate_np<TF><<<blocks, kBlock, 0, st>>>(S));
      if (den) {
        {
          uint32_t pg_, pb_;
          const StepState<TF> Sg_ = pair_shape("press_warm0", pg_, pb_);
          ALB_LAUNCH(e, "press_warm0", 1, st,
                     (wr ? k_p_warm0<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_, P.warm_pred, P.warm_floor) : k_p_warm0<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_, P.warm_pred, P.warm_floor)));
        }
        {
          uint32_t pg_, pb_;
          const StepState<TF> Sg_ = pair_shape("press_warm1", pg_, pb_);
          ALB_LAUNCH(e, "press_warm1", 1, st,
                     (wr ? k_kappa<TF, kPressWarm, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_kappa<TF, kPressWarm, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
        }
        {
          uint32_t pg_, pb_;
          const StepState<TF> Sg_ = pair_shape("press_rho_adv", pg_, pb_);
          ALB_LAUNCH(e, "press_rho_adv", 1, st,
                     (wr ? k_p_rho_adv_init<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_p_rho_adv_init<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
        }
        ALB_TRY(solve(1, P.io.hc->max_den,
                      [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
                        {
                          uint32_t pg_, pb_;
                          const StepState<TF> Sg_ = pair_shape("press_iter", pg_, pb_);
                          ALB_LAUNCH(e, "press_iter", 1, s,
                                     (wr ? k_kappa<TF, kPressIter, true><<<pg_, pb_, 0, s>>>(c, Sg_) : k_kappa<TF, kPressIter, false><<<pg_, pb_, 0, s>>>(c, Sg_)));
                        }
                        {
                          uint32_t pg_, pb_;
                          const StepState<TF> Sg_ = pair_shape("press_residual", pg_, pb_);
                          ALB_LAUNCH(e, "press_residual", 1, s,
                                     (wr ? k_p_residual<TF, true><<<pg_, pb_, 0, s>>>(c, Sg_, h, use) : k_p_residual<TF, false><<<pg_, pb_, 0, s>>>(c, Sg_, h, use)));
                        }
                        return AL_OK;
                      }));
      }
      ALB_LAUNCH(e, "finish", 1, st,
                 (wr ? k_df_finish<TF, true><<<blocks, kBlock, 0, st>>>(
                     c, S, den ? 1 : 0, f->particle_x, f->particle_v, f->particle_a,
                     f->particle_density, f->particle_dfsph_factor, f->particle_kappa,
                     f->particle_kappa_v, f->particle_density_adv, P.warm_floor) : k_df_finish<TF, false><<<blocks, kBlock, 0, st>>>(
                     c, S, den ? 1 : 0, f->particle_x, f->particle_v, f->particle_a,
                     f->particle_density, f->particle_dfsph_factor, f->particle_kappa,
                     f->particle_kappa_v, f->particle_density_adv, P.warm_floor)));
    } else if (P.isph) {
      ALB_LAUNCH(e, "i_advect", 1, st, k_i_advect<TF><<<blocks, kBlock, 0, st>>>(S));
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("i_diag", pg_, pb_);
        ALB_LAUNCH(e, "i_diag", 1, st, (wr ? k_i_diag<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_i_diag<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
      }
      ALB_TRY(solve(1, P.io.hc->max_den,
                    [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
                      {
                        uint32_t pg_, pb_;
                        const StepState<TF> Sg_ = pair_shape("i_iter", pg_, pb_);
                        ALB_LAUNCH(e, "i_iter", 1, s,
                                   (wr ? k_i_iter<TF, true><<<pg_, pb_, 0, s>>>(c, Sg_, h, use) : k_i_iter<TF, false><<<pg_, pb_, 0, s>>>(c, Sg_, h, use)));
                      }
                      return AL_OK;
                    }));
      ALB_LAUNCH(e, "i_final", 1, st,
                 k_i_final<TF><<<blocks, kBlock, 0, st>>>(S));
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("finish", pg_, pb_);
        ALB_LAUNCH(e, "finish", 1, st,
                   (wr ? k_ii_accel_finish<TF, true><<<pg_, pb_, 0, st>>>(
                       c, Sg_, f->particle_x, f->particle_v, f->particle_a, f->particle_density,
                       f->particle_pressure, f->particle_density_adv) : k_ii_accel_finish<TF, false><<<pg_, pb_, 0, st>>>(
                       c, Sg_, f->particle_x, f->particle_v, f->particle_a, f->particle_density,
                       f->particle_pressure, f->particle_density_adv)));
      }
    } else {
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("ii_predict0", pg_, pb_);
        ALB_LAUNCH(e, "ii_predict0", 1, st, (wr ? k_ii_predict0<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_ii_predict0<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
      }
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("ii_predict1", pg_, pb_);
        ALB_LAUNCH(e, "ii_predict1", 1, st, (wr ? k_ii_predict1<TF, true><<<pg_, pb_, 0, st>>>(c, Sg_) : k_ii_predict1<TF, false><<<pg_, pb_, 0, st>>>(c, Sg_)));
      }
      ALB_TRY(solve(1, P.io.hc->max_den,
                    [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
                      {
                        uint32_t pg_, pb_;
                        const StepState<TF> Sg_ = pair_shape("ii_iter0", pg_, pb_);
                        ALB_LAUNCH(e, "ii_iter0", 1, s,
                                   (wr ? k_ii_iter0<TF, true><<<pg_, pb_, 0, s>>>(c, Sg_) : k_ii_iter0<TF, false><<<pg_, pb_, 0, s>>>(c, Sg_)));
                      }
                      {
                        uint32_t pg_, pb_;
                        const StepState<TF> Sg_ = pair_shape("ii_iter1", pg_, pb_);
                        ALB_LAUNCH(e, "ii_iter1", 1, s,
                                   (wr ? k_ii_iter1<TF, true><<<pg_, pb_, 0, s>>>(c, Sg_, h, use) : k_ii_iter1<TF, false><<<pg_, pb_, 0, s>>>(c, Sg_, h, use)));
                      }
                      return AL_OK;
                    }));
      {
        uint32_t pg_, pb_;
        const StepState<TF> Sg_ = pair_shape("finish", pg_, pb_);
        ALB_LAUNCH(e, "finish", 1, st,
                   (wr ? k_ii_accel_finish<TF, true><<<pg_, pb_, 0, st>>>(
                       c, Sg_, f->particle_x, f->particle_v, f->particle_a, f->particle_density,
                       f->particle_pressure, f->particle_density_adv) : k_ii_accel_finish<TF, false><<<pg_, pb_, 0, st>>>(
                       c, Sg_, f->particle_x, f->particle_v, f->particle_a, f->particle_density,
                       f->particle_pressure, f->particle_density_adv)));
      }
    }
  }
  if (nb) {
    if (S.grid > kRigidChunks)
      ALB_LAUNCH(e, "rigid_finish", 2, st,
                 (k_rigid_partial<<<dim3(kRigidChunks, nb), 256, 0, st>>>(S.ft, S.grid, nb, P.ftp),
                  k_rigid_finish<TF><<<nb, 256, 0, st>>>(S, P.ftp, kRigidChunks)));
    else
      ALB_LAUNCH(e, "rigid_finish", 1, st,
                 k_rigid_finish<TF><<<nb, 256, 0, st>>>(S, S.ft, S.grid));
  }
  ALB_CUDA(cudaGetLastError());
  // ---- read back: report, rigid state, anomaly flags
  ALB_CUDA(cudaMemcpyAsync(P.io.hc, S.ctrl, sizeof(Ctrl<TF>), cudaMemcpyDeviceToHost, st));
  if (nb)
    ALB_CUDA(cudaMemcpyAsync(P.io.hr, S.rigid, sizeof(RigidDev<TF>) * nb, cudaMemcpyDeviceToHost,
                             st));
  ALB_CUDA(cudaMemcpyAsync(P.io.hf, P.flags, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  return AL_OK;
}

// Kernels one solver-loop iteration launches: the update and the residual
// (DFSPH, IISPH), one fused pass (implicit SPH).
template <class TF>
uint32_t iteration_launches(const StepPlan<TF>& P) {
  return P.isph ? 1u : 2u;
}

// Captures one step into an executable graph.  Sets `*exec` to null (and
// returns AL_OK) when a scratch buffer moved during the capture.
template <class TF>
int capture_step(al_engine* e, StepPlan<TF>& P, cudaGraphExec_t* exec, uint32_t* fixed) {
  *exec = nullptr;
  ALB_TRY(e->capture_streams());
  cudaStream_t cs = e->capture_stream;
  const uint64_t launches0 = e->launches;
  const uint64_t gen0 = e->generation;
  ALB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int loops = 0;
  const int rc = enqueue_step<TF>(e, P, cs, true, &loops);
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(cs, &graph);
  const uint64_t captured = e->launches - launches0;
  e->launches = launches0;
  if (rc != AL_OK || end != cudaSuccess || e->generation != gen0) {
    if (graph) cudaGraphDestroy(graph);
    if (rc != AL_OK) return rc;
    ALB_CUDA(end);
    return AL_OK;
  }
  const cudaError_t inst = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) *exec = nullptr;
  ALB_CUDA(inst);
  *fixed = uint32_t(captured - iteration_launches(P) * uint32_t(loops) -
                    (P.learned ? kWarmIfLaunches : 0u));
  return AL_OK;
}

// Graph cache key: precision, method, enabled solves, scratch generation
// and the raw bytes of the constants, grid descriptor and fluid buffer
// table (their fields carry no padding).
template <class TF>
std::vector<uint64_t> step_key(const al_engine* e, const StepPlan<TF>& P,
                               const typename FluidT<TF>::cn* cn, const al_consti* cni) {
  std::vector<uint64_t> k{sizeof(TF),         uint64_t(P.iisph), uint64_t(P.isph),
                          uint64_t(P.div),    uint64_t(P.den),   e->generation};
  auto add = [&k](const void* p, size_t bytes) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < bytes; i += 8) {
      uint64_t w = 0;
      std::memcpy(&w, b + i, bytes - i < 8 ? bytes - i : 8);
      k.push_back(w);
    }
  };
  add(cn, sizeof(*cn));
  add(cni, sizeof(*cni));
  add(P.f, sizeof(*P.f));
  k.push_back(uint64_t(P.c.wrap));  // baked into the captured kernels' parameters
  add(&P.c.wrap_len, sizeof(P.c.wrap_len));
  k.push_back(uint64_t(P.learned));
  k.push_back(reinterpret_cast<uint64_t>(P.warm_feat_out));
  if (P.learned) add(&P.net, sizeof(P.net));
  return k;
}

constexpr size_t kMaxGraphs = 8;

// Solver methods of run_step: SolverDf, SolverIi, SolverI.
constexpr int kMethodDf = 0, kMethodIi = 1, kMethodI = 2;

// Host-side arguments of one scene's step (the C ABI's per-call inputs).
template <class TF>
struct StepArgs {
  bool iisph = false;
  bool isph = false;
  const typename FluidT<TF>::cn* cn = nullptr;
  const al_consti* cni = nullptr;
  const typename FluidT<TF>::type* f = nullptr;
  const typename FluidT<TF>::body* bodies = nullptr;
  typename FluidT<TF>::rigid* rigid = nullptr;
  const al_solver_params* sp = nullptr;
  TF* dt = nullptr;
  al_step_report* report = nullptr;
  const al_warm_start* warm = nullptr;
  // launch-shape context: 0 single step, 1 a scene of a batched step
  uint32_t batch = 0;
};

// Validates the arguments, sizes the scene's scratch (under the engine's
// current buffer namespace; with `alloc` false none: a fused batch places
// the scene's state in its shared arena and staging copy) and fills staging
// slot `slot` of `nslots`.
template <class TF>
int prepare_step(al_engine* e, const StepArgs<TF>& A, StepPlan<TF>& P, uint32_t slot,
                 uint32_t nslots, bool alloc = true) {
  ALB_TRY(check_step_args<TF>(A.f, A.cni, A.bodies, A.rigid, A.sp, A.dt));
  const al_solver_params* sp = A.sp;
  const bool iisph = A.iisph || A.isph;
  P.iisph = iisph;
  P.isph = A.isph;
  P.div = !iisph && sp->enable_divergence_solve;
  P.den = iisph || sp->enable_density_solve;
  P.c = to_cn<TF>(*A.cn);
  if (sp->wrap_y) {  // SolverDf / SolverIi / SolverI::step<1>
    ALB_CHECK_ARG(sp->wrap_length > 0, "step: wrap_y needs a positive wrap_length");
    set_wrap(P.c, TF(sp->wrap_length));
  }
  P.g = to_dims(*A.cni);
  P.f = A.f;
  const uint32_t n = A.f->num_particles;
  const uint32_t nb = P.g.nb;
  StepState<TF>& S = P.S;
  S.n = n;
  S.ls = n;
  S.nb = nb;
  S.cap = P.g.cap_nbr;
  P.bucket = n ? uint32_t(31 - __builtin_clz(n)) : 0u;
  P.ctx = A.batch;
  S.tpp = pair_tpp(n);
  // per-block buffers (rigid partials, reduction partials) hold the largest
  // grid any pair pass of this scene launches
  S.grid = pair_blocks(n, S.tpp);
  for (uint32_t k = 0; alloc && k < kNumTunable; ++k) {
    if (!kTunable[k].pair) continue;
    const LaunchShape sh = P.shape(e, kTunable[k].name, true);
    S.grid = std::max(S.grid, pair_blocks(n, sh.tpp, sh.block));
  }
  if (S.grid == 0) S.grid = 1;
  // ---- buffers
  if (alloc) {
    ALB_TRY(e->buf("flags", 4, &P.flags));
    ALB_TRY(e->buf("sorted.x", size_t(n) + kSortedPad, &S.x));
    ALB_TRY(e->buf("sorted.rec", size_t(n) * 2, &S.rec));
    ALB_TRY(e->buf("sorted.a", n, &S.a));
    ALB_TRY(e->buf("sorted.rho", n, &S.rho));
    ALB_TRY(e->buf("sorted.alpha", n, &S.alpha));
    ALB_TRY(e->buf("sorted.rho_adv", n, &S.rho_adv));
    ALB_TRY(e->buf("sorted.kappa", n, &S.kappa));
    ALB_TRY(e->buf("sorted.kappa_v", n, &S.kappa_v));
    if (iisph) {
      ALB_TRY(e->buf("sorted.kk", n, &S.kk));
      ALB_TRY(e->buf("sorted.err", n, &S.err));
    }
    if (iisph && !P.isph) {
      ALB_TRY(e->buf("sorted.dii", n, &S.dii));
      ALB_TRY(e->buf("sorted.dij_pj", n, &S.dij_pj));
    }
    ALB_TRY(e->buf("nbr.list", size_t(n) * P.g.cap_nbr, &S.nbr));
    ALB_TRY(e->buf("nbr.count", n, &S.ncount));
    ALB_TRY(e->buf("bnd.mask", n, &S.mask));
    ALB_TRY(e->buf("bnd.x", size_t(nb ? nb : 1) * n, &S.bx));
    ALB_TRY(e->buf("bnd.k", size_t(nb ? nb : 1) * n, &S.bk));
    ALB_TRY(e->buf("bodies", nb ? nb : 1, &P.bodies_dev));
    ALB_TRY(e->buf("rigid", nb ? nb : 1, &S.rigid));
    ALB_TRY(e->buf("ft", size_t(S.grid) * (nb ? nb : 1) * 6, &S.ft));
    ALB_TRY(e->buf("ftp", size_t(kRigidChunks) * (nb ? nb : 1) * 6, &P.ftp));
    ALB_TRY(e->buf("red", S.grid, &S.red));
    ALB_TRY(e->buf("ctrl", 1, &S.ctrl));
  }
  S.bodies = P.bodies_dev;
  const al_warm_start* warm = A.warm;
  if (warm && (warm->net || warm->features_out)) {
    if (sizeof(TF) != 4 || iisph || !P.div) {
      set_error("learned warm start: float32 DFSPH steps with the divergence solve only");
      return AL_ERR_UNSUPPORTED;
    }
    P.warm_feat_out = warm->features_out;
    if (warm->net) {
      ALB_CHECK_ARG(warm->net->params != nullptr, "learned warm start: params is null");
      P.learned = true;
      P.net = to_warm_dev(*warm->net);
      ALB_TRY(e->buf("warm.feat", size_t(n) * AL_WARM_NUM_FEATURES, &P.warm_feat));
      ALB_TRY(e->buf("warm.pred", size_t(n) * AL_WARM_NUM_OUTPUTS, &P.warm_pred));
      bool fresh = false;
      ALB_TRY(e->buf("warm.floor", 4, &P.warm_floor, &fresh));
      // the gate belongs to a scene: other caller buffers than last time
      // (or a new gate buffer) start it afresh
      const void*& owner = e->warm_owner[e->ns];
      if (fresh || owner != static_cast<const void*>(A.f->particle_x)) {
        ALB_CUDA(cudaMemset(P.warm_floor, 0, 4 * sizeof(uint32_t)));
        owner = A.f->particle_x;
      }
    }
  }
  // ---- host staging: control block, bodies, rigid state
  ALB_TRY(staging<TF>(e, &P.io, slot, nslots));
  Ctrl<TF>* hc = P.io.hc;
  std::memset(hc, 0, sizeof(Ctrl<TF>));
  hc->dt = *A.dt;
  hc->length_scale = P.c.radius * TF(2);
  hc->cfl = TF(sp->cfl);
  hc->max_dt = TF(sp->max_dt);
  hc->min_dt = TF(sp->min_dt);
  hc->tol_div = double(TF(sp->density_change_tolerance));
  hc->tol_den = double(TF(sp->density_error_tolerance));
  hc->min_div = sp->min_divergence_solve;
  hc->max_div = sp->max_divergence_solve;
  hc->min_den = sp->min_density_solve;
  hc->max_den = sp->max_density_solve;
  hc->integrate_rigids = sp->integrate_rigids;
  for (int k = 0; k < 3; ++k) hc->pile_gravity[k] = TF(sp->pile_gravity[k]);
  for (uint32_t b = 0; b < nb; ++b) {
    P.io.hb[b] = to_body_dev<TF>(A.bodies[b]);
    ALB_TRY(validate_body(P.io.hb[b], true, true));
    P.io.hr[b] = to_rigid_dev<TF>(A.rigid[b]);
  }
  return AL_OK;
}

// Reads a completed step back: report, dt, rigid state, status.
template <class TF>
int finish_step(const StepArgs<TF>& A, const StepPlan<TF>& P) {
  al_step_report rep = P.io.hc->rep;
  const uint32_t* hf = P.io.hf;
  for (int k = 0; k < 3; ++k) rep.grid_anomaly[k] = hf[k];
  if (P.S.n == 0) rep.dt = double(*A.dt);
  *A.dt = TF(rep.dt);
  const RigidDev<TF>* hr = P.io.hr;
  for (uint32_t b = 0; b < P.S.nb; ++b) {
    for (int k = 0; k < 3; ++k) {
      A.rigid[b].x[k] = (&hr[b].x.x)[k];
      A.rigid[b].v[k] = (&hr[b].v.x)[k];
      A.rigid[b].omega[k] = (&hr[b].omega.x)[k];
    }
    A.rigid[b].q[0] = hr[b].q.x;
    A.rigid[b].q[1] = hr[b].q.y;
    A.rigid[b].q[2] = hr[b].q.z;
    A.rigid[b].q[3] = hr[b].q.w;
  }
  if (A.report) *A.report = rep;
  if (hf[0]) return AL_ERR_OUT_OF_GRID;
  if (hf[1]) return AL_ERR_CELL_OVERFLOW;
  if (hf[2]) return AL_ERR_NEIGHBOR_OVERFLOW;
  if (hf[3]) {
    set_error("learned warm start: a tensor-core wait timed out");
    return AL_ERR_TIMEOUT;
  }
  return AL_OK;
}

// Cached graph for `key`, capturing it with `capture` when the key ran
// eagerly before.  Returns null (run eagerly) otherwise.
template <class Capture>
int find_or_capture(al_engine* e, const std::vector<uint64_t>& key, Capture&& capture,
                    al_engine::Graph** out) {
  *out = nullptr;
  for (al_engine::Graph& gr : e->graphs)
    if (gr.key == key) *out = &gr;
  if (*out) return AL_OK;
  bool seen = false;
  for (const auto& k : e->seen_keys) seen = seen || k == key;
  if (!seen) return AL_OK;
  al_engine::Graph gr;
  gr.key = key;
  ALB_TRY(capture(&gr.exec, &gr.fixed_launches));
  if (!gr.exec) return AL_OK;
  if (e->graphs.size() >= kMaxGraphs) {
    cudaGraphExecDestroy(e->graphs.front().exec);
    e->graphs.erase(e->graphs.begin());
  }
  e->graphs.push_back(std::move(gr));
  *out = &e->graphs.back();
  ++e->graph_captures;
  return AL_OK;
}

void remember_key(al_engine* e, std::vector<uint64_t> key) {
  if (e->seen_keys.size() >= 2 * kMaxGraphs) e->seen_keys.erase(e->seen_keys.begin());
  e->seen_keys.push_back(std::move(key));
}

template <class TF>
int run_step(al_engine* e, int method, const typename FluidT<TF>::cn* cn, const al_consti* cni,
             const typename FluidT<TF>::type* f, const typename FluidT<TF>::body* bodies,
             typename FluidT<TF>::rigid* rigid, const al_solver_params* sp, TF* dt,
             al_step_report* report, cudaStream_t st, const al_warm_start* warm = nullptr) {
  ALB_TRY(e->activate());
  e->ns.clear();
  StepArgs<TF> A;
  A.iisph = method == kMethodIi;
  A.isph = method == kMethodI;
  A.cn = cn;
  A.cni = cni;
  A.f = f;
  A.bodies = bodies;
  A.rigid = rigid;
  A.sp = sp;
  A.dt = dt;
  A.report = report;
  A.warm = warm;
  StepPlan<TF> P;
  ALB_TRY(prepare_step<TF>(e, A, P, 0, 1));
  // ---- launch: a cached graph when this configuration ran before, else
  // eagerly (the first run of a configuration sizes every scratch buffer)
  const bool use_graph = e->graph_mode && !e->profiling && P.S.n > 0;
  al_engine::Graph* graph = nullptr;
  if (use_graph)
    ALB_TRY(find_or_capture(e, step_key<TF>(e, P, cn, cni),
                            [&](cudaGraphExec_t* x, uint32_t* fl) {
                              return capture_step<TF>(e, P, x, fl);
                            },
                            &graph));
  if (graph) {
    ALB_CUDA(cudaGraphLaunch(graph->exec, st));
    ++e->graph_replays;
  } else {
    ALB_TRY(enqueue_step<TF>(e, P, st, false, nullptr));
  }
  ALB_CUDA(cudaStreamSynchronize(st));
  e->flush_stats();
  // remember the configuration with the scratch generation it left
  if (use_graph && !graph) remember_key(e, step_key<TF>(e, P, cn, cni));
  const al_step_report& r = P.io.hc->rep;
  if (graph)
    e->launches += graph->fixed_launches +
                   uint64_t(iteration_launches(P)) *
                       (uint64_t(r.num_divergence_solve) + r.num_density_solve) +
                   (P.learned && P.io.hc->warm_ran ? kWarmIfLaunches : 0u);
  return finish_step<TF>(A, P);
}

// ------------------------------------------------------------ batched steps
// Every scene of a batch keeps its scratch under its own namespace and its
// own staging slot; a batch is captured as one graph whose branches (one
// per scene, forked from and joined to the capture stream) are the scenes'
// whole steps, each with its own conditional solver loops.  One launch and
// one synchronisation advance every scene; the branches' kernels overlap on
// the GPU.
std::string batch_ns(uint32_t k) { return "batch" + std::to_string(k) + "."; }

template <class TF>
int capture_batch(al_engine* e, std::vector<StepPlan<TF>>& plans, cudaGraphExec_t* exec,
                  uint32_t* fixed) {
  *exec = nullptr;
  const uint32_t K = uint32_t(plans.size());
  ALB_TRY(e->capture_streams());
  ALB_TRY(e->branches(K));
  cudaStream_t cs = e->capture_stream;
  const uint64_t launches0 = e->launches;
  const uint64_t gen0 = e->generation;
  ALB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = AL_OK, loops = 0;
  cudaError_t ce = cudaEventRecord(e->fork_event, cs);
  for (uint32_t k = 0; k < K && rc == AL_OK && ce == cudaSuccess; ++k) {
    cudaStream_t bs = e->branch_streams[k];
    ce = cudaStreamWaitEvent(bs, e->fork_event, 0);
    if (ce != cudaSuccess) break;
    e->ns = batch_ns(k);
    rc = enqueue_step<TF>(e, plans[k], bs, true, &loops);
    if (rc != AL_OK) break;
    ce = cudaEventRecord(e->join_events[k], bs);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cs, e->join_events[k], 0);
  }
  e->ns.clear();
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(cs, &graph);
  const uint64_t captured = e->launches - launches0;
  e->launches = launches0;
  if (rc != AL_OK || ce != cudaSuccess || end != cudaSuccess || e->generation != gen0) {
    if (graph) cudaGraphDestroy(graph);
    if (rc != AL_OK) return rc;
    ALB_CUDA(ce);
    ALB_CUDA(end);
    return AL_OK;
  }
  const cudaError_t inst = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) *exec = nullptr;
  ALB_CUDA(inst);
  *fixed = uint32_t(captured - 2u * uint32_t(loops));
  return AL_OK;
}

template <class TF>
std::vector<uint64_t> batch_key(al_engine* e, const std::vector<StepArgs<TF>>& args,
                                const std::vector<StepPlan<TF>>& plans) {
  std::vector<uint64_t> key{0xBA7C4ull, uint64_t(args.size())};
  for (size_t k = 0; k < args.size(); ++k) {
    const std::vector<uint64_t> kk = step_key<TF>(e, plans[k], args[k].cn, args[k].cni);
    key.insert(key.end(), kk.begin(), kk.end());
  }
  return key;
}

// ------------------------------------------------------------ fused batches
// A fused batch runs each pass of all its scenes as one launch.  The
// scenes' cell-sorted particles share one arena (scene k at slots
// [s0_k, s0_k + n_k), s0_k a multiple of kFusedAlign, so every
// kFusedBlock-slot block belongs to one scene), the neighbor lists and
// boundary terms are slot-major over the whole arena (the lists hold arena
// slots), and each block of a pass finds its scene in a block -> scene
// table (block_scene) for the scene's dt, control block, bodies and
// reductions.  The sort is one counting sort over all scenes' cells
// (grid_build_fused); gather, boundary sampling and the neighbor build take
// each block's scene grid and buffers from per-scene tables; the write-back
// goes to each scene's own buffers; the control blocks, bodies and rigid
// state travel in one device copy of the batch's staging.  The solver
// loops are one WHILE loop over all scenes: a scene whose solve has
// converged sits out the remaining iterations and the loop ends when no
// scene iterates again, so each scene runs exactly its own iterations.
// Pair passes run one thread per particle in kFusedBlock-thread blocks;
// every reduction of a scene covers its own blocks in the order a single
// step's 128-thread launch would, so with those shapes in the shape table's
// batch context the branch and the fused batch give bit-identical results.
constexpr uint32_t kFusedBlock = 128;
constexpr uint32_t kFusedAlign = 256;

static_assert(kFusedBlock == uint32_t(kBlock), "fused passes share the arena's block map");

template <class TF>
struct FusedPlan {
  uint32_t K = 0, N = 0, nblocks = 0, nbmax = 1;
  StepState<TF> S;           // the arena, as the fused passes see it
  const BuildScene* build = nullptr;         // device [K]
  const BoundaryScene<TF>* bnd = nullptr;    // device [K]
  const SortScene<TF>* sort = nullptr;       // device [K]
  uint32_t ncells = 0;       // the scenes' concatenated cells (tails, padding)
  uint32_t* go = nullptr;    // device: 1 while some scene iterates again
  uint32_t* hgo = nullptr;   // pinned readback of `go` (eager loops)
  // the scenes' staging slots (pinned, contiguous) and their device copy
  void* stage_host = nullptr;
  void* stage_dev = nullptr;
  size_t stage_bytes = 0;
  size_t ft_words = 0;       // rigid slots of all scenes (S.ft)
};

// Starts the solver loop of every scene (k_loop_begin) and sets the loop
// condition: some scene iterates.
template <class TF>
__global__ void k_fused_loop_begin(const FusedScene<TF>* __restrict__ sc, uint32_t K,
                                   int density_solve, uint32_t* go,
                                   cudaGraphConditionalHandle handle, int use_handle) {
  uint32_t any = 0;
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) {
    Ctrl<TF>& C = *sc[k].ctrl;
    C.it = 0;
    C.ticket = 0;
    C.keep_going = (density_solve ? C.max_den : C.max_div) > 0 ? 1u : 0u;
    any |= C.keep_going;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    *go = any;
    if (use_handle) cudaGraphSetConditional(handle, any);
  }
}

// Condition of the next iteration of a fused solver loop.
template <class TF>
__global__ void k_fused_loop_cond(const FusedScene<TF>* __restrict__ sc, uint32_t K,
                                  uint32_t* go, cudaGraphConditionalHandle handle,
                                  int use_handle) {
  uint32_t any = 0;
  for (uint32_t k = threadIdx.x; k < K; k += blockDim.x) any |= sc[k].ctrl->keep_going;
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    *go = any;
    if (use_handle) cudaGraphSetConditional(handle, any);
  }
}

// The scene view of the per-scene kernels below.
template <class TF>
__device__ __forceinline__ StepState<TF> scene_view(const FusedScene<TF>& f) {
  StepState<TF> V;
  V.n = f.n;
  V.nb = f.nb;
  V.ctrl = f.ctrl;
  V.bodies = f.bodies;
  V.rigid = f.rigid;
  V.ft = f.ft;
  return V;
}

// Block k: scene k's step initialisation (k_step_init) and cleared anomaly
// flags.
template <class TF>
__global__ void k_fused_step_init(const FusedScene<TF>* __restrict__ sc) {
  const FusedScene<TF>& f = sc[blockIdx.x];
  if (threadIdx.x < 4) f.flags[threadIdx.x] = 0u;
  step_init(scene_view(f));
}

// Rigid totals of every scene (the two stages of a single step's rigid
// finish, in the same chunking): block (c, b, k) sums chunk c of body b of
// scene k when the scene has more slots than kRigidChunks.
template <class TF>
__global__ void k_fused_rigid_partial(const FusedScene<TF>* __restrict__ sc) {
  const FusedScene<TF>& f = sc[blockIdx.z];
  if (blockIdx.y >= f.nb || f.nblk <= kRigidChunks) return;
  rigid_partial(f.ft, f.nblk, f.nb, f.ftp, blockIdx.y, blockIdx.x);
}

// Block (b, k): body b of scene k's totals and integration.
template <class TF>
__global__ void k_fused_rigid_finish(const FusedScene<TF>* __restrict__ sc) {
  const FusedScene<TF>& f = sc[blockIdx.y];
  if (blockIdx.x >= f.nb) return;
  const bool chunked = f.nblk > kRigidChunks;
  rigid_finish(scene_view(f), chunked ? f.ftp : f.ft, chunked ? kRigidChunks : f.nblk,
               blockIdx.x);
}

// Whether a batch can run fused: DFSPH scenes with particles, one set of
// constants, the same solves enabled, no periodic wrap.
template <class TF>
bool fusable(const std::vector<StepArgs<TF>>& args) {
  for (const StepArgs<TF>& a : args) {
    if (a.iisph || a.isph || a.warm || !a.f || !a.sp || !a.cn || !a.cni) return false;
    if (a.f->num_particles == 0 || a.sp->wrap_y) return false;
    if (std::memcmp(a.cn, args[0].cn, sizeof(*a.cn)) != 0) return false;
    if (a.sp->enable_divergence_solve != args[0].sp->enable_divergence_solve ||
        a.sp->enable_density_solve != args[0].sp->enable_density_solve)
      return false;
  }
  return !args.empty();
}

// Places the scenes (prepared without their own particle scratch) in the
// arena, fills the block -> scene table and uploads it when it changed.
template <class TF>
int fused_prepare(al_engine* e, std::vector<StepPlan<TF>>& plans, FusedPlan<TF>& F,
                  cudaStream_t st) {
  const uint32_t K = uint32_t(plans.size());
  std::vector<uint32_t> s0(K);
  uint64_t N = 0;
  std::vector<uint32_t> cell0(K);
  uint64_t C = 0;
  uint32_t nbmax = 1, cap = 1;
  size_t ft_words = 0, ftp_words = 0;
  for (uint32_t k = 0; k < K; ++k) {
    const StepState<TF>& Sk = plans[k].S;
    cell0[k] = uint32_t(C);
    C += uint64_t(plans[k].g.ncells) + 2;  // cells, out-of-grid tail, padding
    ALB_CHECK_ARG(C < (uint64_t(1) << 31), "al_df_batch_step_f32: too many grid cells in all");
    s0[k] = uint32_t(N);
    N = (N + Sk.n + kFusedAlign - 1) / kFusedAlign * kFusedAlign;
    ALB_CHECK_ARG(N < (uint64_t(1) << 31), "al_df_batch_step_f32: too many particles in all");
    nbmax = std::max(nbmax, Sk.nb);
    cap = std::max(cap, Sk.cap);
    const size_t nbk = Sk.nb ? Sk.nb : 1;
    ft_words += size_t(blocks_for(Sk.n, kFusedBlock)) * nbk * 6;
    ftp_words += size_t(kRigidChunks) * nbk * 6;
  }
  F.K = K;
  F.N = uint32_t(N);
  F.nblocks = F.N / kFusedBlock;
  StepState<TF> A = plans[0].S;
  FusedScene<TF>* table = nullptr;
  uint32_t* blk = nullptr;
  double* ftp = nullptr;
  e->ns = "fused.";
  ALB_TRY(e->buf("sorted.x", size_t(N) + kSortedPad, &A.x));
  ALB_TRY(e->buf("sorted.rec", size_t(N) * 2, &A.rec));
  ALB_TRY(e->buf("sorted.a", N, &A.a));
  ALB_TRY(e->buf("sorted.rho", N, &A.rho));
  ALB_TRY(e->buf("sorted.alpha", N, &A.alpha));
  ALB_TRY(e->buf("sorted.rho_adv", N, &A.rho_adv));
  ALB_TRY(e->buf("sorted.kappa", N, &A.kappa));
  ALB_TRY(e->buf("sorted.kappa_v", N, &A.kappa_v));
  ALB_TRY(e->buf("nbr.list", size_t(N) * cap, &A.nbr));
  ALB_TRY(e->buf("nbr.count", N, &A.ncount));
  ALB_TRY(e->buf("bnd.mask", N, &A.mask));
  ALB_TRY(e->buf("bnd.x", size_t(nbmax) * N, &A.bx));
  ALB_TRY(e->buf("bnd.k", size_t(nbmax) * N, &A.bk));
  using L = StagingLayout<TF>;
  char* stage = nullptr;
  ALB_TRY(e->buf("stage", L::bytes * K, &stage));
  ALB_TRY(e->buf("ft", ft_words, &A.ft));
  ALB_TRY(e->buf("ftp", ftp_words, &ftp));
  ALB_TRY(e->buf("red", F.nblocks, &A.red));
  ALB_TRY(e->buf("table", K, &table));
  ALB_TRY(e->buf("blk_scene", F.nblocks, &blk));
  ALB_TRY(e->buf("go", 1, &F.go));
  FusedIo<TF>* io = nullptr;
  BuildScene* build = nullptr;
  BoundaryScene<TF>* bnd = nullptr;
  SortScene<TF>* sort = nullptr;
  ALB_TRY(e->buf("io", K, &io));
  ALB_TRY(e->buf("build", K, &build));
  ALB_TRY(e->buf("bnd", K, &bnd));
  ALB_TRY(e->buf("sort", K, &sort));
  // the buffers grid_build_fused will use for the permutation and cell starts
  uint32_t *perm = nullptr, *cell_start = nullptr;
  ALB_TRY(e->buf("grid.perm", N, &perm));
  ALB_TRY(e->buf("grid.start", size_t(C) + 2, &cell_start));
  e->ns.clear();
  std::vector<FusedScene<TF>> tab(K);
  std::vector<FusedIo<TF>> hio(K);
  std::vector<BuildScene> hbuild(K);
  std::vector<BoundaryScene<TF>> hbnd(K);
  std::vector<SortScene<TF>> hsort(K);
  std::vector<uint32_t> hblk(F.nblocks, K);
  size_t ft_off = 0, ftp_off = 0;
  for (uint32_t k = 0; k < K; ++k) {
    StepPlan<TF>& P = plans[k];
    StepState<TF>& Sk = P.S;
    const uint32_t o = s0[k], n = Sk.n, nb = Sk.nb, nbk = nb ? nb : 1;
    const uint32_t nblk = blocks_for(n, kFusedBlock), blk0 = o / kFusedBlock;
    Sk.ls = F.N;
    Sk.x = A.x + o;
    Sk.rec = A.rec + 2 * size_t(o);
    Sk.a = A.a + o;
    Sk.rho = A.rho + o;
    Sk.alpha = A.alpha + o;
    Sk.rho_adv = A.rho_adv + o;
    Sk.kappa = A.kappa + o;
    Sk.kappa_v = A.kappa_v + o;
    Sk.nbr = A.nbr + o;
    Sk.ncount = A.ncount + o;
    Sk.mask = A.mask + o;
    Sk.bx = A.bx + o;
    Sk.bk = A.bk + o;
    // control block, bodies, rigid state and flags in the device copy of
    // the scene's staging slot
    char* slot = stage + L::bytes * k;
    Sk.ctrl = reinterpret_cast<Ctrl<TF>*>(slot);
    P.bodies_dev = reinterpret_cast<BodyDev<TF>*>(slot + L::bodies);
    Sk.bodies = P.bodies_dev;
    Sk.rigid = reinterpret_cast<RigidDev<TF>*>(slot + L::rigid);
    P.flags = reinterpret_cast<uint32_t*>(slot + L::flag + 64);
    Sk.ft = A.ft + ft_off;
    Sk.grid = nblk;
    Sk.red = A.red + blk0;
    P.ftp = ftp + ftp_off;
    ft_off += size_t(nblk) * nbk * 6;
    ftp_off += size_t(kRigidChunks) * nbk * 6;
    tab[k] = FusedScene<TF>{o,        n,          blk0,  nblk,   nb,      0u,
                            Sk.ctrl,  Sk.bodies,  Sk.rigid, Sk.ft, P.ftp, Sk.red, P.flags};
    const auto* f = P.f;
    hio[k] = FusedIo<TF>{f->particle_x,      f->particle_v,     f->particle_kappa,
                         f->particle_kappa_v, f->particle_x,   f->particle_v,
                         f->particle_a,     f->particle_density, f->particle_dfsph_factor,
                         f->particle_kappa, f->particle_kappa_v, f->particle_density_adv};
    hbuild[k] = BuildScene{P.g, cell_start + cell0[k], P.flags, o, n};
    hbnd[k] = BoundaryScene<TF>{Sk.bodies, Sk.rigid, perm, f->particle_boundary,
                                f->particle_boundary_kernel,
                                &Sk.ctrl->rep.num_active_boundary_pairs, nb, o, n, 0u};
    const uint32_t next = k + 1 < K ? s0[k + 1] : F.N;
    hsort[k] = SortScene<TF>{f->particle_x, P.g, cell0[k], o, n, next - o - n, P.flags};
    for (uint32_t b = blk0; b < blk0 + nblk; ++b) hblk[b] = k;
  }
  A.n = F.N;
  A.ls = F.N;
  A.tpp = 1;
  A.grid = F.nblocks;
  A.perm = perm;
  A.blk_scene = blk;
  A.fused = table;
  A.io = io;
  A.nscenes = K;
  F.S = A;
  F.build = build;
  F.bnd = bnd;
  F.sort = sort;
  F.ncells = uint32_t(C);
  F.hgo = plans[0].io.hflag;
  F.nbmax = nbmax;
  F.stage_host = plans[0].io.hc;  // slot 0 starts the pinned block
  F.stage_dev = stage;
  F.stage_bytes = L::bytes * K;
  F.ft_words = ft_words;
  // upload the tables when they (or their buffers) changed
  struct Part {
    void* dev;
    const void* host;
    size_t bytes;
  };
  const Part parts[] = {{table, tab.data(), sizeof(FusedScene<TF>) * K},
                        {blk, hblk.data(), sizeof(uint32_t) * F.nblocks},
                        {io, hio.data(), sizeof(FusedIo<TF>) * K},
                        {build, hbuild.data(), sizeof(BuildScene) * K},
                        {bnd, hbnd.data(), sizeof(BoundaryScene<TF>) * K},
                        {sort, hsort.data(), sizeof(SortScene<TF>) * K}};
  std::vector<unsigned char> bytes;
  for (const Part& pt : parts) {
    const unsigned char* h = static_cast<const unsigned char*>(pt.host);
    const unsigned char* d = reinterpret_cast<const unsigned char*>(&pt.dev);
    bytes.insert(bytes.end(), d, d + sizeof(pt.dev));
    bytes.insert(bytes.end(), h, h + pt.bytes);
  }
  if (bytes != e->fused_tables) {
    for (const Part& pt : parts)
      ALB_CUDA(cudaMemcpyAsync(pt.dev, pt.host, pt.bytes, cudaMemcpyHostToDevice, st));
    ALB_CUDA(cudaStreamSynchronize(st));
    e->fused_tables.swap(bytes);
  }
  return AL_OK;
}

// The fused passes of a batch after the scenes' grid sorts: gather,
// boundary sampling and neighbor build (with the divergence warm start's
// first pass), each one launch over the arena.
template <class TF>
int enqueue_fused_head(al_engine* e, const StepPlan<TF>& P0, FusedPlan<TF>& F, cudaStream_t st) {
  const Cn<TF>& c = P0.c;
  const StepState<TF>& S = F.S;
  const uint32_t G = F.nblocks, B = kFusedBlock;
  ALB_LAUNCH(e, "gather_state", 1, st,
             (k_gather_state<TF, true, true><<<G, B, 0, st>>>(S, nullptr, nullptr, nullptr)));
  ALB_LAUNCH(e, "boundary", 1, st,
             ALB_TRY(sample_boundaries_fused<TF>(c, S.x, F.N, S.blk_scene, F.bnd, F.K, G, S.mask,
                                                 S.bx, S.bk, st)));
  const SortedBoundaryKernel<TF> sbk{S.mask, S.bk, F.N};
  TF* rho_rec = reinterpret_cast<TF*>(S.rec) + 7;  // rec[2s + 1].w
  const FusedBuild fb{S.blk_scene, F.build, F.K};
  if (P0.div) {
    const WarmDivergence<TF> wd{S, nullptr, nullptr, c.radius * TF(2), c.vol, nullptr};
    ALB_LAUNCH(e, "neighbors", 1, st,
               (k_build_neighbors<TF, SortedBoundaryKernel<TF>, true, WarmDivergence<TF>, false,
                                  true><<<G, B, 0, st>>>(c, GridDims{}, nullptr, S.x, 0u, F.N,
                                                         sbk, S.nbr, S.ncount, S.rho, S.alpha,
                                                         rho_rec, nullptr, wd, fb)));
  } else {
    ALB_LAUNCH(e, "neighbors", 1, st,
               (k_build_neighbors<TF, SortedBoundaryKernel<TF>, true, NoExtra<TF>, false, true>
                    <<<G, B, 0, st>>>(c, GridDims{}, nullptr, S.x, 0u, F.N, sbk, S.nbr, S.ncount,
                                      S.rho, S.alpha, rho_rec, nullptr, NoExtra<TF>{}, fb)));
  }
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

// The fused solves of a batch: every pass one launch over the arena.
template <class TF>
int enqueue_fused_solve(al_engine* e, const StepPlan<TF>& P0, FusedPlan<TF>& F, cudaStream_t st,
                        bool capture, int* loops) {
  const Cn<TF>& c = P0.c;
  const StepState<TF>& S = F.S;
  const uint32_t G = F.nblocks, B = kFusedBlock;
  auto solve = [&](int density_solve, auto&& body) -> int {
    if (capture) {
      ++*loops;
      return capture_while(
          e, st,
          [&](cudaGraphConditionalHandle h) -> int {
            ALB_LAUNCH(e, "loop_begin", 1, st,
                       (k_fused_loop_begin<TF><<<1, 256, 0, st>>>(S.fused, F.K, density_solve,
                                                                   F.go, h, 1)));
            return AL_OK;
          },
          body);
    }
    ALB_LAUNCH(e, "loop_begin", 1, st,
               (k_fused_loop_begin<TF><<<1, 256, 0, st>>>(S.fused, F.K, density_solve, F.go,
                                                           cudaGraphConditionalHandle(0), 0)));
    for (;;) {
      ALB_CUDA(cudaMemcpyAsync(F.hgo, F.go, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
      ALB_CUDA(cudaStreamSynchronize(st));
      if (!*F.hgo) break;
      ALB_TRY(body(st, cudaGraphConditionalHandle(0), 0));
    }
    return AL_OK;
  };
  auto cond = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
    ALB_LAUNCH(e, "loop_cond", 1, s,
               (k_fused_loop_cond<TF><<<1, 256, 0, s>>>(S.fused, F.K, F.go, h, use)));
    return AL_OK;
  };
  const cudaGraphConditionalHandle none(0);
  if (P0.div) {
    ALB_LAUNCH(e, "div_warm1", 1, st, (k_kappa<TF, kDivWarm, false, true><<<G, B, 0, st>>>(c, S)));
    ALB_LAUNCH(e, "div_rho_adv", 1, st,
               (k_df_rho_adv_init<TF, false, true><<<G, B, 0, st>>>(c, S)));
    ALB_TRY(solve(0, [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
      ALB_LAUNCH(e, "div_iter", 1, s, (k_kappa<TF, kDivIter, false, true><<<G, B, 0, s>>>(c, S)));
      ALB_LAUNCH(e, "div_residual", 1, s,
                 (k_df_residual<TF, false, true><<<G, B, 0, s>>>(c, S, none, 0)));
      return cond(s, h, use);
    }));
  }
  ALB_LAUNCH(e, "viscosity", 1, st,
             (k_viscosity<TF, false, true><<<G, B, 0, st>>>(c, S, P0.div ? 1 : 0)));
  ALB_LAUNCH(e, "integrate_np", 1, st, (k_integrate_np<TF, true><<<G, B, 0, st>>>(S)));
  if (P0.den) {
    ALB_LAUNCH(e, "press_warm0", 1, st,
               (k_p_warm0<TF, false, true><<<G, B, 0, st>>>(c, S, nullptr, nullptr)));
    ALB_LAUNCH(e, "press_warm1", 1, st,
               (k_kappa<TF, kPressWarm, false, true><<<G, B, 0, st>>>(c, S)));
    ALB_LAUNCH(e, "press_rho_adv", 1, st,
               (k_p_rho_adv_init<TF, false, true><<<G, B, 0, st>>>(c, S)));
    ALB_TRY(solve(1, [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) -> int {
      ALB_LAUNCH(e, "press_iter", 1, s,
                 (k_kappa<TF, kPressIter, false, true><<<G, B, 0, s>>>(c, S)));
      ALB_LAUNCH(e, "press_residual", 1, s,
                 (k_p_residual<TF, false, true><<<G, B, 0, s>>>(c, S, none, 0)));
      return cond(s, h, use);
    }));
  }
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

// Kernels of one iteration of a fused solver loop (update, residual, loop
// condition).
constexpr uint32_t kFusedIterationLaunches = 3;

// Enqueues a fused batch on `st`: one upload of every scene's staging, one
// counting sort over all scenes' cells, every other pass one launch over all
// scenes, one readback.
template <class TF>
int enqueue_fused_batch(al_engine* e, std::vector<StepPlan<TF>>& plans, FusedPlan<TF>& F,
                        cudaStream_t st, bool capture, int* loops) {
  const uint32_t K = uint32_t(plans.size());
  const StepState<TF>& S = F.S;
  ALB_CUDA(cudaMemcpyAsync(F.stage_dev, F.stage_host, F.stage_bytes, cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemsetAsync(S.ft, 0, F.ft_words * sizeof(double), st));
  ALB_LAUNCH(e, "step_init", 1, st, (k_fused_step_init<TF><<<K, 32, 0, st>>>(S.fused)));
  GridState gs;
  e->ns = "fused.";
  ALB_LAUNCH(e, "grid_sort", grid_fused_kernels(F.ncells), st,
             ALB_TRY(grid_build_fused<TF>(e, plans[0].c.h, S.blk_scene, F.sort, K, F.N, F.ncells,
                                          gs, st)));
  e->ns.clear();
  ALB_TRY(enqueue_fused_head<TF>(e, plans[0], F, st));
  ALB_TRY(enqueue_fused_solve<TF>(e, plans[0], F, st, capture, loops));
  ALB_LAUNCH(e, "finish", 1, st,
             (k_df_finish<TF, false, true><<<F.nblocks, kFusedBlock, 0, st>>>(
                 plans[0].c, S, plans[0].den ? 1 : 0, nullptr, nullptr, nullptr, nullptr, nullptr,
                 nullptr, nullptr, nullptr, nullptr)));
  ALB_LAUNCH(e, "rigid_finish", 2, st,
             (k_fused_rigid_partial<TF><<<dim3(kRigidChunks, F.nbmax, K), 256, 0, st>>>(S.fused),
              k_fused_rigid_finish<TF><<<dim3(F.nbmax, K), 256, 0, st>>>(S.fused)));
  ALB_CUDA(cudaGetLastError());
  ALB_CUDA(cudaMemcpyAsync(F.stage_host, F.stage_dev, F.stage_bytes, cudaMemcpyDeviceToHost, st));
  return AL_OK;
}

template <class TF>
int capture_batch_fused(al_engine* e, std::vector<StepPlan<TF>>& plans, FusedPlan<TF>& F,
                        cudaGraphExec_t* exec, uint32_t* fixed) {
  *exec = nullptr;
  ALB_TRY(e->capture_streams());
  cudaStream_t cs = e->capture_stream;
  const uint64_t launches0 = e->launches;
  const uint64_t gen0 = e->generation;
  ALB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int loops = 0;
  const int rc = enqueue_fused_batch<TF>(e, plans, F, cs, true, &loops);
  e->ns.clear();
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(cs, &graph);
  const uint64_t captured = e->launches - launches0;
  e->launches = launches0;
  if (rc != AL_OK || end != cudaSuccess || e->generation != gen0) {
    if (graph) cudaGraphDestroy(graph);
    if (rc != AL_OK) return rc;
    ALB_CUDA(end);
    return AL_OK;
  }
  const cudaError_t inst = cudaGraphInstantiate(exec, graph, 0);
  cudaGraphDestroy(graph);
  if (inst != cudaSuccess) *exec = nullptr;
  ALB_CUDA(inst);
  *fixed = uint32_t(captured - kFusedIterationLaunches * uint32_t(loops));
  return AL_OK;
}

template <class TF>
int run_batch(al_engine* e, const std::vector<StepArgs<TF>>& args, std::vector<int>& status,
              cudaStream_t st) {
  ALB_TRY(e->activate());
  struct NsReset {
    al_engine* e;
    ~NsReset() { e->ns.clear(); }
  } reset{e};
  const uint32_t K = uint32_t(args.size());
  const bool fused = e->batch_fused && fusable<TF>(args);
  std::vector<StepPlan<TF>> plans(K);
  bool nonempty = true;
  for (uint32_t k = 0; k < K; ++k) {
    e->ns = batch_ns(k);
    ALB_TRY(prepare_step<TF>(e, args[k], plans[k], k, K, !fused));
    nonempty = nonempty && plans[k].S.n > 0;
  }
  e->ns.clear();
  // A fused batch's arena and tables follow from what the key holds (the
  // scenes' buffers and sizes, the scratch generation): a replay of its
  // captured graph needs them placed again only when another fused batch
  // used the tables since.
  FusedPlan<TF> F;
  bool placed = false;
  auto key = [&]() {
    std::vector<uint64_t> k = batch_key<TF>(e, args, plans);
    if (fused) k.push_back(0xF05EDull);
    return k;
  };
  auto place = [&]() -> int {
    if (!placed) ALB_TRY(fused_prepare<TF>(e, plans, F, st));
    placed = true;
    e->fused_key = key();
    return AL_OK;
  };
  const bool use_graph = e->graph_mode && !e->profiling && nonempty;
  const std::vector<uint64_t> key0 = key();
  al_engine::Graph* graph = nullptr;
  if (use_graph)
    ALB_TRY(find_or_capture(e, key0,
                            [&](cudaGraphExec_t* x, uint32_t* fl) -> int {
                              if (!fused) return capture_batch<TF>(e, plans, x, fl);
                              ALB_TRY(place());
                              return capture_batch_fused<TF>(e, plans, F, x, fl);
                            },
                            &graph));
  if (graph) {
    if (fused && e->fused_key != key0) ALB_TRY(place());
    ALB_CUDA(cudaGraphLaunch(graph->exec, st));
    ++e->graph_replays;
  } else if (fused) {
    ALB_TRY(place());
    ALB_TRY(enqueue_fused_batch<TF>(e, plans, F, st, false, nullptr));
  } else {
    for (uint32_t k = 0; k < K; ++k) {
      e->ns = batch_ns(k);
      ALB_TRY(enqueue_step<TF>(e, plans[k], st, false, nullptr));
    }
    e->ns.clear();
  }
  ALB_CUDA(cudaStreamSynchronize(st));
  e->flush_stats();
  if (use_graph && !graph) remember_key(e, key());
  status.assign(K, AL_OK);
  uint64_t iters = 0;
  uint32_t max_div = 0, max_den = 0;
  for (uint32_t k = 0; k < K; ++k) {
    const al_step_report& r = plans[k].io.hc->rep;
    iters += uint64_t(r.num_divergence_solve) + r.num_density_solve;
    max_div = std::max(max_div, r.num_divergence_solve);
    max_den = std::max(max_den, r.num_density_solve);
    status[k] = finish_step<TF>(args[k], plans[k]);
  }
  if (graph)
    e->launches += graph->fixed_launches +
                   (fused ? uint64_t(kFusedIterationLaunches) * (max_div + max_den) : 2ull * iters);
  for (int s : status)
    if (s != AL_OK) return s;
  return AL_OK;
}

}  // namespace

}  // namespace alb

using namespace alb;

extern "C" {

int al_df_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                   const al_fluid_f32* fluid, const al_body_f32* bodies, al_rigid_f32* rigid,
                   const al_solver_params* params, float* dt, al_step_report* report,
                   void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_df_step: null argument");
  return run_step<float>(engine, kMethodDf, cn, cni, fluid, bodies, rigid, params, dt, report,
                         static_cast<cudaStream_t>(stream));
}
int al_df_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                   const al_fluid_f64* fluid, const al_body_f64* bodies, al_rigid_f64* rigid,
                   const al_solver_params* params, double* dt, al_step_report* report,
                   void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_df_step: null argument");
  return run_step<double>(engine, kMethodDf, cn, cni, fluid, bodies, rigid, params, dt, report,
                          static_cast<cudaStream_t>(stream));
}
int al_df_step_warm_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                        const al_fluid_f32* fluid, const al_body_f32* bodies,
                        al_rigid_f32* rigid, const al_solver_params* params,
                        const al_warm_start* warm, float* dt, al_step_report* report,
                        void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_df_step_warm_f32: null argument");
  return run_step<float>(engine, kMethodDf, cn, cni, fluid, bodies, rigid, params, dt, report,
                         static_cast<cudaStream_t>(stream), warm);
}
int al_ii_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                   const al_fluid_f32* fluid, const al_body_f32* bodies, al_rigid_f32* rigid,
                   const al_solver_params* params, float* dt, al_step_report* report,
                   void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_ii_step: null argument");
  return run_step<float>(engine, kMethodIi, cn, cni, fluid, bodies, rigid, params, dt, report,
                         static_cast<cudaStream_t>(stream));
}
int al_ii_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                   const al_fluid_f64* fluid, const al_body_f64* bodies, al_rigid_f64* rigid,
                   const al_solver_params* params, double* dt, al_step_report* report,
                   void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_ii_step: null argument");
  return run_step<double>(engine, kMethodIi, cn, cni, fluid, bodies, rigid, params, dt, report,
                          static_cast<cudaStream_t>(stream));
}

int al_i_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                  const al_fluid_f32* fluid, const al_body_f32* bodies, al_rigid_f32* rigid,
                  const al_solver_params* params, float* dt, al_step_report* report,
                  void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_i_step: null argument");
  return run_step<float>(engine, kMethodI, cn, cni, fluid, bodies, rigid, params, dt, report,
                         static_cast<cudaStream_t>(stream));
}
int al_i_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                  const al_fluid_f64* fluid, const al_body_f64* bodies, al_rigid_f64* rigid,
                  const al_solver_params* params, double* dt, al_step_report* report,
                  void* stream) {
  ALB_CHECK_ARG(engine && cn, "al_i_step: null argument");
  return run_step<double>(engine, kMethodI, cn, cni, fluid, bodies, rigid, params, dt, report,
                          static_cast<cudaStream_t>(stream));
}

int al_engine_set_launch_shape(al_engine* engine, const char* group, uint32_t bucket,
                               uint32_t batch, uint32_t block, uint32_t tpp) {
  ALB_CHECK_ARG(engine && group, "al_engine_set_launch_shape: null argument");
  const TunableGroup* tg = nullptr;
  for (uint32_t k = 0; k < kNumTunable; ++k)
    if (std::string(kTunable[k].name) == group) tg = &kTunable[k];
  if (!tg) {
    set_error(std::string("al_engine_set_launch_shape: no tunable pass group '") + group + "'");
    return AL_ERR_INVALID;
  }
  ALB_CHECK_ARG(bucket < 32 && batch < 2, "al_engine_set_launch_shape: bucket < 32, batch 0 or 1");
  ALB_CHECK_ARG(block == 0 || block == 64 || block == 128 || block == 256,
                "al_engine_set_launch_shape: block must be 64, 128 or 256 (0: default)");
  ALB_CHECK_ARG(tpp == 0 || tpp == 1 || ((tpp == 2 || tpp == 4 || tpp == 8) && tg->pair),
                "al_engine_set_launch_shape: threads per particle 1, 2, 4 or 8 (pair passes "
                "only; 0: default)");
  const auto key = std::make_tuple(std::string(group), bucket, batch);
  if (block == 0 && tpp == 0)
    engine->shapes.erase(key);
  else
    engine->shapes[key] = std::make_pair(block, tpp);
  ALB_CUDA(cudaSetDevice(engine->device));
  engine->drop_graphs();  // captured steps hold the old shapes
  ++engine->generation;
  return AL_OK;
}

int al_engine_get_launch_shape(al_engine* engine, const char* group, uint32_t num_particles,
                               uint32_t batch, uint32_t* block, uint32_t* tpp) {
  ALB_CHECK_ARG(engine && group && block && tpp, "al_engine_get_launch_shape: null argument");
  const TunableGroup* tg = nullptr;
  for (uint32_t k = 0; k < kNumTunable; ++k)
    if (std::string(kTunable[k].name) == group) tg = &kTunable[k];
  if (!tg) {
    set_error(std::string("al_engine_get_launch_shape: no tunable pass group '") + group + "'");
    return AL_ERR_INVALID;
  }
  StepPlan<float> P;
  P.S.n = num_particles;
  P.bucket = num_particles ? uint32_t(31 - __builtin_clz(num_particles)) : 0u;
  P.ctx = batch ? 1u : 0u;
  const LaunchShape sh = P.shape(engine, group, tg->pair);
  *block = sh.block;
  *tpp = sh.tpp;
  return AL_OK;
}

int al_tunable_group(uint32_t index, const char** name, uint32_t* pair) {
  ALB_CHECK_ARG(name && pair, "al_tunable_group: null argument");
  if (index >= kNumTunable) {
    set_error("al_tunable_group: index past the last group");
    return AL_ERR_INVALID;
  }
  *name = kTunable[index].name;
  *pair = kTunable[index].pair ? 1u : 0u;
  return AL_OK;
}

int al_engine_set_batch_fused(al_engine* engine, int enable) {
  ALB_CHECK_ARG(engine, "al_engine_set_batch_fused: null engine");
  engine->batch_fused = enable != 0;
  return AL_OK;
}

int al_df_batch_step_f32(al_engine* engine, al_scene_f32* scenes, uint32_t num_scenes,
                         void* stream) {
  ALB_CHECK_ARG(engine && (num_scenes == 0 || scenes), "al_df_batch_step_f32: null argument");
  ALB_CHECK_ARG(num_scenes <= AL_MAX_BATCH, "al_df_batch_step_f32: too many scenes");
  if (num_scenes == 0) return AL_OK;
  std::vector<StepArgs<float>> args(num_scenes);
  for (uint32_t k = 0; k < num_scenes; ++k) {
    const al_scene_f32& sc = scenes[k];
    ALB_CHECK_ARG(sc.cn != nullptr, "al_df_batch_step_f32: scene constants are null");
    args[k].cn = sc.cn;
    args[k].cni = sc.cni;
    args[k].f = sc.fluid;
    args[k].bodies = sc.bodies;
    args[k].rigid = sc.rigid;
    args[k].sp = sc.params;
    args[k].dt = sc.dt;
    args[k].report = sc.report;
  }
  // launch shapes from the batch context of the shape table
  for (uint32_t k = 0; k < num_scenes; ++k) args[k].batch = 1;
  std::vector<int> status;
  const int rc = run_batch<float>(engine, args, status, static_cast<cudaStream_t>(stream));
  for (uint32_t k = 0; k < num_scenes; ++k)
    scenes[k].status = k < status.size() ? status[k] : rc;
  return rc;
}

}  // extern "C"
