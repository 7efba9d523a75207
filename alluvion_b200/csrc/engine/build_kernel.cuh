// build_kernel.cuh -- the neighbor-list build kernel with fused density
// and DFSPH factor, shared by the standalone neighbor update and the solver
// step (which adds a per-neighbor term through the EX hook).  Internal
// linkage: each translation unit that launches it compiles its own copy.
#pragma once

#include "neighbors.cuh"

namespace alb {

// What phase 2 of the build hands to the EX hook for particle s.
template <class TF>
struct BuildOut {
  uint32_t cnt;    // neighbors in the list
  TF div;          // sum_j V (v_i - v_j) . grad W_ij, list order
  vec3<TF> vi;     // the particle's velocity (EX::self_v)
  TF density;      // rho / rho0 (fluid + boundary terms)
  TF alpha;        // DFSPH factor (0 without FACTOR)
  TF grad_norm2;   // |sum_j V grad W_ij + sum_b (grad W V)_b|^2 (0 without FACTOR)
};

// A build launched over every scene of a fused batch: each scene's grid,
// cell starts, anomaly flags and range [s0, s0 + n) of the shared arena, and
// the scene of each block (nscenes for a block past every scene).
struct BuildScene {
  GridDims g;
  const uint32_t* cell_start;
  uint32_t* flags;
  uint32_t s0, n;
};
struct FusedBuild {
  const uint32_t* blk_scene = nullptr;
  const BuildScene* scenes = nullptr;
  uint32_t nscenes = 0;
};

// EX hook of k_build_neighbors that adds nothing.
template <class TF>
struct NoExtra {
  static constexpr bool kOn = false;
  __device__ __forceinline__ void narrow(uint32_t) {}
  __device__ __forceinline__ vec3<TF> self_v(uint32_t) const { return vec3<TF>{0, 0, 0}; }
  // neighbor t's position and velocity for phase 2 (the velocity unused)
  __device__ __forceinline__ void xv(const vec4<TF>* __restrict__ xs, uint32_t t, vec3<TF>& x,
                                     vec3<TF>& v) const {
    x = xyz(__ldg(xs + t));
    v = vec3<TF>{0, 0, 0};
  }
  __device__ __forceinline__ void finish(uint32_t, const BuildOut<TF>&) const {}
};

namespace {

// Candidates tested per round of the build's scan (loads issued together;
// measured on B200 per build at 8,388,608 / 1,048,576 particles: 2.79 / 0.354
// ms at 8, 2.84 / 0.358 at 4, 2.89 / 0.370 at 2, and 3.18 / 0.381 for a
// branch per candidate).
constexpr uint32_t kScan = 8;
static_assert(32 % kScan == 0 && kScan <= kSortedPad,
              "scan rounds must tile 32 and stay in the pad");

// Two phases per particle.  Phase 1 walks the 3x3 rows of z-contiguous
// cells around the particle's cell and appends every candidate closer than
// h to the list, in ascending sorted index; about 1 in 7 candidates is
// accepted, so the tests run without a branch per candidate and only the
// accepted ones pay for a store.  Phase 2 walks the compact list in
// the same order and evaluates W (and grad W for the DFSPH factor) only
// for neighbors, two list entries in flight at a time.  Both phases form
// d and |d|^2 with the same rounded operations, so phase 2 sees the
// distances phase 1 accepted.
//
// `EX` supplies the neighbors' positions (and velocities) for phase 2 and
// may add one more sum over the list (EX::kOn): it supplies the particle's
// and the neighbors' velocities and receives sum_j V (v_i - v_j) . grad W_ij,
// in list order, at the end.
//
// The list is slot-major with row stride `stride` (n for one scene).  With
// BT the launch covers every scene of a fused batch (fb): xs, the outputs
// and the cell starts are in arena slots, each block takes its scene's grid,
// cell starts and flags, and the scene's particle s0 + i looks only at the
// scene's own cells.
template <class TF, class BK, bool FACTOR, class EX, bool WR = false, bool BT = false>
__global__ void __launch_bounds__(kMaxBlock)
    k_build_neighbors(Cn<TF> c, GridDims g, const uint32_t* __restrict__ cell_start,
                      const vec4<TF>* __restrict__ xs, uint32_t n, uint32_t stride, BK bk,
                      uint32_t* __restrict__ nbr, uint32_t* __restrict__ ncount,
                      TF* __restrict__ rho, TF* __restrict__ alpha, TF* __restrict__ rho_rec,
                      uint32_t* __restrict__ flags, EX ex, FusedBuild fb) {
  if constexpr (!WR) c.wrap = 0;  // non-periodic: the wrap branches fold away
  uint32_t sl = blockIdx.x * blockDim.x + threadIdx.x, s0 = 0;
  if constexpr (BT) {
    const uint32_t k = __ldg(fb.blk_scene + blockIdx.x);
    if (k >= fb.nscenes) return;
    const BuildScene& sc = fb.scenes[k];
    g = sc.g;
    cell_start = sc.cell_start;
    flags = sc.flags;
    s0 = sc.s0;
    n = sc.n;
    sl -= s0;
    ex.narrow(k);
  }
  if (sl >= n) return;
  const uint32_t s = s0 + sl;  // the particle's slot in xs and the outputs
  const vec3<TF> xi = xyz(xs[s]);
  int ip[3];
  cell_coords(c.h, g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  const int z1 = min(ip[2] + 1, int(g.res[2]) - 1);
  uint32_t cnt = 0;
  // ---- phase 1: candidates -> list
  if (z0 <= z1) {
    for (int dx = -1; dx <= 1; ++dx) {
      const int cx = ip[0] + dx;
      if (cx < 0 || cx >= int(g.res[0])) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int cy = ip[1] + dy;
        if (c.wrap) {  // wrap_ipos_y (runner.hpp:689-697)
          if (cy >= int(g.res[1]))
            cy -= int(g.res[1]);
          else if (cy < 0)
            cy += int(g.res[1]);
        }
        if (cy < 0 || cy >= int(g.res[1])) continue;
        const uint32_t b = cell_start[cell_linear(g, cx, cy, z0)];
        const uint32_t e = cell_start[cell_linear(g, cx, cy, z1) + 1];
        // The row's candidates in chunks of 32: the distance tests set one
        // bit per accepted candidate (branch-free, kScan candidates per
        // round; a round may read up to kScan - 1 entries past the row, into
        // the next row or the buffer's kSortedPad spare entries, and their
        // bits are masked off), then the set bits are appended to the list
        // in ascending order.
        for (uint32_t t0 = b; t0 < e; t0 += 32) {
          const uint32_t m = min(e - t0, 32u);
          const vec4<TF>* xt = xs + t0;
          uint32_t acc = 0;
          for (uint32_t q = 0; q < m; q += kScan) {
            vec3<TF> xj[kScan];
#pragma unroll
            for (uint32_t u = 0; u < kScan; ++u) xj[u] = xyz(__ldg(xt + q + u));
            uint32_t bits = 0;
#pragma unroll
            for (uint32_t u = 0; u < kScan; ++u)
              bits |= uint32_t(pdist2(c, xi, xj[u]) < c.h2) << u;
            acc |= bits << q;
          }
          if (m < 32) acc &= (1u << m) - 1u;
          if (s - t0 < m) acc &= ~(1u << (s - t0));  // the particle itself
          for (; acc; acc &= acc - 1) {
            if (cnt < g.cap_nbr)
              nbr[size_t(cnt) * stride + s] = t0 + uint32_t(__ffs(acc) - 1);
            ++cnt;
          }
        }
      }
    }
  }
  if (cnt > g.cap_nbr) {
    flags[2] = 1u;
    cnt = g.cap_nbr;
  }
  ncount[s] = cnt;
  // ---- phase 2: density (+ factor, + EX) over the list, in list order
  TF density = c.vol * c.w0;
  TF sum_grad = 0;
  vec3<TF> grad_i{0, 0, 0};
  TF div = 0;
  const vec3<TF> vi = ex.self_v(s);
  // list entries per round (measured on B200 with the 256-bit record loads,
  // per build at 1,048,576 / 8,388,608 particles: 0.334 / 2.66 ms at 2,
  // 0.338 / 2.71 at 4, 0.367 / 2.90 at 8)
  constexpr uint32_t kB = 2;
  for (uint32_t k0 = 0; k0 < cnt; k0 += kB) {
    uint32_t t[kB];
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q)  // this thread's own stores: plain loads
      t[q] = k0 + q < cnt ? nbr[size_t(k0 + q) * stride + s] : s;
    vec3<TF> xj[kB], vj[kB];
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q) ex.xv(xs, t[q], xj[q], vj[q]);
#pragma unroll
    for (uint32_t q = 0; q < kB; ++q) {
      if (k0 + q >= cnt) break;
      density += c.vol * W_r2(c, pdist2(c, xi, xj[q]));
      if (FACTOR || EX::kOn) {
        const vec3<TF> d = pdisp(c, xi, xj[q]);
        const vec3<TF> gw = gradW(c, d);
        if (FACTOR) {
          const vec3<TF> gpj = (-c.vol) * gw;
          sum_grad += length_sqr(gpj);
          grad_i -= gpj;
        }
        if (EX::kOn) div += c.vol * dot(vi - vj[q], gw);
      }
    }
  }
  density += bk.density_term(s);
  rho[s] = density * c.rho0;
  if (rho_rec) rho_rec[size_t(s) * kRecStride] = density * c.rho0;
  TF a = 0, g2 = 0;
  if (FACTOR) {
    grad_i += bk.grad_term(s);
    g2 = length_sqr(grad_i);
    sum_grad += g2;
    a = sum_grad > c.eps ? TF(-1) / sum_grad : TF(0);
    alpha[s] = a;
  }
  if (EX::kOn) ex.finish(s, BuildOut<TF>{cnt, div, vi, density, a, g2});
}

}  // namespace

}  // namespace alb
