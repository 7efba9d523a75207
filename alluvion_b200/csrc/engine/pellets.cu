// pellets.cu -- the implicit SPH step (SolverI<TF>::step<0>,
// solver_i.hpp:79-327) on the pellet boundary branch: bodies are sampled
// by boundary particles ("pellets") instead of volume maps.
//
// Layout: one array of N + P points, the N fluid particles ("beads") first,
// then the P pellets (world positions from transform_pellets), as the
// reference stores pellets after max_num_particles.  One grid over all
// points; every point gets a bead list and a pellet list, slot-major
// (list[k * (N + P) + i]) in canonical (cell, index) order, of original
// indices.  The per-particle kernels run one thread per point in cell
// order.  Pressures live in two [N + P] arrays whose roles swap with the
// iteration parity (the reference copies pressure into last_pressure after
// every iteration); the pellet part of the array an iteration reads is
// filled just before it by the extrapolation.  With wrap_y (step<1>) the
// lists' cells and displacements wrap in y, rigid torque arms use the
// pellet image x_i - x_ij, and integrated positions wrap; the
// extrapolation's weighted centre uses absolute positions, as the
// reference's does.
#include <cfloat>
#include <cstring>
#include <vector>

#include "body_geometry.cuh"
#include "boundary.cuh"
#include "engine.hpp"
#include "grid.cuh"
#include "step_shared.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

template <class TF>
struct PelletState {
  uint32_t n = 0;   // beads
  uint32_t np = 0;  // pellets
  uint32_t nb = 0;
  uint32_t cap = 0;
  TF* x = nullptr;   // [n + np][3] beads then pellets
  TF* v = nullptr;   // [n + np][3]
  const uint32_t* perm = nullptr;     // sorted slot -> point
  uint32_t* blist = nullptr;          // [cap][n + np] bead neighbors
  uint32_t* bcnt = nullptr;           // [n + np]
  uint32_t* plist = nullptr;          // [cap][n + np] pellet neighbors
  uint32_t* pcnt = nullptr;           // [n + np]
  uint32_t* pbody = nullptr;          // [np] body of each pellet
  TF* rho = nullptr;                  // [n]
  TF* a = nullptr;                    // [n][3]
  TF* p0 = nullptr;                   // [n + np] last pressure on even iterations
  TF* p1 = nullptr;                   // [n + np] pressure on even iterations
  TF* diag = nullptr;                 // [n] Jacobi diagonal (times rho0)
  TF* adv = nullptr;                  // [n] advected density
  TF* force = nullptr;                // [nb][n][3] per-particle rigid force
  TF* torque = nullptr;               // [nb][n][3]
  RigidDev<TF>* rigid = nullptr;      // [nb] device
  Ctrl<TF>* ctrl = nullptr;
  double* red = nullptr;
};

struct BodyOffsets {
  uint32_t start[AL_MAX_BOUNDARIES + 1];
};

template <class TF>
__device__ __forceinline__ vec3<TF> ldv(const TF* p, size_t i) {
  return vec3<TF>{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
template <class TF>
__device__ __forceinline__ void stv(TF* p, size_t i, vec3<TF> v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

// Pressure arrays of the running iteration (see the file comment).
template <class TF>
__device__ __forceinline__ void pressure_roles(const PelletState<TF>& S, uint32_t it,
                                               const TF*& last, TF*& next) {
  const bool odd = (it & 1u) != 0;
  last = odd ? S.p1 : S.p0;
  next = odd ? S.p0 : S.p1;
}
// The array that holds the final pressure after `it` iterations: p1 after
// none (the previous step's pressure) or an odd number, p0 after an even
// number.
template <class TF>
__device__ __forceinline__ TF* final_pressure(const PelletState<TF>& S, uint32_t it) {
  return (it == 0 || (it & 1u)) ? S.p1 : S.p0;
}

// Adds a rigid force / torque to particle i's entry for body b (only the
// thread of particle i writes it).
template <class TF>
__device__ __forceinline__ void add_force(const PelletState<TF>& S, uint32_t b, uint32_t i,
                                          vec3<TF> f, vec3<TF> t) {
  const size_t slot = size_t(b) * S.n + i;
  stv(S.force, slot, ldv(S.force, slot) + f);
  stv(S.torque, slot, ldv(S.torque, slot) + t);
}

// ------------------------------------------------------------------ setup
// Beads copied in; pellets placed by transform_pellets (runner.hpp:4070-4082):
// x = R(q) local + x_b, v = omega x R(q) local + v_b.
template <class TF>
__global__ void k_pel_place(PelletState<TF> S, const TF* __restrict__ px,
                            const TF* __restrict__ pv, const TF* __restrict__ pp,
                            const TF* __restrict__ local, BodyOffsets off) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n + S.np) return;
  if (i < S.n) {
    stv(S.x, i, ldv(px, i));
    stv(S.v, i, ldv(pv, i));
    S.p1[i] = pp[i];
    return;
  }
  const uint32_t p = i - S.n;
  uint32_t b = 0;
  while (b + 1 < S.nb && p >= off.start[b + 1]) ++b;
  const RigidDev<TF> r = S.rigid[b];
  const vec3<TF> rl = rotate(ldv(local, p), r.q);
  stv(S.x, i, rl + r.x);
  stv(S.v, i, cross(r.omega, rl) + r.v);
  S.pbody[p] = b;
}

// make_bead_pellet_neighbor_list (runner.hpp:1912-1966) over every point,
// canonical order, and compute_density_with_pellets (runner.hpp:2074-2098)
// for the beads: rho = m (W(0) + sum_beads W + sum_pellets W).
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_pel_lists(Cn<TF> c, GridDims g, const uint32_t* __restrict__ cell_start,
                const vec4<TF>* __restrict__ xs, PelletState<TF> S, uint32_t* flags) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = S.n + S.np;
  if (t0 >= total) return;
  const uint32_t i = S.perm[t0];
  const vec3<TF> xi = xyz(xs[t0]);
  int ip[3];
  cell_coords(c.h, g, xi, ip);
  const int z0 = max(ip[2] - 1, 0);
  const int z1 = min(ip[2] + 1, int(g.res[2]) - 1);
  uint32_t nbead = 0, npel = 0;
  TF wsum = 0;
  if (z0 <= z1) {
    for (int dx = -1; dx <= 1; ++dx) {
      const int cx = ip[0] + dx;
      if (cx < 0 || cx >= int(g.res[0])) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int cy = ip[1] + dy;
        if (c.wrap) {  // make_bead_pellet_neighbor_list<1>
          if (cy >= int(g.res[1]))
            cy -= int(g.res[1]);
          else if (cy < 0)
            cy += int(g.res[1]);
        }
        if (cy < 0 || cy >= int(g.res[1])) continue;
        const uint32_t b = cell_start[cell_linear(g, cx, cy, z0)];
        const uint32_t e = cell_start[cell_linear(g, cx, cy, z1) + 1];
        for (uint32_t t = b; t < e; ++t) {
          const uint32_t j = S.perm[t];
          if (j == i) continue;
          const TF d2 = pdist2(c, xi, xyz(xs[t]));
          if (!(d2 < c.h2)) continue;
          if (j < S.n) {
            if (nbead < S.cap) S.blist[size_t(nbead) * total + i] = j;
            ++nbead;
          } else {
            if (npel < S.cap) S.plist[size_t(npel) * total + i] = j;
            ++npel;
          }
          if (i < S.n) wsum += W_r2(c, d2);
        }
      }
    }
  }
  if (nbead > S.cap || npel > S.cap) flags[2] = 1u;
  S.bcnt[i] = min(nbead, S.cap);
  S.pcnt[i] = min(npel, S.cap);
  if (i < S.n) S.rho[i] = (c.w0 + wsum) * c.mass;
}

// --------------------------------------------------------- forces and CFL
// clear_acceleration + compute_viscosity_with_pellets
// (runner.hpp:1974-1980, 2251-2299), per-particle rigid force and torque
// (the pellet's body), and calculate_cfl_v2 (runner.hpp:2533-2541) reduced
// to the global max; the last block applies Solver::update_dt.
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_pel_viscosity(Cn<TF> c, PelletState<TF> S) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = S.n + S.np;
  const TF eps = TF(0.01) * c.h2;
  TF v2 = 0;
  const uint32_t i = t0 < total ? S.perm[t0] : 0xffffffffu;
  if (i < S.n) {
    const vec3<TF> xi = ldv(S.x, i), vi = ldv(S.v, i);
    vec3<TF> da{0, 0, 0};
    const uint32_t nbd = S.bcnt[i];
    for (uint32_t k = 0; k < nbd; ++k) {
      const uint32_t j = S.blist[size_t(k) * total + i];
      const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
      da += (c.visc * c.mass / S.rho[j] * dot(d, gradW(c, d)) / (length_sqr(d) + eps)) *
            (vi - ldv(S.v, j));
    }
    const uint32_t npl = S.pcnt[i];
    for (uint32_t k = 0; k < npl; ++k) {
      const uint32_t j = S.plist[size_t(k) * total + i];
      const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
      const vec3<TF> a =
          (c.vol * c.bvisc * dot(d, gradW(c, d)) / (length_sqr(d) + eps)) * (vi - ldv(S.v, j));
      da += a;
      const uint32_t b = S.pbody[j - S.n];
      const vec3<TF> f = (-c.mass) * a;
      // pellet_x = x_i - x_ij (runner.hpp:2289): the pellet's image next to x_i
      add_force(S, b, i, f, cross((xi - d) - S.rigid[b].x, f));
    }
    const vec3<TF> acc = c.g + da;
    stv(S.a, i, acc);
    v2 = length_sqr(vi + acc * S.ctrl->dt);
  }
  // block max, then one ordered-bits atomicMax per block; the last block
  // applies update_dt
  __shared__ TF wmax[kBlock / 32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v2;
  __syncthreads();
  if (threadIdx.x == 0) {
    TF bm = wmax[0];
    for (int w = 1; w < kBlock / 32; ++w) bm = fmax(bm, wmax[w]);
    unsigned long long bits;
    if constexpr (sizeof(TF) == 4)
      bits = __float_as_uint(bm);
    else
      bits = (unsigned long long)__double_as_longlong(bm);
    atomicMax(&S.ctrl->vmax_bits, bits);
    __threadfence();
    last = atomicAdd(&S.ctrl->ticket, 1u) == gridDim.x - 1;
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


// ------------------------------------------------------------ the solve
// advect_and_init_pressure (runner.hpp:2889-2900) for the beads: v += dt a,
// last pressure = pressure / 2.
template <class TF>
__global__ void k_pel_advect(PelletState<TF> S) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S.n) return;
  const TF dt = S.ctrl->dt;
  stv(S.v, i, ldv(S.v, i) + dt * ldv(S.a, i));
  S.p0[i] = S.p1[i] * TF(0.5);
}

// calculate_isph_diagonal_adv_density_with_pellets (runner.hpp:2955-3004).
template <class TF>
__global__ void __launch_bounds__(kBlock) k_pel_diag(Cn<TF> c, PelletState<TF> S) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = S.n + S.np;
  if (t0 >= total) return;
  const uint32_t i = S.perm[t0];
  if (i >= S.n) return;
  const TF dt = S.ctrl->dt;
  const TF eps = TF(0.01) * c.h2;
  const vec3<TF> xi = ldv(S.x, i), vi = ldv(S.v, i);
  const TF rho = S.rho[i];
  TF adv = rho / c.rho0, diag = 0;
  const uint32_t nbd = S.bcnt[i];
  for (uint32_t k = 0; k < nbd; ++k) {
    const uint32_t j = S.blist[size_t(k) * total + i];
    const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
    const TF rj = S.rho[j];
    const vec3<TF> gw = gradW(c, d);
    adv += dt * c.vol * dot(vi - ldv(S.v, j), gw);
    diag += c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gw);
  }
  const uint32_t npl = S.pcnt[i];
  for (uint32_t k = 0; k < npl; ++k) {
    const uint32_t j = S.plist[size_t(k) * total + i];
    const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
    const vec3<TF> gwv = c.vol * gradW(c, d);
    adv += dt * dot(vi - ldv(S.v, j), gwv);
    diag += (rho + c.rho0) / (rho * c.rho0) / (length_sqr(d) + eps) * dot(d, gwv);
  }
  S.diag[i] = diag * c.rho0;
  S.adv[i] = adv;
}

// Eigen-decomposition of the symmetric 3x3 matrix a by cyclic Jacobi
// rotations (Golub and Van Loan, Matrix Computations, sec. 8.5): on return
// a is diagonal (the eigenvalues) and the columns of q the eigenvectors.
// Six sweeps; each rotation zeroes one off-diagonal entry.
template <class TF>
__device__ __forceinline__ void jacobi_eigen3(TF a[3][3], TF q[3][3]) {
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) q[r][k] = r == k ? TF(1) : TF(0);
  for (int sweep = 0; sweep < 6; ++sweep) {
    for (int pr = 0; pr < 3; ++pr) {
      const int p = pr == 2 ? 1 : 0;
      const int r = pr == 0 ? 1 : 2;
      const TF apr = a[p][r];
      if (apr == TF(0)) continue;
      const TF theta = (a[r][r] - a[p][p]) / (TF(2) * apr);
      const TF t = (theta >= TF(0) ? TF(1) : TF(-1)) / (fabs(theta) + sqrt(theta * theta + TF(1)));
      const TF cs = TF(1) / sqrt(t * t + TF(1));
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

// extrapolate_pressure_to_pellet (runner.hpp:2543-2607): the pellet's
// pressure from its bead neighbors, the Shepard average plus a linear
// moving-least-squares term, pseudo-inverting the weighted second moment
// (singular values of magnitude <= 1e-2 dropped; the moment is symmetric
// positive semi-definite, so its singular values are its eigenvalues);
// clamped at 0, and 0 for a pellet without bead neighbors.  Reads the
// beads' part of `pr` and writes the pellets' part.
template <class TF>
__global__ void k_pel_extrapolate(Cn<TF> c, PelletState<TF> S, int final_pass) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= S.np) return;
  const uint32_t it = S.ctrl->it;
  TF* pr;
  if (final_pass) {
    pr = final_pressure(S, it);
  } else {
    const TF* last;
    TF* next;
    pressure_roles(S, it, last, next);
    pr = const_cast<TF*>(last);
  }
  const uint32_t total = S.n + S.np;
  const uint32_t i = S.n + p;
  const vec3<TF> xi = ldv(S.x, i);
  const uint32_t cnt = S.bcnt[i];
  TF wsum = 0;
  vec3<TF> center{0, 0, 0};
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = S.blist[size_t(k) * total + i];
    const vec3<TF> xj = ldv(S.x, j);
    const TF w = W_r2(c, pdist2(c, xi, xj)) * c.vol;  // the list's (wrapped) x_ij
    wsum += w;
    center += w * xj;
  }
  if (!(wsum > TF(0))) {
    pr[i] = TF(0);
    return;
  }
  center = (TF(1) / wsum) * center;
  TF alpha = 0;
  vec3<TF> psum{0, 0, 0};
  TF m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (uint32_t k = 0; k < cnt; ++k) {
    const uint32_t j = S.blist[size_t(k) * total + i];
    const vec3<TF> xj = ldv(S.x, j);
    const vec3<TF> xt = xj - center;
    const TF w = W_r2(c, pdist2(c, xi, xj)) * c.vol;
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
  // plane = Q diag(1 / lambda) Q^T psum over the kept eigenvalues
  vec3<TF> plane{0, 0, 0};
  for (int e = 0; e < 3; ++e) {
    const TF lam = m[e][e];
    if (!(fabs(lam) > TF(1e-2))) continue;
    const vec3<TF> qe{q[0][e], q[1][e], q[2][e]};
    plane += (dot(qe, psum) / lam) * qe;
  }
  const TF pressure = alpha + dot(plane, xi - center);
  pr[i] = fmax(pressure, TF(0));
}

// isph_solve_iteration_with_pellets (runner.hpp:3055-3121) and the mean
// density error of solver_i.hpp:272-274 (double, on the device).
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_pel_iter(Cn<TF> c, PelletState<TF> S) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = S.n + S.np;
  const uint32_t i = t0 < total ? S.perm[t0] : 0xffffffffu;
  const TF* last;
  TF* next;
  pressure_roles(S, S.ctrl->it, last, next);
  double val = 0;
  if (i < S.n) {
    const TF dt = S.ctrl->dt;
    const TF eps = TF(0.01) * c.h2;
    const vec3<TF> xi = ldv(S.x, i);
    const TF rho = S.rho[i];
    TF off = 0;
    const uint32_t nbd = S.bcnt[i];
    for (uint32_t k = 0; k < nbd; ++k) {
      const uint32_t j = S.blist[size_t(k) * total + i];
      const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
      const TF rj = S.rho[j];
      off -= c.vol * (rho + rj) / (rho * rj) / (length_sqr(d) + eps) * dot(d, gradW(c, d)) *
             last[j];
    }
    const uint32_t npl = S.pcnt[i];
    for (uint32_t k = 0; k < npl; ++k) {
      const uint32_t j = S.plist[size_t(k) * total + i];
      const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
      off -= c.vol * (rho + c.rho0) / (rho * c.rho0) / (length_sqr(d) + eps) *
             dot(d, gradW(c, d)) * last[j];
    }
    off *= c.rho0;
    const TF diag = S.diag[i];
    const TF bterm = TF(1) - S.adv[i];
    const TF dt2 = dt * dt;
    const TF denom = diag * dt2;
    const TF w = TF(2) / TF(3);
    TF pv = 0;
    if (fabs(denom) > TF(1.0e-9))
      pv = fmax((TF(1) - w) * last[i] + w * (bterm / denom - off / diag), TF(0));
    const TF err = pv == TF(0) ? TF(0) : (denom * pv + off * dt2 - bterm);
    next[i] = pv;
    val = double(err);
  }
  double totalv;
  if (grid_sum_last(val, S.red, &S.ctrl->ticket, &totalv) && threadIdx.x == 0)
    finish_iteration(*S.ctrl, totalv, S.n, 1, cudaGraphConditionalHandle(0), 0);
}

// compute_pressure_accels_with_pellets (runner.hpp:2819-2871) and
// kinematic_integration<0> (runner.hpp:2873-2887), written back in the
// caller's buffers.  The pellet term's rigid force is m a with a the term
// before the rho0 factor of the particle's acceleration, as in the
// reference.
template <class TF>
__global__ void __launch_bounds__(kBlock)
    k_pel_accel_finish(Cn<TF> c, PelletState<TF> S, TF* __restrict__ x_ref,
                       TF* __restrict__ v_ref, TF* __restrict__ a_ref, TF* __restrict__ rho_ref,
                       TF* __restrict__ p_ref, TF* __restrict__ adv_ref) {
  const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = S.n + S.np;
  if (t0 >= total) return;
  const uint32_t i = S.perm[t0];
  if (i >= S.n) return;
  const TF* pr = final_pressure(S, S.ctrl->it);
  const vec3<TF> xi = ldv(S.x, i);
  const TF rho = S.rho[i];
  const TF dpi = pr[i] / (rho * rho);
  vec3<TF> ai{0, 0, 0};
  const uint32_t nbd = S.bcnt[i];
  for (uint32_t k = 0; k < nbd; ++k) {
    const uint32_t j = S.blist[size_t(k) * total + i];
    const TF rj = S.rho[j];
    const TF dpj = pr[j] / (rj * rj);
    ai -= (c.mass * (dpi + dpj)) * gradW(c, pdisp(c, xi, ldv(S.x, j)));
  }
  const uint32_t npl = S.pcnt[i];
  const TF r02 = c.rho0 * c.rho0;
  for (uint32_t k = 0; k < npl; ++k) {
    const uint32_t j = S.plist[size_t(k) * total + i];
    const vec3<TF> d = pdisp(c, xi, ldv(S.x, j));
    const TF dpj = pr[j] / r02;
    const vec3<TF> a = (c.mass * (dpi + dpj)) * gradW(c, d);
    const vec3<TF> f = c.mass * a;
    ai -= a;
    const uint32_t b = S.pbody[j - S.n];
    add_force(S, b, i, f, cross((xi - d) - S.rigid[b].x, f));  // x_j = x_i - x_ij
  }
  const TF dt = S.ctrl->dt;
  const vec3<TF> v = ldv(S.v, i) + (c.rho0 * ai) * dt;
  vec3<TF> xn = xi + v * dt;
  xn.y = wrap_y(c, xn.y);  // kinematic_integration<wrap>
  stv(x_ref, i, xn);
  stv(v_ref, i, v);
  if (a_ref) stv(a_ref, i, ldv(S.a, i));
  if (rho_ref) rho_ref[i] = rho;
  if (p_ref) p_ref[i] = pr[i];
  if (adv_ref) adv_ref[i] = S.adv[i];
}

// Per-body totals of the per-particle entries, in double: block k sums a
// contiguous chunk of particles in a fixed order into slot k
// (the [grid][nb][6] layout k_rigid_finish reads).
template <class TF>
__global__ void k_pel_force_slots(PelletState<TF> S, double* ft, uint32_t chunk) {
  const uint32_t b = blockIdx.y;
  const uint32_t lo = blockIdx.x * chunk;
  const uint32_t hi = min(lo + chunk, S.n);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const vec3<TF> f = ldv(S.force, size_t(b) * S.n + i);
    const vec3<TF> t = ldv(S.torque, size_t(b) * S.n + i);
    acc[0] += double(f.x);
    acc[1] += double(f.y);
    acc[2] += double(f.z);
    acc[3] += double(t.x);
    acc[4] += double(t.y);
    acc[5] += double(t.z);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double tot = block_sum_double(acc[k]);
    if (threadIdx.x == 0) ft[(size_t(blockIdx.x) * S.nb + b) * 6 + k] = tot;
  }
}

template <class TF>
__global__ void k_pel_outputs(PelletState<TF> S, TF* __restrict__ x_out, TF* __restrict__ p_out,
                              TF* __restrict__ v_out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= S.np) return;
  if (x_out) stv(x_out, p, ldv(S.x, S.n + p));
  if (v_out) stv(v_out, p, ldv(S.v, S.n + p));
  if (p_out) p_out[p] = final_pressure(S, S.ctrl->it)[S.n + p];
}

// ------------------------------------------------------------ host side
template <class TF>
struct PelletTypes;
template <>
struct PelletTypes<float> {
  using cn = al_const_f32;
  using fluid = al_fluid_f32;
  using body = al_body_f32;
  using rigid = al_rigid_f32;
  using pellets = al_pellets_f32;
};
template <>
struct PelletTypes<double> {
  using cn = al_const_f64;
  using fluid = al_fluid_f64;
  using body = al_body_f64;
  using rigid = al_rigid_f64;
  using pellets = al_pellets_f64;
};

template <class TF>
int pellet_step(al_engine* e, const typename PelletTypes<TF>::cn* cn, const al_consti* cni,
                const typename PelletTypes<TF>::fluid* f, const typename PelletTypes<TF>::body* bodies,
                typename PelletTypes<TF>::rigid* rigid,
                const typename PelletTypes<TF>::pellets* pel, const al_solver_params* sp, TF* dt,
                al_step_report* report, cudaStream_t st) {
  ALB_CHECK_ARG(e && cn && cni && f && pel && sp && dt, "al_i_step_pellets: null argument");
  const uint32_t n = f->num_particles;
  const uint32_t np = pel->num_pellets;
  const uint32_t nb = cni->num_boundaries;
  ALB_CHECK_ARG(nb <= AL_MAX_BOUNDARIES, "al_i_step_pellets: too many bodies");
  ALB_CHECK_ARG(nb == 0 || (bodies && rigid), "al_i_step_pellets: bodies / rigid are null");
  ALB_CHECK_ARG(n == 0 || (f->particle_x && f->particle_v && f->particle_pressure),
                "al_i_step_pellets: particle_x / particle_v / particle_pressure are null");
  ALB_CHECK_ARG(np == 0 || pel->local_x, "al_i_step_pellets: pellet local_x is null");
  ALB_CHECK_ARG(np == 0 || nb > 0, "al_i_step_pellets: pellets need bodies");
  ALB_CHECK_ARG(!sp->wrap_y || sp->wrap_length > 0, "al_i_step_pellets: wrap_y needs a length");
  ALB_CHECK_ARG(uint64_t(n) + np < (1ull << 31), "al_i_step_pellets: too many points");
  BodyOffsets off{};
  uint64_t acc = 0;
  for (uint32_t b = 0; b < nb; ++b) {
    off.start[b] = uint32_t(acc);
    acc += pel->count[b];
  }
  off.start[nb] = uint32_t(acc);
  ALB_CHECK_ARG(acc == np, "al_i_step_pellets: pellet counts do not add up to num_pellets");
  for (uint32_t b = 0; b < nb; ++b)
    ALB_CHECK_ARG(bodies[b].shape <= AL_SHAPE_INFINITE_TUBE, "al_i_step_pellets: unknown body shape");
  ALB_TRY(e->activate());
  e->ns.clear();
  struct NsReset {
    al_engine* e;
    ~NsReset() { e->ns.clear(); }
  } reset{e};
  e->ns = "pellet.";
  Cn<TF> c = to_cn<TF>(*cn);
  if (sp->wrap_y) set_wrap(c, TF(sp->wrap_length));  // SolverI::step<1>
  const GridDims g = to_dims(*cni);
  const uint32_t total = n + np;
  PelletState<TF> S;
  S.n = n;
  S.np = np;
  S.nb = nb;
  S.cap = g.cap_nbr;
  uint32_t* flags = nullptr;
  vec4<TF>* xs = nullptr;
  BodyDev<TF>* bodies_dev = nullptr;
  double* ft = nullptr;
  const uint32_t chunk = 4096;
  const uint32_t slots = n ? (n + chunk - 1) / chunk : 1;
  ALB_TRY(e->buf("flags", 4, &flags));
  ALB_TRY(e->buf("x", size_t(total ? total : 1) * 3, &S.x));
  ALB_TRY(e->buf("v", size_t(total ? total : 1) * 3, &S.v));
  ALB_TRY(e->buf("sorted.x", total ? total : 1, &xs));
  ALB_TRY(e->buf("blist", size_t(total ? total : 1) * S.cap, &S.blist));
  ALB_TRY(e->buf("bcnt", total ? total : 1, &S.bcnt));
  ALB_TRY(e->buf("plist", size_t(total ? total : 1) * S.cap, &S.plist));
  ALB_TRY(e->buf("pcnt", total ? total : 1, &S.pcnt));
  ALB_TRY(e->buf("pbody", np ? np : 1, &S.pbody));
  ALB_TRY(e->buf("rho", n ? n : 1, &S.rho));
  ALB_TRY(e->buf("a", size_t(n ? n : 1) * 3, &S.a));
  ALB_TRY(e->buf("p0", total ? total : 1, &S.p0));
  ALB_TRY(e->buf("p1", total ? total : 1, &S.p1));
  ALB_TRY(e->buf("diag", n ? n : 1, &S.diag));
  ALB_TRY(e->buf("adv", n ? n : 1, &S.adv));
  ALB_TRY(e->buf("force", size_t(nb ? nb : 1) * (n ? n : 1) * 3, &S.force));
  ALB_TRY(e->buf("torque", size_t(nb ? nb : 1) * (n ? n : 1) * 3, &S.torque));
  ALB_TRY(e->buf("rigid", AL_MAX_BOUNDARIES, &S.rigid));
  ALB_TRY(e->buf("bodies", AL_MAX_BOUNDARIES, &bodies_dev));
  ALB_TRY(e->buf("ctrl", 1, &S.ctrl));
  ALB_TRY(e->buf("red", blocks_for(total ? total : 1, kBlock), &S.red));
  ALB_TRY(e->buf("ft", size_t(slots) * (nb ? nb : 1) * 6, &ft));
  // control block, bodies and poses
  Ctrl<TF> hc;
  std::memset(&hc, 0, sizeof(hc));
  hc.dt = *dt;
  hc.length_scale = c.radius * TF(2);
  hc.cfl = TF(sp->cfl);
  hc.max_dt = TF(sp->max_dt);
  hc.min_dt = TF(sp->min_dt);
  hc.tol_den = double(TF(sp->density_error_tolerance));
  hc.min_den = sp->min_density_solve;
  hc.max_den = sp->max_density_solve;
  hc.integrate_rigids = sp->integrate_rigids;
  for (int k = 0; k < 3; ++k) hc.pile_gravity[k] = TF(sp->pile_gravity[k]);
  std::vector<BodyDev<TF>> hb(nb ? nb : 1);
  std::vector<RigidDev<TF>> hr(nb ? nb : 1);
  for (uint32_t b = 0; b < nb; ++b) {
    hb[b] = to_body_dev<TF>(bodies[b]);
    hr[b] = to_rigid_dev<TF>(rigid[b]);
  }
  ALB_CUDA(cudaMemcpyAsync(S.ctrl, &hc, sizeof(hc), cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(bodies_dev, hb.data(), sizeof(BodyDev<TF>) * hb.size(),
                           cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemcpyAsync(S.rigid, hr.data(), sizeof(RigidDev<TF>) * hr.size(),
                           cudaMemcpyHostToDevice, st));
  ALB_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), st));
  ALB_CUDA(cudaMemsetAsync(ft, 0, size_t(slots) * (nb ? nb : 1) * 6 * sizeof(double), st));
  if (nb && n) {
    ALB_CUDA(cudaMemsetAsync(S.force, 0, size_t(nb) * n * 3 * sizeof(TF), st));
    ALB_CUDA(cudaMemsetAsync(S.torque, 0, size_t(nb) * n * 3 * sizeof(TF), st));
  }
  // the shared kernels' view of the step
  StepState<TF> SS;
  SS.n = n;
  SS.ls = n;
  SS.nb = nb;
  SS.grid = slots;
  SS.ft = ft;
  SS.red = S.red;
  SS.ctrl = S.ctrl;
  SS.bodies = bodies_dev;
  SS.rigid = S.rigid;
  ALB_LAUNCH(e, "pellet_init", 1, st, k_step_init<TF><<<1, 32, 0, st>>>(SS));
  const uint32_t tb = blocks_for(total ? total : 1, kBlock);
  if (total) {
    ALB_LAUNCH(e, "pellet_place", 1, st,
               (k_pel_place<TF><<<tb, kBlock, 0, st>>>(S, f->particle_x, f->particle_v,
                                                       f->particle_pressure, pel->local_x, off)));
    GridState gs;
    ALB_LAUNCH(e, "pellet_grid", kGridBuildKernels, st,
               ALB_TRY(grid_build<TF>(e, c, g, S.x, total, xs, flags, gs, st)));
    S.perm = gs.perm;
    ALB_LAUNCH(e, "pellet_lists", 1, st,
               (k_pel_lists<TF><<<tb, kBlock, 0, st>>>(c, g, gs.cell_start, xs, S, flags)));
  }
  if (n) {
    ALB_LAUNCH(e, "pellet_viscosity", 1, st,
               (k_pel_viscosity<TF><<<tb, kBlock, 0, st>>>(c, S)));
    ALB_LAUNCH(e, "pellet_advect", 1, st,
               (k_pel_advect<TF><<<blocks_for(n, kBlock), kBlock, 0, st>>>(S)));
    ALB_LAUNCH(e, "pellet_diag", 1, st, (k_pel_diag<TF><<<tb, kBlock, 0, st>>>(c, S)));
    ALB_LAUNCH(e, "pellet_loop_begin", 1, st,
               (k_loop_begin<TF><<<1, 1, 0, st>>>(SS, 1, cudaGraphConditionalHandle(0), 0)));
    uint32_t hflag = 0;
    bool go = sp->max_density_solve > 0;
    while (go) {
      if (np)
        ALB_LAUNCH(e, "pellet_extrapolate", 1, st,
                   (k_pel_extrapolate<TF><<<blocks_for(np, kBlock), kBlock, 0, st>>>(c, S, 0)));
      ALB_LAUNCH(e, "pellet_iter", 1, st, (k_pel_iter<TF><<<tb, kBlock, 0, st>>>(c, S)));
      ALB_TRY(read_keep_going(SS, &hflag, st, &go));
    }
    if (np)
      ALB_LAUNCH(e, "pellet_extrapolate", 1, st,
                 (k_pel_extrapolate<TF><<<blocks_for(np, kBlock), kBlock, 0, st>>>(c, S, 1)));
    ALB_LAUNCH(e, "pellet_finish", 1, st,
               (k_pel_accel_finish<TF><<<tb, kBlock, 0, st>>>(
                   c, S, f->particle_x, f->particle_v, f->particle_a, f->particle_density,
                   f->particle_pressure, f->particle_density_adv)));
    if (nb)
      ALB_LAUNCH(e, "pellet_force_slots", 1, st,
                 (k_pel_force_slots<TF><<<dim3(slots, nb), 256, 0, st>>>(S, ft, chunk)));
  }
  if (nb)
    ALB_LAUNCH(e, "rigid_finish", 1, st,
               k_rigid_finish<TF><<<nb, 256, 0, st>>>(SS, SS.ft, SS.grid));
  if (np && (pel->x || pel->pressure || pel->v))
    ALB_LAUNCH(e, "pellet_outputs", 1, st,
               (k_pel_outputs<TF><<<blocks_for(np, kBlock), kBlock, 0, st>>>(
                   S, pel->x, pel->pressure, pel->v)));
  ALB_CUDA(cudaGetLastError());
  uint32_t hf[4];
  ALB_CUDA(cudaMemcpyAsync(&hc, S.ctrl, sizeof(hc), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaMemcpyAsync(hr.data(), S.rigid, sizeof(RigidDev<TF>) * hr.size(),
                           cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  e->flush_stats();
  al_step_report rep = hc.rep;
  for (int k = 0; k < 3; ++k) rep.grid_anomaly[k] = hf[k];
  if (n == 0) rep.dt = double(*dt);
  *dt = TF(rep.dt);
  for (uint32_t b = 0; b < nb; ++b) {
    for (int k = 0; k < 3; ++k) {
      rigid[b].x[k] = (&hr[b].x.x)[k];
      rigid[b].v[k] = (&hr[b].v.x)[k];
      rigid[b].omega[k] = (&hr[b].omega.x)[k];
    }
    rigid[b].q[0] = hr[b].q.x;
    rigid[b].q[1] = hr[b].q.y;
    rigid[b].q[2] = hr[b].q.z;
    rigid[b].q[3] = hr[b].q.w;
  }
  if (report) *report = rep;
  if (hf[0]) return AL_ERR_OUT_OF_GRID;
  if (hf[1]) return AL_ERR_CELL_OVERFLOW;
  if (hf[2]) return AL_ERR_NEIGHBOR_OVERFLOW;
  return AL_OK;
}

}  // namespace

}  // namespace alb

using namespace alb;

extern "C" {

int al_i_step_pellets_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                          const al_fluid_f32* fluid, const al_body_f32* bodies,
                          al_rigid_f32* rigid, const al_pellets_f32* pellets,
                          const al_solver_params* params, float* dt, al_step_report* report,
                          void* stream) {
  return pellet_step<float>(engine, cn, cni, fluid, bodies, rigid, pellets, params, dt, report,
                            static_cast<cudaStream_t>(stream));
}
int al_i_step_pellets_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                          const al_fluid_f64* fluid, const al_body_f64* bodies,
                          al_rigid_f64* rigid, const al_pellets_f64* pellets,
                          const al_solver_params* params, double* dt, al_step_report* report,
                          void* stream) {
  return pellet_step<double>(engine, cn, cni, fluid, bodies, rigid, pellets, params, dt, report,
                             static_cast<cudaStream_t>(stream));
}

}  // extern "C"
