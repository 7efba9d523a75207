// solver.cuh -- DFSPH and IISPH steps over the cell-sorted particle state.
//
// Replaces SolverDf<TF>::step<0> (solver_df.hpp:74-359) and
// SolverIi<TF>::step<0> (solver_ii.hpp:76-243) with the kernels they launch
// (runner.hpp:1974-2249, 2533-2541, 2609-2887, 3123-3623) and the rigid
// force/torque sums and Pile::integrate_kinematics (pile.hpp:794-815).
//
// Differences in mechanism (same arithmetic per particle):
//  * all passes run on cell-sorted state (gathered once per step, scattered
//    back to the caller's buffers at the end);
//  * the solvers' convergence means are reduced on the device in double,
//    deterministically (fixed block partition, fixed summation order), and
//    the loop decision is taken on the device; the host reads one flag per
//    iteration (eager mode) or nothing at all (graph mode);
//  * rigid force/torque contributions are reduced per block into per-block
//    slots (no atomics) and summed per body in double at the end of the
//    step; per-particle [nb][N] force arrays are not materialised.
#pragma once

#include "boundary.cuh"
#include "common.cuh"
#include "engine.hpp"
#include "grid.cuh"

namespace alb {

// Device control block of one step.
template <class TF>
struct Ctrl {
  TF dt;            // time step in use by the kernels
  TF length_scale;  // 2 r
  TF cfl, max_dt, min_dt;
  TF pad0;
  double tol_div;   // density_change_tolerance
  double tol_den;   // density_error_tolerance
  uint32_t min_div, max_div, min_den, max_den;
  uint32_t it;          // iterations done by the running solve
  uint32_t keep_going;  // 1 while the running solve must iterate again
  uint32_t ticket;      // last-block ticket of grid reductions
  uint32_t integrate_rigids;
  uint32_t warm_ran;    // 1 when the learned warm start's network ran this step
  double mean;          // latest mean of the running solve
  unsigned long long vmax_bits;  // max |v + a dt|^2 as ordered bits
  TF pile_gravity[3];
  TF pad1;
  al_step_report rep;
};

template <class TF>
struct FusedScene;
template <class TF>
struct FusedIo;

template <class TF>
struct StepState {
  uint32_t n = 0, nb = 0, cap = 0, grid = 0;
  uint32_t tpp = 1;  // threads per particle of the pair passes (pair_tpp)
  // Stride of the slot-major arrays (nbr [cap][ls], bx / bk [nb][ls]): n for
  // one scene; the arena's particle count for the scenes of a fused batch.
  uint32_t ls = 0;
  vec4<TF>* x = nullptr;    // sorted positions (grid sort, boundaries, build)
  // Interleaved particle records of the pair passes: rec[2s] = {x, payload},
  // rec[2s + 1] = {v, rho}.  One 32-byte sector (float) holds all a
  // neighbor contributes to any DFSPH pass.  `payload` is the scalar the
  // next k_kappa pass reads from its neighbors (the kappa_v / kappa warm
  // start, or k = b alpha of the running iteration); the kernels that write
  // it read only x from the same half, so the 4-byte store never races
  // with a value another thread uses.
  vec4<TF>* rec = nullptr;
  vec4<TF>* a = nullptr;
  TF* rho = nullptr;
  TF* alpha = nullptr;
  TF* rho_adv = nullptr;
  TF* kappa = nullptr;    // DFSPH kappa, IISPH / implicit SPH pressure
  TF* kappa_v = nullptr;  // DFSPH kappa_v, IISPH / implicit SPH last pressure
  TF* kk = nullptr;       // IISPH aii, implicit SPH diagonal (times rho0)
  TF* err = nullptr;      // IISPH / implicit SPH density error
  vec4<TF>* dii = nullptr;
  vec4<TF>* dij_pj = nullptr;
  uint32_t* nbr = nullptr;
  uint32_t* ncount = nullptr;
  uint32_t* mask = nullptr;
  vec4<TF>* bx = nullptr;
  vec4<TF>* bk = nullptr;
  const BodyDev<TF>* bodies = nullptr;
  RigidDev<TF>* rigid = nullptr;
  double* ft = nullptr;   // [grid][nb][6] rigid force/torque partials
  double* red = nullptr;  // [grid] reduction partials
  Ctrl<TF>* ctrl = nullptr;
  const uint32_t* perm = nullptr;
  // A pass launched over every scene of a fused batch: the scene of each
  // block (nscenes for a block past every scene) and the scenes' ranges.
  const uint32_t* blk_scene = nullptr;
  const FusedScene<TF>* fused = nullptr;
  const FusedIo<TF>* io = nullptr;
  uint32_t nscenes = 0;
};

// One scene of a fused batch: its particles [s0, s0 + n) of the shared
// arena, its blocks [blk0, blk0 + nblk) of a pass launch (128 threads, one
// per particle), and its control block, bodies, rigid state, rigid slots
// ([nblk][nb][6]), their first-stage partials, reduction partials ([nblk])
// and anomaly flags.
template <class TF>
struct FusedScene {
  uint32_t s0, n, blk0, nblk, nb, pad;
  Ctrl<TF>* ctrl;
  const BodyDev<TF>* bodies;
  RigidDev<TF>* rigid;
  double* ft;
  double* ftp;
  double* red;
  uint32_t* flags;
};

// The caller's buffers of one scene of a fused batch (original particle
// order: read by the gather, written by the write-back).
template <class TF>
struct FusedIo {
  const TF* x_in;
  const TF* v_in;
  const TF* kappa_in;
  const TF* kappa_v_in;
  TF* x_out;
  TF* v_out;
  TF* a_out;
  TF* rho_out;
  TF* alpha_out;
  TF* kappa_out;
  TF* kappa_v_out;
  TF* rho_adv_out;
};

}  // namespace alb
