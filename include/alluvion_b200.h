/*
 * alluvion_b200.h -- C ABI of the B200 (sm_100a) SPH fluid-step engine.
 *
 * This is the drop-in boundary underneath alluvion's fluid-step path.  The
 * reference drives that path from templated C++ host code
 * (include/alluvion/solver.hpp, solver_df.hpp, solver_ii.hpp, pile.hpp) that
 * launches kernels from include/alluvion/runner.hpp.  Each entry point below
 * names the reference routine(s) it replaces.
 *
 * Conventions
 *  - Plain C types only: device pointers, sizes, POD parameter blocks passed
 *    by pointer and read once per call.  No CUDA, torch or C++ types.
 *  - Buffers named particle_* use the reference's layouts: particle_x and
 *    particle_v are [N][3] arrays of the solver's real type (float3/double3
 *    AoS), scalars are [N], particle_boundary / particle_boundary_kernel are
 *    [num_boundaries][N][4], particle_neighbors is [N][cap][4] whose 4th
 *    component holds the neighbor's index as raw uint32 bits
 *    (runner.hpp:1896-1897).
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Calls are asynchronous unless documented otherwise.
 *  - Every call returns an al_status.  No call throws or aborts.  Capacity
 *    anomalies (the reference's grid_anomaly flags, runner.hpp:1860-1865,
 *    1907-1909) are reported with their own codes after the outputs have
 *    been written with the reference's truncation semantics.
 *  - The engine owns its scratch memory (cell tables, sorted particle state,
 *    compact neighbor lists); callers own every particle_* buffer.
 */
#ifndef ALLUVION_B200_H
#define ALLUVION_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define AL_API __attribute__((visibility("default")))
#else
#define AL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef enum al_status {
  AL_OK = 0,
  AL_ERR_CUDA = 1,             /* a CUDA runtime call failed (message: al_last_error) */
  AL_ERR_INVALID = 2,          /* bad argument (null pointer, size, capacity) */
  AL_ERR_OUT_OF_GRID = 3,      /* a particle fell outside the grid: grid_anomaly[0] */
  AL_ERR_CELL_OVERFLOW = 4,    /* a cell exceeded max_num_particles_per_cell: grid_anomaly[1] */
  AL_ERR_NEIGHBOR_OVERFLOW = 5,/* a particle exceeded max_num_neighbors_per_particle: grid_anomaly[2] */
  AL_ERR_UNSUPPORTED = 6,      /* option outside the engine's scope */
  AL_ERR_TIMEOUT = 7,          /* a bounded device-side wait gave up */
  AL_ERR_NO_DEVICE = 8,        /* no CUDA device, or not an sm_100 part */
  AL_ERR_ALLOC = 9             /* device allocation failed */
} al_status;

#define AL_MAX_BOUNDARIES 16

/* ------------------------------------------------------- parameter blocks
 * Mirror of the hot-path subset of Const<TF> (constants.hpp:51-137).  The
 * derived kernel constants are computed by the caller exactly as
 * Const::set_kernel_radius / set_particle_attr do (constants.hpp:100-128),
 * so the engine sees the same rounded values the reference would. */
typedef struct al_const_f32 {
  float kernel_radius;       /* h */
  float kernel_radius_sqr;   /* h^2 */
  float cubic_kernel_k;      /* 8 / h^3 / pi */
  float cubic_kernel_l;      /* 48 / h^4 / pi */
  float cubic_kernel_zero;   /* W(0) = k */
  float particle_radius;
  float particle_vol;        /* mass / density0 */
  float particle_mass;
  float density0;
  float viscosity;
  float boundary_viscosity;
  float dfsph_factor_epsilon;
  float gravity[3];
} al_const_f32;

typedef struct al_const_f64 {
  double kernel_radius;
  double kernel_radius_sqr;
  double cubic_kernel_k;
  double cubic_kernel_l;
  double cubic_kernel_zero;
  double particle_radius;
  double particle_vol;
  double particle_mass;
  double density0;
  double viscosity;
  double boundary_viscosity;
  double dfsph_factor_epsilon;
  double gravity[3];
} al_const_f64;

/* Mirror of Consti (constants.hpp:40-49). */
typedef struct al_consti {
  uint32_t max_num_particles_per_cell;
  uint32_t grid_res[3];
  int32_t grid_offset[3];
  uint32_t max_num_neighbors_per_particle;
  uint32_t num_boundaries;
} al_consti;

/* ----------------------------------------------------------- rigid bodies
 * One boundary of the Pile (pile.hpp:98-121).  The analytic distances are
 * those of dg/box_distance.hpp, dg/sphere_distance.hpp and
 * dg/box_shell_distance.hpp; AL_SHAPE_TORUS has no reference counterpart.
 * Grid fields follow Pile::calculate_grid_attributes (pile.hpp:66-78):
 * cell_size = (domain_max - domain_min) / resolution and
 * num_nodes = (rx+1)(ry+1)(rz+1) + 2 * (edge count).
 * Node arrays are device pointers for the engine. */
typedef enum al_shape {
  AL_SHAPE_BOX = 0,       /* shape_params: half widths x y z, outset */
  AL_SHAPE_SPHERE = 1,    /* shape_params: radius */
  AL_SHAPE_BOX_SHELL = 2, /* shape_params: inner half widths xyz, outer half widths xyz, outset */
  AL_SHAPE_TORUS = 3,     /* shape_params: major radius (x-z plane), minor radius */
  AL_SHAPE_MESH = 4,      /* triangle mesh: distance_nodes from al_build_mesh_distance_grid_f32
                             (MeshDistance, dg/mesh_distance.hpp); use_distance_grid must be 1 */
  AL_SHAPE_CYLINDER = 5,  /* shape_params: radius, height, com_y (CylinderDistance,
                             dg/cylinder_distance.hpp; axis y, centre at y = -com_y) */
  AL_SHAPE_CAPSULE = 6,   /* shape_params: radius, height of the straight part (CapsuleDistance,
                             dg/capsule_distance.hpp; axis y) */
  AL_SHAPE_INFINITE_CYLINDER = 7, /* shape_params: radius (InfiniteCylinderDistance,
                             dg/infinite_cylinder_distance.hpp; invariant along y) */
  AL_SHAPE_INFINITE_TUBE = 8 /* shape_params: inner radius, outer radius (InfiniteTubeDistance,
                             dg/infinite_tube_distance.hpp; invariant along y) */
} al_shape;
/* The y-invariant shapes are sampled as the reference's
 * compute_volume_and_boundary_x_analytic<1> does (runner.hpp:1744-1746): the
 * body-frame y of the particle is set to 0, so the volume map is read on its
 * y = 0 slice; they need use_distance_grid = 0. */

typedef struct al_body_f32 {
  uint32_t shape;
  /* 1: distance and normal interpolated from distance_nodes
   *    (compute_particle_boundary, runner.hpp:2004-2025);
   * 0: analytic distance with finite-difference normal
   *    (compute_particle_boundary_analytic<0>, runner.hpp:1982-2002). */
  uint32_t use_distance_grid;
  float sign; /* +1: fluid outside the body; -1: fluid inside (container) */
  float shape_params[8];
  float domain_min[3];
  float domain_max[3];
  float cell_size[3];
  uint32_t resolution[3];
  uint32_t num_nodes;
  const float* distance_nodes; /* [num_nodes]; required when use_distance_grid */
  const float* volume_nodes;   /* [num_nodes] */
  float max_distance;          /* Distance::get_max_distance (CFL bound) */
  float mass;                  /* 0: kinematic body, not integrated */
  float inertia[3];            /* principal moments, body frame */
} al_body_f32;

typedef struct al_body_f64 {
  uint32_t shape;
  uint32_t use_distance_grid;
  double sign;
  double shape_params[8];
  double domain_min[3];
  double domain_max[3];
  double cell_size[3];
  uint32_t resolution[3];
  uint32_t num_nodes;
  const double* distance_nodes;
  const double* volume_nodes;
  double max_distance;
  double mass;
  double inertia[3];
} al_body_f64;

/* Kinematic state of one body (Pile x_, v_, q_, omega_; pile.hpp:103-110).
 * q is {x, y, z, w}. */
typedef struct al_rigid_f32 {
  float x[3];
  float v[3];
  float q[4];
  float omega[3];
} al_rigid_f32;

typedef struct al_rigid_f64 {
  double x[3];
  double v[3];
  double q[4];
  double omega[3];
} al_rigid_f64;

/* ------------------------------------------------------- solver controls
 * Fields of Solver / SolverDf / SolverIi (solver.hpp:261-273,
 * solver_df.hpp:372-379, solver_ii.hpp:259-261) plus Pile::gravity_
 * (pile.hpp:142) used by Pile::integrate_kinematics. */
typedef struct al_solver_params {
  double density_change_tolerance; /* DFSPH divergence solve: mean drho/dt < tol / dt */
  double density_error_tolerance;  /* mean (rho_adv - 1) < tol */
  uint32_t min_density_solve;
  uint32_t max_density_solve;
  uint32_t min_divergence_solve;
  uint32_t max_divergence_solve;
  uint32_t enable_divergence_solve;
  uint32_t enable_density_solve;
  double cfl;
  double max_dt;
  double min_dt;
  double pile_gravity[3];
  uint32_t integrate_rigids; /* 1: apply Pile::integrate_kinematics after the fluid step */
  /* 1: periodic in y, the solvers' step<1> (SolverDf / SolverIi / SolverI
   * step_wrap1): neighbor cells wrap in y (wrap_ipos_y, runner.hpp:689-697),
   * displacements and integrated positions wrap into
   * [-wrap_length/2, wrap_length/2) (wrap_y, runner.hpp:698-707).  The grid's
   * y extent must be the period (grid_res[1] cells of size h). */
  uint32_t wrap_y;
  double wrap_length;        /* Const::wrap_length (constants.hpp:130-136) */
} al_solver_params;

/* What one step reports (the solvers' read-only report fields,
 * solver.hpp:274-279, solver_df.hpp:381-385) plus FP64 rigid totals. */
typedef struct al_step_report {
  uint32_t num_divergence_solve;
  uint32_t num_density_solve;
  double mean_density_change;
  double mean_density_error;
  double particle_max_v2;
  double pile_max_v2;
  double max_v2;
  double cfl_dt;
  double utilized_cfl;
  double dt; /* time step used after update_dt */
  uint32_t grid_anomaly[3];
  uint32_t num_active_boundary_pairs; /* (particle, body) pairs with nonzero volume */
  double force[AL_MAX_BOUNDARIES][3];  /* sum_i particle_force[b][i], FP64 */
  double torque[AL_MAX_BOUNDARIES][3];
} al_step_report;

/* ------------------------------------------------------------- lifecycle */
typedef struct al_engine al_engine;

/* Creates an engine bound to CUDA device `device`.  Allocates no particle
 * memory; scratch grows on first use.  Fails with AL_ERR_NO_DEVICE when the
 * device is absent or not compute capability 10.x. */
AL_API int al_engine_create(int device, al_engine** out);
AL_API int al_engine_destroy(al_engine* engine);
/* Static description of a status code. */
AL_API const char* al_status_string(int status);
/* Thread-local text of the last failing call on this thread ("" if none). */
AL_API const char* al_last_error(void);
/* Blocks until all work the engine queued on `stream` has finished. */
AL_API int al_engine_synchronize(al_engine* engine, void* stream);

/* Device memory on the engine's device, the counterpart of the reference's
 * Allocator (allocator.hpp:13-24, 45-74: allocate, free, copy, set), for
 * hosts without a CUDA runtime of their own (the C++ Store of
 * alluvion_b200_solver.hpp).  al_allocate of 0 bytes gives NULL; al_copy
 * copies between any host or device addresses (unified addressing) and,
 * like al_set, returns after the copy has completed. */
AL_API int al_allocate(al_engine* engine, void** ptr, size_t bytes);
AL_API int al_free(al_engine* engine, void* ptr);
AL_API int al_copy(al_engine* engine, void* dst, const void* src, size_t bytes);
AL_API int al_set(al_engine* engine, void* dst, int value, size_t bytes);

/* Step graphs.  With graph mode on (the default), the second and later
 * al_*_step calls with the same constants, grid descriptor, fluid buffer
 * table, body count and enabled solves replay one captured CUDA graph: the
 * divergence and density loops are conditional WHILE nodes whose condition
 * the residual kernels set on the device, so a step costs one graph launch
 * and one synchronisation instead of one flag readback per solver
 * iteration.  Body descriptors, rigid state, dt and the solver parameters
 * are staged through pinned host memory on every call, so they may change
 * between calls; changing any keyed argument (or a scratch buffer growing)
 * makes the next call eager and the one after it capture again.  Steps run
 * eagerly while profiling is on.  No reference counterpart (the reference
 * launches every kernel from the host). */
AL_API int al_engine_set_graph_mode(al_engine* engine, int enable);
/* Number of step graphs captured and of steps run by replaying one. */
AL_API int al_engine_graph_stats(al_engine* engine, uint64_t* captures, uint64_t* replays);

/* Launch shapes of the step's tunable pass groups, the counterpart of the
 * reference's per-kernel block sizes (Runner::optimal_block_size_dict loaded
 * from .alcache, runner.hpp:4922-4937, found by bin/block_scan:15-36).  A
 * shape applies to scenes of 2^bucket <= N < 2^(bucket+1) particles, in
 * single steps (batch = 0) or as a scene of al_df_batch_step_f32 (batch =
 * 1): `block` threads per block (64, 128 or 256) and, for the pair passes
 * that walk neighbor lists, `tpp` threads per particle (1, 2, 4 or 8; the
 * group's lanes split the list and combine partial sums in a fixed order,
 * so float results depend on tpp in the last bits).  0 keeps a field's
 * default (128-thread blocks; tpp 1 from 2^17 particles up, else the
 * smallest of 2, 4, 8 that gives 2^17 threads); 0 / 0 removes the entry.
 * Setting a shape drops the engine's captured step graphs.  Group names are
 * enumerated by al_tunable_group ("finish" is the acceleration and
 * integration pass of IISPH and implicit SPH).  No reference counterpart
 * for tpp. */
AL_API int al_engine_set_launch_shape(al_engine* engine, const char* group, uint32_t bucket,
                                      uint32_t batch, uint32_t block, uint32_t tpp);
/* The shape a step of `num_particles` particles would use for `group`. */
AL_API int al_engine_get_launch_shape(al_engine* engine, const char* group,
                                      uint32_t num_particles, uint32_t batch, uint32_t* block,
                                      uint32_t* tpp);
/* Name of tunable group `index` (static storage) and whether it is a pair
 * pass; AL_ERR_INVALID past the last group. */
AL_API int al_tunable_group(uint32_t index, const char** name, uint32_t* pair);

/* Launch statistics, the counterpart of Runner's per-kernel event timing
 * (launch_stat_dict_, runner.hpp:4835-4859, 6306-6308).  While profiling
 * is on, every launch group is bracketed with CUDA events on its stream and
 * its elapsed time accumulated under its name; off by default (the
 * reference synchronises after every launch; the engine never does).
 * al_engine_launch_count counts kernel launches whether or not profiling
 * is on.  al_engine_kernel_stat returns AL_ERR_INVALID past the last
 * entry. */
AL_API int al_engine_set_profiling(al_engine* engine, int enable);
AL_API int al_engine_reset_stats(al_engine* engine);
AL_API int al_engine_launch_count(al_engine* engine, uint64_t* count);
AL_API int al_engine_kernel_stat(al_engine* engine, uint32_t index, char* name,
                                 size_t name_len, double* total_ms, uint64_t* count);

/* ------------------------------------------------------------ grid / sort
 * Uniform-grid cell hash and stable counting sort.  Replaces the bucket
 * insert of update_particle_grid (runner.hpp:1840-1867): instead of
 * atomic-order buckets the engine produces the canonical order
 * (cell index, original index), cell index = (ix*gy + iy)*gz + iz with
 * (ix,iy,iz) = floor(x / h) - grid_offset (runner.hpp:1827-1838), IEEE
 * division.  Particles outside the grid get cell index UINT32_MAX and sort
 * after every in-grid particle.
 *
 *   particle_x         [N][3] device, in
 *   particle_cell      [N] device, out: cell index per original particle
 *   sorted_to_original [N] device, out: permutation, sorted slot -> index
 *   cell_start         [gx*gy*gz + 1] device, out (may be NULL): first
 *                      sorted slot of each cell; last entry = in-grid count
 *   pid_length         [gx][gy][gz] device, out (may be NULL): particles per
 *                      cell, uncapped (reference buffer solver.hpp:67-73)
 * Returns AL_ERR_OUT_OF_GRID / AL_ERR_CELL_OVERFLOW after writing outputs
 * when the reference would have raised grid_anomaly[0] / [1]. */
AL_API int al_grid_sort_f32(al_engine* engine, const al_const_f32* cn,
                     const al_consti* cni, const float* particle_x,
                     uint32_t num_particles, uint32_t* particle_cell,
                     uint32_t* sorted_to_original, uint32_t* cell_start,
                     uint32_t* pid_length, void* stream);
AL_API int al_grid_sort_f64(al_engine* engine, const al_const_f64* cn,
                     const al_consti* cni, const double* particle_x,
                     uint32_t num_particles, uint32_t* particle_cell,
                     uint32_t* sorted_to_original, uint32_t* cell_start,
                     uint32_t* pid_length, void* stream);

/* The grid sort of al_grid_sort_f32 for callers that must not let the
 * library allocate device memory (a renderer or game engine that owns the
 * memory budget, a real-time loop avoiding the stalls of cudaMalloc /
 * cudaFree).  No counterpart in the reference.  Allocates nothing: all
 * scratch is one static device array of 12.6 MiB, resident on a device
 * from the first call there (CUDA loads the library's device image lazily)
 * until the process exits.  Limits: at most 1,048,576 particles and
 * 1,048,576 grid cells; larger problems return AL_ERR_INVALID.  Uses the
 * current device.  Its first call on a device looks up the array's device
 * address, so make that first call before any stream capture.  Calls share
 * the array: calls that overlap on the GPU race, so order them.
 * Synchronises `stream` before returning (it reads the anomaly flags);
 * returns AL_ERR_OUT_OF_GRID / AL_ERR_CELL_OVERFLOW like al_grid_sort_f32. */
AL_API int al_grid_sort_noalloc_f32(const al_const_f32* cn, const al_consti* cni,
                                    const float* particle_x, uint32_t num_particles,
                                    uint32_t* particle_cell, uint32_t* sorted_to_original,
                                    uint32_t* cell_start, uint32_t* pid_length, void* stream);

/* ------------------------------------------------ neighbors and density
 * Solver::update_particle_neighbors<0> (solver.hpp:225-260) for the
 * volume-map boundary method: grid sort, neighbor list
 * (make_neighbor_list<0>, runner.hpp:1869-1911) and density
 * (compute_density, runner.hpp:2052-2072).
 *
 *   particle_boundary_kernel [nb][N][4] device in, or NULL when
 *                            cni->num_boundaries == 0
 *   particle_density         [N] device out
 *   particle_num_neighbors   [N] device out (min(count, cap))
 *   particle_neighbors       [N][cap][4] device out or NULL; entries are
 *                            {x_i - x_j, bits(j)} in canonical order
 *                            (ascending (cell, index) of j)
 *   grid_anomaly             [3] device out or NULL (reference flags)
 * When a particle has more than cap neighbors the first cap canonical
 * entries are kept and AL_ERR_NEIGHBOR_OVERFLOW is returned. */
AL_API int al_update_particle_neighbors_f32(
    al_engine* engine, const al_const_f32* cn, const al_consti* cni,
    const float* particle_x, uint32_t num_particles,
    const float* particle_boundary_kernel, float* particle_density,
    uint32_t* particle_num_neighbors, float* particle_neighbors,
    uint32_t* grid_anomaly, void* stream);
AL_API int al_update_particle_neighbors_f64(
    al_engine* engine, const al_const_f64* cn, const al_consti* cni,
    const double* particle_x, uint32_t num_particles,
    const double* particle_boundary_kernel, double* particle_density,
    uint32_t* particle_num_neighbors, double* particle_neighbors,
    uint32_t* grid_anomaly, void* stream);
/* update_particle_neighbors<1> (launch_make_neighbor_list_wrap1): the same,
 * periodic in y -- neighbor cells wrap (wrap_ipos_y, runner.hpp:689-697) and
 * the entries' x_i - x_j are wrapped into [-wrap_length/2, wrap_length/2)
 * (wrap_y, runner.hpp:698-707).  The grid's y extent must be the period. */
AL_API int al_update_particle_neighbors_periodic_f32(
    al_engine* engine, const al_const_f32* cn, const al_consti* cni,
    const float* particle_x, uint32_t num_particles,
    const float* particle_boundary_kernel, float* particle_density,
    uint32_t* particle_num_neighbors, float* particle_neighbors,
    uint32_t* grid_anomaly, double wrap_length, void* stream);
AL_API int al_update_particle_neighbors_periodic_f64(
    al_engine* engine, const al_const_f64* cn, const al_consti* cni,
    const double* particle_x, uint32_t num_particles,
    const double* particle_boundary_kernel, double* particle_density,
    uint32_t* particle_num_neighbors, double* particle_neighbors,
    uint32_t* grid_anomaly, double wrap_length, void* stream);

/* ------------------------------------------------------ boundary sampling
 * compute_all_boundaries (solver.hpp:170-185): for every body b and
 * particle i, {x_b, V} into particle_boundary[b][i] and
 * {grad W(x_i - x_b) V, W(d) V} into particle_boundary_kernel[b][i]
 * (compute_particle_boundary / _analytic<0>, runner.hpp:1982-2025).
 *   bodies  host array [num_boundaries]; node arrays are device pointers
 *   rigid   host array [num_boundaries] (pose at this step) */
AL_API int al_compute_particle_boundary_f32(
    al_engine* engine, const al_const_f32* cn, uint32_t num_boundaries,
    const al_body_f32* bodies, const al_rigid_f32* rigid, const float* particle_x,
    uint32_t num_particles, float* particle_boundary, float* particle_boundary_kernel,
    void* stream);
AL_API int al_compute_particle_boundary_f64(
    al_engine* engine, const al_const_f64* cn, uint32_t num_boundaries,
    const al_body_f64* bodies, const al_rigid_f64* rigid, const double* particle_x,
    uint32_t num_particles, double* particle_boundary, double* particle_boundary_kernel,
    void* stream);

/* Volume-map nodes of one body (update_volume_field, runner.hpp:1616-1694,
 * launched by Pile::build_grid, pile.hpp:523-622): Peirce m = 14 ball
 * quadrature (27,000 samples per node) of the body's distance -- from
 * body->distance_nodes when use_distance_grid, else the analytic shape.
 * volume_nodes: device [body->num_nodes] out. */
AL_API int al_build_volume_field_f32(al_engine* engine, const al_const_f32* cn,
                                     const al_body_f32* body, float* volume_nodes,
                                     void* stream);
AL_API int al_build_volume_field_f64(al_engine* engine, const al_const_f64* cn,
                                     const al_body_f64* body, double* volume_nodes,
                                     void* stream);

/* Distance nodes sampled from the body's analytic shape at the Lagrange
 * node positions -- the role of Pile::construct_distance_grid
 * (pile.hpp:79-94) for mesh bodies.  distance_nodes: device out. */
AL_API int al_build_distance_grid_f32(al_engine* engine, const al_body_f32* body,
                                      float* distance_nodes, void* stream);
AL_API int al_build_distance_grid_f64(al_engine* engine, const al_body_f64* body,
                                      double* distance_nodes, void* stream);

/* Node positions of the body's grid (index_to_node_position,
 * runner.hpp:1131-1178).  positions: device [num_nodes][3] out. */
AL_API int al_node_positions_f32(al_engine* engine, const al_body_f32* body, float* positions,
                                 void* stream);
AL_API int al_node_positions_f64(al_engine* engine, const al_body_f64* body, double* positions,
                                 void* stream);

/* Distance grid of a triangle-mesh body (AL_SHAPE_MESH), on the device: the
 * grid Pile builds on the host for MeshDistance bodies (pile.hpp:79-94,
 * 512-521; MeshDistance::signedDistance, dg/mesh_distance.hpp:186-223):
 * exact point-triangle distance, sign from angle-weighted pseudonormals of
 * the nearest feature, minus `offset`.  The mesh (host arrays, body frame)
 * must be a closed 2-manifold, as the reference requires.  body: domain,
 * resolution and num_nodes; nodes: device [num_nodes].  Synchronous. */
AL_API int al_build_mesh_distance_grid_f32(al_engine* engine, const al_body_f32* body,
                                           const float* vertices, uint32_t num_vertices,
                                           const uint32_t* faces, uint32_t num_faces,
                                           float offset, float* nodes, void* stream);

/* ------------------------------------------------------------ fluid steps
 * The caller-owned particle buffers of one solver (solver.hpp:286-305,
 * solver_df.hpp:367-370, solver_ii.hpp:250-257).  Required: particle_x,
 * particle_v.  Every other pointer may be NULL (not read / not written).
 *   in/out: particle_x, particle_v, particle_kappa, particle_kappa_v
 *           (DFSPH warm-start state), particle_pressure (IISPH)
 *   out:    particle_a (non-pressure acceleration), particle_density,
 *           particle_dfsph_factor, particle_density_adv,
 *           particle_boundary / particle_boundary_kernel ([nb][N][4]) */
typedef struct al_fluid_f32 {
  uint32_t num_particles;
  uint32_t reserved;
  float* particle_x;
  float* particle_v;
  float* particle_a;
  float* particle_density;
  float* particle_dfsph_factor;
  float* particle_kappa;
  float* particle_kappa_v;
  float* particle_density_adv;
  float* particle_pressure;
  float* particle_boundary;
  float* particle_boundary_kernel;
} al_fluid_f32;

typedef struct al_fluid_f64 {
  uint32_t num_particles;
  uint32_t reserved;
  double* particle_x;
  double* particle_v;
  double* particle_a;
  double* particle_density;
  double* particle_dfsph_factor;
  double* particle_kappa;
  double* particle_kappa_v;
  double* particle_density_adv;
  double* particle_pressure;
  double* particle_boundary;
  double* particle_boundary_kernel;
} al_fluid_f64;

/* One DFSPH step: SolverDf<TF>::step<0> (solver_df.hpp:74-359) without
 * contacts (pile.hpp:826-979).  bodies: host [num_boundaries]; rigid: host
 * [num_boundaries] in/out (integrated when params->integrate_rigids);
 * dt: host in/out (in: step's initial dt, out: dt after update_dt);
 * report: host out, may be NULL.  Synchronous: returns after the step has
 * completed on `stream`. */
AL_API int al_df_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                          const al_fluid_f32* fluid, const al_body_f32* bodies,
                          al_rigid_f32* rigid, const al_solver_params* params, float* dt,
                          al_step_report* report, void* stream);
AL_API int al_df_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                          const al_fluid_f64* fluid, const al_body_f64* bodies,
                          al_rigid_f64* rigid, const al_solver_params* params, double* dt,
                          al_step_report* report, void* stream);

/* One IISPH step: SolverIi<TF>::step<0> (solver_ii.hpp:76-243) without
 * contacts.  Same conventions as al_df_step; uses particle_pressure. */
AL_API int al_ii_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                          const al_fluid_f32* fluid, const al_body_f32* bodies,
                          al_rigid_f32* rigid, const al_solver_params* params, float* dt,
                          al_step_report* report, void* stream);
AL_API int al_ii_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                          const al_fluid_f64* fluid, const al_body_f64* bodies,
                          al_rigid_f64* rigid, const al_solver_params* params, double* dt,
                          al_step_report* report, void* stream);

/* One implicit SPH step: SolverI<TF>::step<0> (solver_i.hpp:79-327) with
 * volume-map boundaries, without contacts: advect_and_init_pressure,
 * calculate_isph_diagonal_adv_density and damped-Jacobi
 * isph_solve_iteration (runner.hpp:2889-3053) until the mean density error
 * is under density_error_tolerance (min/max_density_solve), then
 * compute_pressure_accels and kinematic_integration.  Same conventions as
 * al_ii_step: uses particle_pressure (in/out); particle_density_adv receives
 * the advected density. */
AL_API int al_i_step_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                         const al_fluid_f32* fluid, const al_body_f32* bodies,
                         al_rigid_f32* rigid, const al_solver_params* params, float* dt,
                         al_step_report* report, void* stream);
AL_API int al_i_step_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                         const al_fluid_f64* fluid, const al_body_f64* bodies,
                         al_rigid_f64* rigid, const al_solver_params* params, double* dt,
                         al_step_report* report, void* stream);

/* ------------------------------------------------- pellet boundary model
 * Bodies represented by boundary particles ("pellets", Pile with
 * VolumeMethod::pellets): SolverI<TF>::step<0> (solver_i.hpp:79-327) on the
 * pellet branch, without contacts --
 *   transform_pellets (runner.hpp:4070-4082) from each body's pose,
 *   one grid over particles and pellets, bead / pellet neighbor lists
 *   (make_bead_pellet_neighbor_list, runner.hpp:1912-1966: particle j < N
 *   is a bead, j >= N a pellet; pellets get lists too),
 *   compute_density_with_pellets (runner.hpp:2074-2098),
 *   compute_viscosity_with_pellets (runner.hpp:2251-2299),
 *   calculate_isph_diagonal_adv_density_with_pellets (runner.hpp:2955-3004),
 *   per iteration extrapolate_pressure_to_pellet (runner.hpp:2543-2607,
 *   Shepard average + linear moving-least-squares term through a 3x3
 *   pseudo-inverse with singular values below 1e-2 dropped) and
 *   isph_solve_iteration_with_pellets (runner.hpp:3055-3121),
 *   compute_pressure_accels_with_pellets (runner.hpp:2819-2871),
 *   kinematic_integration, per-body totals and Pile::integrate_kinematics.
 * Pellets weigh as fluid particles of rest density rho0.  Bodies need
 * mass, inertia and max_distance; their node arrays are not read.
 * params->wrap_y selects step<1> (periodic in y, as for al_i_step_f32).
 * Eager: the host reads the loop flag after every iteration. */
typedef struct al_pellets_f32 {
  const float* local_x;  /* device [num_pellets][3]: body frame, body after body */
  uint32_t num_pellets;
  uint32_t count[AL_MAX_BOUNDARIES]; /* pellets of each body, in body order */
  float* x;              /* device [num_pellets][3] out or NULL: world positions */
  float* pressure;       /* device [num_pellets] out or NULL: extrapolated pressure */
  float* v;              /* device [num_pellets][3] out or NULL: pellet velocities */
} al_pellets_f32;

typedef struct al_pellets_f64 {
  const double* local_x;
  uint32_t num_pellets;
  uint32_t count[AL_MAX_BOUNDARIES];
  double* x;
  double* pressure;
  double* v;
} al_pellets_f64;

AL_API int al_i_step_pellets_f32(al_engine* engine, const al_const_f32* cn,
                                 const al_consti* cni, const al_fluid_f32* fluid,
                                 const al_body_f32* bodies, al_rigid_f32* rigid,
                                 const al_pellets_f32* pellets, const al_solver_params* params,
                                 float* dt, al_step_report* report, void* stream);
AL_API int al_i_step_pellets_f64(al_engine* engine, const al_const_f64* cn,
                                 const al_consti* cni, const al_fluid_f64* fluid,
                                 const al_body_f64* bodies, al_rigid_f64* rigid,
                                 const al_pellets_f64* pellets, const al_solver_params* params,
                                 double* dt, al_step_report* report, void* stream);

/* Pellet relaxation: SolverPellet<TF>::step<wrap> (solver_pellet.hpp:57-119),
 * the reference's tool that spreads boundary particles ("pellets") over a
 * body by repeated steps of
 *   update_particle_neighbors (pellet branch: density m (W(0) + sum W)),
 *   compute_cohesion_adhesion_displacement (runner.hpp:2453-2532):
 *     dx = -cohesion sum_j m / rho_j (1 - 2r / |x_ij|) W x_ij
 *          - adhesion m / rho_i W(d) d n   (d, n: the body's distance and
 *          normal at x_i minus contact_tolerance on the analytic branch),
 *   compute_dfsph_factor_with_pellets (runner.hpp:3156-3190),
 *   pellet_divergence_solve_iteration (runner.hpp:3365-3395),
 *   cfl = min(cfl_factor 0.4 (2r) / max |dx|, 1) (solver_pellet.hpp:100-103),
 *   move_and_avoid_boundary (runner.hpp:4010-4066): x += cfl dx, pushed back
 *     to distance r from the body.
 * The body is evaluated in its own frame at the particle positions (the
 * reference's pile holds this one body at the origin); a mesh body uses its
 * distance grid, every other shape its analytic distance.  `body` is a host
 * struct (device node arrays); particle_x (device, [n][3]) is updated in
 * place; particle_dx ([n][3], the reference's particle_v) and
 * particle_density ([n]) receive the last step's values when non-NULL. */
typedef struct al_pellet_relax_params {
  double cohesion;          /* SolverPellet::cohesion (default 4) */
  double adhesion;          /* SolverPellet::adhesion (default 2) */
  double cfl_factor;        /* SolverPellet::cfl_factor (default 0.25) */
  double contact_tolerance; /* Const::contact_tolerance */
  uint32_t wrap_y;          /* 1: step<1> (periodic in y) */
  uint32_t reserved;
  double wrap_length;
} al_pellet_relax_params;

AL_API int al_relax_pellets_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                                const al_body_f32* body, float* particle_x, uint32_t num_particles,
                                const al_pellet_relax_params* params, uint32_t steps,
                                float* particle_dx, float* particle_density, void* stream);
AL_API int al_relax_pellets_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                                const al_body_f64* body, double* particle_x,
                                uint32_t num_particles, const al_pellet_relax_params* params,
                                uint32_t steps, double* particle_dx, double* particle_density,
                                void* stream);

/* ---------------------------------------------------- learned warm start
 * No reference counterpart.  A per-particle MLP 12 -> 64 -> 64 -> 2 with
 * GELU (tanh form), BF16 operands and FP32 accumulation on the tensor
 * cores, predicts the converged kappa_v and kappa of a DFSPH step from
 * features available when the step starts; the predictions replace the
 * previous-step warm starts (runner.hpp:3230-3249, 3430-3449) under the
 * same gates (rho_dot > 0, rho_adv > 1).  The solves' tolerances still
 * decide convergence, so the result stays within tolerance and only the
 * iteration counts change.
 *
 * Features (raw FP32, particle order), at the start of the step:
 *   0 rho / rho0 - 1                1 rho_dot * dt (clamped >= 0; 0 if < 20 neighbors)
 *   2 neighbors / 32                3 previous kappa_v (particle_kappa_v / dt)
 *   4 previous kappa (particle_kappa / dt^2)
 *   5 sum of boundary volumes / particle volume
 *   6 |v|                            7 |v| dt / (2 r)
 *   8 DFSPH factor (before the 1/dt scaling)
 *   9 boundary density term sum_b (W V)_b
 *  10 |sum_j V grad W_ij + sum_b (grad W V)_b| * 2 r     11 dt
 * Targets: the converged kappa_v (particle_kappa_v / dt after the step) and
 * kappa (particle_kappa / dt^2 after the step). */
#define AL_WARM_NUM_FEATURES 12
#define AL_WARM_HIDDEN 64
#define AL_WARM_NUM_OUTPUTS 2
/* flat FP32 parameters: W1[64][12], b1[64], W2[64][64], b2[64], W3[2][64], b3[2] */
#define AL_WARM_NUM_PARAMS 5122

typedef struct al_warm_net {
  const float* params;       /* device, AL_WARM_NUM_PARAMS FP32 (rounded to BF16 for the MMAs) */
  float feature_shift[AL_WARM_NUM_FEATURES]; /* input = (feature - shift) * scale */
  float feature_scale[AL_WARM_NUM_FEATURES];
  float output_scale[AL_WARM_NUM_OUTPUTS];   /* kappa_v = y0 * scale0, kappa = y1 * scale1 */
  uint32_t reserved[2];
} al_warm_net;

/* out[p][0..1] = predicted {kappa_v, kappa} of features[p] (device [n][12]
 * raw FP32) for p < n.  AL_ERR_TIMEOUT if a bounded tensor-core wait gave
 * up. */
AL_API int al_warm_net_forward_f32(al_engine* engine, const al_warm_net* net,
                                   const float* features, uint32_t n, float* out,
                                   void* stream);

/* Loss L = 0.5 / n * sum_p |y_p - t_p|^2 of the network outputs y (before
 * output_scale) against targets[p] / output_scale (targets: device [n][2]
 * raw {kappa_v, kappa}), and dL/dparams into grad (device
 * [AL_WARM_NUM_PARAMS]), with the tensor cores' own forward and backward
 * kernels; the gradient is summed over the batch in a fixed order
 * (deterministic).  loss: host out, may be NULL. */
AL_API int al_warm_net_gradient_f32(al_engine* engine, const al_warm_net* net,
                                    const float* features, const float* targets, uint32_t n,
                                    float* grad, double* loss, void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8; step counts from 1) on
 * the FP32 master parameters; m, v: device [AL_WARM_NUM_PARAMS] moments.
 * Asynchronous on `stream`. */
AL_API int al_warm_net_adam_f32(al_engine* engine, float* params, const float* grad, float* m,
                                float* v, uint32_t step, float lr, void* stream);

/* Warm-start options of al_df_step_warm_f32. */
typedef struct al_warm_start {
  const al_warm_net* net; /* NULL: the reference's previous-step warm starts */
  float* features_out;    /* NULL or device [N][12]: this step's features, particle order */
} al_warm_start;

/* al_df_step_f32 with the learned warm start (warm->net) and/or the
 * features of the step written out for training (warm->features_out).
 * The engine keeps a per-scene gate on the device: the network runs on the
 * scene's first step, then only after a step whose solves went beyond their
 * minimum iteration counts and while its last outcome (iterations of the
 * last step that ran it) is no worse than the plain start's last outcome,
 * or when it has not run for 64 steps; other steps use the reference's
 * previous-step warm starts.
 * Float32 DFSPH with the divergence solve enabled only
 * (AL_ERR_UNSUPPORTED otherwise); AL_ERR_TIMEOUT if a bounded tensor-core
 * wait gave up (the step's outputs are then invalid). */
AL_API int al_df_step_warm_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                               const al_fluid_f32* fluid, const al_body_f32* bodies,
                               al_rigid_f32* rigid, const al_solver_params* params,
                               const al_warm_start* warm, float* dt, al_step_report* report,
                               void* stream);

/* ------------------------------------------------------------- contacts
 * Rigid-rigid contacts on the device: Pile::find_contacts (pile.hpp:886-900,
 * volume-map branch) with collision_test (runner.hpp:3833-4010; analytic
 * distance for analytic bodies, the distance grid through
 * collision_find_dist_normal, runner.hpp:1793-1822, for bodies with
 * use_distance_grid) and Pile::solve_contacts (pile.hpp:906-979).  The
 * reference appends contacts with an atomic counter, so its contact order
 * and hence its sequential-impulse result vary from run to run; the
 * engine lists contacts in (i, j, vertex) order, deterministically. */
typedef struct al_contact_body_f32 {
  const float* vertices;  /* device [num_vertices][3], body frame (collision vertices) */
  uint32_t num_vertices;
  float restitution;      /* pair restitution: product of the two bodies' */
  float friction;         /* pair friction: sum of the two bodies' */
  uint32_t reserved;
} al_contact_body_f32;

/* Contact<float3, float> (contact.hpp:8-25). */
typedef struct al_contact_f32 {
  uint32_t i, j;
  float cp_i[3], cp_j[3], n[3], t[3];
  float iiwi_diag[3], iiwi_off_diag[3], iiwj_diag[3], iiwj_off_diag[3];
  float friction, nkninv, pmax, goalu, impulse_sum;
} al_contact_f32;

/* Tests every collision vertex of body i against body j for each ordered
 * pair i != j (not both kinematic, mass 0) and writes the contacts
 * (dist - contact_tolerance < 0) to `contacts` (device, up to
 * max_contacts) in (i, j, vertex) order; *num_found (host) receives the
 * count found, which may exceed max_contacts (the reference then clamps,
 * pile.hpp:908-914).  bodies / rigid / contact_bodies: host arrays. */
AL_API int al_find_contacts_f32(al_engine* engine, const al_body_f32* bodies,
                                const al_rigid_f32* rigid,
                                const al_contact_body_f32* contact_bodies, uint32_t num_bodies,
                                float contact_tolerance, uint32_t max_contacts,
                                al_contact_f32* contacts, uint32_t* num_found, void* stream);
/* Five sequential-impulse sweeps over contacts[0, num_contacts) (device),
 * in order, on the device; rigid (host in/out): v and omega updated. */
AL_API int al_solve_contacts_f32(al_engine* engine, const al_body_f32* bodies,
                                 al_rigid_f32* rigid, uint32_t num_bodies,
                                 al_contact_f32* contacts, uint32_t num_contacts, void* stream);

/* ------------------------------------------------------- batched scenes
 * No reference counterpart (the reference advances one scene per call).
 * Advances every scene by one DFSPH step (each with its own dt, iteration
 * counts and report; same semantics as al_df_step_f32 per scene).  From the
 * second call with the same configuration on, the whole batch is one
 * captured CUDA graph: one launch and one synchronisation for all scenes.
 *
 * Fused (the default, when every scene has particles, the same constants
 * `cn`, the same solves enabled and no periodic wrap): the scenes' particles
 * share one device arena and every solver pass is ONE kernel launch over
 * all scenes, each block finding its scene in a block -> scene table: one
 * counting sort over all scenes' cells, then gather, boundary sampling,
 * neighbor build, every solver pass, write-back and rigid totals.  The
 * solver loops are one device-driven loop in which a scene whose solve has
 * converged sits out the remaining iterations, so each scene runs exactly
 * its own iterations.  Pair passes run one thread per particle in
 * 128-thread blocks.  The scenes' control blocks, bodies and rigid state are
 * uploaded and read back in one copy each.  Out-of-grid particles (an
 * AL_ERR_OUT_OF_GRID step) are ordered by index in their tail bucket.
 * Otherwise (or after al_engine_set_batch_fused(engine, 0)): the graph's
 * parallel branches are the scenes' whole steps, each with its own scratch
 * and launch shapes (the shape table's batch context).
 * With 128-thread blocks and one thread per particle for every pair pass in
 * the batch context, both forms give bit-identical results.
 * Returns AL_OK, or the first scene's failure; every scene's own status is
 * in scenes[k].status. */
AL_API int al_engine_set_batch_fused(al_engine* engine, int enable);
#define AL_MAX_BATCH 256
typedef struct al_scene_f32 {
  const al_const_f32* cn;
  const al_consti* cni;
  const al_fluid_f32* fluid;
  const al_body_f32* bodies;
  al_rigid_f32* rigid;
  const al_solver_params* params;
  float* dt;               /* host in/out */
  al_step_report* report;  /* host out, may be NULL */
  int status;              /* out */
  uint32_t reserved;
} al_scene_f32;

AL_API int al_df_batch_step_f32(al_engine* engine, al_scene_f32* scenes, uint32_t num_scenes,
                                void* stream);

/* ------------------------------------------------------------- sampling
 * Fluid quantities at sample points, with the reference's sample neighbor
 * list (make_neighbor_list over sample_x, runner.hpp:1869-1911: the 27
 * cells around the sample, candidates j != sample index -- the reference
 * compares the particle index with the sample's -- closer than h) and:
 *   sample_density           sample_fluid_density (runner.hpp:4193-4209):
 *                            rho0 sum_j V W
 *   sample_position_density  sample_position_density (runner.hpp:2100-2121):
 *                            rho0 (sum_j V W + sum_b (W V)_b)
 *   sample_quantity          sample_fluid (runner.hpp:4173-4191) of a
 *                            1- or 3-component particle quantity:
 *                            sum_j m / rho_j W q_j
 *   sample_v                 compute_sample_velocity (runner.hpp:4211-4240):
 *                            sum_j m / rho_j W v_j + sum_b v_b (W V)_b
 *   sample_vorticity         compute_sample_vorticity (runner.hpp:4289-4323):
 *                            sum_j m / rho_j (v_j - v_s) x grad W
 *                            + sum_b (v_b - v_s) x (grad W V)_b
 * v_b = omega x (x_b - x) + v of body b at its boundary point x_b.  The
 * body terms run over cni->num_boundaries bodies and read the samples'
 * boundary arrays from al_compute_particle_boundary_f32 called with the
 * sample positions, and `rigid` (host array, the bodies' states).  Each
 * output is computed when its pointer is non-NULL; vorticity needs sample_v.
 * All arrays are device pointers in the reference's layouts.  More than
 * max_num_neighbors_per_particle neighbors return AL_ERR_NEIGHBOR_OVERFLOW
 * (the first ones in canonical order are summed). */
typedef struct al_sample_f32 {
  const float* sample_x;               /* [num_samples][3] */
  uint32_t num_samples;
  uint32_t quantity_dim;               /* 1 or 3 when sample_quantity is set */
  const float* particle_density;       /* [N], for quantity / velocity / vorticity */
  const float* particle_v;             /* [N][3], for velocity / vorticity */
  const float* particle_quantity;      /* [N][quantity_dim] */
  const float* sample_boundary;        /* [num_boundaries][num_samples][4] {x_b, V} */
  const float* sample_boundary_kernel; /* [num_boundaries][num_samples][4] {grad W V, W V} */
  float* sample_density;               /* [num_samples] out or NULL */
  float* sample_position_density;      /* [num_samples] out or NULL */
  float* sample_quantity;              /* [num_samples][quantity_dim] out or NULL */
  float* sample_v;                     /* [num_samples][3] out or NULL */
  float* sample_vorticity;             /* [num_samples][3] out or NULL */
  /* 1: periodic in y (make_neighbor_list<1>): neighbor cells wrap in y
   * (wrap_ipos_y, runner.hpp:689-697) and displacements are wrapped into
   * [-wrap_length/2, wrap_length/2) (wrap_y, runner.hpp:698-707) */
  uint32_t wrap_y;
  float wrap_length;                   /* Const::wrap_length (constants.hpp:130-136) */
  /* pellet boundary model (the *_with_pellets sampling kernels,
   * runner.hpp:2122-2147, 4242-4275, 4325-4357): pellets join the grid after
   * the particles; position density becomes m (sum_particles W + sum_pellets W),
   * velocity adds V W v_p, vorticity V (v_p - v_s) x grad W, and no
   * volume-map body terms are added */
  const float* pellet_x;               /* [num_pellets][3] world positions */
  const float* pellet_v;               /* [num_pellets][3], for velocity / vorticity */
  uint32_t num_pellets;
  uint32_t reserved;
} al_sample_f32;

AL_API int al_sample_fluid_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                               const float* particle_x, uint32_t num_particles,
                               const al_rigid_f32* rigid, const al_sample_f32* request,
                               void* stream);
/* The same in double (Runner<double>): every array and wrap_length double. */
typedef struct al_sample_f64 {
  const double* sample_x;
  uint32_t num_samples;
  uint32_t quantity_dim;
  const double* particle_density;
  const double* particle_v;
  const double* particle_quantity;
  const double* sample_boundary;
  const double* sample_boundary_kernel;
  double* sample_density;
  double* sample_position_density;
  double* sample_quantity;
  double* sample_v;
  double* sample_vorticity;
  uint32_t wrap_y;
  uint32_t reserved0;
  double wrap_length;
  const double* pellet_x;
  const double* pellet_v;
  uint32_t num_pellets;
  uint32_t reserved;
} al_sample_f64;

AL_API int al_sample_fluid_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                               const double* particle_x, uint32_t num_particles,
                               const al_rigid_f64* rigid, const al_sample_f64* request,
                               void* stream);

/* compute_density_mask (runner.hpp:4359-4365): mask[i] = density[i] > 0.
 * Device arrays. */
AL_API int al_density_mask_f32(al_engine* engine, const float* sample_density,
                               uint32_t num_samples, uint32_t* mask, void* stream);
AL_API int al_density_mask_f64(al_engine* engine, const double* sample_density,
                               uint32_t num_samples, uint32_t* mask, void* stream);

/* compute_boundary_mask (runner.hpp:4367-4396, launched by
 * Runner::launch_compute_boundary_mask, runner.hpp:5516-5600):
 * mask[i] *= (sign d(x_i) >= distance_threshold), d the body's signed
 * distance at the sample in its frame -- the distance grid for a mesh
 * body, the analytic shape otherwise.  body, rigid: host; sample_x, mask:
 * device. */
AL_API int al_boundary_mask_f32(al_engine* engine, const al_body_f32* body,
                                const al_rigid_f32* rigid, const float* sample_x,
                                uint32_t num_samples, float distance_threshold, float* mask,
                                void* stream);
AL_API int al_boundary_mask_f64(al_engine* engine, const al_body_f64* body,
                                const al_rigid_f64* rigid, const double* sample_x,
                                uint32_t num_samples, double distance_threshold, double* mask,
                                void* stream);

/* compute_distance_mask_multiple (runner.hpp:4272-4287):
 * mask[k][i] = |buoy_x[k] - grid_x[i]|^2 <= threshold^2.  Device arrays. */
AL_API int al_distance_mask_multiple_f32(al_engine* engine, const float* grid_x,
                                         uint32_t num_grid_points, const float* buoy_x,
                                         uint32_t num_buoys, float distance_threshold,
                                         float* mask, void* stream);
AL_API int al_distance_mask_multiple_f64(al_engine* engine, const double* grid_x,
                                         uint32_t num_grid_points, const double* buoy_x,
                                         uint32_t num_buoys, double distance_threshold,
                                         double* mask, void* stream);

/* Runner::launch_histogram256[_with_mask] (runner.hpp:5849-5889; kernels
 * quantize, histogram256[_with_mask], merge_histogram256,
 * runner.hpp:4399-4536): histogram[b] = number of i < n (with mask[i] == 1
 * when mask is non-NULL) whose byte (floor((v[i] - v_min) * step_inverse)
 * saturated to uint32, low 8 bits) is b, step_inverse =
 * float(256 / (double(v_max) - double(v_min))).  One pass over v (and
 * mask); histogram: device [256] out. */
AL_API int al_histogram256_f32(al_engine* engine, const float* v, const float* mask, uint32_t n,
                               float v_min, float v_max, uint32_t* histogram, void* stream);
/* Runner<double>: step_inverse = 256 / (v_max - v_min) in double, and the
 * quantize kernel's (v - v_min) * step_inverse, formed in double, reaches
 * __float2uint_rd through the implicit conversion to float (round to
 * nearest): byte = floor(float((v - v_min) * step_inverse)) saturated,
 * low 8 bits. */
AL_API int al_histogram256_f64(al_engine* engine, const double* v, const double* mask,
                               uint32_t n, double v_min, double v_max, uint32_t* histogram,
                               void* stream);

/* Runner::calculate_kl_divergence (runner.hpp:4803-4815, KLDivergence
 * runner.hpp:746-762): sum over bins with p > 0 of
 * p / n_p log(p / max(q, q_lower_bound) n_q / n_p), evaluated in double
 * with a fixed-order reduction.  histogram_p, histogram_q: device [num_bins]; result: host. */
AL_API int al_kl_divergence(al_engine* engine, const uint32_t* histogram_p,
                            const uint32_t* histogram_q, uint32_t n_p, uint32_t n_q,
                            double q_lower_bound, uint32_t num_bins, double* result,
                            void* stream);

/* ------------------------------------------------------------- metrics
 * The Runner reductions that score sampled fields against targets
 * (runner.hpp:715-744, 4710-4800).  v0, v1: device [n][dims] (dims 1..4,
 * the reference's scalar or vector element); per-element terms in the
 * arrays' real type (correctly rounded, no contraction), sums in double in
 * a fixed order (the reference sums in the real type with
 * thrust::transform_reduce).  result: host.
 *   al_calculate_se_*           se[i] = |v0[i] - v1[i]|^2 (device [n] out)
 *   al_calculate_se_weighted_*  *result = sum_i weight[i] |v0[i] - v1[i]|^2
 *   al_calculate_se_yz_masked_* *result = sum over mask[i] == 1 of
 *                               (v0 - v1).y^2 + (v0 - v1).z^2  (dims 3)
 *   al_sum_products_*           result[k] = sum_i v0[i][k] v1[i][k], k < dims */
AL_API int al_calculate_se_f32(al_engine* engine, const float* v0, const float* v1, float* se,
                               uint32_t n, uint32_t dims, void* stream);
AL_API int al_calculate_se_f64(al_engine* engine, const double* v0, const double* v1,
                               double* se, uint32_t n, uint32_t dims, void* stream);
AL_API int al_calculate_se_weighted_f32(al_engine* engine, const float* v0, const float* v1,
                                        const float* weight, uint32_t n, uint32_t dims,
                                        double* result, void* stream);
AL_API int al_calculate_se_weighted_f64(al_engine* engine, const double* v0, const double* v1,
                                        const double* weight, uint32_t n, uint32_t dims,
                                        double* result, void* stream);
AL_API int al_calculate_se_yz_masked_f32(al_engine* engine, const float* v0, const float* v1,
                                         const float* mask, uint32_t n, double* result,
                                         void* stream);
AL_API int al_calculate_se_yz_masked_f64(al_engine* engine, const double* v0, const double* v1,
                                         const double* mask, uint32_t n, double* result,
                                         void* stream);
AL_API int al_sum_products_f32(al_engine* engine, const float* v0, const float* v1, uint32_t n,
                               uint32_t dims, double* result, void* stream);
AL_API int al_sum_products_f64(al_engine* engine, const double* v0, const double* v1, uint32_t n,
                               uint32_t dims, double* result, void* stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* ALLUVION_B200_H */
