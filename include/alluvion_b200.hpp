/*
 * alluvion_b200.hpp -- header-only C++ layer over the C ABI of
 * alluvion_b200.h for hosts written in C++ (the reference's compiled
 * solvers).  It adds no entry points: it owns an al_engine, picks the
 * float / double entry point from the template argument, and turns the
 * failure statuses into exceptions the way the reference's
 * Allocator::abort_if_error turns CUDA errors into std::runtime_error
 * (lib/allocator.cu:35-41).  The capacity anomalies (AL_ERR_OUT_OF_GRID,
 * AL_ERR_CELL_OVERFLOW, AL_ERR_NEIGHBOR_OVERFLOW) are the reference's
 * grid_anomaly flags, which it reports without throwing; they come back in
 * the step report and, by default, do not throw here either.
 */
#ifndef ALLUVION_B200_HPP
#define ALLUVION_B200_HPP

#include <stdexcept>
#include <string>
#include <utility>

#include "alluvion_b200.h"

namespace alluvion_b200 {

class error : public std::runtime_error {
 public:
  error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int status() const noexcept { return status_; }

 private:
  int status_;
};

inline bool is_anomaly(int status) {
  return status == AL_ERR_OUT_OF_GRID || status == AL_ERR_CELL_OVERFLOW ||
         status == AL_ERR_NEIGHBOR_OVERFLOW;
}

// Throws for every status but AL_OK (and the anomalies unless
// anomalies_throw).
inline void check(int status, const char* where, bool anomalies_throw = false) {
  if (status == AL_OK || (!anomalies_throw && is_anomaly(status))) return;
  const char* detail = al_last_error();
  std::string msg = std::string(where) + ": " + al_status_string(status);
  if (detail && *detail) msg += std::string(" (") + detail + ")";
  throw error(status, msg);
}

// One al_engine on a CUDA device, released with the object.
class engine {
 public:
  explicit engine(int device = 0) { check(al_engine_create(device, &e_), "al_engine_create"); }
  ~engine() {
    if (e_) al_engine_destroy(e_);
  }
  engine(const engine&) = delete;
  engine& operator=(const engine&) = delete;
  engine(engine&& o) noexcept : e_(std::exchange(o.e_, nullptr)) {}
  engine& operator=(engine&& o) noexcept {
    if (this != &o) {
      if (e_) al_engine_destroy(e_);
      e_ = std::exchange(o.e_, nullptr);
    }
    return *this;
  }
  al_engine* get() const noexcept { return e_; }
  void synchronize(void* stream = nullptr) const {
    check(al_engine_synchronize(e_, stream), "al_engine_synchronize");
  }
  void set_graph_mode(bool on) const {
    check(al_engine_set_graph_mode(e_, on ? 1 : 0), "al_engine_set_graph_mode");
  }

 private:
  al_engine* e_ = nullptr;
};

// The C types and entry points of one real type.
template <class TF>
struct real;
template <>
struct real<float> {
  using cn = al_const_f32;
  using fluid = al_fluid_f32;
  using body = al_body_f32;
  using rigid = al_rigid_f32;
  using pellets = al_pellets_f32;
  static constexpr auto df_step = al_df_step_f32;
  static constexpr auto ii_step = al_ii_step_f32;
  static constexpr auto i_step = al_i_step_f32;
  static constexpr auto i_step_pellets = al_i_step_pellets_f32;
  static constexpr auto relax_pellets = al_relax_pellets_f32;
  static constexpr auto update_particle_neighbors = al_update_particle_neighbors_f32;
  static constexpr auto update_particle_neighbors_periodic =
      al_update_particle_neighbors_periodic_f32;
  static constexpr auto compute_particle_boundary = al_compute_particle_boundary_f32;
  static constexpr auto build_volume_field = al_build_volume_field_f32;
  static constexpr auto build_distance_grid = al_build_distance_grid_f32;
};
template <>
struct real<double> {
  using cn = al_const_f64;
  using fluid = al_fluid_f64;
  using body = al_body_f64;
  using rigid = al_rigid_f64;
  using pellets = al_pellets_f64;
  static constexpr auto df_step = al_df_step_f64;
  static constexpr auto ii_step = al_ii_step_f64;
  static constexpr auto i_step = al_i_step_f64;
  static constexpr auto i_step_pellets = al_i_step_pellets_f64;
  static constexpr auto relax_pellets = al_relax_pellets_f64;
  static constexpr auto update_particle_neighbors = al_update_particle_neighbors_f64;
  static constexpr auto update_particle_neighbors_periodic =
      al_update_particle_neighbors_periodic_f64;
  static constexpr auto compute_particle_boundary = al_compute_particle_boundary_f64;
  static constexpr auto build_volume_field = al_build_volume_field_f64;
  static constexpr auto build_distance_grid = al_build_distance_grid_f64;
};

// The solvers' step<wrap>: SolverDf (df), SolverIi (ii), SolverI (i), each
// one call; wrap is params.wrap_y.
enum class method { df, ii, i };

template <class TF>
al_step_report step(const engine& e, method m, const typename real<TF>::cn& cn,
                    const al_consti& cni, const typename real<TF>::fluid& fluid,
                    const typename real<TF>::body* bodies, typename real<TF>::rigid* rigid,
                    const al_solver_params& params, TF& dt, void* stream = nullptr) {
  al_step_report rep{};
  const auto fn = m == method::df ? real<TF>::df_step
                  : m == method::ii ? real<TF>::ii_step
                                    : real<TF>::i_step;
  check(fn(e.get(), &cn, &cni, &fluid, bodies, rigid, &params, &dt, &rep, stream),
        m == method::df ? "al_df_step" : m == method::ii ? "al_ii_step" : "al_i_step");
  return rep;
}

// SolverI<TF>::step<0> on the pellet branch.
template <class TF>
al_step_report step_pellets(const engine& e, const typename real<TF>::cn& cn,
                            const al_consti& cni, const typename real<TF>::fluid& fluid,
                            const typename real<TF>::body* bodies,
                            typename real<TF>::rigid* rigid,
                            const typename real<TF>::pellets& pellets,
                            const al_solver_params& params, TF& dt, void* stream = nullptr) {
  al_step_report rep{};
  check(real<TF>::i_step_pellets(e.get(), &cn, &cni, &fluid, bodies, rigid, &pellets, &params,
                                 &dt, &rep, stream),
        "al_i_step_pellets");
  return rep;
}

}  // namespace alluvion_b200

#endif /* ALLUVION_B200_HPP */
