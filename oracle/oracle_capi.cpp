// oracle_capi.cpp -- C entry points of the CPU ORACLE (test infrastructure).
//
// Loaded by tests/ (as the checker) and by bench.py's CPU-baseline leg only.
// All pointers are HOST pointers; layouts are the reference's (see
// include/alluvion_b200.h).  Each function restates the reference routine
// named in sph_oracle.hpp.
#include <omp.h>

#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "sph_oracle.hpp"

using namespace oracle;

namespace {

template <class TF>
V3<TF> v3(const TF* p) {
  return V3<TF>{p[0], p[1], p[2]};
}

// Lazily filled volume maps, keyed by their node array (see LazyVolume).
template <class TF>
std::map<const void*, std::unique_ptr<LazyVolume<TF>>>& lazy_registry() {
  static std::map<const void*, std::unique_ptr<LazyVolume<TF>>> reg;
  return reg;
}
std::mutex g_lazy_mutex;

template <class TF>
LazyVolume<TF>* find_lazy(const void* nodes) {
  std::lock_guard<std::mutex> lock(g_lazy_mutex);
  auto& reg = lazy_registry<TF>();
  auto it = reg.find(nodes);
  return it == reg.end() ? nullptr : it->second.get();
}

template <class TF, class B>
Body<TF> make_body(const B& b, const TF* rigid) {
  Body<TF> o{};
  o.shape = b.shape;
  o.use_grid = b.use_distance_grid;
  o.sign = b.sign;
  o.dmin = v3<TF>(b.domain_min);
  o.dmax = v3<TF>(b.domain_max);
  o.cs = v3<TF>(b.cell_size);
  for (int k = 0; k < 3; ++k) o.res[k] = b.resolution[k];
  o.num_nodes = b.num_nodes;
  o.dist_nodes = b.distance_nodes;
  o.vol_nodes = b.volume_nodes;
  o.lazy_vol = find_lazy<TF>(b.volume_nodes);
  o.sdf.kind = b.shape;
  for (int k = 0; k < 8; ++k) o.sdf.p[k] = b.shape_params[k];
  o.max_distance = b.max_distance;
  o.mass = b.mass;
  o.inertia = v3<TF>(b.inertia);
  // rigid: x[3] v[3] q[4] omega[3]
  if (rigid) {
    o.x = v3<TF>(rigid);
    o.v = v3<TF>(rigid + 3);
    o.q = V4<TF>{rigid[6], rigid[7], rigid[8], rigid[9]};
    o.omega = v3<TF>(rigid + 10);
  } else {
    o.x = {0, 0, 0};
    o.v = {0, 0, 0};
    o.q = {0, 0, 0, 1};
    o.omega = {0, 0, 0};
  }
  return o;
}

template <class TF>
void load_fluid(Fluid<TF>& f, uint32_t n, uint32_t nb, const TF* x, const TF* v) {
  f.x.resize(n);
  f.v.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    f.x[i] = v3<TF>(x + 3 * size_t(i));
    f.v[i] = v ? v3<TF>(v + 3 * size_t(i)) : V3<TF>{0, 0, 0};
  }
  f.resize(n, nb);
}

template <class TF, class C>
int grid_sort_impl(const C* cn, const al_consti* cni, const TF* x, uint32_t n, uint32_t* cell,
                   uint32_t* sorted, uint32_t* cell_start, uint32_t* flags) {
  Cn<TF> c = make_cn<TF>(*cn);
  std::vector<V3<TF>> xs(n);
  for (uint32_t i = 0; i < n; ++i) xs[i] = v3<TF>(x + 3 * size_t(i));
  GridSort s = grid_sort(c, *cni, xs.data(), n);
  std::copy(s.cell.begin(), s.cell.end(), cell);
  std::copy(s.sorted.begin(), s.sorted.end(), sorted);
  if (cell_start) std::copy(s.cell_start.begin(), s.cell_start.end(), cell_start);
  flags[0] = s.out_of_grid;
  flags[1] = s.cell_overflow;
  return 0;
}

template <class TF, class C>
int neighbors_impl(const C* cn, const al_consti* cni, const TF* x, uint32_t n,
                   const TF* boundary_kernel, TF* density, uint32_t* count, uint32_t* index,
                   TF* neighbors, uint32_t* flags, double wrap_length = 0) {
  Cn<TF> c = make_cn<TF>(*cn);
  Fluid<TF> f;
  load_fluid<TF>(f, n, cni->num_boundaries, x, nullptr);
  if (wrap_length > 0) {  // update_particle_neighbors<1>
    f.wrap = true;
    f.wrap_len = TF(wrap_length);
  }
  if (boundary_kernel)
    for (size_t k = 0; k < size_t(f.nb) * n; ++k)
      f.bk[k] = V4<TF>{boundary_kernel[4 * k], boundary_kernel[4 * k + 1],
                       boundary_kernel[4 * k + 2], boundary_kernel[4 * k + 3]};
  update_particle_neighbors(c, *cni, f);
  const uint32_t cap = f.nl.cap;
  for (uint32_t i = 0; i < n; ++i) {
    if (density) density[i] = f.density[i];
    count[i] = f.nl.count[i];
    for (uint32_t k = 0; k < cap; ++k) {
      uint32_t j = f.nl.index[size_t(i) * cap + k];
      if (index) index[size_t(i) * cap + k] = k < f.nl.count[i] ? j : 0xffffffffu;
      if (neighbors && k < f.nl.count[i]) {
        TF* e = neighbors + (size_t(i) * cap + k) * 4;
        V3<TF> d = xv(f, i, j);
        e[0] = d.x;
        e[1] = d.y;
        e[2] = d.z;
        std::memcpy(&e[3], &j, sizeof(uint32_t));
      }
    }
  }
  flags[0] = f.gs.out_of_grid;
  flags[1] = f.gs.cell_overflow;
  flags[2] = f.nl.overflow;
  return 0;
}

template <class TF>
void node_positions_impl(const TF* dmin, const uint32_t* res, const TF* cs, TF* out) {
  uint32_t nn = num_grid_nodes(res);
  V3<TF> lo = v3<TF>(dmin), c = v3<TF>(cs);
  for (uint32_t l = 0; l < nn; ++l) {
    V3<TF> p = node_position(lo, res, c, l);
    out[3 * size_t(l)] = p.x;
    out[3 * size_t(l) + 1] = p.y;
    out[3 * size_t(l) + 2] = p.z;
  }
}

// Distance nodes sampled from the analytic SDF at the node positions (the
// role CubicLagrangeDiscreteGrid::addFunction plays for mesh distances,
// pile.hpp:79-94).
template <class TF, class B>
void distance_grid_impl(const B* b, TF* out) {
  Body<TF> body = make_body<TF>(*b, nullptr);
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < int64_t(body.num_nodes); ++l)
    out[l] = body.sdf.sdf(node_position(body.dmin, body.res, body.cs, uint32_t(l)));
}

template <class TF, class C, class B>
void lazy_register_impl(const C* cn, const B* b, TF* out) {
  Cn<TF> c = make_cn<TF>(*cn);
  B geo = *b;
  geo.volume_nodes = nullptr;  // not a lazy map itself
  Body<TF> body = make_body<TF>(geo, nullptr);
  auto lv = std::make_unique<LazyVolume<TF>>(c, body.dmin, body.dmax, body.cs, body.res,
                                             body.use_grid, body.sign, body.sdf,
                                             body.dist_nodes, out);
  std::lock_guard<std::mutex> lock(g_lazy_mutex);
  lazy_registry<TF>()[out] = std::move(lv);
}

// Computes every node of the Lagrange cells within `dilate` cells of each
// particle's cell in the body's frame (the nodes the next steps' boundary
// samples read), so that a timed run afterwards finds them ready.
template <class TF, class B>
void lazy_touch_impl(const B* b, const TF* rigid, const TF* x, uint32_t n, uint32_t dilate) {
  LazyVolume<TF>* lv = find_lazy<TF>(b->volume_nodes);
  if (!lv) return;
  const Body<TF> body = make_body<TF>(*b, rigid);
  const int d = int(dilate);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < int64_t(n); ++i) {
    V3<TF> local = rotate(v3<TF>(x + 3 * i) - body.x, conjugate(body.q));
    if (body.shape == AL_SHAPE_INFINITE_CYLINDER || body.shape == AL_SHAPE_INFINITE_TUBE)
      local.y = 0;
    // cell of the particle in the body's grid, possibly outside it: particles
    // up to `dilate` cells outside the domain may move in
    const V3<TF> rel = local - body.dmin;
    const TF fx = std::floor(rel.x / body.cs.x), fy = std::floor(rel.y / body.cs.y),
             fz = std::floor(rel.z / body.cs.z);
    const TF lim = TF(1 << 20);
    if (!(std::fabs(fx) < lim && std::fabs(fy) < lim && std::fabs(fz) < lim)) continue;
    const int ip[3] = {int(fx), int(fy), int(fz)};
    for (int a = -d; a <= d; ++a)
      for (int bb = -d; bb <= d; ++bb)
        for (int cc = -d; cc <= d; ++cc) {
          int q[3] = {ip[0] + a, ip[1] + bb, ip[2] + cc};
          if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= int(body.res[0]) ||
              q[1] >= int(body.res[1]) || q[2] >= int(body.res[2]))
            continue;
          uint32_t cells[32];
          cell_nodes(body.res, q, cells);
          for (int j = 0; j < 32; ++j) lv->get(cells[j]);
        }
  }
}

template <class TF>
void lazy_counts_impl(const TF* out, uint64_t counts[2]) {
  LazyVolume<TF>* lv = find_lazy<TF>(out);
  counts[0] = lv ? lv->sampled.load() : 0;
  counts[1] = lv ? lv->skipped.load() : 0;
}

template <class TF, class C, class B>
void volume_field_impl(const C* cn, const B* b, TF* out) {
  Cn<TF> c = make_cn<TF>(*cn);
  Body<TF> body = make_body<TF>(*b, nullptr);
  PeirceTables pt = peirce_tables();
  LagrangeGrid<TF> grid{body.dmin, body.dmax, body.cs, {body.res[0], body.res[1], body.res[2]},
                        body.dist_nodes};
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t l = 0; l < int64_t(body.num_nodes); ++l) {
    V3<TF> x = node_position(body.dmin, body.res, body.cs, uint32_t(l));
    if (body.use_grid) {
      LagrangeGrid<TF> g = grid;
      typename LagrangeGrid<TF>::Cache cache;
      g.cache = &cache;
      out[l] = volume_at(c, pt, x, body.sign, [&](V3<TF> p) { return g.value(p); });
    } else {
      out[l] = volume_at(c, pt, x, body.sign, [&](V3<TF> p) { return body.sdf.sdf(p); });
    }
  }
}

template <class TF, class C, class B>
void boundary_impl(const C* cn, const B* bodies, const TF* rigid, uint32_t nb, const TF* x,
                   uint32_t n, TF* bnd, TF* bk) {
  Cn<TF> c = make_cn<TF>(*cn);
  std::vector<Body<TF>> bs;
  for (uint32_t b = 0; b < nb; ++b) bs.push_back(make_body<TF>(bodies[b], rigid + 13 * b));
  Fluid<TF> f;
  load_fluid<TF>(f, n, nb, x, nullptr);
  compute_boundaries(c, bs, f);
  for (size_t k = 0; k < size_t(nb) * n; ++k) {
    bnd[4 * k] = f.bnd[k].x;
    bnd[4 * k + 1] = f.bnd[k].y;
    bnd[4 * k + 2] = f.bnd[k].z;
    bnd[4 * k + 3] = f.bnd[k].w;
    bk[4 * k] = f.bk[k].x;
    bk[4 * k + 1] = f.bk[k].y;
    bk[4 * k + 2] = f.bk[k].z;
    bk[4 * k + 3] = f.bk[k].w;
  }
}

// Runs `steps` solver steps on host arrays.  State arrays are in/out.
// rigid: nb x 13 values (x, v, q, omega).  reports: `steps` entries.
template <class TF, class C, class B>
int run_impl(int method, const C* cn, const al_consti* cni, const B* bodies, TF* rigid,
             uint32_t n, TF* x, TF* v, TF* kappa_or_pressure, TF* kappa_v, TF* density,
             TF* density_adv, TF* a, const al_solver_params* sp_in, TF* dt, uint32_t steps,
             al_step_report* reports, const PelletSet<TF>* pel = nullptr,
             TF* pellet_x = nullptr, TF* pellet_p = nullptr) {
  Cn<TF> c = make_cn<TF>(*cn);
  // 0 DFSPH, 1 IISPH, 2 implicit SPH (SolverI), 3 SolverI with pellets
  const bool iisph = method != 0;
  const uint32_t nb = cni->num_boundaries;
  std::vector<Body<TF>> bs;
  for (uint32_t b = 0; b < nb; ++b) bs.push_back(make_body<TF>(bodies[b], rigid + 13 * b));
  Fluid<TF> f;
  f.x.resize(n);
  f.v.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    f.x[i] = v3<TF>(x + 3 * size_t(i));
    f.v[i] = v3<TF>(v + 3 * size_t(i));
  }
  f.kappa.assign(n, 0);
  f.kappa_v.assign(n, 0);
  f.pressure.assign(n, 0);
  if (iisph) {
    if (kappa_or_pressure) std::copy(kappa_or_pressure, kappa_or_pressure + n, f.pressure.begin());
  } else {
    if (kappa_or_pressure) std::copy(kappa_or_pressure, kappa_or_pressure + n, f.kappa.begin());
    if (kappa_v) std::copy(kappa_v, kappa_v + n, f.kappa_v.begin());
  }
  f.resize(n, nb);
  if (sp_in->wrap_y) {  // step<1>
    f.wrap = true;
    f.wrap_len = TF(sp_in->wrap_length);
  }
  SolverParams sp;
  sp.density_change_tolerance = sp_in->density_change_tolerance;
  sp.density_error_tolerance = sp_in->density_error_tolerance;
  sp.min_density_solve = sp_in->min_density_solve;
  sp.max_density_solve = sp_in->max_density_solve;
  sp.min_divergence_solve = sp_in->min_divergence_solve;
  sp.max_divergence_solve = sp_in->max_divergence_solve;
  sp.enable_divergence_solve = sp_in->enable_divergence_solve != 0;
  sp.enable_density_solve = sp_in->enable_density_solve != 0;
  sp.cfl = sp_in->cfl;
  sp.max_dt = sp_in->max_dt;
  sp.min_dt = sp_in->min_dt;
  V3<TF> pg{TF(sp_in->pile_gravity[0]), TF(sp_in->pile_gravity[1]), TF(sp_in->pile_gravity[2])};
  TF step_dt = *dt;
  for (uint32_t s = 0; s < steps; ++s) {
    std::vector<V3<double>> F, T;
    const bool ib = sp_in->integrate_rigids != 0;
    std::vector<V3<TF>> px;
    std::vector<TF> pp;
    StepReport r = method == 1   ? ii_step(c, *cni, bs, f, sp, step_dt, pg, ib, &F, &T)
                   : method == 2 ? i_step(c, *cni, bs, f, sp, step_dt, pg, ib, &F, &T)
                   : method == 3 ? i_step_pellets(c, *cni, bs, f, *pel, sp, step_dt, pg, ib, &F,
                                                  &T, &px, &pp)
                                 : df_step(c, *cni, bs, f, sp, step_dt, pg, ib, &F, &T);
    for (size_t k = 0; k < px.size(); ++k) {
      if (pellet_x) {
        pellet_x[3 * k] = px[k].x;
        pellet_x[3 * k + 1] = px[k].y;
        pellet_x[3 * k + 2] = px[k].z;
      }
      if (pellet_p) pellet_p[k] = pp[k];
    }
    if (reports) {
      al_step_report& o = reports[s];
      std::memset(&o, 0, sizeof(o));
      o.num_divergence_solve = r.num_divergence_solve;
      o.num_density_solve = r.num_density_solve;
      o.mean_density_change = r.mean_density_change;
      o.mean_density_error = r.mean_density_error;
      o.particle_max_v2 = r.particle_max_v2;
      o.pile_max_v2 = r.pile_max_v2;
      o.max_v2 = r.max_v2;
      o.cfl_dt = r.cfl_dt;
      o.utilized_cfl = r.utilized_cfl;
      o.dt = r.dt;
      for (int k = 0; k < 3; ++k) o.grid_anomaly[k] = r.grid_anomaly[k];
      uint32_t active = 0;
      for (size_t k = 0; k < f.bnd.size(); ++k) active += f.bnd[k].w != 0;
      o.num_active_boundary_pairs = active;
      for (uint32_t b = 0; b < nb && b < AL_MAX_BOUNDARIES; ++b) {
        o.force[b][0] = F[b].x;
        o.force[b][1] = F[b].y;
        o.force[b][2] = F[b].z;
        o.torque[b][0] = T[b].x;
        o.torque[b][1] = T[b].y;
        o.torque[b][2] = T[b].z;
      }
    }
  }
  *dt = step_dt;
  for (uint32_t i = 0; i < n; ++i) {
    x[3 * size_t(i)] = f.x[i].x;
    x[3 * size_t(i) + 1] = f.x[i].y;
    x[3 * size_t(i) + 2] = f.x[i].z;
    v[3 * size_t(i)] = f.v[i].x;
    v[3 * size_t(i) + 1] = f.v[i].y;
    v[3 * size_t(i) + 2] = f.v[i].z;
    if (density) density[i] = f.density[i];
    if (density_adv) density_adv[i] = f.density_adv[i];
    if (a) {
      a[3 * size_t(i)] = f.a[i].x;
      a[3 * size_t(i) + 1] = f.a[i].y;
      a[3 * size_t(i) + 2] = f.a[i].z;
    }
    if (iisph) {
      if (kappa_or_pressure) kappa_or_pressure[i] = f.pressure[i];
    } else {
      if (kappa_or_pressure) kappa_or_pressure[i] = f.kappa[i];
      if (kappa_v) kappa_v[i] = f.kappa_v[i];
    }
  }
  for (uint32_t b = 0; b < nb; ++b) {
    TF* r = rigid + 13 * b;
    const Body<TF>& o = bs[b];
    TF vals[13] = {o.x.x, o.x.y, o.x.z, o.v.x, o.v.y, o.v.z, o.q.x,
                   o.q.y, o.q.z, o.q.w, o.omega.x, o.omega.y, o.omega.z};
    std::copy(vals, vals + 13, r);
  }
  return 0;
}

// SolverI with pellets: pellet_local [P][3] body frame, body after body,
// counts[nb]; pellet_x / pellet_p (may be NULL) receive the last step's
// world positions and extrapolated pressures.
template <class TF, class C, class B>
int run_pellets(const C* cn, const al_consti* cni, const B* bodies, TF* rigid, uint32_t n, TF* x,
                TF* v, TF* pressure, TF* density, TF* density_adv, TF* a, const TF* pellet_local,
                const uint32_t* counts, uint32_t np, const al_solver_params* sp, TF* dt,
                uint32_t steps, al_step_report* reports, TF* pellet_x, TF* pellet_p) {
  PelletSet<TF> pel;
  uint32_t b = 0, left = cni->num_boundaries ? counts[0] : 0;
  for (uint32_t k = 0; k < np; ++k) {
    while (left == 0 && b + 1 < cni->num_boundaries) left = counts[++b];
    pel.local.push_back(v3<TF>(pellet_local + 3 * size_t(k)));
    pel.body.push_back(b);
    if (left) --left;
  }
  return run_impl<TF>(3, cn, cni, bodies, rigid, n, x, v, pressure, nullptr, density,
                      density_adv, a, sp, dt, steps, reports, &pel, pellet_x, pellet_p);
}

}  // namespace

extern "C" {

int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { omp_set_num_threads(n); }

void orc_peirce_tables(double* cosphi, double* sinphi, double* b, double* r, double* c) {
  PeirceTables t = peirce_tables();
  std::copy(t.cosphi, t.cosphi + kNumPhi, cosphi);
  std::copy(t.sinphi, t.sinphi + kNumPhi, sinphi);
  std::copy(t.b, t.b + kNumPhi, b);
  std::copy(t.r, t.r + kNumR, r);
  std::copy(t.c, t.c + kNumR, c);
}

int orc_grid_sort_f32(const al_const_f32* cn, const al_consti* cni, const float* x, uint32_t n,
                      uint32_t* cell, uint32_t* sorted, uint32_t* cell_start, uint32_t* flags) {
  return grid_sort_impl<float>(cn, cni, x, n, cell, sorted, cell_start, flags);
}
int orc_grid_sort_f64(const al_const_f64* cn, const al_consti* cni, const double* x, uint32_t n,
                      uint32_t* cell, uint32_t* sorted, uint32_t* cell_start, uint32_t* flags) {
  return grid_sort_impl<double>(cn, cni, x, n, cell, sorted, cell_start, flags);
}

int orc_update_particle_neighbors_f32(const al_const_f32* cn, const al_consti* cni,
                                      const float* x, uint32_t n, const float* boundary_kernel,
                                      float* density, uint32_t* count, uint32_t* index,
                                      float* neighbors, uint32_t* flags) {
  return neighbors_impl<float>(cn, cni, x, n, boundary_kernel, density, count, index, neighbors,
                               flags);
}
int orc_update_particle_neighbors_f64(const al_const_f64* cn, const al_consti* cni,
                                      const double* x, uint32_t n, const double* boundary_kernel,
                                      double* density, uint32_t* count, uint32_t* index,
                                      double* neighbors, uint32_t* flags) {
  return neighbors_impl<double>(cn, cni, x, n, boundary_kernel, density, count, index, neighbors,
                                flags);
}
int orc_update_particle_neighbors_periodic_f32(const al_const_f32* cn, const al_consti* cni,
                                               const float* x, uint32_t n, const float* bk,
                                               float* density, uint32_t* count, uint32_t* index,
                                               float* neighbors, uint32_t* flags,
                                               double wrap_length) {
  return neighbors_impl<float>(cn, cni, x, n, bk, density, count, index, neighbors, flags,
                               wrap_length);
}
int orc_update_particle_neighbors_periodic_f64(const al_const_f64* cn, const al_consti* cni,
                                               const double* x, uint32_t n, const double* bk,
                                               double* density, uint32_t* count, uint32_t* index,
                                               double* neighbors, uint32_t* flags,
                                               double wrap_length) {
  return neighbors_impl<double>(cn, cni, x, n, bk, density, count, index, neighbors, flags,
                                wrap_length);
}

uint32_t orc_num_grid_nodes(const uint32_t* res) { return num_grid_nodes(res); }
void orc_node_positions_f32(const float* dmin, const uint32_t* res, const float* cs, float* out) {
  node_positions_impl<float>(dmin, res, cs, out);
}
void orc_node_positions_f64(const double* dmin, const uint32_t* res, const double* cs,
                            double* out) {
  node_positions_impl<double>(dmin, res, cs, out);
}

// Shape functions at reference coordinates xi (3 values): N[32], dN[3][32].
void orc_shape_functions_f64(const double* xi, double* N, double* dN) {
  shape_functions<double>(V3<double>{xi[0], xi[1], xi[2]}, N, dN, dN + 32, dN + 64);
}
void orc_cell_nodes(const uint32_t* res, const int* ipos, uint32_t* out) {
  cell_nodes(res, ipos, out);
}

void orc_distance_grid_f32(const al_body_f32* b, float* out) { distance_grid_impl<float>(b, out); }
void orc_distance_grid_f64(const al_body_f64* b, double* out) {
  distance_grid_impl<double>(b, out);
}
void orc_volume_field_f32(const al_const_f32* cn, const al_body_f32* b, float* out) {
  volume_field_impl<float>(cn, b, out);
}
void orc_volume_field_f64(const al_const_f64* cn, const al_body_f64* b, double* out) {
  volume_field_impl<double>(cn, b, out);
}
// Registers `out` (the body's num_nodes volume values) as a lazily filled
// volume map: steps that get a body whose volume_nodes == out compute each
// node on first use.  distance_nodes must stay valid while registered.
void orc_lazy_volume_register_f32(const al_const_f32* cn, const al_body_f32* b, float* out) {
  lazy_register_impl<float>(cn, b, out);
}
void orc_lazy_volume_register_f64(const al_const_f64* cn, const al_body_f64* b, double* out) {
  lazy_register_impl<double>(cn, b, out);
}
// Nodes computed so far: [0] by sampling, [1] by the analytic shortcuts.
void orc_lazy_volume_counts_f32(const float* out, uint64_t counts[2]) {
  lazy_counts_impl<float>(out, counts);
}
void orc_lazy_volume_counts_f64(const double* out, uint64_t counts[2]) {
  lazy_counts_impl<double>(out, counts);
}
void orc_lazy_volume_touch_f32(const al_body_f32* b, const float* rigid, const float* x,
                               uint32_t n, uint32_t dilate) {
  lazy_touch_impl<float>(b, rigid, x, n, dilate);
}
void orc_lazy_volume_touch_f64(const al_body_f64* b, const double* rigid, const double* x,
                               uint32_t n, uint32_t dilate) {
  lazy_touch_impl<double>(b, rigid, x, n, dilate);
}
void orc_lazy_volume_release(const void* out) {
  std::lock_guard<std::mutex> lock(g_lazy_mutex);
  lazy_registry<float>().erase(out);
  lazy_registry<double>().erase(out);
}

void orc_boundary_f32(const al_const_f32* cn, const al_body_f32* bodies, const float* rigid,
                      uint32_t nb, const float* x, uint32_t n, float* bnd, float* bk) {
  boundary_impl<float>(cn, bodies, rigid, nb, x, n, bnd, bk);
}
void orc_boundary_f64(const al_const_f64* cn, const al_body_f64* bodies, const double* rigid,
                      uint32_t nb, const double* x, uint32_t n, double* bnd, double* bk) {
  boundary_impl<double>(cn, bodies, rigid, nb, x, n, bnd, bk);
}

int orc_df_run_f32(const al_const_f32* cn, const al_consti* cni, const al_body_f32* bodies,
                   float* rigid, uint32_t n, float* x, float* v, float* kappa, float* kappa_v,
                   float* density, float* density_adv, float* a, const al_solver_params* sp,
                   float* dt, uint32_t steps, al_step_report* reports) {
  return run_impl<float>(0, cn, cni, bodies, rigid, n, x, v, kappa, kappa_v, density,
                         density_adv, a, sp, dt, steps, reports);
}
int orc_df_run_f64(const al_const_f64* cn, const al_consti* cni, const al_body_f64* bodies,
                   double* rigid, uint32_t n, double* x, double* v, double* kappa,
                   double* kappa_v, double* density, double* density_adv, double* a,
                   const al_solver_params* sp, double* dt, uint32_t steps,
                   al_step_report* reports) {
  return run_impl<double>(0, cn, cni, bodies, rigid, n, x, v, kappa, kappa_v, density,
                          density_adv, a, sp, dt, steps, reports);
}
int orc_ii_run_f32(const al_const_f32* cn, const al_consti* cni, const al_body_f32* bodies,
                   float* rigid, uint32_t n, float* x, float* v, float* pressure, float* density,
                   float* density_adv, float* a, const al_solver_params* sp, float* dt,
                   uint32_t steps, al_step_report* reports) {
  return run_impl<float>(1, cn, cni, bodies, rigid, n, x, v, pressure, nullptr, density,
                         density_adv, a, sp, dt, steps, reports);
}
int orc_ii_run_f64(const al_const_f64* cn, const al_consti* cni, const al_body_f64* bodies,
                   double* rigid, uint32_t n, double* x, double* v, double* pressure,
                   double* density, double* density_adv, double* a, const al_solver_params* sp,
                   double* dt, uint32_t steps, al_step_report* reports) {
  return run_impl<double>(1, cn, cni, bodies, rigid, n, x, v, pressure, nullptr, density,
                          density_adv, a, sp, dt, steps, reports);
}

int orc_i_run_f32(const al_const_f32* cn, const al_consti* cni, const al_body_f32* bodies,
                  float* rigid, uint32_t n, float* x, float* v, float* pressure, float* density,
                  float* density_adv, float* a, const al_solver_params* sp, float* dt,
                  uint32_t steps, al_step_report* reports) {
  return run_impl<float>(2, cn, cni, bodies, rigid, n, x, v, pressure, nullptr, density,
                         density_adv, a, sp, dt, steps, reports);
}
int orc_i_run_f64(const al_const_f64* cn, const al_consti* cni, const al_body_f64* bodies,
                  double* rigid, uint32_t n, double* x, double* v, double* pressure,
                  double* density, double* density_adv, double* a, const al_solver_params* sp,
                  double* dt, uint32_t steps, al_step_report* reports) {
  return run_impl<double>(2, cn, cni, bodies, rigid, n, x, v, pressure, nullptr, density,
                          density_adv, a, sp, dt, steps, reports);
}

int orc_i_run_pellets_f32(const al_const_f32* cn, const al_consti* cni, const al_body_f32* bodies,
                          float* rigid, uint32_t n, float* x, float* v, float* pressure,
                          float* density, float* density_adv, float* a, const float* pellet_local,
                          const uint32_t* counts, uint32_t np, const al_solver_params* sp,
                          float* dt, uint32_t steps, al_step_report* reports, float* pellet_x,
                          float* pellet_p) {
  return run_pellets<float>(cn, cni, bodies, rigid, n, x, v, pressure, density, density_adv, a,
                            pellet_local, counts, np, sp, dt, steps, reports, pellet_x, pellet_p);
}
int orc_i_run_pellets_f64(const al_const_f64* cn, const al_consti* cni, const al_body_f64* bodies,
                          double* rigid, uint32_t n, double* x, double* v, double* pressure,
                          double* density, double* density_adv, double* a,
                          const double* pellet_local, const uint32_t* counts, uint32_t np,
                          const al_solver_params* sp, double* dt, uint32_t steps,
                          al_step_report* reports, double* pellet_x, double* pellet_p) {
  return run_pellets<double>(cn, cni, bodies, rigid, n, x, v, pressure, density, density_adv, a,
                             pellet_local, counts, np, sp, dt, steps, reports, pellet_x, pellet_p);
}

}  // extern "C"

// ------------------------------------------------------------------ contacts
namespace {

template <class TF, class CB>
void load_contact_bodies(const al_body_f32* bodies, const al_rigid_f32* rigid, const CB* cb,
                         uint32_t nb, std::vector<Body<TF>>& B, std::vector<const TF*>& verts,
                         std::vector<uint32_t>& nv, std::vector<TF>& rest, std::vector<TF>& fric) {
  for (uint32_t b = 0; b < nb; ++b) {
    B.push_back(make_body<TF>(bodies[b], reinterpret_cast<const TF*>(&rigid[b])));
    verts.push_back(cb[b].vertices);
    nv.push_back(cb[b].num_vertices);
    rest.push_back(cb[b].restitution);
    fric.push_back(cb[b].friction);
  }
}

void to_abi(const Contact<float>& c, al_contact_f32& o) {
  auto put = [](float* d, V3<float> v) {
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
  };
  o.i = c.i;
  o.j = c.j;
  put(o.cp_i, c.cp_i);
  put(o.cp_j, c.cp_j);
  put(o.n, c.n);
  put(o.t, c.t);
  put(o.iiwi_diag, c.iiwi_diag);
  put(o.iiwi_off_diag, c.iiwi_off);
  put(o.iiwj_diag, c.iiwj_diag);
  put(o.iiwj_off_diag, c.iiwj_off);
  o.friction = c.friction;
  o.nkninv = c.nkninv;
  o.pmax = c.pmax;
  o.goalu = c.goalu;
  o.impulse_sum = c.impulse_sum;
}

Contact<float> from_abi(const al_contact_f32& o) {
  Contact<float> c;
  c.i = o.i;
  c.j = o.j;
  c.cp_i = v3<float>(o.cp_i);
  c.cp_j = v3<float>(o.cp_j);
  c.n = v3<float>(o.n);
  c.t = v3<float>(o.t);
  c.iiwi_diag = v3<float>(o.iiwi_diag);
  c.iiwi_off = v3<float>(o.iiwi_off_diag);
  c.iiwj_diag = v3<float>(o.iiwj_diag);
  c.iiwj_off = v3<float>(o.iiwj_off_diag);
  c.friction = o.friction;
  c.nkninv = o.nkninv;
  c.pmax = o.pmax;
  c.goalu = o.goalu;
  c.impulse_sum = o.impulse_sum;
  return c;
}

}  // namespace

extern "C" {

// Pile::find_contacts with HOST vertex and node pointers; writes up to
// max_contacts contacts in (i, j, vertex) order and returns the count found.
uint32_t orc_find_contacts_f32(const al_body_f32* bodies, const al_rigid_f32* rigid,
                               const al_contact_body_f32* cb, uint32_t nb, float tol,
                               uint32_t max_contacts, al_contact_f32* out) {
  std::vector<Body<float>> B;
  std::vector<const float*> verts;
  std::vector<uint32_t> nv;
  std::vector<float> rest, fric;
  load_contact_bodies<float>(bodies, rigid, cb, nb, B, verts, nv, rest, fric);
  std::vector<Contact<float>> cs;
  find_contacts(B, verts, nv, rest, fric, tol, cs);
  for (size_t k = 0; k < cs.size() && k < max_contacts; ++k) to_abi(cs[k], out[k]);
  return uint32_t(cs.size());
}

// Pile::solve_contacts: updates rigid[b].v / omega in place.
void orc_solve_contacts_f32(const al_body_f32* bodies, al_rigid_f32* rigid, uint32_t nb,
                            const al_contact_f32* contacts, uint32_t num_contacts) {
  std::vector<Body<float>> B;
  for (uint32_t b = 0; b < nb; ++b)
    B.push_back(make_body<float>(bodies[b], reinterpret_cast<const float*>(&rigid[b])));
  std::vector<Contact<float>> cs;
  for (uint32_t k = 0; k < num_contacts; ++k) cs.push_back(from_abi(contacts[k]));
  solve_contacts(B, cs);
  for (uint32_t b = 0; b < nb; ++b) {
    rigid[b].v[0] = B[b].v.x;
    rigid[b].v[1] = B[b].v.y;
    rigid[b].v[2] = B[b].v.z;
    rigid[b].omega[0] = B[b].omega.x;
    rigid[b].omega[1] = B[b].omega.y;
    rigid[b].omega[2] = B[b].omega.z;
  }
}

}  // extern "C"

extern "C" {

// Distance grid of a mesh body: node positions of `b`, signed distances
// to the mesh (host arrays) minus offset.
void orc_mesh_distance_grid_f32(const al_body_f32* b, const float* verts, uint32_t nv,
                                const uint32_t* faces, uint32_t nf, float offset, float* out) {
  const Body<float> body = make_body<float>(*b, nullptr);
  const TriMesh<float> m = make_mesh<float>(verts, nv, faces, nf);
#pragma omp parallel for schedule(static)
  for (int64_t l = 0; l < int64_t(body.num_nodes); ++l)
    out[l] = mesh_signed_distance(m, node_position(body.dmin, body.res, body.cs, uint32_t(l)),
                                  offset);
}

}  // extern "C"

extern "C" {

}  // extern "C"

namespace {

template <class TF, class Req, class ConstT, class RigidT>
int sample_impl(const ConstT* cn, const al_consti* cni, const TF* particle_x, uint32_t n,
                const RigidT* rigid, const Req* req) {
  const Cn<TF> c = make_cn<TF>(*cn);
  std::vector<V3<TF>> px(n);
  for (uint32_t i = 0; i < n; ++i) px[i] = v3<TF>(particle_x + 3 * size_t(i));
  std::vector<V3<TF>> sx(req->num_samples);
  for (uint32_t i = 0; i < req->num_samples; ++i) sx[i] = v3<TF>(req->sample_x + 3 * size_t(i));
  std::vector<Body<TF>> bodies;
  for (uint32_t b = 0; rigid && b < cni->num_boundaries; ++b) {
    Body<TF> o{};
    o.x = v3<TF>(rigid[b].x);
    o.v = v3<TF>(rigid[b].v);
    o.omega = v3<TF>(rigid[b].omega);
    o.q = V4<TF>{rigid[b].q[0], rigid[b].q[1], rigid[b].q[2], rigid[b].q[3]};
    bodies.push_back(o);
  }
  SampleRequest<TF> r;
  r.sx = sx.data();
  r.num = req->num_samples;
  r.rho = req->particle_density;
  r.v = reinterpret_cast<const V3<TF>*>(req->particle_v);
  r.q = req->particle_quantity;
  r.qdim = req->sample_quantity ? req->quantity_dim : 0;
  r.bnd = reinterpret_cast<const V4<TF>*>(req->sample_boundary);
  r.bk = reinterpret_cast<const V4<TF>*>(req->sample_boundary_kernel);
  r.density = req->sample_density;
  r.position_density = req->sample_position_density;
  r.quantity = req->sample_quantity;
  r.vel = reinterpret_cast<V3<TF>*>(req->sample_v);
  r.vort = reinterpret_cast<V3<TF>*>(req->sample_vorticity);
  r.wrap = req->wrap_y != 0;
  r.wrap_length = TF(req->wrap_length);
  r.pel_x = reinterpret_cast<const V3<TF>*>(req->pellet_x);
  r.pel_v = reinterpret_cast<const V3<TF>*>(req->pellet_v);
  r.npel = req->num_pellets;
  return sample_fluid(c, *cni, px.data(), n, bodies, r) ? 1 : 0;
}

template <class TF, class BodyT, class RigidT>
void boundary_mask_impl(const BodyT* body, const RigidT* rigid, const TF* sample_x, uint32_t n,
                        TF threshold, TF* mask) {
  const Body<TF> b = make_body<TF>(*body, reinterpret_cast<const TF*>(rigid));
  std::vector<V3<TF>> sx(n);
  for (uint32_t i = 0; i < n; ++i) sx[i] = v3<TF>(sample_x + 3 * size_t(i));
  boundary_mask(b, sx.data(), n, threshold, mask);
}

}  // namespace

extern "C" {

// Sampling at sample points (sample_fluid and friends) with HOST arrays in
// the layouts of al_sample_f32 / al_sample_f64; `rigid` holds the bodies'
// states (cni->num_boundaries of them).  Returns 1 when a sample had more
// neighbors than the cap, else 0.
int orc_sample_fluid_f32(const al_const_f32* cn, const al_consti* cni, const float* particle_x,
                         uint32_t n, const al_rigid_f32* rigid, const al_sample_f32* req) {
  return sample_impl<float>(cn, cni, particle_x, n, rigid, req);
}
int orc_sample_fluid_f64(const al_const_f64* cn, const al_consti* cni, const double* particle_x,
                         uint32_t n, const al_rigid_f64* rigid, const al_sample_f64* req) {
  return sample_impl<double>(cn, cni, particle_x, n, rigid, req);
}

// compute_boundary_mask with HOST node arrays: mask *= (sign d >= threshold).
void orc_boundary_mask_f32(const al_body_f32* body, const al_rigid_f32* rigid,
                           const float* sample_x, uint32_t n, float threshold, float* mask) {
  boundary_mask_impl<float>(body, rigid, sample_x, n, threshold, mask);
}
void orc_boundary_mask_f64(const al_body_f64* body, const al_rigid_f64* rigid,
                           const double* sample_x, uint32_t n, double threshold, double* mask) {
  boundary_mask_impl<double>(body, rigid, sample_x, n, threshold, mask);
}

// launch_histogram256[_with_mask]: 256 counts of quantized bytes.
void orc_histogram256_f32(const float* v, const float* mask, uint32_t n, float v_min, float v_max,
                          uint32_t* hist) {
  histogram256(v, mask, n, v_min, v_max, hist);
}
void orc_histogram256_f64(const double* v, const double* mask, uint32_t n, double v_min,
                          double v_max, uint32_t* hist) {
  histogram256(v, mask, n, v_min, v_max, hist);
}

// calculate_kl_divergence in double, bins in order.
double orc_kl_divergence(const uint32_t* p, const uint32_t* q, uint32_t n_p, uint32_t n_q,
                         double q_lower_bound, uint32_t num_bins) {
  return kl_divergence(p, q, n_p, n_q, q_lower_bound, num_bins);
}

}  // extern "C"

extern "C" {

// SolverPellet<float>::step repeated `steps` times on host arrays:
// x [n][3] in/out, dx [n][3] / rho [n] (may be NULL) of the last step.
// Returns 1 on a neighbor overflow.
int orc_relax_pellets_f32(const al_const_f32* cn, const al_consti* cni, const al_body_f32* body,
                          float* x, uint32_t n, const al_pellet_relax_params* p, uint32_t steps,
                          float* dx, float* rho) {
  const Cn<float> c = make_cn<float>(*cn);
  const Body<float> b = make_body<float>(*body, nullptr);
  std::vector<V3<float>> xs(n);
  for (uint32_t i = 0; i < n; ++i) xs[i] = v3<float>(x + 3 * size_t(i));
  RelaxParams rp;
  rp.cohesion = p->cohesion;
  rp.adhesion = p->adhesion;
  rp.cfl_factor = p->cfl_factor;
  rp.tolerance = p->contact_tolerance;
  rp.wrap = p->wrap_y != 0;
  rp.wrap_length = p->wrap_length;
  std::vector<V3<float>> d;
  std::vector<float> r;
  const bool over = relax_pellets(c, *cni, b, xs, rp, steps, &d, &r);
  for (uint32_t i = 0; i < n; ++i) {
    x[3 * size_t(i)] = xs[i].x;
    x[3 * size_t(i) + 1] = xs[i].y;
    x[3 * size_t(i) + 2] = xs[i].z;
    if (dx && !d.empty()) {
      dx[3 * size_t(i)] = d[i].x;
      dx[3 * size_t(i) + 1] = d[i].y;
      dx[3 * size_t(i) + 2] = d[i].z;
    }
    if (rho && !r.empty()) rho[i] = r[i];
  }
  return over ? 1 : 0;
}

}  // extern "C"
