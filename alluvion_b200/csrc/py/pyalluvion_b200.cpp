// pyalluvion_b200.cpp -- pybind11 module with the reference's Python class
// names (lib/pyalluvion.cu: Store, Const<suffix>, ConstiN, Runner, Pile,
// Solver, SolverDf, SolverIi, SolverI, SolverPellet and the dg distances, suffixed
// "float" / "double") over the C++ layer of alluvion_b200_solver.hpp.
// Variables expose the numpy get / set of the reference's Coated variables
// (alluvion/variable.py:22-44) and __cuda_array_interface__ for zero-copy
// views from torch or cupy.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include "alluvion_b200_solver.hpp"

namespace py = pybind11;
using namespace alluvion_b200;

namespace {

py::dtype dtype_of(NumericType t) {
  switch (t) {
    case NumericType::f32: return py::dtype::of<float>();
    case NumericType::f64: return py::dtype::of<double>();
    case NumericType::i32: return py::dtype::of<int32_t>();
    default: return py::dtype::of<uint32_t>();
  }
}

const char* typestr_of(NumericType t) {
  switch (t) {
    case NumericType::f32: return "<f4";
    case NumericType::f64: return "<f8";
    case NumericType::i32: return "<i4";
    default: return "<u4";
  }
}

NumericType type_from_name(const std::string& s) {
  if (s == "float32" || s == "float" || s == "f32") return NumericType::f32;
  if (s == "float64" || s == "double" || s == "f64") return NumericType::f64;
  if (s == "int32" || s == "i32") return NumericType::i32;
  if (s == "uint32" || s == "u32") return NumericType::u32;
  throw error(AL_ERR_INVALID, "unknown numeric type " + s);
}

std::vector<py::ssize_t> element_shape(const Variable& v) {
  std::vector<py::ssize_t> shape(v.get_shape().begin(), v.get_shape().end());
  if (v.get_num_primitives_per_element() > 1) shape.push_back(v.get_num_primitives_per_element());
  return shape;
}

// Coated variable get (variable.py:22-35): a host copy shaped [shape..., n].
py::array variable_get(const Variable& v) {
  py::array out(dtype_of(v.get_type()), element_shape(v));
  if (v.get_num_bytes()) v.get_bytes(out.mutable_data(), v.get_num_bytes());
  return out;
}

// Coated variable set (variable.py:38-42): casts to the variable's type and
// copies the array's bytes starting at `offset` bytes.
void variable_set(Variable& v, py::array src, size_t offset) {
  py::array a = py::array::ensure(src.attr("astype")(dtype_of(v.get_type())),
                                  py::array::c_style | py::array::forcecast);
  v.set_bytes(a.data(), size_t(a.nbytes()), offset);
}

template <class TF>
std::array<TF, 3> t3(py::object o) {
  auto s = o.cast<std::vector<TF>>();
  if (s.size() != 3) throw error(AL_ERR_INVALID, "expected 3 components");
  return {s[0], s[1], s[2]};
}
template <class TF>
std::array<TF, 4> t4(py::object o) {
  auto s = o.cast<std::vector<TF>>();
  if (s.size() != 4) throw error(AL_ERR_INVALID, "expected 4 components");
  return {s[0], s[1], s[2], s[3]};
}

template <class TF>
void declare_real(py::module& m, py::module& dg_m, const char* sfx) {
  using T3 = std::array<TF, 3>;
  const std::string s(sfx);

  py::class_<Const<TF>>(m, ("Const" + s).c_str())
      .def(py::init<>())
      .def("set_kernel_radius", &Const<TF>::set_kernel_radius)
      .def("set_particle_attr", &Const<TF>::set_particle_attr)
      .def("set_wrap_length", &Const<TF>::set_wrap_length)
      .def_property_readonly("kernel_radius", [](const Const<TF>& c) { return c.kernel_radius; })
      .def_property_readonly("particle_radius",
                             [](const Const<TF>& c) { return c.particle_radius; })
      .def_property_readonly("particle_vol", [](const Const<TF>& c) { return c.particle_vol; })
      .def_property_readonly("particle_mass", [](const Const<TF>& c) { return c.particle_mass; })
      .def_property_readonly("density0", [](const Const<TF>& c) { return c.density0; })
      .def_readonly("wrap_length", &Const<TF>::wrap_length)
      .def_readonly("wrap_min", &Const<TF>::wrap_min)
      .def_readonly("wrap_max", &Const<TF>::wrap_max)
      .def_property(
          "viscosity", [](const Const<TF>& c) { return c.viscosity; },
          [](Const<TF>& c, TF v) { c.viscosity = v; })
      .def_property(
          "boundary_viscosity", [](const Const<TF>& c) { return c.boundary_viscosity; },
          [](Const<TF>& c, TF v) { c.boundary_viscosity = v; })
      .def_property(
          "dfsph_factor_epsilon", [](const Const<TF>& c) { return c.dfsph_factor_epsilon; },
          [](Const<TF>& c, TF v) { c.dfsph_factor_epsilon = v; })
      .def_readwrite("contact_tolerance", &Const<TF>::contact_tolerance)
      .def_property(
          "gravity",
          [](const Const<TF>& c) { return T3{c.gravity[0], c.gravity[1], c.gravity[2]}; },
          [](Const<TF>& c, py::object g) {
            const T3 v = t3<TF>(g);
            for (int k = 0; k < 3; ++k) c.gravity[k] = v[k];
          });

  using R = Runner<TF>;
  py::class_<R>(m, ("Runner" + s).c_str())
      .def(py::init<>())
      .def_static("calculate_se", &R::calculate_se, py::arg("v0"), py::arg("v1"),
                  py::arg("se"), py::arg("n"), py::arg("offset") = 0)
      .def_static("calculate_se_weighted", &R::calculate_se_weighted, py::arg("v0"),
                  py::arg("v1"), py::arg("weight0"), py::arg("n"), py::arg("offset") = 0)
      .def_static("calculate_se_yz_masked", &R::calculate_se_yz_masked, py::arg("v0"),
                  py::arg("v1"), py::arg("mask"), py::arg("n"), py::arg("offset") = 0)
      .def_static(
          "sum_products",
          [](const Variable& v0, const Variable& v1, uint32_t n, uint32_t offset) -> py::object {
            auto r = R::sum_products(v0, v1, n, offset);
            if (r.size() == 1) return py::float_(r[0]);
            return py::cast(r);
          },
          py::arg("v0"), py::arg("v1"), py::arg("n"), py::arg("offset") = 0)
      .def_static("calculate_kl_divergence", &R::calculate_kl_divergence,
                  py::arg("histogram_p"), py::arg("histogram_q"), py::arg("n_p"), py::arg("n_q"),
                  py::arg("q_lower_bound") = TF(1e-6), py::arg("num_bins") = 256);

  py::class_<dg::Distance<TF>, std::shared_ptr<dg::Distance<TF>>>(dg_m, ("Distance" + s).c_str())
      .def_readonly("aabb_min", &dg::Distance<TF>::aabb_min)
      .def_readonly("aabb_max", &dg::Distance<TF>::aabb_max)
      .def_readonly("max_distance", &dg::Distance<TF>::max_distance);
  py::class_<dg::SphereDistance<TF>, dg::Distance<TF>, std::shared_ptr<dg::SphereDistance<TF>>>(
      dg_m, ("SphereDistance" + s).c_str())
      .def(py::init<TF>(), py::arg("radius"))
      .def_static("create", [](TF r) { return std::make_shared<dg::SphereDistance<TF>>(r); },
                  py::arg("radius"))
      .def_readonly("radius", &dg::SphereDistance<TF>::radius);
  py::class_<dg::BoxDistance<TF>, dg::Distance<TF>, std::shared_ptr<dg::BoxDistance<TF>>>(
      dg_m, ("BoxDistance" + s).c_str())
      .def_static(
          "create",
          [](py::object w, TF outset) {
            return std::make_shared<dg::BoxDistance<TF>>(t3<TF>(w), outset);
          },
          py::arg("widths"), py::arg("outset") = TF(0))
      .def_readonly("half_widths", &dg::BoxDistance<TF>::half_widths)
      .def_readonly("outset", &dg::BoxDistance<TF>::outset);
  py::class_<dg::BoxShellDistance<TF>, dg::Distance<TF>,
             std::shared_ptr<dg::BoxShellDistance<TF>>>(dg_m, ("BoxShellDistance" + s).c_str())
      .def_static(
          "create",
          [](py::object w, TF thickness, TF outset) {
            return std::make_shared<dg::BoxShellDistance<TF>>(t3<TF>(w), thickness, outset);
          },
          py::arg("widths"), py::arg("thickness"), py::arg("outset") = TF(0))
      .def_readonly("half_inner_widths", &dg::BoxShellDistance<TF>::half_inner_widths)
      .def_readonly("half_outer_widths", &dg::BoxShellDistance<TF>::half_outer_widths)
      .def_readonly("outset", &dg::BoxShellDistance<TF>::outset);
  py::class_<dg::CylinderDistance<TF>, dg::Distance<TF>,
             std::shared_ptr<dg::CylinderDistance<TF>>>(dg_m, ("CylinderDistance" + s).c_str())
      .def_static(
          "create",
          [](TF r, TF h, TF com_y) { return std::make_shared<dg::CylinderDistance<TF>>(r, h, com_y); },
          py::arg("radius"), py::arg("height"), py::arg("com_y") = TF(0));
  py::class_<dg::CapsuleDistance<TF>, dg::Distance<TF>, std::shared_ptr<dg::CapsuleDistance<TF>>>(
      dg_m, ("CapsuleDistance" + s).c_str())
      .def_static(
          "create", [](TF r, TF h) { return std::make_shared<dg::CapsuleDistance<TF>>(r, h); },
          py::arg("radius"), py::arg("height"));
  py::class_<dg::InfiniteCylinderDistance<TF>, dg::Distance<TF>,
             std::shared_ptr<dg::InfiniteCylinderDistance<TF>>>(
      dg_m, ("InfiniteCylinderDistance" + s).c_str())
      .def_static(
          "create", [](TF r) { return std::make_shared<dg::InfiniteCylinderDistance<TF>>(r); },
          py::arg("radius"));
  py::class_<dg::InfiniteTubeDistance<TF>, dg::Distance<TF>,
             std::shared_ptr<dg::InfiniteTubeDistance<TF>>>(
      dg_m, ("InfiniteTubeDistance" + s).c_str())
      .def_static(
          "create",
          [](TF ri, TF ro, TF half) {
            return std::make_shared<dg::InfiniteTubeDistance<TF>>(ri, ro, half);
          },
          py::arg("inner_radius"), py::arg("outer_radius"), py::arg("aabb_half_length") = TF(0));
  py::class_<dg::TriangleMesh<TF>>(dg_m, ("TriangleMesh" + s).c_str())
      .def(py::init([](py::array_t<TF, py::array::c_style | py::array::forcecast> v,
                       py::array_t<uint32_t, py::array::c_style | py::array::forcecast> f) {
             if (v.ndim() != 2 || v.shape(1) != 3 || f.ndim() != 2 || f.shape(1) != 3)
               throw error(AL_ERR_INVALID, "TriangleMesh: vertices [n][3], faces [m][3]");
             dg::TriangleMesh<TF> m;
             m.vertices.resize(v.shape(0));
             m.faces.resize(f.shape(0));
             std::memcpy(m.vertices.data(), v.data(), v.nbytes());
             std::memcpy(m.faces.data(), f.data(), f.nbytes());
             return m;
           }),
           py::arg("vertices"), py::arg("faces"));
  py::class_<dg::MeshDistance<TF>, dg::Distance<TF>, std::shared_ptr<dg::MeshDistance<TF>>>(
      dg_m, ("MeshDistance" + s).c_str())
      .def_static(
          "create",
          [](const dg::TriangleMesh<TF>& mesh, TF offset, bool) {
            return std::make_shared<dg::MeshDistance<TF>>(mesh, offset);
          },
          py::arg("mesh"), py::arg("offset") = TF(0), py::arg("precompute_normals") = true);

  py::class_<Mesh<TF>>(m, ("Mesh" + s).c_str())
      .def(py::init<>())
      .def_property(
          "vertices",
          [](const Mesh<TF>& me) {
            py::array_t<TF> a({py::ssize_t(me.vertices.size()), py::ssize_t(3)});
            if (!me.vertices.empty())
              std::memcpy(a.mutable_data(), me.vertices.data(), me.vertices.size() * 3 * sizeof(TF));
            return a;
          },
          [](Mesh<TF>& me, py::array_t<TF, py::array::c_style | py::array::forcecast> v) {
            if (v.ndim() != 2 || v.shape(1) != 3)
              throw error(AL_ERR_INVALID, "Mesh.vertices: [n][3]");
            me.vertices.resize(v.shape(0));
            std::memcpy(me.vertices.data(), v.data(), v.nbytes());
          });

  using P = Pile<TF>;
  py::class_<P>(m, ("Pile" + s).c_str())
      .def(py::init<Store&, Runner<TF>&, uint32_t, VolumeMethod, uint32_t, const Const<TF>*,
                    const ConstiN*>(),
           py::arg("store"), py::arg("runner"), py::arg("max_num_contacts"),
           py::arg("volume_method") = VolumeMethod::volume_map,
           py::arg("max_num_pellets") = 10000, py::arg("cn") = nullptr, py::arg("cni") = nullptr,
           py::keep_alive<1, 2>(), py::keep_alive<1, 3>())
      .def(
          "add",
          [](P& p, std::shared_ptr<dg::Distance<TF>> d, py::object resolution, TF cell_width,
             TF margin, TF sign, py::object collision_mesh, py::object pellets, TF mass,
             TF restitution, TF friction, py::object inertia, py::object x, py::object q,
             py::object) {
            auto r = resolution.cast<std::vector<uint32_t>>();
            if (r.size() != 3) throw error(AL_ERR_INVALID, "resolution: 3 components");
            if (!pellets.is_none()) {  // the pellet overload: numpy [n][3] or a Variable
              std::vector<std::array<TF, 3>> pl;
              if (py::isinstance<Variable>(pellets)) {
                const Variable& v = pellets.cast<const Variable&>();
                if (v.get_num_primitives_per_element() != 3 ||
                    v.get_type() != numeric_type_of<TF>())
                  throw error(AL_ERR_INVALID, "pellets: a [n] x 3 variable of the pile's type");
                pl.resize(v.get_linear_shape());
                if (!pl.empty()) v.get_bytes(pl.data(), pl.size() * sizeof(pl[0]));
              } else {
                py::array_t<TF, py::array::c_style | py::array::forcecast> a(pellets);
                if (a.ndim() != 2 || a.shape(1) != 3)
                  throw error(AL_ERR_INVALID, "pellets: [n][3]");
                pl.resize(a.shape(0));
                if (!pl.empty()) std::memcpy(pl.data(), a.data(), a.nbytes());
              }
              return p.add(std::move(d), {r[0], r[1], r[2]}, cell_width, margin, sign, pl, mass,
                           restitution, friction, t3<TF>(inertia), t3<TF>(x), t4<TF>(q));
            }
            Mesh<TF> cm;
            if (!collision_mesh.is_none()) cm = collision_mesh.cast<Mesh<TF>>();
            return p.add(std::move(d), {r[0], r[1], r[2]}, cell_width, margin, sign, cm, mass,
                         restitution, friction, t3<TF>(inertia), t3<TF>(x), t4<TF>(q));
          },
          py::arg("distance"), py::arg("resolution") = std::vector<uint32_t>{0, 0, 0},
          py::arg("cell_width") = TF(0), py::arg("margin") = std::numeric_limits<TF>::infinity(),
          py::arg("sign") = TF(1), py::arg("collision_mesh") = py::none(),
          py::arg("pellets") = py::none(), py::arg("mass") = TF(0),
          py::arg("restitution") = TF(1), py::arg("friction") = TF(0),
          py::arg("inertia_tensor") = std::vector<TF>{1, 1, 1},
          py::arg("x") = std::vector<TF>{0, 0, 0}, py::arg("q") = std::vector<TF>{0, 0, 0, 1},
          py::arg("display_mesh") = py::none())
      .def_property_readonly("num_pellets", &P::num_pellets)
      .def_readonly("max_num_pellets", &P::max_num_pellets_)
      .def("get_size", &P::get_size)
      .def("set_gravity", [](P& p, py::object g) { p.set_gravity(t3<TF>(g)); })
      .def("copy_kinematics_to_device", &P::copy_kinematics_to_device)
      .def("write_file", &P::write_file, py::arg("filename"), py::arg("x_scale") = TF(1),
           py::arg("v_scale") = TF(1), py::arg("omega_scale") = TF(1))
      .def("read_file", &P::read_file, py::arg("filename"), py::arg("num_rigids") = -1,
           py::arg("dst_offset") = 0, py::arg("src_offset") = 0)
      .def_static("get_size_from_file", &P::get_size_from_file, py::arg("filename"))
      .def_readwrite("mass", &P::mass_)
      .def_readwrite("x", &P::x_)
      .def_readwrite("v", &P::v_)
      .def_readwrite("q", &P::q_)
      .def_readwrite("omega", &P::omega_)
      .def_readwrite("restitution", &P::restitution_)
      .def_readwrite("friction", &P::friction_)
      .def_readwrite("inertia_tensor", &P::inertia_tensor_)
      .def_readonly("force", &P::force_)
      .def_readonly("torque", &P::torque_)
      .def_readonly("domain_min_list", &P::domain_min_list_)
      .def_readonly("domain_max_list", &P::domain_max_list_)
      .def_readonly("resolution_list", &P::resolution_list_)
      .def_readonly("cell_size_list", &P::cell_size_list_)
      .def_readonly("sign_list", &P::sign_list_)
      .def_readonly("grid_size_list", &P::grid_size_list_)
      .def_property_readonly("distance_grids", &P::get_distance_grids,
                             py::return_value_policy::reference_internal)
      .def_property_readonly("volume_grids", &P::get_volume_grids,
                             py::return_value_policy::reference_internal);

  using S = Solver<TF>;
  const auto ref = py::return_value_policy::reference_internal;
  py::class_<S>(m, ("Solver" + s).c_str())
      .def_readonly("max_num_particles", &S::max_num_particles)
      .def_readonly("particle_max_v2", &S::particle_max_v2)
      .def_readonly("pile_max_v2", &S::pile_max_v2)
      .def_readonly("max_v2", &S::max_v2)
      .def_readonly("cfl_dt", &S::cfl_dt)
      .def_readonly("utilized_cfl", &S::utilized_cfl)
      .def_readwrite("num_particles", &S::num_particles)
      .def_readwrite("t", &S::t)
      .def_readwrite("dt", &S::dt)
      .def_readwrite("initial_dt", &S::initial_dt)
      .def_readwrite("max_dt", &S::max_dt)
      .def_readwrite("min_dt", &S::min_dt)
      .def_readwrite("cfl", &S::cfl)
      .def_readwrite("particle_radius", &S::particle_radius)
      .def_property_readonly("particle_x", [](const S& x) { return x.particle_x; }, ref)
      .def_property_readonly("particle_v", [](const S& x) { return x.particle_v; }, ref)
      .def_property_readonly("particle_a", [](const S& x) { return x.particle_a; }, ref)
      .def_property_readonly("particle_density", [](const S& x) { return x.particle_density; },
                             ref)
      .def_property_readonly("particle_boundary", [](const S& x) { return x.particle_boundary; },
                             ref)
      .def_property_readonly("particle_boundary_kernel",
                             [](const S& x) { return x.particle_boundary_kernel; }, ref)
      .def_property_readonly("particle_neighbors",
                             [](const S& x) { return x.particle_neighbors; }, ref)
      .def_property_readonly("particle_num_neighbors",
                             [](const S& x) { return x.particle_num_neighbors; }, ref)
      .def_property_readonly("grid_anomaly", [](const S& x) { return x.grid_anomaly; }, ref)
      .def_property_readonly("pile", [](const S& x) { return &x.pile; }, ref)
      .def("reset_solving_var", &S::reset_solving_var)
      .def("reset_t", &S::reset_t)
      .def("compute_all_boundaries", &S::compute_all_boundaries)
      .def("sample_all_boundaries", &S::sample_all_boundaries, py::arg("sample_x"),
           py::arg("sample_boundary"), py::arg("sample_boundary_kernel"),
           py::arg("num_samples"))
      .def("update_particle_neighbors", &S::template update_particle_neighbors<0>)
      .def("update_particle_neighbors_wrap1", &S::template update_particle_neighbors<1>);

  using Df = SolverDf<TF>;
  py::class_<Df, S>(m, ("SolverDf" + s).c_str())
      .def(py::init<Runner<TF>&, P&, Store&, uint32_t, uint32_t, bool, bool, const Const<TF>*,
                    const ConstiN*, bool>(),
           py::arg("runner"), py::arg("pile"), py::arg("store"), py::arg("max_num_particles"),
           py::arg("num_ushers") = 0, py::arg("enable_surface_tension") = false,
           py::arg("enable_vorticity") = false, py::arg("cn") = nullptr, py::arg("cni") = nullptr,
           py::arg("graphical") = false, py::keep_alive<1, 2>(), py::keep_alive<1, 3>(),
           py::keep_alive<1, 4>())
      .def_readonly("num_divergence_solve", &Df::num_divergence_solve)
      .def_readonly("num_density_solve", &Df::num_density_solve)
      .def_readonly("mean_density_change", &Df::mean_density_change)
      .def_readonly("mean_density_error", &Df::mean_density_error)
      .def_readwrite("enable_divergence_solve", &Df::enable_divergence_solve)
      .def_readwrite("enable_density_solve", &Df::enable_density_solve)
      .def_readwrite("density_change_tolerance", &Df::density_change_tolerance)
      .def_readwrite("density_error_tolerance", &Df::density_error_tolerance)
      .def_readwrite("min_density_solve", &Df::min_density_solve)
      .def_readwrite("max_density_solve", &Df::max_density_solve)
      .def_readwrite("min_divergence_solve", &Df::min_divergence_solve)
      .def_readwrite("max_divergence_solve", &Df::max_divergence_solve)
      .def_property_readonly("particle_dfsph_factor",
                             [](const Df& x) { return x.particle_dfsph_factor; }, ref)
      .def_property_readonly("particle_kappa", [](const Df& x) { return x.particle_kappa; }, ref)
      .def_property_readonly("particle_kappa_v", [](const Df& x) { return x.particle_kappa_v; },
                             ref)
      .def_property_readonly("particle_density_adv",
                             [](const Df& x) { return x.particle_density_adv; }, ref)
      .def("step", &Df::template step<0>)
      .def("step_wrap1", &Df::template step<1>);

  auto declare_pressure = [&](auto tag, const std::string& name) {
    using Sp = typename decltype(tag)::type;
    py::class_<Sp, S>(m, (name + s).c_str())
        .def(py::init<Runner<TF>&, P&, Store&, uint32_t, uint32_t, bool, bool, const Const<TF>*,
                      const ConstiN*, bool>(),
             py::arg("runner"), py::arg("pile"), py::arg("store"), py::arg("max_num_particles"),
             py::arg("num_ushers") = 0, py::arg("enable_surface_tension") = false,
             py::arg("enable_vorticity") = false, py::arg("cn") = nullptr,
             py::arg("cni") = nullptr, py::arg("graphical") = false, py::keep_alive<1, 2>(),
             py::keep_alive<1, 3>(), py::keep_alive<1, 4>())
        .def_readonly("num_density_solve", &Sp::num_density_solve)
        .def_readonly("mean_density_error", &Sp::mean_density_error)
        .def_readwrite("density_error_tolerance", &Sp::density_error_tolerance)
        .def_readwrite("min_density_solve", &Sp::min_density_solve)
        .def_readwrite("max_density_solve", &Sp::max_density_solve)
        .def_property_readonly("particle_pressure",
                               [](const Sp& x) { return x.particle_pressure; }, ref)
        .def_property_readonly("particle_adv_density",
                               [](const Sp& x) { return x.particle_adv_density; }, ref)
        .def("step", &Sp::template step<0>)
        .def("step_wrap1", &Sp::template step<1>);
  };
  using Pel = SolverPellet<TF>;
  py::class_<Pel, S>(m, ("SolverPellet" + s).c_str())
      .def(py::init<Runner<TF>&, P&, Store&, uint32_t, const Const<TF>*, const ConstiN*, bool>(),
           py::arg("runner"), py::arg("pile"), py::arg("store"), py::arg("max_num_particles"),
           py::arg("cn") = nullptr, py::arg("cni") = nullptr, py::arg("graphical") = false,
           py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>())
      .def_readwrite("cfl_factor", &Pel::cfl_factor)
      .def_readwrite("cohesion", &Pel::cohesion)
      .def_readwrite("adhesion", &Pel::adhesion)
      .def_property_readonly("particle_dfsph_factor",
                             [](const Pel& x) { return x.particle_dfsph_factor; }, ref)
      .def("set_pellets", &Pel::set_pellets)
      .def("step", &Pel::template step<0>)
      .def("step_wrap1", &Pel::template step<1>);

  struct IiTag {
    using type = SolverIi<TF>;
  };
  struct ITag {
    using type = SolverI<TF>;
  };
  declare_pressure(IiTag{}, "SolverIi");
  declare_pressure(ITag{}, "SolverI");
}

}  // namespace

PYBIND11_MODULE(_alluvion_b200, m) {
  m.doc() = "The reference's Python object model for the SPH step over the alluvion_b200 engine";
  py::register_exception<error>(m, "Error", PyExc_RuntimeError);

  py::enum_<NumericType>(m, "NumericType")
      .value("f32", NumericType::f32)
      .value("f64", NumericType::f64)
      .value("i32", NumericType::i32)
      .value("u32", NumericType::u32);
  py::enum_<VolumeMethod>(m, "VolumeMethod")
      .value("volume_map", VolumeMethod::volume_map)
      .value("pellets", VolumeMethod::pellets);

  py::class_<Variable>(m, "Variable")
      .def("get_shape", &Variable::get_shape)
      .def("get_linear_shape", &Variable::get_linear_shape)
      .def("get_num_primitives_per_element", &Variable::get_num_primitives_per_element)
      .def("get_type", &Variable::get_type)
      .def("get_num_bytes", &Variable::get_num_bytes)
      .def("get_bytes",
           [](const Variable& v, py::array dst, size_t offset) {
             if (!(dst.flags() & py::array::c_style) || !dst.writeable())
               throw error(AL_ERR_INVALID, "get_bytes: a writeable contiguous array");
             v.get_bytes(dst.mutable_data(), size_t(dst.nbytes()), offset);
           },
           py::arg("dst"), py::arg("offset") = 0)
      .def("set_bytes",
           [](Variable& v, py::array src, size_t offset) {
             py::array a = py::array::ensure(src, py::array::c_style);
             v.set_bytes(a.data(), size_t(a.nbytes()), offset);
           },
           py::arg("src"), py::arg("offset") = 0)
      .def("write_file", &Variable::write_file, py::arg("filename"),
           py::arg("shape_outermost") = 0, py::arg("offset") = 0)
      .def("read_file", &Variable::read_file, py::arg("filename"))
      .def("set_zero", &Variable::set_zero)
      .def("set_from", &Variable::set_from)
      .def("get", &variable_get)
      .def("set", &variable_set, py::arg("src"), py::arg("offset") = 0)
      .def_property_readonly("ptr", [](const Variable& v) { return uintptr_t(v.ptr()); })
      .def_property_readonly("__cuda_array_interface__", [](const Variable& v) {
        py::dict d;
        py::tuple shape = py::cast(element_shape(v));
        d["shape"] = shape;
        d["typestr"] = typestr_of(v.get_type());
        d["data"] = py::make_tuple(uintptr_t(v.ptr()), false);
        d["version"] = 3;
        return d;
      });

  py::class_<ConstiN>(m, "ConstiN")
      .def(py::init<>())
      .def_readonly("max_num_contacts", &ConstiN::max_num_contacts)
      .def_property(
          "num_boundaries", [](const ConstiN& c) { return c.num_boundaries; },
          [](ConstiN& c, uint32_t v) { c.num_boundaries = v; })
      .def_property(
          "max_num_particles_per_cell", [](const ConstiN& c) { return c.max_num_particles_per_cell; },
          [](ConstiN& c, uint32_t v) { c.max_num_particles_per_cell = v; })
      .def_property(
          "max_num_neighbors_per_particle",
          [](const ConstiN& c) { return c.max_num_neighbors_per_particle; },
          [](ConstiN& c, uint32_t v) { c.max_num_neighbors_per_particle = v; })
      .def_property(
          "grid_res",
          [](const ConstiN& c) {
            return std::array<uint32_t, 3>{c.grid_res[0], c.grid_res[1], c.grid_res[2]};
          },
          [](ConstiN& c, std::array<uint32_t, 3> v) {
            for (int k = 0; k < 3; ++k) c.grid_res[k] = v[k];
          })
      .def_property(
          "grid_offset",
          [](const ConstiN& c) {
            return std::array<int32_t, 3>{c.grid_offset[0], c.grid_offset[1], c.grid_offset[2]};
          },
          [](ConstiN& c, std::array<int32_t, 3> v) {
            for (int k = 0; k < 3; ++k) c.grid_offset[k] = v[k];
          });

  py::module dg_m = m.def_submodule("dg", "signed distances (Discregrid)");
  declare_real<float>(m, dg_m, "float");
  declare_real<double>(m, dg_m, "double");

  const auto ref = py::return_value_policy::reference_internal;
  py::class_<Store>(m, "Store")
      .def(py::init<int>(), py::arg("device") = 0)
      .def("create",
           [](Store& s, std::vector<uint32_t> shape, uint32_t n, const std::string& type) {
             return s.create(std::move(shape), n, type_from_name(type));
           },
           py::arg("shape"), py::arg("n"), py::arg("dtype") = "float32", ref)
      .def("remove", &Store::remove)
      .def("has_display", &Store::has_display)
      .def_property_readonly("cnfloat", [](Store& s) { return &s.get_cn<float>(); }, ref)
      .def_property_readonly("cndouble", [](Store& s) { return &s.get_cn<double>(); }, ref)
      .def_property_readonly("cni", [](Store& s) { return &s.get_cni(); }, ref)
      .def("copy_cnfloat", &Store::copy_cn<float>)
      .def("copy_cndouble", &Store::copy_cn<double>)
      .def("copy_cn_externalfloat", &Store::copy_cn_external<float>)
      .def("copy_cn_externaldouble", &Store::copy_cn_external<double>)
      .def("create_cnfloat", [](Store&) { return std::make_pair(Const<float>(), ConstiN()); })
      .def("create_cndouble", [](Store&) { return std::make_pair(Const<double>(), ConstiN()); })
      .def("synchronize", [](Store& s) { s.get_engine().synchronize(); });
}
