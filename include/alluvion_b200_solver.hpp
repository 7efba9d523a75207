/*
 * alluvion_b200_solver.hpp -- the reference's host object model for the
 * fluid step, restated over the C ABI of alluvion_b200.h: Store and
 * Variable (store.hpp, variable.hpp), Const / ConstiN (constants.hpp),
 * the analytic and mesh distances (the dg distance headers), Pile (pile.hpp),
 * Runner (a tag: launches are the engine's), and Solver / SolverDf /
 * SolverIi / SolverI / SolverPellet (solver.hpp, solver_df.hpp,
 * solver_ii.hpp, solver_i.hpp, solver_pellet.hpp) with the reference's
 * field names, defaults and step<wrap>.
 * Header-only; the pybind11 module alluvion_b200/_alluvion_b200 exposes it
 * with the reference's Python class names.
 *
 * Differences that follow from the engine:
 *  - Const / ConstiN travel by value with every call: copy_cn and
 *    copy_cn_external only record which block a solver uses (the
 *    reference uploads them to __constant__ symbols, store.hpp:142-164).
 *  - Pile kinematics are read by value at each step, so
 *    copy_kinematics_to_device has nothing to copy; rigid integration runs
 *    on the device inside the step and writes back x_, v_, q_, omega_;
 *    the per-body force and torque totals land in force_ / torque_ (FP64
 *    sums, narrowed), and no per-particle particle_force / particle_torque
 *    buffers exist.
 *  - Options outside the engine's scope (ushers, surface tension,
 *    vorticity, graphical buffers) throw error(AL_ERR_UNSUPPORTED); a
 *    pile with VolumeMethod::pellets steps with SolverI (its pellet branch)
 *    and relaxes with SolverPellet, as in the reference.
 */
#ifndef ALLUVION_B200_SOLVER_HPP
#define ALLUVION_B200_SOLVER_HPP

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "alluvion_b200.hpp"

namespace alluvion_b200 {

enum class NumericType { f32, f64, i32, u32 };

inline size_t numeric_size(NumericType t) { return t == NumericType::f64 ? 8 : 4; }

template <class T>
constexpr NumericType numeric_type_of();
template <>
constexpr NumericType numeric_type_of<float>() { return NumericType::f32; }
template <>
constexpr NumericType numeric_type_of<double>() { return NumericType::f64; }
template <>
constexpr NumericType numeric_type_of<int32_t>() { return NumericType::i32; }
template <>
constexpr NumericType numeric_type_of<uint32_t>() { return NumericType::u32; }

class Store;

// Variable<D, M> (variable.hpp): a view {shape, primitives per element,
// numeric type, device pointer} of memory the Store owns.  Offsets and
// sizes of the byte copies are in bytes, as in Variable::get_bytes /
// set_bytes.
class Variable {
 public:
  Variable() = default;
  Variable(al_engine* e, void* p, std::vector<uint32_t> shape, uint32_t num_primitives,
           NumericType type)
      : engine_(e), ptr_(p), shape_(std::move(shape)), n_(num_primitives), type_(type) {}
  void* ptr() const { return ptr_; }
  al_engine* engine_handle() const { return engine_; }
  template <class T>
  T* data() const { return static_cast<T*>(ptr_); }
  const std::vector<uint32_t>& get_shape() const { return shape_; }
  uint32_t get_linear_shape() const {
    uint32_t n = 1;
    for (uint32_t s : shape_) n *= s;
    return shape_.empty() ? 0 : n;
  }
  uint32_t get_num_primitives_per_element() const { return n_; }
  NumericType get_type() const { return type_; }
  size_t get_num_primitives() const { return size_t(get_linear_shape()) * n_; }
  size_t get_num_bytes() const { return get_num_primitives() * numeric_size(type_); }
  void get_bytes(void* dst, size_t num_bytes, size_t offset = 0) const {
    bounds(num_bytes, offset, "Variable::get_bytes");
    check(al_copy(engine_, dst, static_cast<const char*>(ptr_) + offset, num_bytes),
          "Variable::get_bytes");
  }
  void set_bytes(const void* src, size_t num_bytes, size_t offset = 0) {
    bounds(num_bytes, offset, "Variable::set_bytes");
    check(al_copy(engine_, static_cast<char*>(ptr_) + offset, src, num_bytes),
          "Variable::set_bytes");
  }
  void get_bytes(void* dst) const { get_bytes(dst, get_num_bytes()); }
  void set_bytes(const void* src) { set_bytes(src, get_num_bytes()); }
  void set_zero() { check(al_set(engine_, ptr_, 0, get_num_bytes()), "Variable::set_zero"); }
  // Copies min(bytes of src, bytes of this) from another variable.
  void set_from(const Variable& src) {
    const size_t b = std::min(src.get_num_bytes(), get_num_bytes());
    check(al_copy(engine_, ptr_, src.ptr_, b), "Variable::set_from");
  }
  // Variable::write_file (variable.hpp:132-167): the shape (outermost entry
  // shape_outermost, 0 = all), a 0 terminator, the primitives per element,
  // the type label, then the elements from element `offset` on.  (With
  // shape_outermost 0 the reference writes the header of the whole variable
  // but no elements; here the elements follow, as the header says.)
  void write_file(const std::string& filename, uint32_t shape_outermost = 0,
                  uint32_t offset = 0) const {
    if (shape_.empty()) throw error(AL_ERR_INVALID, "write_file: empty variable");
    if (shape_outermost > shape_[0])
      throw error(AL_ERR_INVALID, "Writing more than the outermost shape (" +
                                      std::to_string(shape_outermost) + ">" +
                                      std::to_string(shape_[0]) + ").");
    if (shape_outermost == 0) shape_outermost = shape_[0];
    const size_t esize = numeric_size(type_) * n_;
    const size_t per_outer = size_t(get_linear_shape()) / shape_[0];
    const size_t bytes = per_outer * shape_outermost * esize, boff = size_t(offset) * esize;
    if (bytes + boff > get_num_bytes())
      throw error(AL_ERR_INVALID, "Writing more than allocated: " + std::to_string(bytes + boff) +
                                      " " + std::to_string(get_num_bytes()));
    std::ofstream f(filename, std::ios::binary | std::ios::trunc);
    if (!f) throw error(AL_ERR_INVALID, "Failed to open alu file: " + filename);
    for (size_t i = 0; i < shape_.size(); ++i) {
      const uint32_t v = i == 0 ? shape_outermost : shape_[i];
      f.write(reinterpret_cast<const char*>(&v), 4);
    }
    const uint32_t end = 0;
    f.write(reinterpret_cast<const char*>(&end), 4);
    f.write(reinterpret_cast<const char*>(&n_), 4);
    const char label = type_label(type_);
    f.write(&label, 1);
    std::vector<char> host(bytes);
    if (bytes) get_bytes(host.data(), bytes, boff);
    f.write(host.data(), std::streamsize(bytes));
  }
  // Variable::read_file (variable.hpp:169-262): checks the dimensions, the
  // inner shape and the primitives per element, converts float <-> double,
  // and returns the outermost shape read.
  uint32_t read_file(const std::string& filename) {
    std::ifstream f(filename, std::ios::binary);
    if (!f.is_open()) throw error(AL_ERR_INVALID, "Failed to open alu file: " + filename);
    uint32_t outer = 0;
    for (size_t i = 0; i < shape_.size(); ++i) {
      uint32_t v = 0;
      f.read(reinterpret_cast<char*>(&v), 4);
      if (v == 0) throw error(AL_ERR_INVALID, "Shape mismatch when reading " + filename);
      if (i == 0) {
        outer = v;
        if (outer > shape_[0])
          throw error(AL_ERR_INVALID, "Reading more than the outermost shape: " + filename);
      } else if (v != shape_[i]) {
        throw error(AL_ERR_INVALID, "Shape mismatch for shape item " + std::to_string(i) +
                                        ": " + filename);
      }
    }
    uint32_t end = 1, p = 0;
    f.read(reinterpret_cast<char*>(&end), 4);
    if (end != 0) throw error(AL_ERR_INVALID, "Dimension mismatch when reading " + filename);
    f.read(reinterpret_cast<char*>(&p), 4);
    if (p != n_)
      throw error(AL_ERR_INVALID, "Num primitives per unit mismatch when reading " + filename);
    char label = 0;
    f.read(&label, 1);
    const size_t prims = size_t(get_linear_shape()) / shape_[0] * outer * n_;
    const char mine = type_label(type_);
    std::vector<char> host(prims * numeric_size(type_));
    if (label == mine) {
      f.read(host.data(), std::streamsize(host.size()));
    } else if (label == 'f' && mine == 'd') {
      std::vector<float> src(prims);
      f.read(reinterpret_cast<char*>(src.data()), std::streamsize(prims * 4));
      for (size_t i = 0; i < prims; ++i) reinterpret_cast<double*>(host.data())[i] = src[i];
    } else if (label == 'd' && mine == 'f') {
      std::vector<double> src(prims);
      f.read(reinterpret_cast<char*>(src.data()), std::streamsize(prims * 8));
      for (size_t i = 0; i < prims; ++i)
        reinterpret_cast<float*>(host.data())[i] = static_cast<float>(src[i]);
    } else {
      throw error(AL_ERR_INVALID, "Data type mismatch when reading " + filename);
    }
    if (!host.empty()) set_bytes(host.data(), host.size());
    return outer;
  }

 private:
  friend class Store;
  static char type_label(NumericType t) {
    switch (t) {
      case NumericType::f32: return 'f';
      case NumericType::f64: return 'd';
      case NumericType::i32: return 'i';
      default: return 'u';
    }
  }
  void bounds(size_t num_bytes, size_t offset, const char* where) const {
    if (offset > get_num_bytes() || num_bytes > get_num_bytes() - offset)
      throw error(AL_ERR_INVALID, std::string(where) + ": range past the end of the variable");
  }
  al_engine* engine_ = nullptr;
  void* ptr_ = nullptr;
  std::vector<uint32_t> shape_;
  uint32_t n_ = 1;
  NumericType type_ = NumericType::f32;
};

// Const<TF> (constants.hpp:51-137): the engine's al_const plus the wrap
// fields and the setters.
template <class TF>
struct Const : real<TF>::cn {
  TF wrap_length = 0, wrap_min = 0, wrap_max = 0;
  TF contact_tolerance = 0;
  Const() { std::memset(static_cast<typename real<TF>::cn*>(this), 0, sizeof(typename real<TF>::cn)); }
  const typename real<TF>::cn* c() const { return this; }
  // Const::set_kernel_radius (constants.hpp:100-120), the cubic-spline part.
  void set_kernel_radius(TF h) {
    const TF h2 = h * h, h3 = h2 * h, h4 = h2 * h2;
    const TF pi = TF(3.14159265358979323846);
    this->kernel_radius = h;
    this->kernel_radius_sqr = h2;
    this->cubic_kernel_k = TF(8.0) / h3 / pi;
    this->cubic_kernel_l = TF(48.0) / h4 / pi;
    this->cubic_kernel_zero = this->cubic_kernel_k;
  }
  // Const::set_particle_attr (constants.hpp:122-128).
  void set_particle_attr(TF radius, TF mass, TF density) {
    this->particle_radius = radius;
    this->particle_mass = mass;
    this->density0 = density;
    this->particle_vol = mass / density;
  }
  // Const::set_wrap_length (constants.hpp:130-136).
  void set_wrap_length(TF l) {
    wrap_length = l;
    wrap_min = l * TF(-0.5);
    wrap_max = l * TF(0.5);
  }
};

// Consti (constants.hpp:40-49) with its max_num_contacts.
struct ConstiN : al_consti {
  uint32_t max_num_contacts = 0;
  ConstiN() { std::memset(static_cast<al_consti*>(this), 0, sizeof(al_consti)); }
};

// Store (store.hpp): owns every device buffer and the default Const /
// ConstiN blocks.
class Store {
 public:
  explicit Store(int device = 0) : engine_(device) {}
  Store(const Store&) = delete;
  Store& operator=(const Store&) = delete;
  ~Store() {
    for (auto& v : vars_)
      if (v && v->ptr_) al_free(engine_.get(), v->ptr_);
  }
  al_engine* eng() const { return engine_.get(); }
  const engine& get_engine() const { return engine_; }
  Variable* create(std::vector<uint32_t> shape, uint32_t num_primitives, NumericType type) {
    size_t n = 1;
    for (uint32_t s : shape) n *= s;
    void* p = nullptr;
    const size_t bytes = n * num_primitives * numeric_size(type);
    check(al_allocate(engine_.get(), &p, bytes), "Store::create");
    // zero-filled (the reference's Allocator leaves new memory undefined)
    const int st = al_set(engine_.get(), p, 0, bytes);
    if (st != AL_OK) {
      al_free(engine_.get(), p);
      check(st, "Store::create");
    }
    vars_.emplace_back(new Variable(engine_.get(), p, std::move(shape), num_primitives, type));
    return vars_.back().get();
  }
  template <class T>
  Variable* create(std::vector<uint32_t> shape, uint32_t num_primitives = 1) {
    return create(std::move(shape), num_primitives, numeric_type_of<T>());
  }
  // Frees the variable's memory; the view becomes empty.
  void remove(Variable& v) {
    if (v.ptr_) al_free(engine_.get(), v.ptr_);
    v.ptr_ = nullptr;
    v.shape_.clear();
  }
  bool has_display() const { return false; }
  template <class TF>
  Const<TF>& get_cn();
  ConstiN& get_cni() { return cni_; }
  template <class TF>
  void copy_cn() {}
  template <class TF>
  void copy_cn_external(const Const<TF>&, const ConstiN&) {}

 private:
  engine engine_;
  std::vector<std::unique_ptr<Variable>> vars_;
  Const<float> cnf_;
  Const<double> cnd_;
  ConstiN cni_;
};
template <>
inline Const<float>& Store::get_cn<float>() { return cnf_; }
template <>
inline Const<double>& Store::get_cn<double>() { return cnd_; }

namespace dg {
// Distance (dg/distance.hpp): shape code, parameters, bounding box and
// max_distance of one signed-distance body.
template <class TF>
struct Distance {
  using T3 = std::array<TF, 3>;
  uint32_t shape = 0;
  std::array<TF, 8> params{};
  T3 aabb_min{}, aabb_max{};
  TF max_distance = 0;
  virtual ~Distance() = default;
};
template <class TF>
struct SphereDistance : Distance<TF> {  // dg/sphere_distance.hpp
  TF radius;
  explicit SphereDistance(TF r) : radius(r) {
    this->shape = AL_SHAPE_SPHERE;
    this->params[0] = r;
    this->aabb_min = {-r, -r, -r};
    this->aabb_max = {r, r, r};
    this->max_distance = r;
  }
};
template <class TF>
struct BoxDistance : Distance<TF> {  // dg/box_distance.hpp
  std::array<TF, 3> half_widths;
  TF outset;
  explicit BoxDistance(std::array<TF, 3> widths, TF outset_arg = 0) : outset(outset_arg) {
    this->shape = AL_SHAPE_BOX;
    TF n2 = 0;
    for (int i = 0; i < 3; ++i) {
      half_widths[i] = widths[i] * TF(0.5);
      this->params[i] = half_widths[i];
      this->aabb_min[i] = -half_widths[i] - outset;
      this->aabb_max[i] = half_widths[i] + outset;
      n2 += half_widths[i] * half_widths[i];
    }
    this->params[3] = outset;
    this->max_distance = std::sqrt(n2) + outset;
  }
};
template <class TF>
struct BoxShellDistance : Distance<TF> {  // dg/box_shell_distance.hpp
  std::array<TF, 3> half_inner_widths, half_outer_widths;
  TF outset;
  BoxShellDistance(std::array<TF, 3> widths, TF thickness, TF outset_arg = 0)
      : outset(outset_arg) {
    this->shape = AL_SHAPE_BOX_SHELL;
    TF n2 = 0;
    for (int i = 0; i < 3; ++i) {
      half_inner_widths[i] = widths[i] * TF(0.5);
      half_outer_widths[i] = half_inner_widths[i] + thickness;
      this->params[i] = half_inner_widths[i];
      this->params[3 + i] = half_outer_widths[i];
      this->aabb_min[i] = -half_outer_widths[i] - outset;
      this->aabb_max[i] = half_outer_widths[i] + outset;
      n2 += half_outer_widths[i] * half_outer_widths[i];
    }
    this->params[6] = outset;
    this->max_distance = std::sqrt(n2) + outset;
  }
};
template <class TF>
struct CylinderDistance : Distance<TF> {  // dg/cylinder_distance.hpp
  CylinderDistance(TF radius, TF height, TF com_y = 0) {
    this->shape = AL_SHAPE_CYLINDER;
    this->params[0] = radius;
    this->params[1] = height;
    this->params[2] = com_y;
    const TF hh = height * TF(0.5);
    this->aabb_min = {-radius, -hh - com_y, -radius};
    this->aabb_max = {radius, hh - com_y, radius};
    const TF a = hh + std::fabs(com_y);
    this->max_distance = std::sqrt(radius * radius + a * a);
  }
};
template <class TF>
struct CapsuleDistance : Distance<TF> {  // dg/capsule_distance.hpp
  CapsuleDistance(TF radius, TF height) {
    this->shape = AL_SHAPE_CAPSULE;
    this->params[0] = radius;
    this->params[1] = height;
    const TF hh = height * TF(0.5);
    this->aabb_min = {-radius, -hh - radius, -radius};
    this->aabb_max = {radius, hh + radius, radius};
    this->max_distance = hh + radius;
  }
};
template <class TF>
struct InfiniteCylinderDistance : Distance<TF> {  // dg/infinite_cylinder_distance.hpp
  explicit InfiniteCylinderDistance(TF radius) {
    this->shape = AL_SHAPE_INFINITE_CYLINDER;
    this->params[0] = radius;
    this->aabb_min = {-radius, -radius, -radius};
    this->aabb_max = {radius, radius, radius};
    this->max_distance = radius;
  }
};
template <class TF>
struct InfiniteTubeDistance : Distance<TF> {  // dg/infinite_tube_distance.hpp
  InfiniteTubeDistance(TF inner_radius, TF outer_radius, TF aabb_half_length = 0) {
    this->shape = AL_SHAPE_INFINITE_TUBE;
    this->params[0] = inner_radius;
    this->params[1] = outer_radius;
    this->params[2] = aabb_half_length;
    const TF half = aabb_half_length != 0 ? aabb_half_length : outer_radius;
    this->aabb_min = {-outer_radius, -half, -outer_radius};
    this->aabb_max = {outer_radius, half, outer_radius};
    this->max_distance = std::max(half, outer_radius);
  }
};
// TriangleMesh (dg/triangle_mesh.hpp): vertices and faces.
template <class TF>
struct TriangleMesh {
  std::vector<std::array<TF, 3>> vertices;
  std::vector<std::array<uint32_t, 3>> faces;
};
// MeshDistance (dg/mesh_distance.hpp:105-125 for the box and max_distance).
template <class TF>
struct MeshDistance : Distance<TF> {
  TriangleMesh<TF> mesh;
  TF offset;
  explicit MeshDistance(TriangleMesh<TF> m, TF offset_arg = 0)
      : mesh(std::move(m)), offset(offset_arg) {
    if (mesh.vertices.empty() || mesh.faces.empty())
      throw error(AL_ERR_INVALID, "MeshDistance: empty mesh");
    this->shape = AL_SHAPE_MESH;
    TF r2 = 0;
    this->aabb_min = mesh.vertices[0];
    this->aabb_max = mesh.vertices[0];
    for (const auto& v : mesh.vertices) {
      for (int i = 0; i < 3; ++i) {
        this->aabb_min[i] = std::min(this->aabb_min[i], v[i]);
        this->aabb_max[i] = std::max(this->aabb_max[i], v[i]);
      }
      r2 = std::max(r2, v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
    for (int i = 0; i < 3; ++i) {
      this->aabb_min[i] -= offset;
      this->aabb_max[i] += offset;
    }
    this->max_distance = std::sqrt(r2) + offset;
  }
};
}  // namespace dg

// Mesh (mesh.hpp): collision vertices of a pile body (its faces are not
// used by the contact search).
template <class TF>
struct Mesh {
  std::vector<std::array<TF, 3>> vertices;
  std::vector<std::array<uint32_t, 3>> faces;
};

// Runner<TF>: the reference's launcher.  Every launch is the engine's here,
// so it carries no state; its static reductions over variables
// (runner.hpp:4710-4815) run on the device through the metric entries,
// summing in double, and return the real type as the reference does.
template <class TF>
class Runner {
 public:
  // calculate_se: se[offset + i] = |v0 - v1|^2 of element offset + i.
  static void calculate_se(const Variable& v0, const Variable& v1, Variable& se, uint32_t n,
                           uint32_t offset = 0) {
    const uint32_t d = dims_of(v0, v1, n, offset, "Runner::calculate_se");
    if (se.get_type() != numeric_type_of<TF>() || se.get_num_primitives_per_element() != 1 ||
        size_t(offset) + n > se.get_linear_shape())
      throw error(AL_ERR_INVALID, "Runner::calculate_se: se must be a scalar variable of n");
    check(real_se(v0.engine_handle(), at(v0, offset), at(v1, offset), at(se, offset), n, d),
          "Runner::calculate_se");
  }
  static TF calculate_se_weighted(const Variable& v0, const Variable& v1, const Variable& weight,
                                  uint32_t n, uint32_t offset = 0) {
    const uint32_t d = dims_of(v0, v1, n, offset, "Runner::calculate_se_weighted");
    scalar_of(weight, n, offset, "Runner::calculate_se_weighted");
    double r = 0;
    check(real_se_weighted(v0.engine_handle(), at(v0, offset), at(v1, offset),
                           at(weight, offset), n, d, &r),
          "Runner::calculate_se_weighted");
    return TF(r);
  }
  static TF calculate_se_yz_masked(const Variable& v0, const Variable& v1, const Variable& mask,
                                   uint32_t n, uint32_t offset = 0) {
    if (dims_of(v0, v1, n, offset, "Runner::calculate_se_yz_masked") != 3)
      throw error(AL_ERR_INVALID, "Runner::calculate_se_yz_masked: 3-vectors");
    scalar_of(mask, n, offset, "Runner::calculate_se_yz_masked");
    double r = 0;
    check(real_se_yz(v0.engine_handle(), at(v0, offset), at(v1, offset), at(mask, offset), n,
                     &r),
          "Runner::calculate_se_yz_masked");
    return TF(r);
  }
  // sum_products: the component-wise sum of v0 v1 (one value per primitive).
  static std::vector<TF> sum_products(const Variable& v0, const Variable& v1, uint32_t n,
                                      uint32_t offset = 0) {
    const uint32_t d = dims_of(v0, v1, n, offset, "Runner::sum_products");
    double r[4] = {0, 0, 0, 0};
    check(real_sum_products(v0.engine_handle(), at(v0, offset), at(v1, offset), n, d, r),
          "Runner::sum_products");
    return std::vector<TF>(r, r + d);
  }
  // calculate_kl_divergence (runner.hpp:4803-4815) of two uint32 histograms.
  static TF calculate_kl_divergence(const Variable& p, const Variable& q, uint32_t n_p,
                                    uint32_t n_q, TF q_lower_bound = TF(1e-6),
                                    uint32_t num_bins = 256) {
    if (p.get_type() != NumericType::u32 || q.get_type() != NumericType::u32 ||
        p.get_linear_shape() < num_bins || q.get_linear_shape() < num_bins)
      throw error(AL_ERR_INVALID, "Runner::calculate_kl_divergence: uint32 histograms");
    double r = 0;
    check(al_kl_divergence(p.engine_handle(), p.template data<uint32_t>(),
                           q.template data<uint32_t>(), n_p, n_q, double(q_lower_bound),
                           num_bins, &r, nullptr),
          "Runner::calculate_kl_divergence");
    return TF(r);
  }

 private:
  static const TF* at(const Variable& v, uint32_t offset) {
    return v.template data<TF>() + size_t(offset) * v.get_num_primitives_per_element();
  }
  static TF* at(Variable& v, uint32_t offset) {
    return v.template data<TF>() + size_t(offset) * v.get_num_primitives_per_element();
  }
  static uint32_t dims_of(const Variable& a, const Variable& b, uint32_t n, uint32_t offset,
                          const char* where) {
    const uint32_t d = a.get_num_primitives_per_element();
    if (a.get_type() != numeric_type_of<TF>() || b.get_type() != numeric_type_of<TF>() ||
        b.get_num_primitives_per_element() != d || d < 1 || d > 4 ||
        size_t(offset) + n > a.get_linear_shape() || size_t(offset) + n > b.get_linear_shape())
      throw error(AL_ERR_INVALID, std::string(where) + ": mismatched variables");
    return d;
  }
  static void scalar_of(const Variable& v, uint32_t n, uint32_t offset, const char* where) {
    if (v.get_type() != numeric_type_of<TF>() || v.get_num_primitives_per_element() != 1 ||
        size_t(offset) + n > v.get_linear_shape())
      throw error(AL_ERR_INVALID, std::string(where) + ": a scalar variable of n");
  }
  static int real_se(al_engine* e, const TF* a, const TF* b, TF* se, uint32_t n, uint32_t d) {
    if constexpr (std::is_same_v<TF, float>) return al_calculate_se_f32(e, a, b, se, n, d, nullptr);
    else return al_calculate_se_f64(e, a, b, se, n, d, nullptr);
  }
  static int real_se_weighted(al_engine* e, const TF* a, const TF* b, const TF* w, uint32_t n,
                              uint32_t d, double* r) {
    if constexpr (std::is_same_v<TF, float>)
      return al_calculate_se_weighted_f32(e, a, b, w, n, d, r, nullptr);
    else
      return al_calculate_se_weighted_f64(e, a, b, w, n, d, r, nullptr);
  }
  static int real_se_yz(al_engine* e, const TF* a, const TF* b, const TF* m, uint32_t n,
                        double* r) {
    if constexpr (std::is_same_v<TF, float>)
      return al_calculate_se_yz_masked_f32(e, a, b, m, n, r, nullptr);
    else
      return al_calculate_se_yz_masked_f64(e, a, b, m, n, r, nullptr);
  }
  static int real_sum_products(al_engine* e, const TF* a, const TF* b, uint32_t n, uint32_t d,
                               double* r) {
    if constexpr (std::is_same_v<TF, float>) return al_sum_products_f32(e, a, b, n, d, r, nullptr);
    else return al_sum_products_f64(e, a, b, n, d, r, nullptr);
  }
};

enum class VolumeMethod { volume_map = 0, pellets = 1 };

// Pile<TF> (pile.hpp): the rigid bodies, their grids and kinematics.
template <class TF>
class Pile {
 public:
  using T3 = std::array<TF, 3>;
  using TQ = std::array<TF, 4>;
  using Body = typename real<TF>::body;
  using Rigid = typename real<TF>::rigid;

  Pile(Store& store, Runner<TF>& runner, uint32_t max_num_contacts,
       VolumeMethod volume_method = VolumeMethod::volume_map, uint32_t max_num_pellets = 10000,
       const Const<TF>* cn = nullptr, const ConstiN* cni = nullptr)
      : max_num_contacts_(max_num_contacts),
        max_num_pellets_(volume_method == VolumeMethod::pellets ? max_num_pellets : 0),
        volume_method_(volume_method),
        store_(store),
        runner_(runner),
        cn_(cn ? cn : &store.get_cn<TF>()),
        cni_(cni ? cni : &store.get_cni()) {}
  Pile(const Pile&) = delete;
  Pile& operator=(const Pile&) = delete;
  ~Pile() {
    for (Variable* v : distance_grids_)
      if (v) store_.remove(*v);
    for (Variable* v : volume_grids_)
      if (v) store_.remove(*v);
    if (pellet_x_) store_.remove(*pellet_x_);
  }

  // Pile::add (pile.hpp:217-284, 285-349): grid domain and resolution by
  // calculate_domain_and_resolution (pile.hpp:40-65), the mesh distance
  // grid on the device, the volume map on the device.  Returns the index.
  uint32_t add(std::shared_ptr<dg::Distance<TF>> distance,
               std::array<uint32_t, 3> resolution = {0, 0, 0}, TF cell_width = 0,
               TF margin = std::numeric_limits<TF>::infinity(), TF sign = 1,
               const Mesh<TF>& collision_mesh = Mesh<TF>(), TF mass = 0, TF restitution = 1,
               TF friction = 0, T3 inertia_tensor = {1, 1, 1}, T3 x = {0, 0, 0},
               TQ q = {0, 0, 0, 1}) {
    return add_impl(std::move(distance), resolution, cell_width, margin, sign,
                    collision_mesh.vertices, {}, mass, restitution, friction, inertia_tensor, x,
                    q);
  }
  // The pellet overload (pile.hpp:217-284): with VolumeMethod::pellets the
  // body-frame pellets are the body's boundary particles and its collision
  // vertices; the pile's pellet count may not pass max_num_pellets.
  uint32_t add(std::shared_ptr<dg::Distance<TF>> distance, std::array<uint32_t, 3> resolution,
               TF cell_width, TF margin, TF sign, const std::vector<T3>& pellets, TF mass = 0,
               TF restitution = 1, TF friction = 0, T3 inertia_tensor = {1, 1, 1},
               T3 x = {0, 0, 0}, TQ q = {0, 0, 0, 1}) {
    if (volume_method_ != VolumeMethod::pellets && !pellets.empty())
      throw error(AL_ERR_INVALID, "Pile::add: pellets need VolumeMethod::pellets");
    if (num_pellets_ + pellets.size() > max_num_pellets_)
      throw error(AL_ERR_INVALID, "Pile::add: the pellet count " +
                                      std::to_string(num_pellets_ + pellets.size()) +
                                      " exceeds the limit " + std::to_string(max_num_pellets_));
    return add_impl(std::move(distance), resolution, cell_width, margin, sign, pellets, pellets,
                    mass, restitution, friction, inertia_tensor, x, q);
  }

 private:
  uint32_t add_impl(std::shared_ptr<dg::Distance<TF>> distance,
                    std::array<uint32_t, 3> resolution, TF cell_width, TF margin, TF sign,
                    const std::vector<T3>& collision_vertices, const std::vector<T3>& pellets,
                    TF mass, TF restitution, TF friction, T3 inertia_tensor, T3 x, TQ q) {
    if (!distance) throw error(AL_ERR_INVALID, "Pile::add: distance is null");
    if (get_size() >= AL_MAX_BOUNDARIES)
      throw error(AL_ERR_UNSUPPORTED, "Pile::add: at most AL_MAX_BOUNDARIES bodies");
    const uint32_t i = get_size();
    distance_list_.push_back(distance);
    mass_.push_back(mass);
    restitution_.push_back(restitution);
    friction_.push_back(friction);
    inertia_tensor_.push_back(inertia_tensor);
    x_.push_back(x);
    v_.push_back({0, 0, 0});
    q_.push_back(q);
    omega_.push_back({0, 0, 0});
    force_.push_back({0, 0, 0});
    torque_.push_back({0, 0, 0});
    sign_list_.push_back(sign);
    collision_vertex_list_.push_back(collision_vertices);
    pellet_list_.push_back(pellets);
    num_pellets_ += static_cast<uint32_t>(pellets.size());
    pellets_dirty_ = true;
    // calculate_domain_and_resolution
    if (std::isinf(margin)) margin = sign < 0 ? cn_->kernel_radius : cn_->kernel_radius * 2;
    T3 dmin, dmax;
    for (int k = 0; k < 3; ++k) {
      dmin[k] = distance->aabb_min[k] - margin;
      dmax[k] = distance->aabb_max[k] + margin;
    }
    if (resolution[0] == 0 || resolution[1] == 0 || resolution[2] == 0) {
      if (cell_width == 0) cell_width = cn_->particle_radius;
      for (int k = 0; k < 3; ++k)
        if (resolution[k] == 0) resolution[k] = static_cast<uint32_t>((dmax[k] - dmin[k]) / cell_width);
    }
    domain_min_list_.push_back(dmin);
    domain_max_list_.push_back(dmax);
    resolution_list_.push_back(resolution);
    distance_grids_.push_back(nullptr);
    volume_grids_.push_back(nullptr);
    grid_size_list_.push_back(0);
    cell_size_list_.push_back({0, 0, 0});
    build_grid(i);
    return i;
  }

 public:
  // The reference's add(Distance*): the pile takes ownership.
  template <class... A>
  uint32_t add(dg::Distance<TF>* distance, A&&... rest) {
    return add(std::shared_ptr<dg::Distance<TF>>(distance), std::forward<A>(rest)...);
  }
  uint32_t get_size() const { return static_cast<uint32_t>(distance_list_.size()); }
  void set_gravity(T3 g) { gravity_ = g; }
  const T3& gravity() const { return gravity_; }
  // Kinematics travel by value with each step.
  void copy_kinematics_to_device() {}
  // Pile::write_file / read_file / get_size_from_file (pile.hpp:757-793):
  // per body x, v, q, omega of the real type; x, v and omega scaled on
  // writing.
  void write_file(const std::string& filename, TF x_scale = 1, TF v_scale = 1,
                  TF omega_scale = 1) const {
    std::ofstream f(filename, std::ios::binary | std::ios::trunc);
    if (!f) throw error(AL_ERR_INVALID, "Pile::write_file: cannot open " + filename);
    for (uint32_t i = 0; i < get_size(); ++i) {
      TF rec[13];
      for (int k = 0; k < 3; ++k) {
        rec[k] = x_[i][k] * x_scale;
        rec[3 + k] = v_[i][k] * v_scale;
        rec[10 + k] = omega_[i][k] * omega_scale;
      }
      for (int k = 0; k < 4; ++k) rec[6 + k] = q_[i][k];
      f.write(reinterpret_cast<const char*>(rec), sizeof(rec));
    }
  }
  void read_file(const std::string& filename, int num_rigids = -1, uint32_t dst_offset = 0,
                 uint32_t src_offset = 0) {
    std::ifstream f(filename, std::ios::binary);
    uint32_t n = get_size();
    if (num_rigids >= 0) n = std::min(n, uint32_t(num_rigids));
    f.seekg(std::streamoff(13 * sizeof(TF)) * src_offset, std::ios_base::cur);
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t d = dst_offset + i;
      if (d >= get_size()) throw error(AL_ERR_INVALID, "Pile::read_file: past the last body");
      TF rec[13];
      f.read(reinterpret_cast<char*>(rec), sizeof(rec));
      for (int k = 0; k < 3; ++k) {
        x_[d][k] = rec[k];
        v_[d][k] = rec[3 + k];
        omega_[d][k] = rec[10 + k];
      }
      for (int k = 0; k < 4; ++k) q_[d][k] = rec[6 + k];
      if (f.peek() == std::ifstream::traits_type::eof()) break;
    }
  }
  static uint32_t get_size_from_file(const std::string& filename) {
    std::ifstream f(filename, std::ifstream::ate | std::ifstream::binary);
    return f ? uint32_t(f.tellg() / std::streamoff(13 * sizeof(TF))) : 0u;
  }
  const std::vector<Variable*>& get_distance_grids() const { return distance_grids_; }
  const std::vector<Variable*>& get_volume_grids() const { return volume_grids_; }

  // The engine's body table and kinematic state.
  std::vector<Body> bodies() const {
    std::vector<Body> out(get_size());
    for (uint32_t i = 0; i < get_size(); ++i) {
      Body& b = out[i];
      std::memset(&b, 0, sizeof(Body));
      const dg::Distance<TF>& d = *distance_list_[i];
      b.shape = d.shape;
      b.use_distance_grid = d.shape == AL_SHAPE_MESH ? 1u : 0u;
      b.sign = sign_list_[i];
      for (int k = 0; k < 8; ++k) b.shape_params[k] = d.params[k];
      for (int k = 0; k < 3; ++k) {
        b.domain_min[k] = domain_min_list_[i][k];
        b.domain_max[k] = domain_max_list_[i][k];
        b.cell_size[k] = cell_size_list_[i][k];
        b.resolution[k] = resolution_list_[i][k];
        b.inertia[k] = inertia_tensor_[i][k];
      }
      b.num_nodes = grid_size_list_[i];
      b.distance_nodes = distance_grids_[i] ? distance_grids_[i]->template data<TF>() : nullptr;
      b.volume_nodes = volume_grids_[i] ? volume_grids_[i]->template data<TF>() : nullptr;
      b.max_distance = d.max_distance;
      b.mass = mass_[i];
    }
    return out;
  }
  std::vector<Rigid> rigid() const {
    std::vector<Rigid> out(get_size());
    for (uint32_t i = 0; i < get_size(); ++i) {
      for (int k = 0; k < 3; ++k) {
        out[i].x[k] = x_[i][k];
        out[i].v[k] = v_[i][k];
        out[i].omega[k] = omega_[i][k];
      }
      for (int k = 0; k < 4; ++k) out[i].q[k] = q_[i][k];
    }
    return out;
  }
  void set_rigid(const std::vector<Rigid>& r) {
    for (uint32_t i = 0; i < get_size() && i < r.size(); ++i) {
      for (int k = 0; k < 3; ++k) {
        x_[i][k] = r[i].x[k];
        v_[i][k] = r[i].v[k];
        omega_[i][k] = r[i].omega[k];
      }
      for (int k = 0; k < 4; ++k) q_[i][k] = r[i].q[k];
    }
  }
  // Body-frame pellets of every body, body after body, on the device (the
  // reference's concatenated pellet buffer), and each body's count.
  const Variable* local_pellets() {
    if (pellets_dirty_) {
      if (pellet_x_) store_.remove(*pellet_x_);
      pellet_x_ = nullptr;
      if (num_pellets_) {
        std::vector<T3> all;
        all.reserve(num_pellets_);
        for (const auto& p : pellet_list_) all.insert(all.end(), p.begin(), p.end());
        pellet_x_ = store_.create<TF>({num_pellets_}, 3);
        pellet_x_->set_bytes(all.data(), all.size() * sizeof(T3));
      }
      pellets_dirty_ = false;
    }
    return pellet_x_;
  }
  uint32_t num_pellets() const { return num_pellets_; }
  bool pellet_mode() const { return volume_method_ == VolumeMethod::pellets; }
  bool has_collision_vertices() const {
    for (const auto& c : collision_vertex_list_)
      if (!c.empty()) return true;
    return false;
  }

  // Kinematic fields (pile.hpp:98-121), public as the reference binds them.
  std::vector<TF> mass_, restitution_, friction_, sign_list_;
  std::vector<T3> x_, v_, omega_, inertia_tensor_, force_, torque_;
  std::vector<TQ> q_;
  std::vector<T3> domain_min_list_, domain_max_list_, cell_size_list_;
  std::vector<std::array<uint32_t, 3>> resolution_list_;
  std::vector<uint32_t> grid_size_list_;
  std::vector<std::vector<std::array<TF, 3>>> collision_vertex_list_;
  std::vector<std::vector<std::array<TF, 3>>> pellet_list_;
  uint32_t max_num_contacts_;
  uint32_t max_num_pellets_;
  VolumeMethod volume_method_;

 private:
  // Pile::build_grid (pile.hpp:497-622) with calculate_grid_attributes
  // (pile.hpp:66-78).
  void build_grid(uint32_t i) {
    const auto& res = resolution_list_[i];
    for (int k = 0; k < 3; ++k) {
      if (res[k] == 0) throw error(AL_ERR_INVALID, "Pile::add: zero grid resolution");
      cell_size_list_[i][k] = (domain_max_list_[i][k] - domain_min_list_[i][k]) / TF(res[k]);
    }
    const uint32_t nv = (res[0] + 1) * (res[1] + 1) * (res[2] + 1);
    const uint32_t ne = res[0] * (res[1] + 1) * (res[2] + 1) +
                        (res[0] + 1) * res[1] * (res[2] + 1) +
                        (res[0] + 1) * (res[1] + 1) * res[2];
    grid_size_list_[i] = nv + 2 * ne;
    const dg::Distance<TF>& d = *distance_list_[i];
    if (d.shape == AL_SHAPE_MESH) {
      if constexpr (!std::is_same_v<TF, float>) {
        throw error(AL_ERR_UNSUPPORTED, "Pile::add: mesh distance grids are float32");
      } else {
        const auto& md = static_cast<const dg::MeshDistance<TF>&>(d);
        distance_grids_[i] = store_.create<TF>({grid_size_list_[i]});
        const Body b = bodies()[i];
        check(al_build_mesh_distance_grid_f32(
                  store_.eng(), &b, md.mesh.vertices.front().data(),
                  static_cast<uint32_t>(md.mesh.vertices.size()), md.mesh.faces.front().data(),
                  static_cast<uint32_t>(md.mesh.faces.size()), md.offset,
                  distance_grids_[i]->template data<TF>(), nullptr),
              "Pile::add (mesh distance grid)");
      }
    }
    if (volume_method_ != VolumeMethod::volume_map) return;  // pellets need no volume map
    volume_grids_[i] = store_.create<TF>({grid_size_list_[i]});
    const Body b = bodies()[i];
    check(real<TF>::build_volume_field(store_.eng(), cn_->c(), &b,
                                       volume_grids_[i]->template data<TF>(), nullptr),
          "Pile::add (volume map)");
  }

  Store& store_;
  Runner<TF>& runner_;
  const Const<TF>* cn_;
  const ConstiN* cni_;
  std::vector<std::shared_ptr<dg::Distance<TF>>> distance_list_;
  std::vector<Variable*> distance_grids_, volume_grids_;
  T3 gravity_{0, 0, 0};
  uint32_t num_pellets_ = 0;
  bool pellets_dirty_ = false;
  Variable* pellet_x_ = nullptr;
};

// Solver<TF> (solver.hpp): particle buffers, time stepping fields, the
// neighbor update and the boundary sampling.
template <class TF>
class Solver {
 public:
  using T3 = std::array<TF, 3>;

  Solver(Runner<TF>& runner, Pile<TF>& pile, Store& store, uint32_t max_num_particles,
         uint32_t num_ushers = 0, bool enable_surface_tension = false,
         bool enable_vorticity = false, const Const<TF>* cn = nullptr,
         const ConstiN* cni = nullptr, bool graphical = false)
      : max_num_particles(max_num_particles),
        store(store),
        runner(runner),
        pile(pile),
        cn_(cn ? cn : &store.get_cn<TF>()),
        cni_(cni ? cni : &store.get_cni()) {
    if (num_ushers != 0 || enable_surface_tension || enable_vorticity || graphical)
      throw error(AL_ERR_UNSUPPORTED,
                  "Solver: ushers, surface tension, vorticity and graphical buffers are outside "
                  "the engine's scope");
    particle_radius = cn_->particle_radius;
    const uint32_t n = max_num_particles, nb = std::max<uint32_t>(pile.get_size(), 1);
    // the pellets' world positions and velocities follow the particles
    // (solver.hpp:30-36)
    particle_x = store.create<TF>({n + pile.max_num_pellets_}, 3);
    particle_v = store.create<TF>({n + pile.max_num_pellets_}, 3);
    particle_a = store.create<TF>({n}, 3);
    particle_density = store.create<TF>({n});
    particle_boundary = store.create<TF>({nb, n}, 4);
    particle_boundary_kernel = store.create<TF>({nb, n}, 4);
    particle_neighbors = store.create<TF>({n, cni_->max_num_neighbors_per_particle}, 4);
    particle_num_neighbors = store.create<uint32_t>({n});
    grid_anomaly = store.create<uint32_t>({3});
  }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;
  virtual ~Solver() {
    for (Variable* v : {particle_x, particle_v, particle_a, particle_density, particle_boundary,
                        particle_boundary_kernel, particle_neighbors, particle_num_neighbors,
                        grid_anomaly})
      store.remove(*v);
  }

  virtual void reset_solving_var() {}
  virtual void reset_t() {
    t = 0;
    dt = initial_dt;
  }
  // Solver::compute_all_boundaries (solver.hpp:170-185).  Rows of
  // particle_boundary / particle_boundary_kernel are num_particles long:
  // body b's entries start at b * num_particles (the reference indexes them
  // with the variable's max_num_particles stride; the two agree while
  // num_particles == max_num_particles, and update_particle_neighbors and
  // the steps read the rows with the same num_particles stride).
  void compute_all_boundaries() {
    check_counts();
    const auto bodies = pile.bodies();
    const auto rig = pile.rigid();
    check(real<TF>::compute_particle_boundary(
              store.eng(), cn_->c(), pile.get_size(), bodies.data(), rig.data(),
              particle_x->template data<TF>(), num_particles,
              particle_boundary->template data<TF>(),
              particle_boundary_kernel->template data<TF>(), nullptr),
          "Solver::compute_all_boundaries");
  }
  // Solver::sample_all_boundaries (solver.hpp:186-203): the bodies' volume
  // and kernel terms at sample points, in the particle_boundary layout
  // ([num_bodies][num_samples] x 4).
  void sample_all_boundaries(const Variable& sample_x, Variable& sample_boundary,
                             Variable& sample_boundary_kernel, uint32_t num_samples) {
    const size_t need = size_t(pile.get_size()) * num_samples * 4;
    if (sample_x.get_linear_shape() < num_samples ||
        sample_boundary.get_num_primitives() < need ||
        sample_boundary_kernel.get_num_primitives() < need)
      throw error(AL_ERR_INVALID, "Solver::sample_all_boundaries: variables too small");
    // the rows are written num_samples apart; a [num_bodies][capacity]
    // variable with capacity != num_samples would be indexed with another
    // stride by the reference's Variable<2> (variable.hpp:281-290)
    for (const Variable* v : {&sample_boundary, &sample_boundary_kernel}) {
      const auto& sh = v->get_shape();
      if (sh.size() == 2 && sh[1] != num_samples)
        throw error(AL_ERR_INVALID,
                    "Solver::sample_all_boundaries: sample_boundary variables must have shape "
                    "[num_bodies][num_samples]");
    }
    const auto bodies = pile.bodies();
    const auto rig = pile.rigid();
    check(real<TF>::compute_particle_boundary(
              store.eng(), cn_->c(), pile.get_size(), bodies.data(), rig.data(),
              sample_x.template data<TF>(), num_samples,
              sample_boundary.template data<TF>(), sample_boundary_kernel.template data<TF>(),
              nullptr),
          "Solver::sample_all_boundaries");
  }
  // Solver::update_particle_neighbors<wrap> (solver.hpp:225-260): grid,
  // neighbor list in the reference layout and the density with the
  // boundary terms of the last compute_all_boundaries.
  template <uint32_t wrap>
  void update_particle_neighbors() {
    check_counts();
    ConstiN ci = *cni_;
    ci.num_boundaries = pile.get_size();
    int st;
    if constexpr (wrap == 0) {
      st = real<TF>::update_particle_neighbors(
          store.eng(), cn_->c(), &ci, particle_x->template data<TF>(), num_particles,
          pile.get_size() ? particle_boundary_kernel->template data<TF>() : nullptr,
          particle_density->template data<TF>(), particle_num_neighbors->template data<uint32_t>(),
          particle_neighbors->template data<TF>(), grid_anomaly->template data<uint32_t>(),
          nullptr);
    } else {
      st = real<TF>::update_particle_neighbors_periodic(
          store.eng(), cn_->c(), &ci, particle_x->template data<TF>(), num_particles,
          pile.get_size() ? particle_boundary_kernel->template data<TF>() : nullptr,
          particle_density->template data<TF>(), particle_num_neighbors->template data<uint32_t>(),
          particle_neighbors->template data<TF>(), grid_anomaly->template data<uint32_t>(),
          double(cn_->wrap_length), nullptr);
    }
    check(st, "Solver::update_particle_neighbors");
  }

  uint32_t max_num_particles;
  uint32_t num_particles = 0;
  TF t = 0, dt = 0, initial_dt = 0, max_dt = 0, min_dt = 0, cfl = 0, particle_radius = 0;
  TF particle_max_v2 = 0, pile_max_v2 = 0, max_v2 = 0, cfl_dt = 0, utilized_cfl = 0;
  Store& store;
  Runner<TF>& runner;
  Pile<TF>& pile;
  Variable *particle_x, *particle_v, *particle_a, *particle_density, *particle_boundary,
      *particle_boundary_kernel, *particle_neighbors, *particle_num_neighbors, *grid_anomaly;
  // The last step's anomaly status (AL_OK or one of the grid anomalies,
  // which the reference reports through grid_anomaly without throwing).
  int last_status = AL_OK;

 protected:
  void check_counts() const {
    if (num_particles > max_num_particles)
      throw error(AL_ERR_INVALID, "Solver: num_particles exceeds max_num_particles");
  }
  al_solver_params base_params(uint32_t wrap) const {
    al_solver_params p;
    std::memset(&p, 0, sizeof(p));
    p.cfl = cfl;
    p.max_dt = max_dt;
    p.min_dt = min_dt;
    for (int k = 0; k < 3; ++k) p.pile_gravity[k] = pile.gravity()[k];
    p.integrate_rigids = 1;
    p.wrap_y = wrap;
    p.wrap_length = double(cn_->wrap_length);
    return p;
  }
  typename real<TF>::fluid fluid_table(TF* dfsph_factor, TF* kappa, TF* kappa_v,
                                      TF* density_adv, TF* pressure) const {
    typename real<TF>::fluid f;
    std::memset(&f, 0, sizeof(f));
    f.num_particles = num_particles;
    f.particle_x = particle_x->template data<TF>();
    f.particle_v = particle_v->template data<TF>();
    f.particle_a = particle_a->template data<TF>();
    f.particle_density = particle_density->template data<TF>();
    f.particle_dfsph_factor = dfsph_factor;
    f.particle_kappa = kappa;
    f.particle_kappa_v = kappa_v;
    f.particle_density_adv = density_adv;
    f.particle_pressure = pressure;
    if (pile.get_size()) {
      f.particle_boundary = particle_boundary->template data<TF>();
      f.particle_boundary_kernel = particle_boundary_kernel->template data<TF>();
    }
    return f;
  }
  // Runs one engine step: dt in/out, t += dt, rigid state and per-body
  // totals written back, the step's grid anomalies copied into
  // grid_anomaly, contacts between collision meshes found and solved.
  template <class Fn>
  al_step_report run_step(Fn&& fn, const al_solver_params& p, const char* where) {
    check_counts();
    ConstiN ci = *cni_;
    ci.num_boundaries = pile.get_size();
    auto bodies = pile.bodies();
    auto rig = pile.rigid();
    al_step_report rep;
    std::memset(&rep, 0, sizeof(rep));
    TF d = dt;
    const int st = fn(store.eng(), cn_->c(), &ci, bodies.empty() ? nullptr : bodies.data(),
                      rig.empty() ? nullptr : rig.data(), &p, &d, &rep);
    check(st, where);
    last_status = st;
    dt = d;
    particle_max_v2 = TF(rep.particle_max_v2);
    pile_max_v2 = TF(rep.pile_max_v2);
    max_v2 = TF(rep.max_v2);
    cfl_dt = TF(rep.cfl_dt);
    utilized_cfl = TF(rep.utilized_cfl);
    grid_anomaly->set_bytes(rep.grid_anomaly, sizeof(rep.grid_anomaly));
    pile.set_rigid(rig);
    for (uint32_t b = 0; b < pile.get_size(); ++b)
      for (int k = 0; k < 3; ++k) {
        pile.force_[b][k] = TF(rep.force[b][k]);
        pile.torque_[b][k] = TF(rep.torque[b][k]);
      }
    solve_contacts();
    t += dt;
    return rep;
  }
  // pile.find_contacts + pile.solve_contacts (solver_df.hpp:356-357) for
  // bodies with collision vertices (float32).
  void solve_contacts() {
    if (!pile.has_collision_vertices() || pile.max_num_contacts_ == 0) return;
    if constexpr (!std::is_same_v<TF, float>) {
      throw error(AL_ERR_UNSUPPORTED, "Pile contacts are float32");
    } else {
      const uint32_t nb = pile.get_size();
      std::vector<Variable*> verts(nb, nullptr);
      std::vector<al_contact_body_f32> cb(nb);
      for (uint32_t b = 0; b < nb; ++b) {
        const auto& cv = pile.collision_vertex_list_[b];
        std::memset(&cb[b], 0, sizeof(cb[b]));
        if (!cv.empty()) {
          verts[b] = store.create<float>({uint32_t(cv.size())}, 3);
          verts[b]->set_bytes(cv.front().data(), cv.size() * 3 * sizeof(float));
          cb[b].vertices = verts[b]->template data<float>();
          cb[b].num_vertices = uint32_t(cv.size());
        }
        cb[b].restitution = pile.restitution_[b];
        cb[b].friction = pile.friction_[b];
      }
      Variable* contacts = store.create<uint32_t>(
          {pile.max_num_contacts_}, uint32_t(sizeof(al_contact_f32) / 4));
      auto bodies = pile.bodies();
      auto rig = pile.rigid();
      uint32_t found = 0;
      int st = al_find_contacts_f32(store.eng(), bodies.data(), rig.data(), cb.data(), nb,
                                    cn_->contact_tolerance, pile.max_num_contacts_,
                                    static_cast<al_contact_f32*>(contacts->ptr()), &found,
                                    nullptr);
      if (st == AL_OK && found)
        st = al_solve_contacts_f32(store.eng(), bodies.data(), rig.data(), nb,
                                   static_cast<al_contact_f32*>(contacts->ptr()),
                                   std::min(found, pile.max_num_contacts_), nullptr);
      for (Variable* v : verts)
        if (v) store.remove(*v);
      store.remove(*contacts);
      check(st, "Pile::find_contacts / solve_contacts");
      pile.set_rigid(rig);
    }
  }

  const Const<TF>* cn_;
  const ConstiN* cni_;
};

// SolverDf<TF> (solver_df.hpp): DFSPH.
template <class TF>
class SolverDf : public Solver<TF> {
 public:
  using Base = Solver<TF>;
  SolverDf(Runner<TF>& runner, Pile<TF>& pile, Store& store, uint32_t max_num_particles,
           uint32_t num_ushers = 0, bool enable_surface_tension = false,
           bool enable_vorticity = false, const Const<TF>* cn = nullptr,
           const ConstiN* cni = nullptr, bool graphical = false)
      : Base(runner, pile, store, max_num_particles, num_ushers, enable_surface_tension,
             enable_vorticity, cn, cni, graphical) {
    particle_dfsph_factor = store.create<TF>({max_num_particles});
    particle_kappa = store.create<TF>({max_num_particles});
    particle_kappa_v = store.create<TF>({max_num_particles});
    particle_density_adv = store.create<TF>({max_num_particles});
  }
  ~SolverDf() override {
    for (Variable* v : {particle_dfsph_factor, particle_kappa, particle_kappa_v,
                        particle_density_adv})
      this->store.remove(*v);
  }
  // SolverDf::step<wrap> (solver_df.hpp:74-359).
  template <uint32_t wrap>
  void step() {
    if (this->pile.pellet_mode())
      throw error(AL_ERR_UNSUPPORTED, "SolverDf::step: pellet piles step with SolverI");
    al_solver_params p = this->base_params(wrap);
    p.density_change_tolerance = density_change_tolerance;
    p.density_error_tolerance = density_error_tolerance;
    p.min_density_solve = min_density_solve;
    p.max_density_solve = max_density_solve;
    p.min_divergence_solve = min_divergence_solve;
    p.max_divergence_solve = max_divergence_solve;
    p.enable_divergence_solve = enable_divergence_solve;
    p.enable_density_solve = enable_density_solve;
    const auto f = this->fluid_table(
        particle_dfsph_factor->template data<TF>(), particle_kappa->template data<TF>(),
        particle_kappa_v->template data<TF>(), particle_density_adv->template data<TF>(), nullptr);
    const al_step_report rep = this->run_step(
        [&](al_engine* e, auto* cn, auto* ci, auto* b, auto* r, auto* pp, TF* d, auto* rp) {
          return real<TF>::df_step(e, cn, ci, &f, b, r, pp, d, rp, nullptr);
        },
        p, "SolverDf::step");
    num_divergence_solve = rep.num_divergence_solve;
    num_density_solve = rep.num_density_solve;
    mean_density_change = TF(rep.mean_density_change);
    mean_density_error = TF(rep.mean_density_error);
  }
  void reset_solving_var() override {
    particle_kappa->set_zero();
    particle_kappa_v->set_zero();
  }

  uint32_t num_divergence_solve = 0, num_density_solve = 0;
  TF mean_density_change = 0, mean_density_error = 0;
  bool enable_divergence_solve = true, enable_density_solve = true;
  TF density_change_tolerance = TF(1e-3), density_error_tolerance = TF(1e-3);
  uint32_t min_density_solve = 2, max_density_solve = 100;
  uint32_t min_divergence_solve = 1, max_divergence_solve = 100;
  Variable *particle_dfsph_factor, *particle_kappa, *particle_kappa_v, *particle_density_adv;
};

// The pressure solvers SolverIi (solver_ii.hpp, IISPH) and SolverI
// (solver_i.hpp, implicit SPH with damped Jacobi): one pressure field.
template <class TF, bool Implicit>
class SolverPressure : public Solver<TF> {
 public:
  using Base = Solver<TF>;
  SolverPressure(Runner<TF>& runner, Pile<TF>& pile, Store& store, uint32_t max_num_particles,
                 uint32_t num_ushers = 0, bool enable_surface_tension = false,
                 bool enable_vorticity = false, const Const<TF>* cn = nullptr,
                 const ConstiN* cni = nullptr, bool graphical = false)
      : Base(runner, pile, store, max_num_particles, num_ushers, enable_surface_tension,
             enable_vorticity, cn, cni, graphical) {
    particle_pressure = store.create<TF>({max_num_particles + pile.max_num_pellets_});
    particle_adv_density = store.create<TF>({max_num_particles});
  }
  ~SolverPressure() override {
    this->store.remove(*particle_pressure);
    this->store.remove(*particle_adv_density);
  }
  // SolverIi::step<wrap> (solver_ii.hpp:76-243) / SolverI::step<wrap>
  // (solver_i.hpp) on the volume-map branch.
  template <uint32_t wrap>
  void step() {
    al_solver_params p = this->base_params(wrap);
    p.density_error_tolerance = density_error_tolerance;
    p.min_density_solve = min_density_solve;
    p.max_density_solve = max_density_solve;
    p.enable_density_solve = 1;
    auto f = this->fluid_table(nullptr, nullptr, nullptr,
                               particle_adv_density->template data<TF>(),
                               particle_pressure->template data<TF>());
    al_step_report rep;
    if (this->pile.pellet_mode()) {
      if (!Implicit)
        throw error(AL_ERR_UNSUPPORTED, "SolverIi::step: pellet piles step with SolverI");
      // the pellet branch of SolverI::step (solver_i.hpp:79-327): pellet
      // world positions, velocities and pressures land after the particles
      f.particle_boundary = nullptr;
      f.particle_boundary_kernel = nullptr;
      typename real<TF>::pellets pel;
      std::memset(&pel, 0, sizeof(pel));
      const Variable* lp = this->pile.local_pellets();
      const uint32_t n = this->num_particles;
      pel.local_x = lp ? lp->template data<TF>() : nullptr;
      pel.num_pellets = this->pile.num_pellets();
      for (uint32_t b = 0; b < this->pile.get_size(); ++b)
        pel.count[b] = uint32_t(this->pile.pellet_list_[b].size());
      pel.x = this->particle_x->template data<TF>() + size_t(n) * 3;
      pel.v = this->particle_v->template data<TF>() + size_t(n) * 3;
      pel.pressure = particle_pressure->template data<TF>() + n;
      rep = this->run_step(
          [&](al_engine* e, auto* cn, auto* ci, auto* b, auto* r, auto* pp, TF* d, auto* rp) {
            return real<TF>::i_step_pellets(e, cn, ci, &f, b, r, &pel, pp, d, rp, nullptr);
          },
          p, "SolverI::step (pellets)");
    } else {
      rep = this->run_step(
          [&](al_engine* e, auto* cn, auto* ci, auto* b, auto* r, auto* pp, TF* d, auto* rp) {
            return Implicit ? real<TF>::i_step(e, cn, ci, &f, b, r, pp, d, rp, nullptr)
                            : real<TF>::ii_step(e, cn, ci, &f, b, r, pp, d, rp, nullptr);
          },
          p, Implicit ? "SolverI::step" : "SolverIi::step");
    }
    num_density_solve = rep.num_density_solve;
    mean_density_error = TF(rep.mean_density_error);
  }
  void reset_solving_var() override { particle_pressure->set_zero(); }

  uint32_t num_density_solve = 0;
  TF mean_density_error = 0;
  TF density_error_tolerance = TF(1e-3);
  uint32_t min_density_solve = 2, max_density_solve = 100;
  Variable *particle_pressure, *particle_adv_density;
};
template <class TF>
using SolverIi = SolverPressure<TF, false>;
template <class TF>
using SolverI = SolverPressure<TF, true>;

// SolverPellet<TF> (solver_pellet.hpp): spreads pellets inside or around
// the pile's one body by relaxation steps (cohesion / adhesion
// displacement, the pellet DFSPH divergence iteration, a CFL-limited move
// that keeps them off the boundary).  particle_v receives each step's
// displacement and particle_density the pellets' density, as in the
// reference.
template <class TF>
class SolverPellet : public Solver<TF> {
 public:
  using Base = Solver<TF>;
  SolverPellet(Runner<TF>& runner, Pile<TF>& pile, Store& store, uint32_t max_num_particles,
               const Const<TF>* cn = nullptr, const ConstiN* cni = nullptr,
               bool graphical = false)
      : Base(runner, pile, store, max_num_particles, 0, false, false, cn, cni, graphical) {
    particle_dfsph_factor = store.create<TF>({max_num_particles});
  }
  ~SolverPellet() override { this->store.remove(*particle_dfsph_factor); }
  // SolverPellet::set_pellets (solver_pellet.hpp:53-56).
  void set_pellets(const Variable& x) {
    const uint32_t n = x.get_linear_shape();
    if (n > this->max_num_particles)
      throw error(AL_ERR_INVALID, "SolverPellet::set_pellets: more pellets than max_num_particles");
    this->num_particles = n;
    this->particle_x->set_from(x);
  }
  // SolverPellet::step<wrap> (solver_pellet.hpp:57-119).
  template <uint32_t wrap>
  void step() {
    this->check_counts();
    if (this->pile.get_size() != 1)
      throw error(AL_ERR_INVALID, "SolverPellet::step: the pile must hold one body");
    const auto bodies = this->pile.bodies();
    al_pellet_relax_params p;
    std::memset(&p, 0, sizeof(p));
    p.cohesion = cohesion;
    p.adhesion = adhesion;
    p.cfl_factor = cfl_factor;
    p.contact_tolerance = this->cn_->contact_tolerance;
    p.wrap_y = wrap;
    p.wrap_length = double(this->cn_->wrap_length);
    ConstiN ci = *this->cni_;
    ci.num_boundaries = 0;
    check(real<TF>::relax_pellets(this->store.eng(), this->cn_->c(), &ci, bodies.data(),
                                  this->particle_x->template data<TF>(), this->num_particles, &p,
                                  1u, this->particle_v->template data<TF>(),
                                  this->particle_density->template data<TF>(), nullptr),
          "SolverPellet::step");
  }

  TF cohesion = 4, adhesion = 2, cfl_factor = TF(0.25);
  Variable* particle_dfsph_factor;
};

}  // namespace alluvion_b200

#endif /* ALLUVION_B200_SOLVER_HPP */
