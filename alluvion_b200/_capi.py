"""ctypes view of the engine's C ABI (include/alluvion_b200.h).

The structures here mirror the header field for field.  Loading fails
loudly when liballuvion_b200.so is missing: there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "liballuvion_b200.so")

AL_MAX_BOUNDARIES = 16

STATUS = {
    0: "AL_OK", 1: "AL_ERR_CUDA", 2: "AL_ERR_INVALID", 3: "AL_ERR_OUT_OF_GRID",
    4: "AL_ERR_CELL_OVERFLOW", 5: "AL_ERR_NEIGHBOR_OVERFLOW", 6: "AL_ERR_UNSUPPORTED",
    7: "AL_ERR_TIMEOUT", 8: "AL_ERR_NO_DEVICE", 9: "AL_ERR_ALLOC",
}
AL_OK = 0
AL_ERR_INVALID = 2
AL_ERR_OUT_OF_GRID = 3
AL_ERR_CELL_OVERFLOW = 4
AL_ERR_NEIGHBOR_OVERFLOW = 5
ANOMALY_STATUSES = (AL_ERR_OUT_OF_GRID, AL_ERR_CELL_OVERFLOW, AL_ERR_NEIGHBOR_OVERFLOW)

SHAPE_BOX, SHAPE_SPHERE, SHAPE_BOX_SHELL, SHAPE_TORUS, SHAPE_MESH = 0, 1, 2, 3, 4
SHAPE_CYLINDER, SHAPE_CAPSULE, SHAPE_INFINITE_CYLINDER, SHAPE_INFINITE_TUBE = 5, 6, 7, 8


def _const_struct(name, real):
    fields = [(f, real) for f in (
        "kernel_radius", "kernel_radius_sqr", "cubic_kernel_k", "cubic_kernel_l",
        "cubic_kernel_zero", "particle_radius", "particle_vol", "particle_mass", "density0",
        "viscosity", "boundary_viscosity", "dfsph_factor_epsilon")]
    fields.append(("gravity", real * 3))
    return type(name, (ctypes.Structure,), {"_fields_": fields})


ConstF32 = _const_struct("al_const_f32", ctypes.c_float)
ConstF64 = _const_struct("al_const_f64", ctypes.c_double)


class ConstI(ctypes.Structure):
    _fields_ = [("max_num_particles_per_cell", ctypes.c_uint32),
                ("grid_res", ctypes.c_uint32 * 3),
                ("grid_offset", ctypes.c_int32 * 3),
                ("max_num_neighbors_per_particle", ctypes.c_uint32),
                ("num_boundaries", ctypes.c_uint32)]


def _body_struct(name, real):
    return type(name, (ctypes.Structure,), {"_fields_": [
        ("shape", ctypes.c_uint32),
        ("use_distance_grid", ctypes.c_uint32),
        ("sign", real),
        ("shape_params", real * 8),
        ("domain_min", real * 3),
        ("domain_max", real * 3),
        ("cell_size", real * 3),
        ("resolution", ctypes.c_uint32 * 3),
        ("num_nodes", ctypes.c_uint32),
        ("distance_nodes", ctypes.c_void_p),
        ("volume_nodes", ctypes.c_void_p),
        ("max_distance", real),
        ("mass", real),
        ("inertia", real * 3),
    ]})


BodyF32 = _body_struct("al_body_f32", ctypes.c_float)
BodyF64 = _body_struct("al_body_f64", ctypes.c_double)


def _rigid_struct(name, real):
    return type(name, (ctypes.Structure,), {"_fields_": [
        ("x", real * 3), ("v", real * 3), ("q", real * 4), ("omega", real * 3)]})


RigidF32 = _rigid_struct("al_rigid_f32", ctypes.c_float)
RigidF64 = _rigid_struct("al_rigid_f64", ctypes.c_double)


class SolverParams(ctypes.Structure):
    _fields_ = [("density_change_tolerance", ctypes.c_double),
                ("density_error_tolerance", ctypes.c_double),
                ("min_density_solve", ctypes.c_uint32),
                ("max_density_solve", ctypes.c_uint32),
                ("min_divergence_solve", ctypes.c_uint32),
                ("max_divergence_solve", ctypes.c_uint32),
                ("enable_divergence_solve", ctypes.c_uint32),
                ("enable_density_solve", ctypes.c_uint32),
                ("cfl", ctypes.c_double),
                ("max_dt", ctypes.c_double),
                ("min_dt", ctypes.c_double),
                ("pile_gravity", ctypes.c_double * 3),
                ("integrate_rigids", ctypes.c_uint32),
                ("wrap_y", ctypes.c_uint32),
                ("wrap_length", ctypes.c_double)]


WARM_NUM_FEATURES, WARM_HIDDEN, WARM_NUM_OUTPUTS, WARM_NUM_PARAMS = 12, 64, 2, 5122


class WarmNet(ctypes.Structure):
    """al_warm_net: device parameter pointer plus input/output scalings."""
    _fields_ = [("params", ctypes.c_void_p),
                ("feature_shift", ctypes.c_float * WARM_NUM_FEATURES),
                ("feature_scale", ctypes.c_float * WARM_NUM_FEATURES),
                ("output_scale", ctypes.c_float * WARM_NUM_OUTPUTS),
                ("reserved", ctypes.c_uint32 * 2)]


def make_warm_net(params, shift, scale, out_scale):
    """WarmNet over a device tensor of WARM_NUM_PARAMS floats."""
    w = WarmNet()
    w.params = params.data_ptr()
    for k in range(WARM_NUM_FEATURES):
        w.feature_shift[k] = float(shift[k])
        w.feature_scale[k] = float(scale[k])
    for k in range(WARM_NUM_OUTPUTS):
        w.output_scale[k] = float(out_scale[k])
    return w


class WarmStart(ctypes.Structure):
    """al_warm_start: optional network and optional feature output."""
    _fields_ = [("net", ctypes.c_void_p), ("features_out", ctypes.c_void_p)]


class SceneF32(ctypes.Structure):
    """al_scene_f32: one scene of a batched step."""
    _fields_ = [("cn", ctypes.c_void_p), ("cni", ctypes.c_void_p), ("fluid", ctypes.c_void_p),
                ("bodies", ctypes.c_void_p), ("rigid", ctypes.c_void_p),
                ("params", ctypes.c_void_p), ("dt", ctypes.c_void_p), ("report", ctypes.c_void_p),
                ("status", ctypes.c_int), ("reserved", ctypes.c_uint32)]


class ContactBodyF32(ctypes.Structure):
    """al_contact_body_f32: collision vertices (device, body frame) and
    contact coefficients of one body."""
    _fields_ = [("vertices", ctypes.c_void_p), ("num_vertices", ctypes.c_uint32),
                ("restitution", ctypes.c_float), ("friction", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


class ContactF32(ctypes.Structure):
    """al_contact_f32 (Contact<float3, float>, contact.hpp:8-25)."""
    _fields_ = [("i", ctypes.c_uint32), ("j", ctypes.c_uint32),
                ("cp_i", ctypes.c_float * 3), ("cp_j", ctypes.c_float * 3),
                ("n", ctypes.c_float * 3), ("t", ctypes.c_float * 3),
                ("iiwi_diag", ctypes.c_float * 3), ("iiwi_off_diag", ctypes.c_float * 3),
                ("iiwj_diag", ctypes.c_float * 3), ("iiwj_off_diag", ctypes.c_float * 3),
                ("friction", ctypes.c_float), ("nkninv", ctypes.c_float),
                ("pmax", ctypes.c_float), ("goalu", ctypes.c_float),
                ("impulse_sum", ctypes.c_float)]


CONTACT_FLOATS = ctypes.sizeof(ContactF32) // 4


def _pellets_struct(real):
    class Pellets(ctypes.Structure):
        _fields_ = [("local_x", ctypes.c_void_p), ("num_pellets", ctypes.c_uint32),
                    ("count", ctypes.c_uint32 * AL_MAX_BOUNDARIES), ("x", ctypes.c_void_p),
                    ("pressure", ctypes.c_void_p), ("v", ctypes.c_void_p)]
    Pellets.__name__ = "Pellets" + ("F32" if real is ctypes.c_float else "F64")
    return Pellets


PelletsF32 = _pellets_struct(ctypes.c_float)
PelletsF64 = _pellets_struct(ctypes.c_double)


class PelletRelaxParams(ctypes.Structure):
    """al_pellet_relax_params (SolverPellet's coefficients)."""
    _fields_ = [("cohesion", ctypes.c_double), ("adhesion", ctypes.c_double),
                ("cfl_factor", ctypes.c_double), ("contact_tolerance", ctypes.c_double),
                ("wrap_y", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("wrap_length", ctypes.c_double)]


def pellet_relax_params(cohesion=4.0, adhesion=2.0, cfl_factor=0.25, contact_tolerance=0.0,
                        wrap_length=None):
    """SolverPellet's defaults (solver_pellet.hpp:47-50)."""
    p = PelletRelaxParams()
    p.cohesion, p.adhesion, p.cfl_factor = cohesion, adhesion, cfl_factor
    p.contact_tolerance = contact_tolerance
    if wrap_length is not None:
        p.wrap_y, p.wrap_length = 1, wrap_length
    return p


class SampleF32(ctypes.Structure):
    """al_sample_f32: sample points, particle inputs and the outputs wanted
    (device pointers; None where unused)."""
    _fields_ = [("sample_x", ctypes.c_void_p), ("num_samples", ctypes.c_uint32),
                ("quantity_dim", ctypes.c_uint32), ("particle_density", ctypes.c_void_p),
                ("particle_v", ctypes.c_void_p), ("particle_quantity", ctypes.c_void_p),
                ("sample_boundary", ctypes.c_void_p),
                ("sample_boundary_kernel", ctypes.c_void_p),
                ("sample_density", ctypes.c_void_p),
                ("sample_position_density", ctypes.c_void_p),
                ("sample_quantity", ctypes.c_void_p), ("sample_v", ctypes.c_void_p),
                ("sample_vorticity", ctypes.c_void_p), ("wrap_y", ctypes.c_uint32),
                ("wrap_length", ctypes.c_float), ("pellet_x", ctypes.c_void_p),
                ("pellet_v", ctypes.c_void_p), ("num_pellets", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class SampleF64(ctypes.Structure):
    """al_sample_f64: the double-precision request (wrap_length double)."""
    _fields_ = [("sample_x", ctypes.c_void_p), ("num_samples", ctypes.c_uint32),
                ("quantity_dim", ctypes.c_uint32), ("particle_density", ctypes.c_void_p),
                ("particle_v", ctypes.c_void_p), ("particle_quantity", ctypes.c_void_p),
                ("sample_boundary", ctypes.c_void_p),
                ("sample_boundary_kernel", ctypes.c_void_p),
                ("sample_density", ctypes.c_void_p),
                ("sample_position_density", ctypes.c_void_p),
                ("sample_quantity", ctypes.c_void_p), ("sample_v", ctypes.c_void_p),
                ("sample_vorticity", ctypes.c_void_p), ("wrap_y", ctypes.c_uint32),
                ("reserved0", ctypes.c_uint32), ("wrap_length", ctypes.c_double),
                ("pellet_x", ctypes.c_void_p), ("pellet_v", ctypes.c_void_p),
                ("num_pellets", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


def sample_struct(dtype):
    return SampleF64 if np.dtype(dtype) == np.float64 else SampleF32


class StepReport(ctypes.Structure):
    _fields_ = [("num_divergence_solve", ctypes.c_uint32),
                ("num_density_solve", ctypes.c_uint32),
                ("mean_density_change", ctypes.c_double),
                ("mean_density_error", ctypes.c_double),
                ("particle_max_v2", ctypes.c_double),
                ("pile_max_v2", ctypes.c_double),
                ("max_v2", ctypes.c_double),
                ("cfl_dt", ctypes.c_double),
                ("utilized_cfl", ctypes.c_double),
                ("dt", ctypes.c_double),
                ("grid_anomaly", ctypes.c_uint32 * 3),
                ("num_active_boundary_pairs", ctypes.c_uint32),
                ("force", (ctypes.c_double * 3) * AL_MAX_BOUNDARIES),
                ("torque", (ctypes.c_double * 3) * AL_MAX_BOUNDARIES)]


_FLUID_PTRS = ("particle_x", "particle_v", "particle_a", "particle_density",
               "particle_dfsph_factor", "particle_kappa", "particle_kappa_v",
               "particle_density_adv", "particle_pressure", "particle_boundary",
               "particle_boundary_kernel")


class Fluid(ctypes.Structure):
    """al_fluid_f32 / al_fluid_f64 (identical layout: pointers)."""
    _fields_ = [("num_particles", ctypes.c_uint32), ("reserved", ctypes.c_uint32)] + \
               [(name, ctypes.c_void_p) for name in _FLUID_PTRS]


def make_fluid(num_particles, **buffers):
    """al_fluid from device buffers (torch tensors or raw addresses)."""
    f = Fluid()
    f.num_particles = num_particles
    for name, t in buffers.items():
        assert name in _FLUID_PTRS, name
        if t is None:
            continue
        setattr(f, name, t if isinstance(t, int) else t.data_ptr())
    return f


def real_types(dtype):
    """(ConstT, BodyT, RigidT, ctypes real) for np.float32 / np.float64."""
    if np.dtype(dtype) == np.float32:
        return ConstF32, BodyF32, RigidF32, ctypes.c_float
    if np.dtype(dtype) == np.float64:
        return ConstF64, BodyF64, RigidF64, ctypes.c_double
    raise TypeError("unsupported real type %r" % (dtype,))


def suffix(dtype):
    return "f32" if np.dtype(dtype) == np.float32 else "f64"


_lib = None

# name -> (restype, argtypes); pointer arguments are passed as c_void_p.
_P = ctypes.c_void_p
_U = ctypes.c_uint32
_SIGNATURES = {
    "al_engine_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "al_engine_destroy": (ctypes.c_int, [_P]),
    "al_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "al_last_error": (ctypes.c_char_p, []),
    "al_engine_synchronize": (ctypes.c_int, [_P, _P]),
    "al_allocate": (ctypes.c_int, [_P, _P, ctypes.c_size_t]),
    "al_free": (ctypes.c_int, [_P, _P]),
    "al_copy": (ctypes.c_int, [_P, _P, _P, ctypes.c_size_t]),
    "al_set": (ctypes.c_int, [_P, _P, ctypes.c_int, ctypes.c_size_t]),
    "al_engine_set_graph_mode": (ctypes.c_int, [_P, ctypes.c_int]),
    "al_engine_set_batch_fused": (ctypes.c_int, [_P, ctypes.c_int]),
    "al_engine_set_launch_shape": (ctypes.c_int, [_P, ctypes.c_char_p, _U, _U, _U, _U]),
    "al_engine_get_launch_shape": (ctypes.c_int, [_P, ctypes.c_char_p, _U, _U, _P, _P]),
    "al_tunable_group": (ctypes.c_int, [_U, ctypes.POINTER(ctypes.c_char_p), _P]),
    "al_engine_graph_stats": (ctypes.c_int, [_P, _P, _P]),
    "al_engine_set_profiling": (ctypes.c_int, [_P, ctypes.c_int]),
    "al_warm_net_forward_f32": (ctypes.c_int, [_P, _P, _P, _U, _P, _P]),
    "al_df_step_warm_f32": (ctypes.c_int, [_P] * 8 + [_P, _P, _P]),
    "al_df_batch_step_f32": (ctypes.c_int, [_P, _P, _U, _P]),
    "al_build_mesh_distance_grid_f32": (ctypes.c_int, [_P, _P, _P, _U, _P, _U, ctypes.c_float,
                                                       _P, _P]),
    "al_find_contacts_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, ctypes.c_float, _U, _P, _P,
                                            _P]),
    "al_solve_contacts_f32": (ctypes.c_int, [_P, _P, _P, _U, _P, _U, _P]),
    "al_warm_net_gradient_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P]),
    "al_warm_net_adam_f32": (ctypes.c_int, [_P, _P, _P, _P, _P, _U, ctypes.c_float, _P]),
    "al_engine_reset_stats": (ctypes.c_int, [_P]),
    "al_engine_launch_count": (ctypes.c_int, [_P, _P]),
    "al_engine_kernel_stat": (ctypes.c_int, [_P, _U, ctypes.c_char_p, ctypes.c_size_t, _P, _P]),
    "al_grid_sort_noalloc_f32": (ctypes.c_int, [_P, _P, _P, _U, _P, _P, _P, _P, _P]),
    "al_sample_fluid_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P]),
    "al_sample_fluid_f64": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P]),
    "al_density_mask_f32": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "al_density_mask_f64": (ctypes.c_int, [_P, _P, _U, _P, _P]),
    "al_boundary_mask_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, ctypes.c_float, _P, _P]),
    "al_boundary_mask_f64": (ctypes.c_int, [_P, _P, _P, _P, _U, ctypes.c_double, _P, _P]),
    "al_distance_mask_multiple_f64": (ctypes.c_int, [_P, _P, _U, _P, _U, ctypes.c_double, _P,
                                                     _P]),
    "al_histogram256_f64": (ctypes.c_int, [_P, _P, _P, _U, ctypes.c_double, ctypes.c_double,
                                           _P, _P]),
    "al_distance_mask_multiple_f32": (ctypes.c_int, [_P, _P, _U, _P, _U, ctypes.c_float, _P,
                                                     _P]),
    "al_histogram256_f32": (ctypes.c_int, [_P, _P, _P, _U, ctypes.c_float, ctypes.c_float, _P,
                                           _P]),
    "al_kl_divergence": (ctypes.c_int, [_P, _P, _P, _U, _U, ctypes.c_double, _U, _P, _P]),
    "al_calculate_se_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P]),
    "al_calculate_se_f64": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P]),
    "al_calculate_se_weighted_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P, _P]),
    "al_calculate_se_weighted_f64": (ctypes.c_int, [_P, _P, _P, _P, _U, _U, _P, _P]),
    "al_calculate_se_yz_masked_f32": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P]),
    "al_calculate_se_yz_masked_f64": (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P]),
    "al_sum_products_f32": (ctypes.c_int, [_P, _P, _P, _U, _U, _P, _P]),
    "al_sum_products_f64": (ctypes.c_int, [_P, _P, _P, _U, _U, _P, _P]),
}
for _s in ("f32", "f64"):
    _SIGNATURES["al_grid_sort_" + _s] = (ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P, _P, _P])
    _SIGNATURES["al_update_particle_neighbors_" + _s] = (
        ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P, _P, _P, _P])
    _SIGNATURES["al_update_particle_neighbors_periodic_" + _s] = (
        ctypes.c_int, [_P, _P, _P, _P, _U, _P, _P, _P, _P, _P, ctypes.c_double, _P])
    _SIGNATURES["al_compute_particle_boundary_" + _s] = (
        ctypes.c_int, [_P, _P, _U, _P, _P, _P, _U, _P, _P, _P])
    _SIGNATURES["al_build_volume_field_" + _s] = (ctypes.c_int, [_P, _P, _P, _P, _P])
    _SIGNATURES["al_build_distance_grid_" + _s] = (ctypes.c_int, [_P, _P, _P, _P])
    _SIGNATURES["al_node_positions_" + _s] = (ctypes.c_int, [_P, _P, _P, _P])
    _SIGNATURES["al_df_step_" + _s] = (ctypes.c_int, [_P] * 10)
    _SIGNATURES["al_ii_step_" + _s] = (ctypes.c_int, [_P] * 10)
    _SIGNATURES["al_i_step_" + _s] = (ctypes.c_int, [_P] * 10)
    _SIGNATURES["al_i_step_pellets_" + _s] = (ctypes.c_int, [_P] * 11)
    _SIGNATURES["al_relax_pellets_" + _s] = (ctypes.c_int, [_P] * 5 + [_U, _P, _U, _P, _P, _P])


def declared_symbols():
    """Names of every entry point this module binds (all of include/*.h)."""
    return sorted(_SIGNATURES)


def lib():
    """Loads liballuvion_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "liballuvion_b200.so not found at %s; run `python -m alluvion_b200.build` "
                "(there is no CPU fallback)" % LIB_PATH)
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


class EngineError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = lib().al_last_error().decode() or lib().al_status_string(status).decode()
        super().__init__("%s failed: %s (%s)" % (where, STATUS.get(status, status), msg))


def check(status, where, allow=()):
    """Raises EngineError for a non-OK status not listed in `allow`."""
    if status != AL_OK and status not in allow:
        raise EngineError(status, where)
    return status


class Engine:
    """Owns one al_engine* bound to a CUDA device."""

    def __init__(self, device=0):
        h = ctypes.c_void_p()
        check(lib().al_engine_create(device, ctypes.byref(h)), "al_engine_create")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().al_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self, stream=None):
        check(lib().al_engine_synchronize(self.handle, stream), "al_engine_synchronize")

    def set_graph_mode(self, enable):
        """Replay captured step graphs for repeated step configurations."""
        check(lib().al_engine_set_graph_mode(self.handle, int(bool(enable))), "set_graph_mode")

    def graph_stats(self):
        """(step graphs captured, steps run by replaying one)."""
        c, r = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().al_engine_graph_stats(self.handle, ctypes.byref(c), ctypes.byref(r)),
              "graph_stats")
        return c.value, r.value

    def set_profiling(self, enable):
        check(lib().al_engine_set_profiling(self.handle, int(bool(enable))), "set_profiling")

    def reset_stats(self):
        check(lib().al_engine_reset_stats(self.handle), "al_engine_reset_stats")

    def launch_count(self):
        c = ctypes.c_uint64()
        check(lib().al_engine_launch_count(self.handle, ctypes.byref(c)), "launch_count")
        return c.value

    def set_launch_shape(self, group, bucket, batch, block, tpp):
        """Launch shape of a tunable pass group for scenes of 2^bucket..2^(bucket+1)
        particles in single (batch=0) or batched (batch=1) steps; 0 keeps a default."""
        check(lib().al_engine_set_launch_shape(self.handle, group.encode(), int(bucket),
                                               int(batch), int(block), int(tpp)),
              "al_engine_set_launch_shape")

    def set_batch_fused(self, enable):
        """Batched steps run fused (one launch per solver pass over all scenes,
        the default where the scenes allow it) or as one graph branch per
        scene."""
        check(lib().al_engine_set_batch_fused(self.handle, 1 if enable else 0),
              "al_engine_set_batch_fused")

    def launch_shape(self, group, num_particles, batch=0):
        """(block, threads per particle) a step of num_particles would use."""
        b, t = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().al_engine_get_launch_shape(self.handle, group.encode(), int(num_particles),
                                               int(batch), ctypes.byref(b), ctypes.byref(t)),
              "al_engine_get_launch_shape")
        return b.value, t.value

    def kernel_stats(self):
        """{launch group name: (total_ms, count)} recorded while profiling."""
        out = {}
        buf = ctypes.create_string_buffer(128)
        ms = ctypes.c_double()
        cnt = ctypes.c_uint64()
        i = 0
        while lib().al_engine_kernel_stat(self.handle, i, buf, 128, ctypes.byref(ms),
                                          ctypes.byref(cnt)) == AL_OK:
            out[buf.value.decode()] = (ms.value, cnt.value)
            i += 1
        return out


def tunable_groups():
    """[(name, is_pair_pass)] of the step's pass groups with a settable shape."""
    out = []
    name, pair = ctypes.c_char_p(), ctypes.c_uint32()
    k = 0
    while lib().al_tunable_group(k, ctypes.byref(name), ctypes.byref(pair)) == AL_OK:
        out.append((name.value.decode(), bool(pair.value)))
        k += 1
    return out


def ptr(t):
    """Address of a torch tensor, numpy array or ctypes object (None -> NULL)."""
    if t is None:
        return None
    if isinstance(t, (ctypes.Structure, ctypes.Array, ctypes._SimpleCData)):
        return ctypes.cast(ctypes.pointer(t), ctypes.c_void_p)
    if hasattr(t, "data_ptr"):
        return ctypes.c_void_p(t.data_ptr())
    return ctypes.c_void_p(t.ctypes.data)
