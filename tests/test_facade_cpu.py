"""CPU checks of the pybind11 module that restates the reference's Python
object model (lib/pyalluvion.cu, alluvion/depot.py): the class names a
reference script looks up, the distances' bounding boxes and max_distance
(against the restatement the scene helpers use), the Const setters
(constants.hpp:100-136), and failure as RuntimeError without a device."""
import numpy as np
import pytest

from alluvion_b200 import _alluvion_b200 as al, _capi, scenes
from alluvion_b200.depot import Depot


def test_reference_class_names():
    for sfx in ("float", "double"):
        for name in ("Const", "Runner", "Pile", "Solver", "SolverDf", "SolverIi", "SolverI"):
            assert hasattr(al, name + sfx), name + sfx
        for name in ("Distance", "SphereDistance", "BoxDistance", "BoxShellDistance",
                     "CylinderDistance", "CapsuleDistance", "InfiniteCylinderDistance",
                     "InfiniteTubeDistance", "MeshDistance", "TriangleMesh"):
            assert hasattr(al.dg, name + sfx), name + sfx
    for name in ("Store", "ConstiN", "Variable", "NumericType", "VolumeMethod"):
        assert hasattr(al, name)
    for name in ("step", "step_wrap1", "update_particle_neighbors",
                 "update_particle_neighbors_wrap1", "compute_all_boundaries", "reset_t",
                 "reset_solving_var"):
        assert hasattr(al.SolverDffloat, name)
    assert issubclass(al.Error, RuntimeError)


@pytest.mark.parametrize("sfx,dtype", [("float", np.float32), ("double", np.float64)])
def test_distance_boxes_match_scene_restatement(sfx, dtype):
    dg = al.dg
    cases = [
        (getattr(dg, "BoxDistance" + sfx).create([0.4, 0.2, 0.6], 0.01), _capi.SHAPE_BOX,
         scenes.box_params([0.4, 0.2, 0.6], 0.01)),
        (getattr(dg, "SphereDistance" + sfx).create(0.3), _capi.SHAPE_SPHERE, [0.3]),
        (getattr(dg, "BoxShellDistance" + sfx).create([0.4, 0.2, 0.6], 0.02, 0.01),
         _capi.SHAPE_BOX_SHELL, scenes.box_shell_params([0.4, 0.2, 0.6], 0.02, 0.01)),
        (getattr(dg, "CylinderDistance" + sfx).create(0.1, 0.5, 0.05), _capi.SHAPE_CYLINDER,
         [0.1, 0.5, 0.05]),
        (getattr(dg, "CapsuleDistance" + sfx).create(0.1, 0.5), _capi.SHAPE_CAPSULE, [0.1, 0.5]),
        (getattr(dg, "InfiniteCylinderDistance" + sfx).create(0.2),
         _capi.SHAPE_INFINITE_CYLINDER, [0.2]),
        (getattr(dg, "InfiniteTubeDistance" + sfx).create(0.1, 0.15, 0.4),
         _capi.SHAPE_INFINITE_TUBE, [0.1, 0.15, 0.4]),
    ]
    for d, shape, params in cases:
        lo, hi, maxd = scenes.shape_aabb(shape, params)
        np.testing.assert_allclose(d.aabb_min, lo, rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(d.aabb_max, hi, rtol=1e-6, atol=1e-7)
        assert d.max_distance == pytest.approx(maxd, rel=1e-6)
    v, f = scenes.cube_mesh(0.25)
    mesh = getattr(dg, "TriangleMesh" + sfx)(v, f)
    md = getattr(dg, "MeshDistance" + sfx).create(mesh, 0.01)
    lo, hi, maxd = scenes.mesh_aabb(v, 0.01)
    np.testing.assert_allclose(md.aabb_min, lo, rtol=1e-6)
    np.testing.assert_allclose(md.aabb_max, hi, rtol=1e-6)
    assert md.max_distance == pytest.approx(maxd, rel=1e-6)


@pytest.mark.parametrize("sfx,dtype", [("float", np.float32), ("double", np.float64)])
def test_const_setters_match_make_const(sfx, dtype):
    c = getattr(al, "Const" + sfx)()
    r = 0.005
    c.set_kernel_radius(4 * r)
    c.set_particle_attr(r, 1000.0 * (2 * r) ** 3, 1000.0)
    c.set_wrap_length(0.6)
    ref = scenes.make_const(dtype, r)
    T = np.dtype(dtype).type
    assert T(c.kernel_radius) == ref.kernel_radius
    assert T(c.particle_vol) == pytest.approx(float(ref.particle_vol), rel=1e-6)
    assert (c.wrap_length, c.wrap_min, c.wrap_max) == pytest.approx((0.6, -0.3, 0.3))
    c.gravity = (0.0, -9.81, 0.0)
    assert c.gravity[1] == pytest.approx(-9.81)


def test_store_without_device_raises_runtime_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        Depot(np.float32)


def test_cpp_object_model_compiles(tmp_path):
    """include/alluvion_b200_solver.hpp compiles for both real types with
    g++ against the library (every class template instantiated), and a
    Store without a device throws alluvion_b200::error(AL_ERR_NO_DEVICE)
    the way the reference's Allocator throws std::runtime_error."""
    import os
    import subprocess
    import torch
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "model.cpp"
    src.write_text(r"""
#include <cstdio>
#include "alluvion_b200_solver.hpp"
namespace ab = alluvion_b200;
template class ab::Pile<float>;
template class ab::Pile<double>;
template class ab::SolverDf<float>;
template class ab::SolverDf<double>;
template class ab::SolverPressure<float, false>;
template class ab::SolverPressure<double, true>;
template void ab::SolverDf<float>::step<1>();
template void ab::SolverI<double>::step<1>();
template void ab::Solver<float>::update_particle_neighbors<1>();
int main() {
  ab::dg::BoxDistance<float> box({0.4f, 0.2f, 0.6f}, 0.01f);
  ab::Const<double> cn;
  cn.set_kernel_radius(0.02);
  cn.set_particle_attr(0.005, 0.001, 1000.0);
  int status = 0;
  try {
    ab::Store store(0);
    ab::Runner<float> runner;
    ab::Pile<float> pile(store, runner, 0);
  } catch (const ab::error& e) {
    status = e.status();
  }
  std::printf("%d %.6f %.9f\n", status, double(box.aabb_max[2]), cn.particle_vol);
  return 0;
}
""")
    exe = tmp_path / "model"
    libdir = os.path.join(root, "alluvion_b200")
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(root, "include"), str(src),
                    "-L", libdir, "-lalluvion_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert int(out[0]) == (0 if torch.cuda.is_available() else 8)
    assert float(out[1]) == pytest.approx(0.31)
    assert float(out[2]) == pytest.approx(1e-6)


def test_launch_shape_table_round_trip(tmp_path):
    """alluvion_b200.autotune tables: JSON round trip, validation of names
    and ranges, and load() applying every entry (a stand-in engine records
    the calls; no device is needed)."""
    from alluvion_b200 import autotune

    class Recorder:
        def __init__(self):
            self.calls = []

        def set_launch_shape(self, *args):
            self.calls.append(args)

    table = {"device": "test", "entries": [
        {"group": "press_iter", "bucket": 20, "batch": 0, "block": 256, "tpp": 1, "ms": 0.1},
        {"group": "neighbors", "bucket": 20, "batch": 1, "block": 64, "tpp": 1, "ms": 0.3}]}
    path = str(tmp_path / "t.json")
    autotune.save(table, path)
    rec = Recorder()
    loaded = autotune.load(rec, path)
    assert loaded["entries"] == table["entries"]
    assert rec.calls == [("press_iter", 20, 0, 256, 1), ("neighbors", 20, 1, 64, 1)]
    assert autotune.bucket_of(1 << 20) == 20 and autotune.bucket_of((1 << 20) - 1) == 19
    bad = {"entries": [dict(table["entries"][0], block=96)]}
    with pytest.raises(ValueError):
        autotune.validate(bad)
    dup = {"entries": [table["entries"][0], dict(table["entries"][0])]}
    with pytest.raises(ValueError):
        autotune.validate(dup)
