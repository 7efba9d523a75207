"""Depot: the reference's Python entry object (alluvion/depot.py:8-117) over
the pybind11 module _alluvion_b200.

A Depot is a Store that picks the float or double classes by name suffix,
as the reference's does, so that user scripts written against the reference
keep their shape:

    dp = Depot(np.float32)
    cn, cni = dp.cn, dp.cni
    cn.set_kernel_radius(4 * r); cn.set_particle_attr(r, m, 1000.0)
    runner = dp.Runner()
    pile = dp.Pile(dp, runner, 0)
    pile.add(dp.BoxDistance.create([1, 1, 1]), [32, 32, 32], sign=-1, x=[.5, .5, .5])
    solver = dp.SolverDf(runner, pile, dp, max_num_particles=n)
    solver.particle_x.set(x); solver.num_particles = n
    solver.dt = solver.max_dt = 2e-4; solver.cfl = 0.4
    solver.step()

Variables returned by create() and by the solvers carry the Coated get / set
of alluvion/variable.py directly, plus __cuda_array_interface__ for
zero-copy torch views (torch.as_tensor(var, device="cuda")).
"""
import numpy as np

from . import _alluvion_b200 as _al
from ._alluvion_b200 import NumericType, Store, VolumeMethod  # noqa: F401

_FLOAT_TYPED = ["Runner", "Pile", "SolverDf", "SolverIi", "SolverI", "SolverPellet", "Solver",
                "Mesh", "Const"]
_FLOAT_TYPED_DG = ["BoxDistance", "BoxShellDistance", "CapsuleDistance", "CylinderDistance",
                   "Distance", "InfiniteCylinderDistance", "InfiniteTubeDistance",
                   "SphereDistance", "MeshDistance", "TriangleMesh"]


def dtype_to_string(dtype):
    """'float' or 'double' (Store::dtype_to_string in the reference)."""
    dt = np.dtype(dtype)
    if dt == np.float32:
        return "float"
    if dt == np.float64:
        return "double"
    raise ValueError("Depot: float32 or float64, not %s" % dt)


class Depot(Store):

    def __init__(self, default_dtype=np.float32, device=0):
        super().__init__(device)
        self.default_dtype = np.dtype(default_dtype)
        sfx = dtype_to_string(self.default_dtype)
        for name in _FLOAT_TYPED:
            setattr(self, name, getattr(_al, name + sfx))
        for name in _FLOAT_TYPED_DG:
            setattr(self, name, getattr(_al.dg, name + sfx))
        self.cn = getattr(self, "cn" + sfx)
        self.copy_cn = getattr(self, "copy_cn" + sfx)
        self.copy_cn_external = getattr(self, "copy_cn_external" + sfx)
        self.create_cn = getattr(self, "create_cn" + sfx)

    def create(self, shape, n, dtype=None):
        """A device variable of `shape` elements of n primitives
        (Depot.create, depot.py:70-71); dtype defaults to the depot's."""
        if isinstance(shape, int):
            shape = [shape]
        dt = np.dtype(self.default_dtype if dtype is None else dtype)
        return super().create(list(shape), int(n), dt.name)

    def create_coated(self, shape, n, dtype=None):
        return self.create(shape, n, dtype)

    def coat(self, var):
        """Variables already carry get / set."""
        return var

    def create_coated_like(self, var):
        return self.create(var.get_shape(), var.get_num_primitives_per_element(),
                           type_enum_to_dtype(var.get_type()))


def type_enum_to_dtype(numeric_type):
    """numpy dtype of a NumericType (variable.py:6-16)."""
    return {NumericType.f32: np.float32, NumericType.f64: np.float64,
            NumericType.i32: np.int32, NumericType.u32: np.uint32}[numeric_type]
