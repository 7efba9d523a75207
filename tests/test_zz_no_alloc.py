"""The allocation-free grid sort (al_grid_sort_noalloc_f32).

Callers such as a renderer that owns the device memory budget, or a
real-time loop that cannot take the stalls of cudaMalloc / cudaFree, cannot
let the library allocate; this entry point keeps its scratch in one static
device array.  The test calls it through the C ABI twice in a row, on two
different particle sets, and checks each result against the allocating
al_grid_sort_f32 (integer outputs: bit-exact, the bar of the grid tests).
The second call must see no stale counts from the first, and must not
change the device's free memory (the first call may: CUDA loads the
library's device image, and with it the static array, lazily).  The
anomaly statuses (a particle outside the grid, a cell above its capacity)
must equal the allocating sort's.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes

pytestmark = pytest.mark.gpu


def _inputs(seed, dims):
    cn = scenes.make_const(np.float32, 0.01)
    x = scenes.fluid_block(dims, (0.0, 0.0, 0.0), 0.01, np.float32, seed=seed)
    rng = np.random.default_rng(seed)
    x = x[rng.permutation(len(x))]
    cni = scenes.make_consti(x.min(0), x.max(0), cn.kernel_radius)
    return cn, cni, x


def _run(fn, pre_args, cn, cni, x):
    n = x.shape[0]
    ncells = cni.grid_res[0] * cni.grid_res[1] * cni.grid_res[2]
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    outs = [torch.full((n,), -1, dtype=torch.int32, device="cuda"),
            torch.full((n,), -1, dtype=torch.int32, device="cuda"),
            torch.full((ncells + 1,), -1, dtype=torch.int32, device="cuda"),
            torch.full((ncells,), -1, dtype=torch.int32, device="cuda")]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    status = fn(*pre_args, ctypes.byref(cn), ctypes.byref(cni), _capi.ptr(xd), n,
                *[_capi.ptr(t) for t in outs], None)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    return status, [t.cpu().numpy().view(np.uint32) for t in outs], free_before - free_after


def test_noalloc_grid_sort_matches_allocating_sort_twice():
    assert torch.cuda.is_available()
    lib = _capi.lib()
    engine = _capi.Engine(0)
    try:
        for call, (seed, dims) in enumerate([(21, (20, 16, 18)), (22, (12, 14, 10))]):
            cn, cni, x = _inputs(seed, dims)
            s_ref, ref, _ = _run(lib.al_grid_sort_f32, (engine.handle,), cn, cni, x)
            assert s_ref == _capi.AL_OK
            s_na, got, used = _run(lib.al_grid_sort_noalloc_f32, (), cn, cni, x)
            assert s_na == _capi.AL_OK, lib.al_last_error()
            for name, a, b in zip(("cell", "perm", "cell_start", "pid_length"), got, ref):
                assert np.array_equal(a, b), "call %d: %s differs" % (call, name)
            if call == 1:
                # the static scratch is already resident: nothing is allocated
                assert used == 0
    finally:
        engine.close()


def test_noalloc_rejects_sizes_beyond_the_static_limit():
    cn = scenes.make_const(np.float32, 0.01)
    cni = scenes.make_consti((0, 0, 0), (0.1, 0.1, 0.1), cn.kernel_radius)
    cni.grid_res[0] = 2048
    cni.grid_res[1] = 1024
    cni.grid_res[2] = 1  # 2,097,152 cells > 1,048,576
    status = _capi.lib().al_grid_sort_noalloc_f32(ctypes.byref(cn), ctypes.byref(cni), None, 0,
                                                  None, None, None, None, None)
    assert status == 2  # AL_ERR_INVALID
    assert b"static scratch limit" in _capi.lib().al_last_error()
    status = _capi.lib().al_grid_sort_noalloc_f32(ctypes.byref(cn), ctypes.byref(cni), None,
                                                  (1 << 20) + 1, None, None, None, None, None)
    assert status == 2


@pytest.mark.parametrize("case", ["out_of_grid", "cell_overflow"])
def test_noalloc_reports_the_same_anomalies(case):
    """A particle far outside the grid (AL_ERR_OUT_OF_GRID) and a cell
    capacity below the lattice's ~8 particles per cell
    (AL_ERR_CELL_OVERFLOW): both entry points return the same status and
    the same outputs."""
    lib = _capi.lib()
    engine = _capi.Engine(0)
    try:
        cn, cni, x = _inputs(23, (8, 8, 8))
        x = x.copy()
        if case == "out_of_grid":
            x[5] = (50.0, 50.0, 50.0)
            expect = _capi.AL_ERR_OUT_OF_GRID
        else:
            cni.max_num_particles_per_cell = 4
            expect = _capi.AL_ERR_CELL_OVERFLOW
        s_ref, ref, _ = _run(lib.al_grid_sort_f32, (engine.handle,), cn, cni, x)
        s_na, got, _ = _run(lib.al_grid_sort_noalloc_f32, (), cn, cni, x)
        assert s_ref == expect and s_na == expect
        inside = int(ref[2][-1])
        for name, a, b in zip(("cell", "perm", "cell_start", "pid_length"), got, ref):
            if name == "perm":
                # out-of-grid particles sit after the in-grid ones, in any order
                assert np.array_equal(a[:inside], b[:inside]), name
                assert set(a[inside:]) == set(b[inside:]), name
            else:
                assert np.array_equal(a, b), name
        # a clean call afterwards starts from cleared flags
        cn2, cni2, x2 = _inputs(24, (6, 6, 6))
        s2, _, _ = _run(lib.al_grid_sort_noalloc_f32, (), cn2, cni2, x2)
        assert s2 == _capi.AL_OK
    finally:
        engine.close()
