"""GPU parity of the grid hash / counting sort and the neighbor list + density
(Solver::update_particle_neighbors, solver.hpp:225-260) against the oracle,
through the C ABI.  Bar: bit-exact cell ids, permutation, neighbor lists and
counts; density within 1e-6 relative (float32) / 1e-13 (float64)."""
import ctypes

import numpy as np
import pytest
import torch

from alluvion_b200 import _capi, scenes
from oracle import binding as orc
from conftest import dev, host

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.float64]
RTOL = {np.float32: 1e-6, np.float64: 1e-13}


def _block(dtype, dims=(12, 9, 10), r=0.01, seed=0, jitter=0.1):
    cn = scenes.make_const(dtype, r)
    x = scenes.fluid_block(dims, (0.0, 0.0, 0.0), r, dtype, jitter=jitter, seed=seed)
    cni = scenes.make_consti(x.min(0), x.max(0), cn.kernel_radius)
    return cn, cni, x


def _grid_sort(engine, cn, cni, x):
    n = x.shape[0]
    ncells = cni.grid_res[0] * cni.grid_res[1] * cni.grid_res[2]
    xd = dev(x)
    cell = torch.zeros(n, dtype=torch.int32, device="cuda")
    perm = torch.zeros(n, dtype=torch.int32, device="cuda")
    start = torch.zeros(ncells + 1, dtype=torch.int32, device="cuda")
    plen = torch.zeros(ncells, dtype=torch.int32, device="cuda")
    fn = getattr(_capi.lib(), "al_grid_sort_" + _capi.suffix(x.dtype))
    status = fn(engine.handle, ctypes.byref(cn), ctypes.byref(cni), _capi.ptr(xd), n,
                _capi.ptr(cell), _capi.ptr(perm), _capi.ptr(start), _capi.ptr(plen), None)
    u = lambda t: host(t).view(np.uint32)
    return status, u(cell), u(perm), u(start), u(plen)


def _neighbors(engine, cn, cni, x, bk=None):
    n = x.shape[0]
    cap = cni.max_num_neighbors_per_particle
    xd = dev(x)
    rho = torch.zeros(n, dtype=xd.dtype, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    nbr = torch.zeros((n, cap, 4), dtype=xd.dtype, device="cuda")
    anomaly = torch.zeros(3, dtype=torch.int32, device="cuda")
    bkd = dev(bk) if bk is not None else None
    fn = getattr(_capi.lib(), "al_update_particle_neighbors_" + _capi.suffix(x.dtype))
    status = fn(engine.handle, ctypes.byref(cn), ctypes.byref(cni), _capi.ptr(xd), n,
                _capi.ptr(bkd), _capi.ptr(rho), _capi.ptr(cnt), _capi.ptr(nbr),
                _capi.ptr(anomaly), None)
    return status, host(rho), host(cnt).view(np.uint32), host(nbr), host(anomaly)


def _index_bits(nbrs, dtype):
    w = np.ascontiguousarray(nbrs[..., 3])
    if np.dtype(dtype) == np.float32:
        return w.view(np.uint32)
    return (w.view(np.uint64) & 0xffffffff).astype(np.uint32)


@pytest.mark.parametrize("dtype", DTYPES)
def test_grid_sort_bit_exact(engine, dtype):
    cn, cni, x = _block(dtype, seed=11)
    rng = np.random.default_rng(5)
    x = x[rng.permutation(len(x))]  # scramble the input order
    status, cell, perm, start, plen = _grid_sort(engine, cn, cni, x)
    assert status == _capi.AL_OK
    o_cell, o_perm, o_start, o_flags = orc.grid_sort(cn, cni, x)
    assert np.array_equal(cell, o_cell)
    assert np.array_equal(perm, o_perm)
    assert np.array_equal(start, o_start)
    assert np.array_equal(plen, np.diff(o_start).astype(np.uint32))
    assert not o_flags.any()


@pytest.mark.parametrize("dtype", DTYPES)
def test_neighbors_and_density_parity(engine, dtype):
    cn, cni, x = _block(dtype, seed=7)
    status, rho, cnt, nbrs, anomaly = _neighbors(engine, cn, cni, x)
    assert status == _capi.AL_OK and not anomaly.any()
    o_rho, o_cnt, o_idx, o_nbrs, o_flags = orc.update_particle_neighbors(cn, cni, x)
    assert np.array_equal(cnt, o_cnt)
    idx = _index_bits(nbrs, dtype)
    for i in range(len(x)):
        c = cnt[i]
        assert np.array_equal(idx[i, :c], o_idx[i, :c]), i  # same canonical order
        assert np.array_equal(nbrs[i, :c, :3], o_nbrs[i, :c, :3]), i  # bit-exact x_i - x_j
    np.testing.assert_allclose(rho, o_rho, rtol=RTOL[dtype])
    # interior lattice particles see the 26 lattice neighbours at |d| < 2 spacings
    assert np.median(cnt) >= 18 and cnt.max() <= 64


@pytest.mark.parametrize("dtype", DTYPES)
def test_density_with_boundary_kernel_term(engine, dtype):
    cn, cni, x = _block(dtype, dims=(8, 8, 8), seed=3)
    cni.num_boundaries = 2
    rng = np.random.default_rng(9)
    bk = rng.uniform(0, 1e-3, size=(2, len(x), 4)).astype(dtype)
    status, rho, cnt, _, _ = _neighbors(engine, cn, cni, x, bk)
    assert status == _capi.AL_OK
    o_rho, o_cnt, *_ = orc.update_particle_neighbors(cn, cni, x, bk)
    np.testing.assert_allclose(rho, o_rho, rtol=RTOL[dtype])


def test_empty_input(engine):
    cn, cni, x = _block(np.float32)
    x = x[:0]
    status, cell, perm, start, plen = _grid_sort(engine, cn, cni, x)
    assert status == _capi.AL_OK
    assert start.max() == 0 and plen.max() == 0


def test_single_particle_and_duplicates(engine):
    cn, cni, x = _block(np.float32, dims=(4, 4, 4))
    one = x[:1].copy()
    status, rho, cnt, _, _ = _neighbors(engine, cn, cni, one)
    assert status == _capi.AL_OK and cnt[0] == 0
    np.testing.assert_allclose(rho[0], np.float32(cn.particle_vol * cn.cubic_kernel_zero *
                                                  cn.density0), rtol=1e-6)
    # coincident particles are neighbors of each other (d2 = 0 < h^2)
    two = np.repeat(x[:1], 2, axis=0)
    status, rho, cnt, nbrs, _ = _neighbors(engine, cn, cni, two)
    assert status == _capi.AL_OK and list(cnt) == [1, 1]


def test_out_of_grid_flag(engine):
    cn, cni, x = _block(np.float32, dims=(6, 6, 6), seed=2)
    x = x.copy()
    x[5] = (50.0, 50.0, 50.0)  # far outside the grid
    status, cell, perm, start, plen = _grid_sort(engine, cn, cni, x)
    assert status == _capi.AL_ERR_OUT_OF_GRID
    o_cell, o_perm, o_start, o_flags = orc.grid_sort(cn, cni, x)
    assert o_flags[0] == 1
    assert cell[5] == 0xffffffff and np.array_equal(cell, o_cell)
    inside = o_start[-1]
    assert np.array_equal(perm[:inside], o_perm[:inside])
    assert set(perm[inside:]) == set(o_perm[inside:])
    status, rho, cnt, _, anomaly = _neighbors(engine, cn, cni, x)
    assert status == _capi.AL_ERR_OUT_OF_GRID and anomaly[0] == 1
    assert cnt[5] == 0


def test_cell_overflow_flag(engine):
    cn, cni, x = _block(np.float32, dims=(6, 6, 6), seed=2)
    cni.max_num_particles_per_cell = 4  # ~8 per cell at rest density
    status, *_ = _grid_sort(engine, cn, cni, x)
    assert status == _capi.AL_ERR_CELL_OVERFLOW
    _, _, _, o_flags = orc.grid_sort(cn, cni, x)
    assert o_flags[1] == 1


@pytest.mark.parametrize("dtype", DTYPES)
def test_neighbor_overflow_truncates_canonically(engine, dtype):
    cn, cni, x = _block(dtype, dims=(6, 6, 6), seed=4)
    cni.max_num_neighbors_per_particle = 16
    status, rho, cnt, nbrs, anomaly = _neighbors(engine, cn, cni, x)
    assert status == _capi.AL_ERR_NEIGHBOR_OVERFLOW and anomaly[2] == 1
    o_rho, o_cnt, o_idx, _, o_flags = orc.update_particle_neighbors(cn, cni, x)
    assert o_flags[2] == 1
    assert np.array_equal(cnt, o_cnt) and cnt.max() == 16
    idx = _index_bits(nbrs, dtype)
    for i in range(len(x)):
        assert np.array_equal(idx[i, :cnt[i]], o_idx[i, :cnt[i]])
    np.testing.assert_allclose(rho, o_rho, rtol=RTOL[dtype])


def test_large_block_properties(engine):
    """At 262,144 particles (above the oracle's quick range for full lists):
    permutation is a bijection sorted by cell, counts match the oracle."""
    cn, cni, x = _block(np.float32, dims=(64, 64, 64), r=0.005, seed=1)
    status, cell, perm, start, plen = _grid_sort(engine, cn, cni, x)
    assert status == _capi.AL_OK
    assert np.array_equal(np.sort(perm), np.arange(len(x), dtype=np.uint32))
    sc = cell[perm]
    assert np.all(np.diff(sc.astype(np.int64)) >= 0)
    same = sc[1:] == sc[:-1]
    assert np.all(perm[1:][same] > perm[:-1][same])  # stable within a cell
    o_cell, o_perm, o_start, _ = orc.grid_sort(cn, cni, x)
    assert np.array_equal(perm, o_perm)


@pytest.mark.parametrize("dtype", DTYPES)
def test_periodic_neighbors_bit_exact(engine, dtype):
    """update_particle_neighbors<1>: a slab filling a period of 8 cells in y;
    lists (order, wrapped displacement bits) bit-exact against the oracle,
    and particles on both sides of the seam see each other."""
    r = 0.01
    cn = scenes.make_const(dtype, r)
    h = float(cn.kernel_radius)
    L = 8 * h
    x = scenes.fluid_block((6, 16, 6), (0.0, -L / 2 - 2 * r + 0.5 * r, 0.0), r, dtype, seed=9)
    cni = scenes.make_consti((0.0, -L / 2, 0.0), (0.15, L / 2, 0.15), h)
    cni.grid_offset[1] = -4
    cni.grid_res[1] = 8
    n, cap = len(x), cni.max_num_neighbors_per_particle
    xd = dev(x)
    rho = torch.zeros(n, dtype=xd.dtype, device="cuda")
    cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
    nbr = torch.zeros((n, cap, 4), dtype=xd.dtype, device="cuda")
    fn = getattr(_capi.lib(), "al_update_particle_neighbors_periodic_" + _capi.suffix(dtype))
    st = fn(engine.handle, ctypes.byref(cn), ctypes.byref(cni), _capi.ptr(xd), n, None,
            _capi.ptr(rho), _capi.ptr(cnt), _capi.ptr(nbr), None, ctypes.c_double(L), None)
    assert st == _capi.AL_OK
    o_rho, o_cnt, o_idx, o_nbrs, o_flags = orc.update_particle_neighbors(cn, cni, x,
                                                                        wrap_length=L)
    g_cnt = host(cnt).view(np.uint32)
    g_nbr = host(nbr)
    assert np.array_equal(g_cnt, o_cnt)
    idx = _index_bits(g_nbr, dtype)
    for i in range(n):
        c = g_cnt[i]
        assert np.array_equal(idx[i, :c], o_idx[i, :c]), i
        assert np.array_equal(g_nbr[i, :c, :3], o_nbrs[i, :c, :3]), i
    np.testing.assert_allclose(host(rho), o_rho, rtol=RTOL[dtype])
    # across the seam: the bottom layer's neighbours include top-layer particles,
    # at wrapped (small) displacements
    bottom = x[:, 1] < -L / 2 + 0.01
    top_ids = set(np.nonzero(x[:, 1] > L / 2 - 0.02)[0].tolist())
    i = int(np.nonzero(bottom)[0][len(np.nonzero(bottom)[0]) // 2])
    ids = set(idx[i, :g_cnt[i]].tolist())
    assert ids & top_ids
    assert np.abs(g_nbr[i, :g_cnt[i], 1]).max() < h


@pytest.mark.parametrize("crowd", [40, 300, 5000])
def test_crowded_cells_sorted_canonically(engine, crowd):
    """A cell holding many particles: 40 extra members (within the 64-member
    capacity of the per-thread ordering), 300 (the block-cooperative bitonic
    path) and 5000 (above its shared-memory size, one thread in place).  The
    permutation equals the oracle's canonical (cell, index) order; beyond
    the cell capacity the overflow is reported, as the reference's
    grid_anomaly[1]."""
    cn, cni, x = _block(np.float32, dims=(8, 8, 8), seed=5)
    h = float(cn.kernel_radius)
    corner = (np.floor(x[100] / h)) * h
    rng = np.random.default_rng(crowd)
    pile = (corner + rng.uniform(0.1 * h, 0.9 * h, size=(crowd, 3))).astype(np.float32)
    xs = np.concatenate([x, pile])
    xs = xs[rng.permutation(len(xs))]
    status, cell, perm, start, plen = _grid_sort(engine, cn, cni, xs)
    o_cell, o_perm, o_start, o_flags = orc.grid_sort(cn, cni, xs)
    assert np.array_equal(cell, o_cell)
    assert np.array_equal(start, o_start)
    assert np.array_equal(perm, o_perm)
    assert plen.max() >= crowd
    if plen.max() > cni.max_num_particles_per_cell:
        assert status == _capi.AL_ERR_CELL_OVERFLOW and o_flags[1] == 1
    else:
        assert status == _capi.AL_OK
