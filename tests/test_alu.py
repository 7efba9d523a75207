"""Checkpoint formats (alluvion_b200/alu.py) against the byte layouts of
Variable::write_file / read_file (variable.hpp:132-262) and Pile::write_file
/ read_file (pile.hpp:757-793), built here byte by byte."""
import struct

import numpy as np
import pytest

from alluvion_b200 import alu


def test_alu_bytes_match_reference_layout(tmp_path):
    # a Variable<2, float3> of shape (4, 5): header 4, 5, 0, 3, 'f', data
    a = np.arange(4 * 5 * 3, dtype=np.float32).reshape(4, 5, 3)
    path = tmp_path / "x.alu"
    alu.write_alu(path, a, primitives_per_element=3)
    raw = path.read_bytes()
    assert raw[:16] == struct.pack("<4I", 4, 5, 0, 3)
    assert raw[16:17] == b"f"
    assert raw[17:] == a.tobytes()
    back = alu.read_alu(path, dims=2)
    assert back.dtype == np.float32 and np.array_equal(back, a)


def test_alu_prefix_and_scalar(tmp_path):
    a = np.arange(10, dtype=np.uint32)
    path = tmp_path / "u.alu"
    alu.write_alu(path, a, shape_outermost=6)
    raw = path.read_bytes()
    assert raw[:12] == struct.pack("<3I", 6, 0, 1) and raw[12:13] == b"u"
    assert np.array_equal(alu.read_alu(path), a[:6])
    with pytest.raises(alu.AluError):
        alu.write_alu(path, a, shape_outermost=11)


def test_alu_float_double_conversion_and_errors(tmp_path):
    a = np.linspace(0, 1, 7)
    path = tmp_path / "d.alu"
    alu.write_alu(path, a)
    assert path.read_bytes()[12:13] == b"d"
    f = alu.read_alu(path, dtype=np.float32)
    assert f.dtype == np.float32 and np.allclose(f, a)
    with pytest.raises(alu.AluError):
        alu.read_alu(path, dtype=np.int32)
    with pytest.raises(alu.AluError):
        alu.read_alu(path, dims=2)
    with pytest.raises(alu.AluError):
        alu.read_alu(tmp_path / "missing.alu")


def test_pile_state_round_trip(tmp_path):
    rng = np.random.Generator(np.random.PCG64(1))
    r = rng.normal(size=(3, 13)).astype(np.float32)
    path = tmp_path / "pile.bin"
    alu.write_pile(path, r, x_scale=2.0)
    raw = path.read_bytes()
    assert len(raw) == 3 * 13 * 4 and alu.pile_size(path) == 3
    # per body: x * 2, v, q, omega in float32
    first = np.frombuffer(raw[:52], np.float32)
    assert np.allclose(first[:3], 2 * r[0, :3]) and np.array_equal(first[3:], r[0, 3:])
    back = alu.read_pile(path, num_rigids=2, src_offset=1)
    assert back.shape == (2, 13) and np.array_equal(back[0, 3:], r[1, 3:])
