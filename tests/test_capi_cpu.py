"""CPU checks of the C ABI library: it builds, loads, and exports every
entry point include/alluvion_b200.h declares; host-side argument and device
checks return status codes instead of crashing (no GPU needed)."""
import ctypes
import os
import re

import pytest

from alluvion_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"^AL_API\s+[\w\s\*]+?\b(al_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    declared = header_functions()
    assert declared, "no AL_API declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    # the ctypes binding covers exactly the header
    assert set(_capi.declared_symbols()) == set(declared)


def test_status_strings():
    lib = _capi.lib()
    for code in _capi.STATUS:
        assert lib.al_status_string(code)


def test_engine_create_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    status = _capi.lib().al_engine_create(0, ctypes.byref(h))
    assert status == 8  # AL_ERR_NO_DEVICE
    assert not h.value
    assert _capi.lib().al_last_error()


def test_null_arguments_rejected():
    lib = _capi.lib()
    assert lib.al_grid_sort_f32(None, None, None, None, 0, None, None, None, None, None) == 2
    assert lib.al_engine_create(0, None) == 2


# ctypes mirror -> C typedef of include/alluvion_b200.h
ABI_STRUCTS = {
    "ConstF32": "al_const_f32", "ConstF64": "al_const_f64", "ConstI": "al_consti",
    "BodyF32": "al_body_f32", "BodyF64": "al_body_f64", "RigidF32": "al_rigid_f32",
    "RigidF64": "al_rigid_f64", "SolverParams": "al_solver_params",
    "StepReport": "al_step_report", "Fluid": "al_fluid_f32", "WarmNet": "al_warm_net",
    "WarmStart": "al_warm_start", "SceneF32": "al_scene_f32",
    "ContactBodyF32": "al_contact_body_f32", "ContactF32": "al_contact_f32",
    "SampleF32": "al_sample_f32", "SampleF64": "al_sample_f64", "PelletsF32": "al_pellets_f32",
    "PelletsF64": "al_pellets_f64", "PelletRelaxParams": "al_pellet_relax_params",
}


def test_ctypes_structs_match_the_header_layout(tmp_path):
    """Every ctypes mirror has the C struct's size and field offsets (gcc
    compiles a probe of sizeof / offsetof from the header)."""
    import subprocess
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "alluvion_b200.h"',
             'int main(void) {']
    for py, c in ABI_STRUCTS.items():
        cls = getattr(_capi, py)
        lines.append('  printf("%s size %%zu\\n", sizeof(%s));' % (py, c))
        for name, _ in cls._fields_:
            lines.append('  printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (py, name, c, name))
    lines += ['  return 0;', '}']
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for py in ABI_STRUCTS:
        cls = getattr(_capi, py)
        assert int(got["%s size" % py]) == ctypes.sizeof(cls), py
        for name, _ in cls._fields_:
            assert int(got["%s.%s" % (py, name)]) == getattr(cls, name).offset, (py, name)


def test_cpp_layer_compiles_and_maps_statuses(tmp_path):
    """include/alluvion_b200.hpp: compiles with g++ against the library; a
    failed engine creation throws alluvion_b200::error with the status; the
    capacity anomalies stay quiet unless asked (the reference reports its
    grid_anomaly flags without throwing)."""
    import subprocess
    import torch
    src = tmp_path / "shim.cpp"
    src.write_text(r"""
#include <cstdio>
#include "alluvion_b200.hpp"
namespace ab = alluvion_b200;
// every step template instantiates for both real types
template al_step_report ab::step<float>(const ab::engine&, ab::method, const al_const_f32&,
    const al_consti&, const al_fluid_f32&, const al_body_f32*, al_rigid_f32*,
    const al_solver_params&, float&, void*);
template al_step_report ab::step<double>(const ab::engine&, ab::method, const al_const_f64&,
    const al_consti&, const al_fluid_f64&, const al_body_f64*, al_rigid_f64*,
    const al_solver_params&, double&, void*);
template al_step_report ab::step_pellets<float>(const ab::engine&, const al_const_f32&,
    const al_consti&, const al_fluid_f32&, const al_body_f32*, al_rigid_f32*,
    const al_pellets_f32&, const al_solver_params&, float&, void*);
int main() {
  int created = -1;
  try {
    ab::engine e(0);
    created = 0;
  } catch (const ab::error& err) {
    created = err.status();
  }
  bool quiet = true, loud = false;
  try { ab::check(AL_ERR_NEIGHBOR_OVERFLOW, "x"); } catch (...) { quiet = false; }
  try { ab::check(AL_ERR_NEIGHBOR_OVERFLOW, "x", true); }
  catch (const ab::error& e) { loud = e.status() == AL_ERR_NEIGHBOR_OVERFLOW; }
  int invalid = 0;
  try { ab::check(AL_ERR_INVALID, "y"); } catch (const ab::error& e) { invalid = e.status(); }
  std::printf("%d %d %d %d\n", created, int(quiet), int(loud), invalid);
  return 0;
}
""")
    exe = tmp_path / "shim"
    libdir = os.path.dirname(_capi.lib()._name)
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src),
                    "-L", libdir, "-lalluvion_b200", "-Wl,-rpath," + libdir, "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    created, quiet, loud, invalid = map(int, out)
    assert created == (0 if torch.cuda.is_available() else 8)
    assert quiet == 1 and loud == 1 and invalid == 2
