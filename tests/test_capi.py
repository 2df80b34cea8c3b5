"""C-ABI checks that need no GPU: the library loads, exports every entry point include/*.h declares,
reports the reference defaults, and refuses to run without a CUDA device (no CPU fallback)."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from slosh_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names += re.findall(r"SLOSH_API\s+[\w\s\*]+?\b(slosh_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(slosh):
    lib_path = slosh.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT\s+(slosh_\w+)", out))
    declared = declared_functions()
    assert declared, "no declarations found"
    missing = [n for n in declared if n not in exported]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(slosh.SIGNATURES) == set(declared)
    lib = slosh.load_library()
    for n in declared:
        assert hasattr(lib, n)


def test_abi_version_and_struct_sizes(slosh):
    lib = slosh.load_library()
    assert lib.slosh_abi_version() == 3
    assert C.sizeof(A.Particle) == 48
    assert C.sizeof(A.Collider) == 80
    assert C.sizeof(A.Manipulator) == 80


def test_defaults_are_the_reference_defaults(slosh, oracle_mod):
    """FSloshSolverSettings defaults (SloshTypes.h:113-160)."""
    s = slosh.settings_default()
    o = oracle_mod.settings_default()
    assert bytes(s) == bytes(o)
    assert list(s.grid_dim) == [64, 64, 48]
    assert s.cell_size == pytest.approx(0.05)
    assert s.particle_capacity == 262144
    assert s.transfer_mode == A.TRANSFER_APIC
    assert s.flip_ratio == pytest.approx(0.95)
    assert s.pressure_solver == A.SOLVER_MGPCG
    assert (s.pressure_iterations, s.pcg_iterations, s.mg_coarse_iterations) == (60, 8, 16)
    assert s.sor_weight == pytest.approx(1.7)
    assert (s.sort_interval, s.extrapolation_layers, s.min_substeps, s.max_substeps) == (4, 2, 1, 4)
    assert s.cfl == pytest.approx(2.0)
    assert list(s.gravity) == pytest.approx([0.0, 0.0, -9.81])
    assert s.two_sided_density_projection == 1 and s.ghost_fluid == 1
    assert s.density_relaxation == pytest.approx(0.5)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_loudly(slosh):
    s = slosh.settings_default()
    with pytest.raises(slosh.SloshError) as e:
        slosh.Simulation(s)
    assert e.value.status == A.ERR_NO_DEVICE


def test_invalid_arguments_are_rejected(slosh):
    lib = slosh.load_library()
    assert lib.slosh_get_results(None, None) == A.ERR_INVALID_ARG
    assert lib.slosh_step_frame(None, None) == A.ERR_INVALID_ARG
    assert b"NULL" in lib.slosh_last_error_string()
    ctx = C.c_void_p()
    assert lib.slosh_create(None, 0, C.byref(ctx)) == A.ERR_INVALID_ARG
