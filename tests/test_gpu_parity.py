"""GPU parity: the CUDA substep against the CPU oracle on the same seeded scenes, step by step.

Bar: particles, permutation, brick tables, cell types, flags and stats bit-exact; floating buffers
bit-exact as well (same FP32 operation order on both sides), with 1e-5 relative L2 as the stated
tolerance should a single rounding ever differ."""
import numpy as np
import pytest

from slosh_b200 import _abi as A
from slosh_b200 import scenes

from parity import compare_state, pair, run_frames

pytestmark = pytest.mark.gpu

FLOAT_TOL = 1e-5  # stated float tolerance (relative L2); the states match bit for bit


def _pair(slosh, oracle_mod, sc):
    return pair(slosh, oracle_mod, sc)


def _run_frames(g, o, sc, frames, check_every_substep=True):
    return run_frames(g, o, sc, frames, check_every_substep, FLOAT_TOL)


def test_emission_bit_exact(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=16)
    g, o = _pair(slosh, oracle_mod, sc)
    for e in sc["emits"]:
        g.emit(e)
        o.emit(e)
    pg, po = g.particles(), o.read("PARTICLES")
    assert len(pg) == len(po) == sc["particles"]
    assert np.array_equal(pg.view(np.uint32), po.view(np.uint32))
    assert np.array_equal(g.read("BRICK_TOUCH"), o.read("BRICK_TOUCH"))


def test_sort_permutation_bit_exact(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=32)
    g, o = _pair(slosh, oracle_mod, sc)
    rng = np.random.default_rng(7)
    n = 20000
    p = np.zeros(n, dtype=A.PARTICLE_DTYPE)
    p["pos"] = rng.uniform(0.0, 1.0, size=(n, 3)).astype(np.float32)
    p["age"] = np.where(rng.uniform(size=n) < 0.1, -1.0, 0.5).astype(np.float32)
    p["vel"] = rng.normal(size=(n, 3)).astype(np.float32)
    g.upload_particles(p)
    o.upload_particles(p)
    g.sort_particles()
    o.sort_particles()
    assert np.array_equal(g.read("SORT_PERM"), o.read("SORT_PERM"))
    assert np.array_equal(g.read("SORT_COUNTS"), o.read("SORT_COUNTS"))
    assert np.array_equal(g.read("SORT_OFFSETS"), o.read("SORT_OFFSETS"))
    assert np.array_equal(g.read("PARTICLE_COUNT")[0], o.read("PARTICLE_COUNT")[0])
    assert np.array_equal(g.read("PARTICLES").view(np.uint32), o.read("PARTICLES").view(np.uint32))


@pytest.mark.parametrize("solver", [A.SOLVER_MGPCG, A.SOLVER_RBGS])
def test_tiny_dam_break_substeps(slosh, oracle_mod, solver):
    sc = scenes.tiny(slosh.settings_default, n=16, solver=solver)
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=6)


def test_tiny_over_relaxed_smoother(slosh, oracle_mod):
    """The over-relaxed finest smoother on a hierarchy of only a few small levels (the tail and the coarsest
    solve right below level 0), one sweep pair: bit-exact against the oracle."""
    sc = scenes.tiny(slosh.settings_default, n=16)
    sc["settings"].mg_smoother_weight = 1.3
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=4)


@pytest.mark.parametrize("n,tuned", [(64, False), (96, False), (100, True)])
def test_sparse_sphere_coarse_levels(slosh, oracle_mod, n, tuned):
    """Sparse dam break + falling sphere large enough that MGPCG visits coarse levels through the
    active bricks' footprints (64^3: levels 1 and the single-CTA tail from level 2; 96^3: levels 1-2,
    tail from level 3; 100^3: bricks cut by the grid's faces, so the footprint walks meet cells outside the
    grid), bit-exact substep by substep; 100^3 with the benchmark's preconditioner (correction scale 1.9, two
    sweep pairs, 4 coarsest iterations, finest sweeps over-relaxed by 1.15)."""
    sc = scenes.dam_break_sphere(slosh.settings_default, n=n)
    sc["settings"].max_substeps = 16
    if tuned:
        s = sc["settings"]
        s.mg_correction_scale, s.mg_smoothing_sweeps, s.mg_coarse_iterations, s.mg_smoother_weight = 1.9, 2, 4, 1.15
    g, o = _pair(slosh, oracle_mod, sc)
    assert g.layout().num_mg_levels >= 4
    _run_frames(g, o, sc, frames=2)


def test_dam_break_64_per_substep(slosh, oracle_mod):
    """The 64^3 dam break (cells [1,26) x [1,39) x [1,63), 8 per cell: 471,200 particles), APIC, MGPCG to
    1e-6, g = -9.81 y, CFL 1, frame dt 1/120: bit-exact after every substep for 4 frames."""
    sc = scenes.dam_break(slosh.settings_default, n=64)
    assert sc["particles"] == 471200
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=4)


def test_tiny_with_collider(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24, colliders=True)
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=5)


def test_fp64_error(slosh, oracle_mod):
    """The GPU result's error against the FP64 oracle of the same substep (same starting state)."""
    from test_oracle_pins import fp64_step_errors
    sc = scenes.tiny(slosh.settings_default, n=24)
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=3, check_every_substep=False)
    fi = A.frame_input(sc["settings"])
    g.begin_frame(fi)
    errs = fp64_step_errors(oracle_mod, o, fi, extra=g)
    assert errs[("gpu", "PRESSURE")] == errs[("oracle32", "PRESSURE")]  # bit-exact FP32 on both sides
    assert errs[("gpu", "PRESSURE")] < 1e-4, errs
    assert errs[("gpu", "VEL")] < 1e-5, errs


def test_pool_overflow_parity_and_status(slosh, oracle_mod):
    """Injected pool exhaustion (storage budget below what the liquid needs): bricks left on the null
    brick move ballistically, the overflow is counted, and the frame reports SLOSH_WARN_POOL_OVERFLOW."""
    sc = scenes.tiny(slosh.settings_default, n=32)
    sc["settings"].sparse_storage_budget = 0.2
    g, o = _pair(slosh, oracle_mod, sc)
    fi = A.frame_input(sc["settings"], emits=sc["emits"])
    rc = g.step_frame(fi)
    o.step_frame(fi)
    assert rc == A.WARN_POOL_OVERFLOW
    assert g.results().pool_overflow_bricks > 0
    assert g.results().pool_overflow_bricks == o.results().pool_overflow_bricks
    fi = A.frame_input(sc["settings"])
    for _ in range(3):
        g.step_frame(fi)
        o.step_frame(fi)
        r = compare_state(g, o)
        assert not r.failures(FLOAT_TOL), str(r)


def test_iteration_cap_reports_not_converged(slosh, oracle_mod):
    """Injected non-convergence (tolerance far below reach with a 3-iteration cap)."""
    sc = scenes.tiny(slosh.settings_default, n=16, tolerance=1e-12)
    sc["settings"].max_iterations = 3
    g, o = _pair(slosh, oracle_mod, sc)
    fi = A.frame_input(sc["settings"], emits=sc["emits"])
    rc = g.step_frame(fi)
    o.step_frame(fi)
    assert rc == A.ERR_NOT_CONVERGED
    assert g.results().last_solve_iterations == 3 == o.results().last_solve_iterations
    r = compare_state(g, o)
    assert not r.failures(FLOAT_TOL), str(r)


def test_fixed_iteration_mode_matches_reference_semantics(slosh, oracle_mod):
    """tolerance <= 0: the reference's fixed PCGIterations (8) and no stopping test."""
    sc = scenes.tiny(slosh.settings_default, n=16, tolerance=0.0)
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=3)
    assert g.results().last_solve_iterations == 8
