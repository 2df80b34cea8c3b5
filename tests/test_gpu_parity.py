"""GPU parity: the CUDA substep against the CPU oracle on the same seeded scenes, step by step.

Bar: particles, permutation, brick tables, cell types, flags and stats bit-exact; floating buffers
bit-exact as well (same FP32 operation order on both sides), with 1e-5 relative L2 as the stated
tolerance should a single rounding ever differ."""
import numpy as np
import pytest

from slosh_b200 import _abi as A
from slosh_b200 import scenes

from parity import compare_state

pytestmark = pytest.mark.gpu

FLOAT_TOL = 1e-5


def _pair(slosh, oracle_mod, sc):
    g = slosh.Simulation(sc["settings"])
    o = oracle_mod.Oracle(sc["settings"])
    g.set_emit_seed(sc["seed"])
    o.set_emit_seed(sc["seed"])
    return g, o


def _run_frames(g, o, sc, frames, check_every_substep=True):
    fi = A.frame_input(sc["settings"], emits=sc["emits"], colliders=sc.get("colliders", []))
    reports = []
    for f in range(frames):
        ng, dtg = g.begin_frame(fi)
        no, dto = o.begin_frame(fi)
        assert (ng, dtg) == (no, dto), f"frame {f}: substeps/dt differ {ng, dtg} vs {no, dto}"
        for s in range(ng):
            g.substep(s)
            o.substep(s)
            if check_every_substep:
                r = compare_state(g, o)
                bad = r.failures(FLOAT_TOL)
                assert not bad, f"frame {f} substep {s}:\n{r}"
                reports.append(r)
        g.end_frame()
        o.end_frame()
        rg, ro = g.results(), o.results()
        assert rg.fluid_cells == ro.fluid_cells
        assert rg.max_particle_speed == ro.max_particle_speed
        assert rg.last_solve_iterations == ro.last_solve_iterations
        fi = A.frame_input(sc["settings"], colliders=sc.get("colliders", []))
    return reports


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


def test_tiny_with_collider(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24, colliders=True)
    g, o = _pair(slosh, oracle_mod, sc)
    _run_frames(g, o, sc, frames=5)
