"""GPU parity at the benchmark configurations themselves (not only at reduced sizes): the CUDA substep
against the CPU oracle on the same seeded scenes, whole state compared bit for bit (1e-5 relative L2 is
the stated float tolerance).

* 64^3 dam break (471,200 particles): 100 substeps, each compared.
* 256^3 dam break + falling sphere (20,583,872 particles): the emission frame's first two substeps,
  compared after each, with the benchmark's hierarchy (6 MG levels) and pool (> 6,000 active bricks).
* 512 x 256 x 256 boxes with static collider spheres (34.5 M particles): the first substep with FP32 and
  with BF16 storage of the coarse levels, each against the oracle at the same storage precision, plus
  the error of that substep's pressure and face velocity against the FP64 oracle and the final relative
  residual of its solve.

The scenes restate the reference's demo scenes (SloshDemo/Source/SloshDemo/SloshDemoGameMode.cpp:90-293)
as seeded generators; each substep follows Step_RenderThread (SloshProxy.cpp:339-737)."""
import numpy as np
import pytest

from slosh_b200 import _abi as A
from slosh_b200 import scenes

from parity import active_slots, compare_state, pair, run_frames, slot_mask

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

FLOAT_TOL = 1e-5


def _substeps_compared(g, o, sc, count, fi):
    """Begins one frame on both sides and compares the whole state after each of its first `count` substeps."""
    ng, dtg = g.begin_frame(fi)
    no, dto = o.begin_frame(fi)
    assert (ng, dtg) == (no, dto)
    assert ng >= count
    for s in range(count):
        g.substep(s)
        o.substep(s)
        r = compare_state(g, o)
        bad = r.failures(FLOAT_TOL)
        assert not bad, f"substep {s}:\n{r}"


def test_dam_break_64_100_substeps(slosh, oracle_mod):
    sc = scenes.dam_break(slosh.settings_default, n=64)
    assert sc["particles"] == 471200
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=200, tol=FLOAT_TOL, substeps=100)
    assert g.results().last_solve_rel_residual <= 1e-6


def test_dam_break_sphere_256_first_substeps(slosh, oracle_mod):
    sc = scenes.dam_break_sphere(slosh.settings_default, n=256)
    sc["settings"].max_substeps = 16
    assert sc["particles"] == 20583872
    g, o = pair(slosh, oracle_mod, sc)
    assert g.layout().num_mg_levels == 6
    _substeps_compared(g, o, sc, 2, A.frame_input(sc["settings"], emits=sc["emits"]))
    assert int(g.read("ACTIVE_BRICKS")[0]) > 6000
    g.close()
    o.close()


@pytest.mark.parametrize("mode", [A.PRECISION_FP32, A.PRECISION_BF16_STORAGE])
def test_boxes_512_first_substep(slosh, oracle_mod, mode):
    sc = scenes.boxes_512(slosh.settings_default)
    sc["settings"].precision_mode = mode
    g, o = pair(slosh, oracle_mod, sc)
    fi = A.frame_input(sc["settings"], emits=sc["emits"], colliders=sc["colliders"])
    ng, dtg = g.begin_frame(fi)
    no, dto = o.begin_frame(fi)
    assert (ng, dtg) == (no, dto)
    o64 = oracle_mod.Oracle(o.settings, fp64=True)
    o64.copy_state_from(o)
    g.substep(0)
    o.substep(0)
    o64.substep(0)
    r = compare_state(g, o)
    assert not r.failures(FLOAT_TOL), str(r)
    g.end_frame()  # the frame epilogue reads the solve's statistics back
    res = g.results()
    assert res.last_solve_rel_residual <= 1e-6
    # error of the FP32-arithmetic step against the FP64 oracle of the same step (same starting state)
    L = g.layout()
    slots = active_slots(o)
    errs = {}
    for name, planes in (("PRESSURE", 1), ("VEL", 3)):
        m = slot_mask(slots, L.pool_cells, planes)
        ref = o64.read_f64(name)[m]
        got = g.read(name)[m].astype(np.float64)
        errs[name] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    print(f"boxes_512 precision {mode}: iterations {res.last_solve_iterations}, final relative residual "
          f"{res.last_solve_rel_residual:.3e}, pressure rel L2 vs FP64 {errs['PRESSURE']:.3e}, velocity {errs['VEL']:.3e}")
    assert errs["PRESSURE"] < 1e-4, errs
    assert errs["VEL"] < 1e-5, errs
    o64.close()
    o.close()
    g.close()
