"""GPU parity of the paths the default scene does not exercise, each against the oracle, state compared
after every substep (bit-exact; 1e-5 relative L2 is the stated float tolerance): FLIP transfer, viscosity,
manipulators and drains, sphere/box emission with velocity spread and speed jitter, one-sided density
correction, warm start from zero, the dense (non-sparse) pool, red-black SOR on a sparse scene large
enough to use every pool path, and two-way collider coupling (the per-collider integer accumulators and
their decoded feedback)."""
import os

import numpy as np
import pytest

from slosh_b200 import _abi as A
from slosh_b200 import scenes

from parity import pair, run_frames

pytestmark = pytest.mark.gpu


def _manip(kind, shape, center, extent=(0.2, 0.2, 0.2), axis=(0.0, 1.0, 0.0), strength=5.0, falloff=0.1,
           param0=0.0, param1=0.0):
    m = A.Manipulator()
    m.center[:] = list(center)
    m.kind = kind
    m.rotation[:] = [0.0, 0.0, 0.0, 1.0]
    m.extent[:] = list(extent)
    m.shape = shape
    m.axis[:] = list(axis)
    m.strength = strength
    m.falloff = falloff
    m.param0 = param0
    m.param1 = param1
    return m


def _emit(shape, center, extent, velocity, count, spread=0.3, jitter=0.2):
    e = A.EmitRequest()
    e.shape = shape
    e.center[:] = list(center)
    e.extent[:] = list(extent)
    e.velocity[:] = list(velocity)
    e.rotation[:] = [0.0, 0.38268343, 0.0, 0.92387953]
    e.velocity_spread = spread
    e.speed_jitter = jitter
    e.count = count
    e.fill_jitter = 0.8
    return e


def test_flip_transfer(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=16)
    sc["settings"].transfer_mode = A.TRANSFER_FLIP
    sc["settings"].flip_ratio = 0.95
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=4)


def test_viscosity(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=16)
    sc["settings"].kinematic_viscosity = 0.05
    sc["settings"].viscosity_iterations = 4
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=4)


def test_manipulators_and_drain(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24)
    sc["manipulators"] = [
        _manip(A.MANIP_DIRECTIONAL, A.SHAPE_SPHERE, (0.25, 0.3, 0.5), extent=(0.15, 0, 0), axis=(1.0, 0.0, 0.0)),
        _manip(A.MANIP_RADIAL, A.SHAPE_BOX, (0.6, 0.2, 0.5), extent=(0.1, 0.1, 0.3), strength=-3.0),
        _manip(A.MANIP_SWIRL, A.SHAPE_EVERYWHERE, (0.5, 0.5, 0.5), axis=(0.0, 1.0, 0.0), strength=2.0, param0=0.5),
        _manip(A.MANIP_DRAG, A.SHAPE_CAPSULE, (0.3, 0.2, 0.5), extent=(0.08, 0.2, 0), strength=4.0),
        _manip(A.MANIP_DRAIN, A.SHAPE_BOX, (0.1, 0.08, 0.5), extent=(0.08, 0.06, 0.2), param0=20.0),
    ]
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=5)
    assert g.results().drained_particles == o.results().drained_particles


def test_sphere_and_box_emission(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24)
    sc["settings"].particle_capacity = sc["particles"] + 20000
    sc["emits"] = list(sc["emits"]) + [
        _emit(A.EMIT_SPHERE, (0.7, 0.7, 0.5), (0.12, 0, 0), (0.0, -1.5, 0.3), 6000),
        _emit(A.EMIT_BOX, (0.75, 0.35, 0.4), (0.08, 0.05, 0.1), (-0.5, 0.0, 0.0), 5000, spread=0.0, jitter=0.5),
    ]
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=4)


def test_one_sided_density_correction(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=16)
    sc["settings"].two_sided_density_projection = 0
    sc["settings"].density_correction = 0.15
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=4)


def test_warm_start_zero(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=16)
    sc["settings"].warm_start = A.WARM_START_ZERO
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=3)


def test_dense_pool(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24)
    sc["settings"].sparse_bricks = 0
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=3)


def test_rbgs_sparse_scene(slosh, oracle_mod):
    sc = scenes.dam_break_sphere(slosh.settings_default, n=64, solver=A.SOLVER_RBGS, sor_iterations=60)
    sc["settings"].max_substeps = 16
    run_frames(*pair(slosh, oracle_mod, sc), sc, frames=2)


def _collider(ctype, center, extent, two_way=True, velocity=(0.0, 0.0, 0.0), spin=(0.0, 0.0, 0.0)):
    c = A.Collider()
    c.center[:] = list(center)
    c.type = ctype
    c.rotation[:] = [0.0, 0.0, 0.0, 1.0]
    c.extent[:] = list(extent)
    c.flags = 1 if two_way else 0
    c.linear_velocity[:] = list(velocity)
    c.angular_velocity[:] = list(spin)
    return c


@pytest.mark.parametrize("smooth", [1, 0])
def test_two_way_coupling(slosh, oracle_mod, smooth):
    sc = scenes.tiny(slosh.settings_default, n=24)
    sc["settings"].smooth_coupling_force = smooth
    sc["colliders"] = [
        _collider(A.COLLIDER_SPHERE, (0.25, 0.22, 0.5), (0.09, 0.0, 0.0), spin=(0.0, 0.0, 1.0)),
        _collider(A.COLLIDER_BOX, (0.55, 0.12, 0.5), (0.07, 0.09, 0.12), velocity=(0.1, 0.0, 0.0)),
        _collider(A.COLLIDER_CAPSULE, (0.3, 0.4, 0.3), (0.05, 0.1, 0.0), two_way=False),
    ]
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=4)
    acc = g.read("COUPLING").reshape(A.MAX_COLLIDERS, -1)
    assert np.any(acc[0, :6] != 0) and acc[0, 6] > 0, "the submerged sphere collected no force or wetted faces"
    assert acc[0, 11] > 0 and acc[1, 11] > 0, "solid cells of the two-way bodies were not counted"
    assert not np.any(acc[2, :7]) and not np.any(acc[2, 8:11]), "a one-way collider received coupling terms"


def test_step_frames_matches_individual_frames(slosh):
    """slosh_step_frames overlaps several tanks on the device; every tank must end bit-identical to the
    same tank stepped alone with slosh_step_frame."""
    tanks = scenes.tank_batch(slosh.settings_default, count=3, lo=16, hi=28)
    batch = [slosh.Simulation(t["settings"]) for t in tanks]
    alone = [slosh.Simulation(t["settings"]) for t in tanks]
    for sims in (batch, alone):
        for sim, t in zip(sims, tanks):
            sim.set_emit_seed(t["seed"])
    for f in range(4):
        fis = [A.frame_input(t["settings"], emits=t["emits"] if f == 0 else ()) for t in tanks]
        st = slosh.step_frames(batch, fis)
        assert all(s in (A.OK,) + A.WARNINGS for s in st)
        for sim, fi in zip(alone, fis):
            sim.step_frame(fi)
    for a, b in zip(batch, alone):
        assert np.array_equal(a.particles().view(np.uint32), b.particles().view(np.uint32))
        assert np.array_equal(a.read("PRESSURE").view(np.uint32), b.read("PRESSURE").view(np.uint32))
        assert a.results().substeps == b.results().substeps


@pytest.mark.parametrize("mode", [A.PRECISION_FP16_STORAGE, A.PRECISION_BF16_STORAGE])
@pytest.mark.parametrize("n", [64, 96])
def test_coarse_storage_precision(slosh, oracle_mod, mode, n):
    """FP16 / BF16 storage of the V-cycle's coarse levels: bit-exact against the oracle run at the same
    storage precision, and the solve still reaches its tolerance."""
    sc = scenes.dam_break_sphere(slosh.settings_default, n=n)
    sc["settings"].max_substeps = 16
    sc["settings"].precision_mode = mode
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=2)
    r = g.results()
    assert r.last_solve_rel_residual <= 1e-6


def test_launch_shape_does_not_change_results(slosh):
    """The brick passes' grid size (CTAs per SM, chosen by slosh_autotune) changes only speed: a scene
    stepped with 2 and with 16 CTAs per SM ends bit-identical; the autotuner reports every candidate
    and keeps one of them."""
    sc = scenes.dam_break_sphere(slosh.settings_default, n=96)
    runs = []
    for per_sm in (2, 16):
        sim = slosh.Simulation(sc["settings"])
        sim.set_emit_seed(sc["seed"])
        sim.set_ctas_per_sm(per_sm)
        sim.step_frame(A.frame_input(sc["settings"], emits=sc["emits"]))
        for _ in range(2):
            sim.step_frame(A.frame_input(sc["settings"]))
        runs.append((sim.particles().view(np.uint32).copy(), sim.read("PRESSURE").view(np.uint32).copy()))
        if per_sm == 16:
            r = sim.autotune(A.frame_input(sc["settings"]), frames=1)
            assert r.num_candidates == 5 and r.best_ctas_per_sm in list(r.ctas_per_sm)[:5]
            assert all(r.ms_per_substep[k] > 0 for k in range(5))
        sim.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


@pytest.mark.parametrize("scale,sweeps,flexible,mode,weight", [
    (1.7, 1, 0, A.PRECISION_FP32, 1.0),
    (1.7, 2, 1, A.PRECISION_FP32, 1.0),
    (1.0, 3, 1, A.PRECISION_FP32, 1.0),
    (1.9, 1, 1, A.PRECISION_BF16_STORAGE, 1.0),
    (1.9, 2, 0, A.PRECISION_FP32, 1.15),
    (1.9, 1, 0, A.PRECISION_FP32, 1.3),
    (1.7, 3, 1, A.PRECISION_FP16_STORAGE, 1.15),
])
def test_preconditioner_options(slosh, oracle_mod, scale, sweeps, flexible, mode, weight):
    """The multigrid preconditioner's options (coarse-grid correction scale, red-black sweep pairs per
    smoothing, flexible PCG, over-relaxation of the finest level's sweeps, with FP32, BF16 and FP16 coarse
    storage) on a 96^3 sparse scene whose hierarchy uses footprint levels, the shared-memory tail and the
    coarsest solve: bit-exact against the oracle run with the same options, every solve to its tolerance. One
    sweep pair with over-relaxation makes the first red sweep after the prolongation the one that also forms
    rho."""
    sc = scenes.dam_break_sphere(slosh.settings_default, n=96)
    s = sc["settings"]
    s.max_substeps = 16
    s.mg_correction_scale = scale
    s.mg_smoothing_sweeps = sweeps
    s.pcg_flexible = flexible
    s.precision_mode = mode
    s.mg_smoother_weight = weight
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=2)
    assert g.results().last_solve_rel_residual <= 1e-6


def test_gather_p2g_matches_oracle():
    """P2G as a per-brick gather (SLOSH_P2G_GATHER=1, read once per process: a per-cell particle index, then one CTA
    per brick over the particles of its cells and of the one-cell layer around it, no global atomics): the parity
    tests that reach P2G's edge cases run in a child process on the gather path, bit-exact against the oracle --
    bricks cut by the grid's faces (100^3), particles left in unallocated bricks (pool overflow), colliders, the
    64^3 dam break, the RBGS and MGPCG tiny scenes."""
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sel = "tiny_dam_break or sparse_sphere or pool_overflow or collider or dam_break_64 or emission"
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "gpu", "-p", "no:cacheprovider",
                        os.path.join(here, "test_gpu_parity.py"), "-k", sel],
                       env=dict(os.environ, SLOSH_P2G_GATHER="1"), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and " failed" not in r.stdout, r.stdout[-2000:]


@pytest.mark.parametrize("env", [{"SLOSH_MG_STAGED": "1"}, {"SLOSH_MG_CLUSTER": "2"}, {"SLOSH_PDL": "0"}],
                         ids=["staged_level0", "cluster_levels", "no_pdl"])
def test_alternative_solver_paths_give_identical_results(slosh, env):
    """The MGPCG solve has measured alternatives, each read once per process from the environment: level-0 passes
    that read their bricks from shared-memory stages filled by bulk async copies (SLOSH_MG_STAGED=1), levels 2 to
    the tail in one thread-block cluster (SLOSH_MG_CLUSTER=2) and plain stream order instead of programmatic
    dependent launch (SLOSH_PDL=0). A 96^3 scene (levels 2 and 3 below the tail) stepped in a child process with
    the alternative must end bit-identical to the default path here."""
    import subprocess
    import sys
    code = (
        "import sys, numpy as np\n"
        "sys.path.insert(0, %r)\n"
        "import slosh_b200 as S\n"
        "from slosh_b200 import _abi as A, scenes\n"
        "sc = scenes.dam_break_sphere(S.settings_default, n=96)\n"
        "s = sc['settings']; s.max_substeps = 16; s.mg_correction_scale = 1.9; s.mg_smoothing_sweeps = 2\n"
        "sim = S.Simulation(s); sim.set_emit_seed(sc['seed'])\n"
        "sim.step_frame(A.frame_input(s, emits=sc['emits']))\n"
        "for _ in range(2): sim.step_frame(A.frame_input(s))\n"
        "np.save(sys.argv[1], np.concatenate([sim.particles().view(np.uint32).ravel(), sim.read('PRESSURE').view(np.uint32)]))\n"
    ) % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),)
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "alt.npy")
        r = subprocess.run([sys.executable, "-c", code, out], env=dict(os.environ, **env), capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        alt = np.load(out)
    sc = scenes.dam_break_sphere(slosh.settings_default, n=96)
    s = sc["settings"]
    s.max_substeps = 16
    s.mg_correction_scale = 1.9
    s.mg_smoothing_sweeps = 2
    sim = slosh.Simulation(s)
    sim.set_emit_seed(sc["seed"])
    sim.step_frame(A.frame_input(s, emits=sc["emits"]))
    for _ in range(2):
        sim.step_frame(A.frame_input(s))
    plain = np.concatenate([sim.particles().view(np.uint32).ravel(), sim.read("PRESSURE").view(np.uint32)])
    sim.close()
    assert np.array_equal(alt, plain)
