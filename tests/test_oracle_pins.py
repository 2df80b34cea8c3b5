"""Pins of the CPU oracle against independent computations (CPU only).

The reference has no unit tests or golden vectors and its HLSL cannot run here, so the oracle is pinned
by checks that do not share its code: numpy's IEEE float16 conversion, an independent restatement of
the PCG hash, numpy's stable argsort, scipy's direct sparse solve of the assembled pressure system,
analytic P2G weight sums and a hydrostatic pool."""
import ctypes as C

import numpy as np
import pytest

from slosh_b200 import _abi as A
from slosh_b200 import scenes


def test_f16_rounding_matches_numpy(oracle_mod):
    lib = oracle_mod.lib()
    rng = np.random.default_rng(0)
    vals = np.concatenate([
        rng.normal(scale=s, size=4000).astype(np.float32) for s in (1e-6, 1e-4, 1e-2, 1.0, 100.0, 3e4)
    ] + [np.array([0.0, -0.0, 65000.0, -65000.0, 65504.0, 65519.0, 65520.0, 5.96e-8, 2.98e-8, 1e-30, 6.1e-5],
                  dtype=np.float32)])
    # exact ties between halves
    h = np.arange(0, 0x7BFF, 37, dtype=np.uint16).view(np.float16).astype(np.float32)
    nxt = (np.arange(0, 0x7BFF, 37, dtype=np.uint16) + 1).view(np.float16).astype(np.float32)
    vals = np.concatenate([vals, ((h.astype(np.float64) + nxt) / 2).astype(np.float32)])
    mine = np.array([lib.oracle_f32_to_f16(float(v)) for v in vals], dtype=np.uint16)
    ref = vals.astype(np.float16).view(np.uint16)
    assert np.array_equal(mine, ref)


def test_f16_to_f32_all_halves(oracle_mod):
    lib = oracle_mod.lib()
    hs = np.arange(65536, dtype=np.uint32)
    finite = (hs & 0x7C00) != 0x7C00
    mine = np.array([lib.oracle_f16_to_f32(int(x)) for x in hs[finite]], dtype=np.float32)
    ref = hs[finite].astype(np.uint16).view(np.float16).astype(np.float32)
    assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))


def _pcg_hash_py(v):
    # PCG-RXS-M-XS 32/32 as published by Jarzynski & Olano (JCGT 2020), restated independently.
    M = 0xFFFFFFFF
    state = (v * 747796405 + 2891336453) & M
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M
    return ((word >> 22) ^ word) & M


def test_pcg_hash(oracle_mod):
    lib = oracle_mod.lib()
    rng = np.random.default_rng(1)
    for v in list(range(64)) + [int(x) for x in rng.integers(0, 2**32, size=500, dtype=np.uint64)]:
        assert lib.oracle_pcg_hash(v) == _pcg_hash_py(v)
        h = _pcg_hash_py(v)
        assert lib.oracle_hash_to_unit(h) == np.float32((h & 0xFFFFFF) / 16777216.0)


def _emit_fill_numpy(e, h, seed, grid):
    """FillCells emission (Slosh.usf:295-311, 328-350) restated in numpy float32."""
    dims = list(e.cell_dims)
    n = dims[0] * dims[1] * dims[2] * 8
    i = np.arange(n, dtype=np.uint64)
    M = 0xFFFFFFFF

    def pcg(v):
        v = v.astype(np.uint64)
        state = (v * 747796405 + 2891336453) & M
        word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & M
        return ((word >> 22) ^ word) & M

    h0 = pcg((i * 3 + seed * 7919) & M)
    h1 = pcg(h0)
    h2 = pcg(h1)
    rnd = np.stack([(x & 0xFFFFFF).astype(np.float32) / np.float32(16777216.0) for x in (h0, h1, h2)], axis=1)
    cell = i // 8
    sub = i % 8
    local = np.stack([cell % dims[0], (cell // dims[0]) % dims[1], cell // (dims[0] * dims[1])], axis=1)
    so = np.stack([sub & 1, (sub >> 1) & 1, (sub >> 2) & 1], axis=1).astype(np.float32)
    j = np.float32(e.fill_jitter)
    incell = ((so + np.float32(0.5)) + j * (rnd - np.float32(0.5))) * np.float32(0.5)
    base = (np.array(list(e.cell_min))[None, :] + local).astype(np.float32)
    p = (base + incell) * np.float32(h)
    lo = np.float32(h) * np.float32(1.01)
    hi = (np.array(grid, dtype=np.float32) - np.float32(1.01)) * np.float32(h)
    return np.minimum(np.maximum(p, lo), hi)


def test_fill_emission_matches_numpy(oracle_mod):
    sc = scenes.tiny(oracle_mod.settings_default, n=16)
    o = oracle_mod.Oracle(sc["settings"])
    o.set_emit_seed(5)
    e = sc["emits"][0]
    o.emit(e)
    p = o.read("PARTICLES")
    ref = _emit_fill_numpy(e, sc["settings"].cell_size, 5, list(sc["settings"].grid_dim))
    assert np.array_equal(p["pos"].view(np.uint32), ref.view(np.uint32))
    assert np.all(p["age"] == 0) and np.all(p["vel"] == 0) and np.all(p["c"] == 0)


def _sort_keys_numpy(p, h, grid):
    inv = np.float32(1.0) / np.float32(h)
    c = np.floor(p["pos"] * inv).astype(np.int64)
    c = np.clip(c, 0, np.array(grid) - 1)
    sd = (np.array(grid) + 3) // 4
    nk = int(np.prod(sd)) + 1
    b = c >> 2
    k = np.minimum(b[:, 0] + sd[0] * (b[:, 1] + sd[1] * b[:, 2]), nk - 2)
    dead = ~(p["age"] >= 0)
    k[dead] = nk - 1
    return k, nk


def test_sort_is_stable_counting_sort(oracle_mod):
    sc = scenes.tiny(oracle_mod.settings_default, n=32)
    o = oracle_mod.Oracle(sc["settings"])
    rng = np.random.default_rng(3)
    n = 30000
    p = np.zeros(n, dtype=A.PARTICLE_DTYPE)
    p["pos"] = rng.uniform(-0.05, 1.05, size=(n, 3)).astype(np.float32)
    p["age"] = np.where(rng.uniform(size=n) < 0.1, np.float32(-1.0), np.float32(0.25))
    p["age"][:7] = np.nan
    p["vel"] = rng.normal(size=(n, 3)).astype(np.float32)
    o.upload_particles(p)
    o.sort_particles()
    keys, nk = _sort_keys_numpy(p, sc["settings"].cell_size, list(sc["settings"].grid_dim))
    perm_ref = np.argsort(keys, kind="stable")
    assert np.array_equal(o.read("SORT_PERM"), perm_ref)
    assert np.array_equal(o.read("PARTICLES").view(np.uint32), p[perm_ref].view(np.uint32))
    counts = np.bincount(keys, minlength=nk)
    assert np.array_equal(o.read("SORT_COUNTS"), counts)
    assert np.array_equal(o.read("SORT_OFFSETS"), np.concatenate([[0], np.cumsum(counts)[:-1]]))
    assert o.read("PARTICLE_COUNT")[0] == n - counts[-1]


def _run_tiny(oracle_mod, frames=3, n=16, solver=A.SOLVER_MGPCG, colliders=False):
    sc = scenes.tiny(oracle_mod.settings_default, n=n, solver=solver, colliders=colliders)
    o = oracle_mod.Oracle(sc["settings"])
    o.set_emit_seed(sc["seed"])
    fi = A.frame_input(sc["settings"], emits=sc["emits"], colliders=sc["colliders"])
    for _ in range(frames):
        o.step_frame(fi)
        fi = A.frame_input(sc["settings"], colliders=sc["colliders"])
    return o, sc


def test_p2g_weight_sums(oracle_mod):
    """Every particle's trilinear weights sum to 1 per MAC component: the 2^20 fixed-point weight sums
    over all faces equal the particle count up to the rounding of each of the 8 weights."""
    o, sc = _run_tiny(oracle_mod, frames=2)
    n = sc["particles"]
    L = o.layout()
    fw = o.read("FACE_WEIGHT").reshape(3, L.pool_cells).astype(np.float64)
    # FaceWeight holds this substep's P2G weights (before G2P moved the particles), so compare the
    # weights with the particle count that produced them.
    for a in range(3):
        assert abs(fw[a].sum() - n) <= 8 * n / 2**20 + 1e-9


def _assemble(o, fp64=False):
    """Pressure system of the oracle's last solve, assembled from its own buffers (scipy CSR); with fp64 from the
    FP64 oracle's double buffers (diagonal + double(1e-4f), as that oracle forms it)."""
    import scipy.sparse as sp
    L = o.layout()
    bd = np.array(list(L.brick_dim))
    gd = np.array(list(L.grid_dim))
    ab = o.read("ACTIVE_BRICKS")
    bt = o.read("BRICK_TABLE")
    ct = o.read("CELL_TYPE") & 3
    diag = (o.read_f64 if fp64 else o.read)("CELL_DIAG").astype(np.float64)
    div = (o.read_f64 if fp64 else o.read)("DIVERGENCE").astype(np.float64)
    idx_of = {}
    cells = []
    for e in range(int(ab[0])):
        b = int(ab[1 + e])
        slot = int(bt[b])
        bc = np.array([b % bd[0], (b // bd[0]) % bd[1], b // (bd[0] * bd[1])])
        for l in range(512):
            lc = np.array([l % 8, (l // 8) % 8, l // 64])
            c = bc * 8 + lc
            if np.any(c >= gd):
                continue
            i = slot * 512 + l
            if ct[i] == 1:
                idx_of[tuple(c)] = len(cells)
                cells.append((tuple(c), i))
    rows, cols, vals = [], [], []
    b = np.zeros(len(cells))
    for k, (c, i) in enumerate(cells):
        rows.append(k); cols.append(k)
        vals.append(float(diag[i] + np.float64(np.float32(1e-4))) if fp64 else float(np.float32(diag[i]) + np.float32(1e-4)))
        b[k] = -div[i]
        for d in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            nb = (c[0] + d[0], c[1] + d[1], c[2] + d[2])
            j = idx_of.get(nb)
            if j is not None:
                rows.append(k); cols.append(j); vals.append(-1.0)
    A_ = sp.csr_matrix((vals, (rows, cols)), shape=(len(cells), len(cells)))
    return A_, b, [i for _, i in cells]


def test_mgpcg_matches_direct_solve(oracle_mod):
    import scipy.sparse.linalg as spla
    o, sc = _run_tiny(oracle_mod, frames=3, n=24)
    A_, b, idx = _assemble(o)
    p = o.read_f64("PRESSURE")[idx]
    # the last frame ran the density projection after the pressure solve; the pressure buffer keeps p
    exact = spla.spsolve(A_.tocsc(), b)
    r = b - A_ @ p
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-5
    assert np.linalg.norm(p - exact) / np.linalg.norm(exact) < 1e-3
    res = o.results()
    assert res.last_solve_rel_residual <= 1e-6
    assert res.last_solve_iterations > 0


def test_hydrostatic_calm_pool(oracle_mod):
    """A resting pool: the projection must cancel gravity, so vertical pressure differences in the
    interior equal |g| dt per cell (p_hat = p dt / (rho h)) and velocities stay near zero."""
    s = scenes.base_settings(oracle_mod.settings_default, (16, 16, 16), 16 * 16 * 16 * 8)
    s.tolerance = 1e-7
    s.max_iterations = 400
    mn, dims = scenes.box_cells((16, 16, 16), (0, 0, 0), (1.0, 0.5, 1.0))
    emit = scenes.fill_cells(mn, dims, jitter=0.0)
    o = oracle_mod.Oracle(s)
    o.set_emit_seed(1)
    fi = A.frame_input(s, emits=[emit])
    n, dt = o.begin_frame(fi)
    for k in range(n):
        o.substep(k)
    o.end_frame()
    L = o.layout()
    p = o.read_f64("PRESSURE")
    ct = o.read("CELL_TYPE") & 3
    bt = o.read("BRICK_TABLE")
    bd = list(L.brick_dim)

    def idx(x, y, z):
        b = (x >> 3) + bd[0] * ((y >> 3) + bd[1] * (z >> 3))
        return int(bt[b]) * 512 + (x & 7) + 8 * ((y & 7) + 8 * (z & 7))

    g_dt = 9.81 * dt
    diffs = []
    for x in range(3, 13):
        for z in range(3, 13):
            for y in range(2, 5):
                a, c = idx(x, y, z), idx(x, y + 1, z)
                if ct[a] == 1 and ct[c] == 1:
                    diffs.append(p[a] - p[c])
    diffs = np.array(diffs)
    assert diffs.size > 50
    assert np.allclose(diffs, g_dt, rtol=0.03), (diffs.min(), diffs.max(), g_dt)
    r = o.results()
    assert r.max_particle_speed < 0.05


def test_allocator_invariants(oracle_mod):
    o, sc = _run_tiny(oracle_mod, frames=4, n=32)
    L = o.layout()
    bt, sb = o.read("BRICK_TABLE"), o.read("SLOT_BRICK")
    ab, fs = o.read("ACTIVE_BRICKS"), o.read("FREE_SLOTS")
    act = ab[1:1 + ab[0]]
    assert np.all(np.diff(act.astype(np.int64)) > 0)  # ascending brick order
    used = bt[bt != 0]
    assert len(np.unique(used)) == len(used)
    for b in np.nonzero(bt)[0]:
        assert sb[bt[b]] == b
    free = set(int(x) for x in fs[1:1 + fs[0]])
    assert free.isdisjoint(set(int(x) for x in used))
    assert len(free) + len(used) == L.num_pool_bricks - 1
    assert set(int(b) for b in act) == set(int(b) for b in np.nonzero(bt)[0])


def test_canonical_reductions(oracle_mod):
    lib = oracle_mod.lib()
    rng = np.random.default_rng(9)
    v = rng.normal(size=512) * 10.0 ** rng.integers(-8, 8, size=512)
    lanes = np.zeros(32)
    for t in range(32):
        acc = 0.0
        h, y = t & 1, (t >> 1) & 7
        for k in range(4):
            z = 2 * k + (t >> 4)
            for j in range(4):
                acc = acc + v[4 * h + j + 8 * y + 64 * z]
        lanes[t] = acc
    for off in (16, 8, 4, 2, 1):
        lanes[:off] = lanes[:off] + lanes[off:2 * off]
    total = lanes[0]
    vv = np.ascontiguousarray(v)
    assert lib.oracle_reduce_brick(vv.ctypes.data) == total
    for n in (1, 7, 1024, 3000, 7001):
        p = np.ascontiguousarray(rng.normal(size=n))
        lanes = np.zeros(1024)
        for t in range(1024):
            acc = 0.0
            for e in range(t, n, 1024):
                acc = acc + p[e]
            lanes[t] = acc
        tot = None
        for w in range(32):
            lane = lanes[32 * w:32 * w + 32].copy()
            for off in (16, 8, 4, 2, 1):
                lane[:off] = lane[:off] + lane[off:2 * off]
            tot = lane[0] if w == 0 else tot + lane[0]
        assert lib.oracle_reduce_final(p.ctypes.data, n) == tot


def test_rbgs_and_mgpcg_both_reduce_divergence(oracle_mod):
    for solver in (A.SOLVER_MGPCG, A.SOLVER_RBGS):
        o, _ = _run_tiny(oracle_mod, frames=3, n=16, solver=solver)
        r = o.results()
        assert r.fluid_cells > 100
        assert r.max_divergence < (0.05 if solver == A.SOLVER_MGPCG else 5.0)


def fp64_step_errors(oracle_mod, o32, fi, extra=None):
    """Runs one substep from o32's state in FP32 (o32) and FP64 (a copy); returns relative L2 errors of
    the FP32 pressure and face velocity against FP64 over the active cells."""
    from parity import active_slots, slot_mask
    n, _ = o32.begin_frame(fi)
    o64 = oracle_mod.Oracle(o32.settings, fp64=True)
    o64.copy_state_from(o32)
    o32.substep(0)
    o64.substep(0)
    if extra is not None:
        extra.substep(0)
    L = o32.layout()
    slots = active_slots(o32)
    errs = {}
    for name, planes in (("PRESSURE", 1), ("VEL", 3), ("DIVERGENCE", 1)):
        m = slot_mask(slots, L.pool_cells, planes)
        ref = o64.read_f64(name)[m]
        for tag, src in (("oracle32", o32), ("gpu", extra)):
            if src is None:
                continue
            a = src.read(name)[m].astype(np.float64)
            den = np.linalg.norm(ref)
            errs[(tag, name)] = float(np.linalg.norm(a - ref) / den) if den > 0 else float(np.linalg.norm(a - ref))
    o64.close()
    return errs


def test_fp32_error_against_fp64_oracle(oracle_mod):
    o, sc = _run_tiny(oracle_mod, frames=3, n=24)
    errs = fp64_step_errors(oracle_mod, o, A.frame_input(sc["settings"], colliders=sc["colliders"]))
    # MGPCG stops at a 1e-6 relative residual; FP32 storage adds ~1e-7 relative rounding per pass.
    assert errs[("oracle32", "PRESSURE")] < 1e-4, errs
    assert errs[("oracle32", "VEL")] < 1e-5, errs


def test_bf16_conversion_matches_torch(oracle_mod):
    """The oracle's FP32 -> BF16 rounding (coarse-level storage) against torch's round-to-nearest-even."""
    import torch
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.normal(size=20000).astype(np.float32) * np.float32(10.0) ** rng.integers(-6, 6, 20000),
                        np.array([0.0, -0.0, 1.0, 65504.0, 3.4e38, -3.4e38, 1e-40], dtype=np.float32)]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    lib = oracle_mod.lib()
    got = np.array([lib.oracle_f32_to_bf16(float(v)) for v in x], dtype=np.uint16)
    assert np.array_equal(got, want)


def test_overcorrected_vcycle_needs_fewer_iterations(oracle_mod):
    """The piecewise-constant prolongation under-corrects smooth errors; scaling each coarse-grid correction
    by 1.7 (mg_correction_scale) and a second red-black sweep pair (mg_smoothing_sweeps) must each reach the
    same 1e-6 relative residual in fewer PCG iterations than the reference's V-cycle on the same scene,
    and flexible PCG must not change the count of a linear preconditioner by more than one."""
    from slosh_b200 import scenes
    counts = {}
    for key, (scale, sweeps, flex) in {"ref": (1.0, 1, 0), "scaled": (1.7, 1, 0), "two": (1.7, 2, 0),
                                       "flex": (1.7, 1, 1)}.items():
        sc = scenes.dam_break_sphere(oracle_mod.settings_default, n=48)
        s = sc["settings"]
        s.max_substeps = 16
        s.mg_correction_scale, s.mg_smoothing_sweeps, s.pcg_flexible = scale, sweeps, flex
        o = oracle_mod.Oracle(s)
        o.set_emit_seed(sc["seed"])
        fi = A.frame_input(s, emits=sc["emits"])
        its = []
        for _ in range(3):
            o.step_frame(fi)
            fi = A.frame_input(s)
            r = o.results()
            assert r.last_solve_rel_residual <= 1e-6
            its.append(r.last_solve_iterations)
        o.close()
        counts[key] = its
    assert sum(counts["scaled"]) < sum(counts["ref"]), counts
    assert sum(counts["two"]) < sum(counts["scaled"]), counts
    assert all(abs(a - b) <= 1 for a, b in zip(counts["flex"], counts["scaled"])), counts


@pytest.mark.parametrize("scale,sweeps,flexible,weight", [(1.0, 1, 0, 1.0), (1.9, 2, 1, 1.0), (1.9, 2, 0, 1.15)])
def test_mgpcg_matches_direct_solve_sparse_64(oracle_mod, scale, sweeps, flexible, weight):
    """The solve's mathematics pinned independently of any reduction order: the FP64 oracle's MGPCG on the sparse
    64^3 dam break + falling sphere (ghost-fluid diagonals at the free surface, several MG levels through the
    footprints and the shared tail), with the reference's V-cycle and with the tuned options (over-relaxed finest
    sweeps included), against scipy's direct sparse solve of the same assembled system (diag_f + 1e-4 on the
    fluid cells, -1 per fluid neighbour)."""
    import scipy.sparse.linalg as spla
    sc = scenes.dam_break_sphere(oracle_mod.settings_default, n=64)
    s = sc["settings"]
    s.max_substeps = 16
    s.mg_correction_scale, s.mg_smoothing_sweeps, s.pcg_flexible = scale, sweeps, flexible
    s.mg_smoother_weight = weight
    o = oracle_mod.Oracle(s, fp64=True)
    o.set_emit_seed(sc["seed"])
    fi = A.frame_input(s, emits=sc["emits"])
    for _ in range(2):
        o.step_frame(fi)
        fi = A.frame_input(s)
    A_, b, idx = _assemble(o, fp64=True)
    assert len(idx) > 30000
    diag = A_.diagonal()
    assert np.any(np.abs(diag - np.round(diag)) > 1e-3), "no ghost-fluid (fractional) diagonal in the system"
    p = o.read_f64("PRESSURE")[idx]
    exact = spla.spsolve(A_.tocsc(), b)
    rel = np.linalg.norm(b - A_ @ p) / np.linalg.norm(b)
    res = o.results()
    assert res.last_solve_rel_residual <= 1e-6
    # FP64: the true residual equals the recursive one (no FP32 floor)
    assert rel <= 1.01e-6, rel
    assert np.linalg.norm(p - exact) / np.linalg.norm(exact) < 1e-4
    o.close()
