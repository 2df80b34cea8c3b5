"""Seeded synthetic scenes, expressed as the plugin's own emission requests.

A scene is (settings, emit requests, colliders). Liquid blocks are FillCells requests
(ESloshEmitShape::FillCells: 8 stratified, jittered particles per cell, Slosh.usf:301-312), sized the
way ASloshVolume::QueueFillLocalBox turns a box into a cell range (SloshVolume.cpp:120-146: floor of
the minimum and ceil of the maximum, clamped to [1, N - 1] so the wall layer stays empty). A liquid
sphere is the union of FillCells rows of the cells whose centres lie inside it. The emission seed of
the first request is the scene seed; each further request takes the next seed (SloshProxy.cpp:529).

No public dataset stands behind these scenes: the dam-break, sphere and box shapes, sizes, particle
densities and seeds are the workload definitions the benchmark is quoted on, generated here.
"""
import math

import numpy as np

from . import _abi as A


def fill_cells(cell_min, cell_dims, velocity=(0.0, 0.0, 0.0), jitter=1.0):
    e = A.EmitRequest()
    e.shape = A.EMIT_FILL_CELLS
    e.cell_min[:] = [int(v) for v in cell_min]
    e.cell_dims[:] = [int(v) for v in cell_dims]
    e.velocity[:] = [float(v) for v in velocity]
    e.rotation[:] = [0.0, 0.0, 0.0, 1.0]
    e.fill_jitter = float(jitter)
    return e


def box_cells(grid, lo_frac, hi_frac):
    """Cell range [min, max) of a box given as fractions of the domain, QueueFillLocalBox style."""
    mn, mx = [], []
    for a in range(3):
        n = grid[a]
        lo = min(max(math.floor(lo_frac[a] * n), 1), n - 1)
        hi = min(max(math.ceil(hi_frac[a] * n), 1), n - 1)
        mn.append(lo)
        mx.append(hi)
    return mn, [mx[a] - mn[a] for a in range(3)]


def sphere_rows(grid, center_frac, radius_frac, velocity=(0.0, 0.0, 0.0), jitter=1.0):
    """FillCells rows covering the cells of the domain's interior whose centres lie in the sphere."""
    n = grid
    emits = []
    cx, cy, cz = (center_frac[a] * n[a] for a in range(3))
    r = radius_frac * n[0]
    for z in range(1, n[2] - 1):
        for y in range(1, n[1] - 1):
            dy, dz = (y + 0.5) - cy, (z + 0.5) - cz
            rem = r * r - dy * dy - dz * dz
            if rem < 0:
                continue
            half = math.sqrt(rem)
            x0 = max(math.ceil(cx - half - 0.5), 1)
            x1 = min(math.floor(cx + half - 0.5), n[0] - 2)
            xs = [x for x in range(x0, x1 + 1) if ((x + 0.5) - cx) ** 2 + dy * dy + dz * dz <= r * r]
            if not xs:
                continue
            emits.append(fill_cells((xs[0], y, z), (xs[-1] - xs[0] + 1, 1, 1), velocity, jitter))
    return emits


def base_settings(lib_default, grid, capacity):
    s = lib_default()
    s.grid_dim[:] = list(grid)
    s.cell_size = 1.0 / grid[0]
    s.particle_capacity = int(capacity)
    s.gravity[:] = [0.0, -9.81, 0.0]
    s.cfl = 1.0
    s.max_frame_dt = 1.0 / 120.0
    s.sort_interval = 1
    return s


def dam_break(lib_default, n=64, x_frac=0.4, y_frac=0.6, seed=0, tolerance=1e-6, solver=A.SOLVER_MGPCG,
              extra_capacity=0):
    """Small dam break: n^3 box, h = 1/n, liquid block x < x_frac, y < y_frac, full z, 8 particles per
    cell jittered +-0.25 cell, MGPCG to a relative residual of `tolerance`."""
    grid = (n, n, n)
    mn, dims = box_cells(grid, (0.0, 0.0, 0.0), (x_frac, y_frac, 1.0))
    emits = [fill_cells(mn, dims)]
    count = dims[0] * dims[1] * dims[2] * 8
    s = base_settings(lib_default, grid, count + extra_capacity)
    s.pressure_solver = solver
    s.tolerance = tolerance
    s.max_iterations = 200
    return dict(settings=s, emits=emits, seed=seed, particles=count, name=f"dam_break_{n}")


def dam_break_sphere(lib_default, n=256, seed=1, tolerance=1e-6, solver=A.SOLVER_MGPCG, sor_iterations=200):
    """Sparse-brick dam break plus falling sphere: block x < 0.3, y < 0.5; sphere radius 0.12 at
    (0.7, 0.75, 0.5) moving at -2 m/s in y; 8 particles per fluid cell."""
    grid = (n, n, n)
    mn, dims = box_cells(grid, (0.0, 0.0, 0.0), (0.3, 0.5, 1.0))
    emits = [fill_cells(mn, dims)]
    emits += sphere_rows(grid, (0.7, 0.75, 0.5), 0.12, velocity=(0.0, -2.0, 0.0))
    count = sum(e.cell_dims[0] * e.cell_dims[1] * e.cell_dims[2] * 8 for e in emits)
    s = base_settings(lib_default, grid, count)
    s.pressure_solver = solver
    s.tolerance = tolerance
    s.max_iterations = 200
    s.sor_weight = 1.9
    s.pressure_iterations = sor_iterations
    s.sort_interval = 4
    return dict(settings=s, emits=emits, seed=seed, particles=count, name=f"dam_break_sphere_{n}")


def tiny(lib_default, n=16, seed=0, solver=A.SOLVER_MGPCG, tolerance=1e-6, colliders=False):
    """Few-thousand-particle dam break for fast parity tests (optionally with static solid spheres)."""
    sc = dam_break(lib_default, n=n, x_frac=0.5, y_frac=0.6, seed=seed, tolerance=tolerance, solver=solver)
    sc["colliders"] = []
    if colliders:
        c = A.Collider()
        c.center[:] = [0.7, 0.3, 0.5]
        c.type = A.COLLIDER_SPHERE
        c.rotation[:] = [0, 0, 0, 1]
        c.extent[:] = [0.15, 0, 0]
        sc["colliders"] = [c]
    return sc


def tank_batch(lib_default, count=64, seed=3, lo=32, hi=128, tolerance=1e-6):
    """Independent tanks for batched stepping: per-axis size log-uniform in [lo, hi] cells, h = 1/64 m
    (the same cell for every tank), dam block x < U[0.2, 0.5], y < U[0.3, 0.7], full z, 8 particles per
    cell, MGPCG to `tolerance`, sort every 4 frames. Returns a list of scene dicts (seeds seed * 1000 + k)."""
    rng = np.random.default_rng(seed)
    tanks = []
    for k in range(count):
        grid = tuple(int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(3))
        xf, yf = float(rng.uniform(0.2, 0.5)), float(rng.uniform(0.3, 0.7))
        mn, dims = box_cells(grid, (0.0, 0.0, 0.0), (xf, yf, 1.0))
        n = dims[0] * dims[1] * dims[2] * 8
        s = base_settings(lib_default, grid, n)
        s.cell_size = 1.0 / 64.0
        s.tolerance = tolerance
        s.max_iterations = 200
        s.sort_interval = 4
        s.max_substeps = 16
        tanks.append(dict(settings=s, emits=[fill_cells(mn, dims)], seed=seed * 1000 + k, particles=n,
                          name=f"tank{k}_{grid[0]}x{grid[1]}x{grid[2]}", cost=float(grid[0] * grid[1] * grid[2] + n)))
    return tanks


def boxes_512(lib_default, seed=2, tolerance=1e-6, box_count=(6, 10), size=(0.1, 0.4), spheres=3):
    """512 x 256 x 256 cells (h = 1/256 m): `box_count` non-overlapping liquid boxes (drawn in order, a box
    that overlaps an earlier one is redrawn), each side a fraction U[size] of the domain side, 8 particles
    per cell, plus `spheres` static collider spheres (radius U[0.04, 0.08] m) above the liquid's floor."""
    rng = np.random.default_rng(seed)
    grid = (512, 256, 256)
    n_boxes = int(rng.integers(box_count[0], box_count[1] + 1))
    boxes = []
    attempts = 0
    while len(boxes) < n_boxes and attempts < 1000:
        attempts += 1
        fr = rng.uniform(size[0], size[1], size=3)
        lo = rng.uniform(0.0, 1.0 - fr)
        mn, dims = box_cells(grid, tuple(lo), tuple(lo + fr))
        if any(all(mn[a] < b[0][a] + b[1][a] and b[0][a] < mn[a] + dims[a] for a in range(3)) for b in boxes):
            continue
        boxes.append((mn, dims))
    emits = [fill_cells(mn, dims) for mn, dims in boxes]
    count = sum(d[0] * d[1] * d[2] * 8 for _, d in boxes)
    s = base_settings(lib_default, grid, count)
    s.cell_size = 1.0 / 256.0
    s.tolerance = tolerance
    s.max_iterations = 200
    s.sort_interval = 4
    s.max_substeps = 16
    colliders = []
    for _ in range(spheres):
        c = A.Collider()
        r = float(rng.uniform(0.04, 0.08))
        c.center[:] = [float(rng.uniform(0.2, 1.8)), float(rng.uniform(0.1, 0.6)), float(rng.uniform(0.2, 0.8))]
        c.type = A.COLLIDER_SPHERE
        c.rotation[:] = [0.0, 0.0, 0.0, 1.0]
        c.extent[:] = [r, 0.0, 0.0]
        colliders.append(c)
    return dict(settings=s, emits=emits, seed=seed, particles=count, colliders=colliders, name="boxes_512x256x256")
