"""Headless surface (density splat, f16 field with brick occupancy, surface nets) of the GPU against the
oracle on the same particles: field, occupancy, vertex positions, normals, tangents and triangle indices
bit for bit, vertices and triangles in cell order. Covers field resolutions 1 and 1.5, a finer iso level,
and capacity limits that cut the vertex and index lists."""
import numpy as np
import pytest

import slosh_b200 as S
from slosh_b200 import _abi as A
from slosh_b200 import scenes

from parity import pair, run_frames

pytestmark = pytest.mark.gpu

SURFACE_BUFFERS = ("SURFACE_FIELD", "SURFACE_BRICKS", "SURFACE_POSITIONS", "SURFACE_NORMALS", "SURFACE_TANGENTS",
                   "SURFACE_INDICES")


def _compare(g, o, q):
    ig, io = g.build_surface(q), o.build_surface(q)
    for f, _ in A.SurfaceInfo._fields_:
        vg, vo = getattr(ig, f), getattr(io, f)
        if hasattr(vg, "__len__"):
            vg, vo = list(vg), list(vo)
        assert vg == vo, f"info.{f}: {vg} != {vo}"
    for name in SURFACE_BUFFERS:
        a, b = g.read(name), o.read(name)
        assert a.shape == b.shape, name
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"{name}: {np.count_nonzero(a != b)} differ"
    return ig


def test_surface_bit_exact(slosh, oracle_mod):
    sc = scenes.tiny(slosh.settings_default, n=24)
    g, o = pair(slosh, oracle_mod, sc)
    run_frames(g, o, sc, frames=3)
    q = S.surface_params_default()
    info = _compare(g, o, q)
    assert info.num_vertices > 100 and info.num_indices > 300, "no surface found"
    tri = g.read("SURFACE_INDICES").reshape(-1, 3)
    assert tri.max() < info.num_vertices
    n = g.read("SURFACE_NORMALS").reshape(-1, 3)
    assert np.allclose(np.linalg.norm(n, axis=1), 1.0, atol=1e-5)
    q.field_resolution, q.iso_level = 1.5, 0.35
    _compare(g, o, q)
    q.max_vertices, q.max_indices = info.num_vertices // 2, info.num_indices // 3 + 1
    cut = _compare(g, o, q)
    assert cut.vertices_requested > cut.num_vertices and cut.num_indices % 6 == 0
    q.build_mesh = 0
    _compare(g, o, q)
