"""slosh_sort_particles_static: the allocation-free sort of caller-owned device particles.

It must give exactly what the context's sort (slosh_sort_particles) gives on the same particles --
sorted records, permutation, per-key offsets and live count, all integer or copied bytes, so the bar
is bit-exact -- on two calls in a row (the second smaller than the first, so stale scratch from the
first call would show), and it must refuse inputs above its static scratch size before touching the
device. Calls after the first in a context must not allocate device memory: neither the device's free
memory nor torch's allocator may change across them. With the optional outputs left NULL the scratch
stands in for them, and an empty input gives a live count of 0. This file is collected last so that
the GPU test also runs after every other test."""
import ctypes as C

import numpy as np
import pytest

from slosh_b200 import _abi as A

GRID = (48, 40, 36)
CELL = 0.05
MAX_PARTICLES = 262144  # SLOSH_STATIC_SORT_MAX_PARTICLES


def _settings(slosh, capacity):
    s = slosh.settings_default()
    s.grid_dim[0], s.grid_dim[1], s.grid_dim[2] = GRID
    s.cell_size = CELL
    s.particle_capacity = capacity
    return s


def _particles(seed, n):
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=A.PARTICLE_DTYPE)
    ext = np.array(GRID, dtype=np.float64) * CELL
    # a margin outside the grid exercises the key clamp; 10 % dead records go to the last key
    p["pos"] = rng.uniform(-0.05, 1.05, size=(n, 3)) * ext
    p["age"] = np.where(rng.uniform(size=n) < 0.1, -1.0, rng.uniform(0.0, 3.0, size=n)).astype(np.float32)
    p["vel"] = rng.normal(size=(n, 3)).astype(np.float32)
    p["c"] = rng.integers(0, 2**32, size=(n, 5), dtype=np.uint32)
    return p


def test_static_sort_rejects_oversize(slosh):
    lib = slosh.load_library()
    dims = (C.c_int32 * 3)(*GRID)
    fake = C.c_void_p(0x1000)
    rc = lib.slosh_sort_particles_static(fake, C.c_void_p(0x2000), MAX_PARTICLES + 1, dims, CELL, None, None, None, None)
    assert rc == A.ERR_CAPACITY
    assert b"static scratch maximum" in lib.slosh_last_error_string()
    big = (C.c_int32 * 3)(1024, 1024, 1024)
    rc = lib.slosh_sort_particles_static(fake, C.c_void_p(0x2000), 10, big, CELL, None, None, None, None)
    assert rc == A.ERR_CAPACITY
    assert b"sort keys" in lib.slosh_last_error_string()


@pytest.mark.gpu
def test_static_sort_matches_context_sort(slosh):
    import torch

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n_max = 120000
    sim = slosh.Simulation(_settings(slosh, n_max), device=0)
    num_keys = int(sim.layout().num_sort_keys)
    d_in = torch.empty(n_max * 48, dtype=torch.uint8, device=dev)
    d_out = torch.empty(n_max * 48, dtype=torch.uint8, device=dev)
    d_perm = torch.empty(n_max, dtype=torch.int32, device=dev)
    d_off = torch.empty(num_keys, dtype=torch.int32, device=dev)
    d_live = torch.empty(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def sort_static(n, perm, off, live):
        slosh.sort_particles_static(d_in.data_ptr(), d_out.data_ptr(), n, GRID, CELL, perm, off, live, stream.cuda_stream)

    for call, (seed, n) in enumerate(((11, n_max), (12, 70001))):
        p = _particles(seed, n)
        sim.upload_particles(p)
        sim.sort_particles()
        want = sim.particles()
        want_perm = sim.read("SORT_PERM")[:n]
        want_off = sim.read("SORT_OFFSETS")
        want_live = int(sim.read("PARTICLE_COUNT")[0])

        d_in[: n * 48].copy_(torch.from_numpy(p.view(np.uint8).reshape(-1)))
        d_out.fill_(0xAB)
        d_perm.fill_(-1)
        d_off.fill_(-1)
        d_live.fill_(-1)
        torch.cuda.synchronize(dev)
        free0, alloc0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
        sort_static(n, d_perm.data_ptr(), d_off.data_ptr(), d_live.data_ptr())
        torch.cuda.synchronize(dev)
        if call > 0:  # the first call in this context may load the library's device code; later ones allocate nothing
            assert torch.cuda.mem_get_info(dev)[0] == free0, "device free memory changed across the call"
            assert torch.cuda.memory_allocated(dev) == alloc0
        got = d_out[: n * 48].cpu().numpy().view(A.PARTICLE_DTYPE)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"records differ (seed {seed})"
        assert np.array_equal(d_perm[:n].cpu().numpy().view(np.uint32), want_perm)
        assert np.array_equal(d_off.cpu().numpy().view(np.uint32), want_off)
        assert int(d_live.item()) == want_live
        assert want_live == int((p["age"] >= 0).sum())

        # the optional outputs left NULL: the records alone, through the scratch's own copies
        d_out.fill_(0xCD)
        torch.cuda.synchronize(dev)
        sort_static(n, 0, 0, 0)
        torch.cuda.synchronize(dev)
        got = d_out[: n * 48].cpu().numpy().view(A.PARTICLE_DTYPE)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"records differ without optional outputs (seed {seed})"

    # an empty input: nothing to move, a live count of 0 and all-zero key offsets
    d_live.fill_(-1)
    d_off.fill_(-1)
    torch.cuda.synchronize(dev)
    sort_static(0, 0, d_off.data_ptr(), d_live.data_ptr())
    torch.cuda.synchronize(dev)
    assert int(d_live.item()) == 0
    assert not d_off.any().item()
    sim.close()
