"""Pins of the U-Net oracle (CPU): the convolution against straight loops, its data and weight
gradients by the adjoint identities, BF16 rounding on known values, and the whole network's backward
pass against central finite differences of its loss (exact FP64 mode)."""
import os
import sys

import numpy as np
import pytest

from oracle import unet_oracle as U  # noqa: E402


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -3.0, 65504.0, 1e-40], np.float32)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7 -> even (1); 1 + 3 * 2^-8 -> 1 + 2^-6 (even)
    want = np.array([1.0, 1.0, 1.0078125, 1.015625, -3.0, 65536.0, 0.0], np.float32)
    got = U.bf16(x)
    assert np.array_equal(got[:6], want[:6])
    assert abs(got[6]) < 1e-38
    assert np.array_equal(U.from_bits(U.bf16_bits(x)), got)


def test_conv3d_matches_direct_loops():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 3, 4, 5, 3))
    w = rng.standard_normal((27, 4, 3))
    b = rng.standard_normal(4)
    ref = U.conv3d_direct(x, w, b)
    got = U.conv3d([x], w, b, relu=False, round_out=False)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_conv3d_gradients_are_adjoints():
    rng = np.random.default_rng(2)
    x1 = rng.standard_normal((1, 4, 3, 5, 2))
    x2 = rng.standard_normal((1, 4, 3, 5, 3))
    w = rng.standard_normal((27, 4, 5))
    g = rng.standard_normal((1, 4, 3, 5, 4))
    y = U.conv3d([x1, x2], w, None, relu=False, round_out=False)
    lhs = float((y * g).sum())
    d1, d2 = U.conv3d_dgrad(g, w, [2, 3])
    assert np.isclose(lhs, float((x1 * d1).sum() + (x2 * d2).sum()), rtol=1e-10)
    dw, db = U.conv3d_wgrad([x1, x2], g)
    assert np.isclose(lhs, float((w * dw).sum()), rtol=1e-10)
    assert np.allclose(db, g.reshape(-1, 4).sum(0))


def test_pool_and_upsample_gradients_are_adjoints():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((1, 4, 4, 4, 8))
    g = rng.standard_normal((1, 2, 2, 2, 8))
    assert np.isclose(float((U.pool_exact(x) * g).sum()), float((x * U.pool_bwd_exact(g)).sum()), rtol=1e-12)
    gu = rng.standard_normal((1, 4, 4, 4, 8))
    assert np.isclose(float((U.upsample(g) * gu).sum()), float((g * U.upsample_bwd_exact(gu)).sum()), rtol=1e-12)


def _small_problem(seed, dim=8):
    rng = np.random.default_rng(seed)
    lay, head_off, n = U.layout()
    p = np.zeros(n, np.float32)
    for (w_off, b_off, cout, cins) in lay:
        cin = sum(cins)
        p[w_off:w_off + 27 * cout * cin] = rng.normal(0, np.sqrt(2.0 / (27 * cin)), 27 * cout * cin)
        p[b_off:b_off + cout] = rng.normal(0, 0.05, cout)
    p[head_off:head_off + 16] = rng.normal(0, 0.25, 16)
    inp = np.zeros((1, dim, dim, dim, U.IN_CHANNELS), np.float32)
    fluid = rng.random((1, dim, dim, dim)) < 0.6
    inp[..., 0] = np.where(fluid, rng.uniform(-1, 1, fluid.shape), 0.0)
    inp[..., 1] = fluid
    inp[..., 2] = (~fluid) & (rng.random(fluid.shape) < 0.3)
    target = np.where(fluid, rng.normal(0, 0.3, fluid.shape), 0.0)
    return p, inp, target


def test_network_gradients_match_finite_differences():
    p, inp, target = _small_problem(4)
    net = U.Network(p, exact=True)
    loss, grads, _ = net.loss_and_grads(inp, target)
    assert loss > 0
    rng = np.random.default_rng(5)
    lay, head_off, n = U.layout()
    # a few parameters of every layer (weights and biases) and the head
    picks = []
    for (w_off, b_off, cout, cins) in lay:
        picks += list(rng.integers(w_off, b_off, 2)) + [b_off]
    picks += [head_off + 3, head_off + 16]
    eps = 1e-4
    checked = 0
    for i in picks:
        pp = p.astype(np.float64).copy()
        pp[i] += eps
        lp = U.Network(pp, exact=True).loss_and_grads(inp, target)[0]
        pp[i] -= 2 * eps
        lm = U.Network(pp, exact=True).loss_and_grads(inp, target)[0]
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grads[i]) <= 1e-4 * max(1.0, abs(fd)) + 2e-6, (i, fd, grads[i])
        checked += 1
    assert checked == len(picks)


def test_network_bf16_storage_is_close_to_exact():
    p, inp, target = _small_problem(6)
    l1, g1, y1 = U.Network(p, exact=False).loss_and_grads(inp, target)
    l2, g2, y2 = U.Network(p, exact=True).loss_and_grads(inp, target)
    # BF16 activations and activation gradients: the loss agrees closely, the parameter gradients to
    # the BF16 storage noise (about 10-15 % relative L2 on this small random network)
    assert abs(l1 - l2) <= 0.01 * l2
    assert np.linalg.norm(g1 - g2) <= 0.25 * np.linalg.norm(g2)
    assert float(g1 @ g2) >= 0.95 * np.linalg.norm(g1) * np.linalg.norm(g2)


def test_shipped_weights_match_the_layout():
    """The trained weights in the package have the network's parameter count, finite values, and BF16-
    rounded convolution weights exactly where the oracle's layout puts them."""
    from slosh_b200 import train_warmstart as TW
    lay, head_off, n = U.layout()
    path = os.path.join(os.path.dirname(__file__), "..", "slosh_b200", "warmstart_128.npz")
    p = TW.load_weights(path)
    assert p.shape == (n,) and np.all(np.isfinite(p))
    mask = TW.conv_weight_mask(n)
    want = np.zeros(n, bool)
    for (w_off, b_off, cout, cins) in lay:
        want[w_off:b_off] = True
    assert np.array_equal(mask, want)
    assert np.array_equal(U.bf16(p[mask]), p[mask])


def test_random_scenes_are_seeded():
    """The warm-start scene generator is a pure function of its seed (held-out seeds never repeat training
    ones), with 1-4 boxes inside the domain and 0-3 spheres."""
    import slosh_b200 as S
    from slosh_b200 import warmstart as W
    a = W.random_scene(S.settings_default, 10001, 128)
    b = W.random_scene(S.settings_default, 10001, 128)
    assert [list(e.cell_min) + list(e.cell_dims) + list(e.velocity) for e in a[1]] == \
           [list(e.cell_min) + list(e.cell_dims) + list(e.velocity) for e in b[1]]
    for seed in range(10000, 10040):
        s, emits, cols = W.random_scene(S.settings_default, seed, 128)
        assert 1 <= len(emits) <= 4 and 0 <= len(cols) <= 3
        for e in emits:
            assert min(e.cell_min) >= 1 and all(m + d <= 127 for m, d in zip(e.cell_min, e.cell_dims))
