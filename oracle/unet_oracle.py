"""CPU oracle of the learned warm-start network (test infrastructure only: the tests and smoke() compare
the GPU results with it; nothing in the product path calls it).

A numpy restatement of the U-Net the library trains and runs on the GPU (slosh_b200/csrc/unet.cu):
the same layers, parameter layout and BF16 storage points, with FP64 accumulation. The network is
not part of the Slosh plugin (its pressure solvers start from zero or the previous solution,
Slosh.usf MarkCellsCS); the oracle is pinned by a direct-loop convolution and by central finite
differences of its own loss (tests/test_unet_oracle.py), not by reference vectors.

Layout: dense [batch][z][y][x][channel]. A 3x3x3 convolution with zero padding 1 is the sum over
the 27 taps (tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) of the input shifted by (dz, dy, dx) times W[tap]^T,
W[tap] = [cout][cin]. BF16 rounding (round to nearest even) applies where the GPU stores BF16:
activations, activation gradients and the BF16 weight copies; weight gradients and the head stay
FP32/FP64.
"""
import numpy as np

IN_CHANNELS = 16


def bf16(x):
    """Rounds float32 values to BF16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def bf16_bits(x):
    """BF16 bit patterns (uint16) of float32 values, round to nearest even."""
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bits(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def _shift(x, dz, dy, dx):
    """y[b, z, y, x] = x[b, z + dz, y + dy, x + dx] with zeros outside."""
    B, D, H, W, C = x.shape
    p = np.zeros((B, D + 2, H + 2, W + 2, C), dtype=x.dtype)
    p[:, 1:-1, 1:-1, 1:-1] = x
    return p[:, 1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def conv3d(xs, w, b, relu=True, round_out=True):
    """relu(sum_tap shift(concat(xs)) @ W[tap]^T + b); w [27][cout][cin] (BF16 values)."""
    x = np.concatenate([np.asarray(v, np.float64) for v in xs], axis=-1)
    wd = np.asarray(w, np.float64)
    acc = np.zeros(x.shape[:-1] + (wd.shape[1],), np.float64)
    for t, dz, dy, dx in taps():
        acc += _shift(x, dz, dy, dx) @ wd[t].T
    if b is not None:
        acc += np.asarray(b, np.float64)
    if relu:
        acc = np.maximum(acc, 0.0)
    return bf16(acc.astype(np.float32)) if round_out else acc


def conv3d_dgrad(dz, w, splits):
    """Input gradient of conv3d for output gradient dz: sum_tap shift(dz, -tap) @ W[tap], split by
    input block sizes; FP64 accumulation (unrounded)."""
    g = np.asarray(dz, np.float64)
    wd = np.asarray(w, np.float64)
    acc = np.zeros(g.shape[:-1] + (wd.shape[2],), np.float64)
    for t, ddz, ddy, ddx in taps():
        acc += _shift(g, -ddz, -ddy, -ddx) @ wd[t]
    out, o = [], 0
    for c in splits:
        out.append(acc[..., o:o + c])
        o += c
    return out


def conv3d_wgrad(xs, dz):
    """dW[tap][co][ci] = sum_v dz[v][co] x[v + tap][ci]; db[co] = sum_v dz[v][co] (FP64)."""
    x = np.concatenate([np.asarray(v, np.float64) for v in xs], axis=-1)
    g = np.asarray(dz, np.float64).reshape(-1, dz.shape[-1])
    dw = np.zeros((27, g.shape[1], x.shape[-1]), np.float64)
    for t, ddz, ddy, ddx in taps():
        dw[t] = g.T @ _shift(x, ddz, ddy, ddx).reshape(-1, x.shape[-1])
    return dw, g.sum(axis=0)


def conv3d_direct(x, w, b):
    """Straight loops over output voxel, tap, cout and cin (pin of conv3d on tiny inputs)."""
    B, D, H, W, C = x.shape
    n = w.shape[1]
    y = np.zeros((B, D, H, W, n), np.float64)
    for bb in range(B):
        for z in range(D):
            for yy in range(H):
                for xx in range(W):
                    for t, dz, dy, dx in taps():
                        zz, y2, x2 = z + dz, yy + dy, xx + dx
                        if 0 <= zz < D and 0 <= y2 < H and 0 <= x2 < W:
                            y[bb, z, yy, xx] += w[t] @ x[bb, zz, y2, x2]
                    y[bb, z, yy, xx] += b
    return y


def pool(x):
    """Mean of the 2^3 children, summed in child order (x fastest) in FP32, then * 0.125."""
    x = np.asarray(x, np.float32)
    s = np.zeros((x.shape[0], x.shape[1] // 2, x.shape[2] // 2, x.shape[3] // 2, x.shape[4]), np.float32)
    for o in range(8):
        oz, oy, ox = (o >> 2) & 1, (o >> 1) & 1, o & 1
        s = s + x[:, oz::2, oy::2, ox::2]
    return bf16(s * np.float32(0.125))


def pool_bwd(g):
    g = np.asarray(g, np.float32) * np.float32(0.125)
    return np.repeat(np.repeat(np.repeat(g, 2, 1), 2, 2), 2, 3)


def upsample(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def upsample_bwd(g):
    g = np.asarray(g, np.float32)
    s = np.zeros((g.shape[0], g.shape[1] // 2, g.shape[2] // 2, g.shape[3] // 2, g.shape[4]), np.float32)
    for o in range(8):
        oz, oy, ox = (o >> 2) & 1, (o >> 1) & 1, o & 1
        s = s + g[:, oz::2, oy::2, ox::2]
    return s


# Convolutions in network order: (inputs, cout); inputs name tensors.
LAYERS = [
    (("in",), 16, "e0a"), (("e0a",), 16, "e0"),
    (("p1",), 32, "e1a"), (("e1a",), 32, "e1"),
    (("p2",), 64, "e2a"), (("e2a",), 64, "e2"),
    (("p3",), 64, "e3a"), (("e3a",), 64, "e3"),
    (("u2", "e2"), 64, "d2a"), (("d2a",), 64, "d2"),
    (("u1", "e1"), 32, "d1a"), (("d1a",), 32, "d1"),
    (("u0", "e0"), 16, "d0a"), (("d0a",), 16, "d0"),
]
CHANNELS = {"in": 16, "p1": 16, "p2": 32, "p3": 64, "u2": 64, "u1": 64, "u0": 32}
RESAMPLE_AFTER = {1: ("pool", "e0", "p1"), 3: ("pool", "e1", "p2"), 5: ("pool", "e2", "p3"),
                  7: ("up", "e3", "u2"), 9: ("up", "d2", "u1"), 11: ("up", "d1", "u0")}


def layout():
    """[(w_offset, b_offset, cout, [cin per block])] and the head offset; num_params."""
    ch = dict(CHANNELS)
    off, out = 0, []
    for ins, n, name in LAYERS:
        cins = [ch[i] for i in ins]
        cin = sum(cins)
        out.append((off, off + 27 * n * cin, n, cins))
        off += 27 * n * cin + n
        ch[name] = n
    return out, off, off + 17


class Network:
    """Forward and backward of the U-Net with the GPU's storage points. exact=True drops every BF16
    rounding (the finite-difference pin)."""

    def __init__(self, params, exact=False):
        self.lay, self.head_off, self.num_params = layout()
        assert len(params) == self.num_params
        self.p = np.asarray(params, np.float32)
        self.exact = exact

    def r(self, x):
        return np.asarray(x, np.float64) if self.exact else bf16(np.asarray(x, np.float32))

    def weights(self, i):
        w_off, b_off, n, cins = self.lay[i]
        cin = sum(cins)
        w = self.p[w_off:w_off + 27 * n * cin].reshape(27, n, cin)
        return (w.astype(np.float64) if self.exact else bf16(w)), self.p[b_off:b_off + n].astype(np.float64), cins

    def forward(self, inp):
        a = {"in": np.asarray(inp, np.float64 if self.exact else np.float32)}
        for i, (ins, n, name) in enumerate(LAYERS):
            w, b, _ = self.weights(i)
            a[name] = conv3d([a[k] for k in ins], w, b, relu=True, round_out=not self.exact)
            if i in RESAMPLE_AFTER:
                kind, src, dst = RESAMPLE_AFTER[i]
                if kind == "pool":
                    a[dst] = pool(a[src]) if not self.exact else pool_exact(a[src])
                else:
                    a[dst] = upsample(a[src])
        hw = self.p[self.head_off:self.head_off + 16].astype(np.float64)
        hb = float(self.p[self.head_off + 16])
        guess = a["d0"].astype(np.float64) @ hw + hb
        self.a = a
        return guess if self.exact else guess.astype(np.float32)

    def loss_and_grads(self, inp, target):
        guess = self.forward(inp)
        a = self.a
        fluid = np.asarray(inp)[..., 1] > 0.5
        nf = max(int(fluid.sum()), 1)
        diff = np.where(fluid, guess.astype(np.float64) - np.asarray(target, np.float64), 0.0)
        loss = float((diff * diff).sum() / nf)
        dy = 2.0 * diff / nf
        grads = np.zeros(self.num_params, np.float64)
        hw = self.p[self.head_off:self.head_off + 16].astype(np.float64)
        d0 = a["d0"].astype(np.float64)
        grads[self.head_off:self.head_off + 16] = (d0 * dy[..., None]).reshape(-1, 16).sum(axis=0)
        grads[self.head_off + 16] = dy.sum()
        g = {"d0": self.r(np.where(d0 > 0, dy[..., None] * hw, 0.0))}
        for i in range(len(LAYERS) - 1, -1, -1):
            ins, n, name = LAYERS[i]
            w, b, cins = self.weights(i)
            dz = g[name]
            dw, db = conv3d_wgrad([a[k] for k in ins], dz)
            w_off, b_off, _, _ = self.lay[i]
            grads[w_off:w_off + dw.size] = dw.reshape(-1)
            grads[b_off:b_off + n] = db
            if i == 0:
                break
            parts = conv3d_dgrad(dz, w, cins)
            for k, src in enumerate(ins):
                v = parts[k]
                if k == 0 and src not in CHANNELS:  # a ReLU tensor whose only consumer is this layer
                    v = np.where(a[src] > 0, v, 0.0)
                g[src] = self.r(v)
            # resampling before layer i, backwards
            back = {12: ("up", "u0", "d1"), 10: ("up", "u1", "d2"), 8: ("up", "u2", "e3"),
                    6: ("pool", "p3", "e2"), 4: ("pool", "p2", "e1"), 2: ("pool", "p1", "e0")}
            if i in back:
                kind, src, dst = back[i]
                if kind == "up":
                    v = upsample_bwd(g[src]) if not self.exact else upsample_bwd_exact(g[src])
                    g[dst] = self.r(np.where(a[dst] > 0, v, 0.0))
                else:
                    v = pool_bwd(g[src]) if not self.exact else pool_bwd_exact(g[src])
                    # the skip connection's contribution (from the decoder) was stored first
                    tot = (np.asarray(g[dst], np.float64 if self.exact else np.float32) + v)
                    g[dst] = self.r(np.where(a[dst] > 0, tot, 0.0))
        return loss, grads, guess


def pool_exact(x):
    x = np.asarray(x, np.float64)
    s = sum(x[:, (o >> 2) & 1::2, (o >> 1) & 1::2, o & 1::2] for o in range(8))
    return s * 0.125


def pool_bwd_exact(g):
    g = np.asarray(g, np.float64) * 0.125
    return np.repeat(np.repeat(np.repeat(g, 2, 1), 2, 2), 2, 3)


def upsample_bwd_exact(g):
    g = np.asarray(g, np.float64)
    return sum(g[:, (o >> 2) & 1::2, (o >> 1) & 1::2, o & 1::2] for o in range(8))
