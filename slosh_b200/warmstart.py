"""Learned warm start of the pressure solve: ctypes binding of the U-Net C ABI (include/slosh_cuda.h,
slosh_unet_*) and the randomised training scenes.

The network (4 levels, 16/32/64/64 channels, 3x3x3 convolutions, BF16 weights and activations, FP32
accumulation) runs and trains on the GPU with the library's own tcgen05 kernels; this module only
moves host arrays and drives the steps. A simulation with settings.warm_start = WARM_START_LEARNED and
a network attached (Simulation.set_warm_start_network) starts each pressure solve from the network's
guess and still iterates to its stopping test.
"""
import ctypes as C

import numpy as np

from . import _abi, load_library, _check, SloshError
from ._abi import Collider, ConvTest, EmitRequest, UnetConfig

_VP = C.c_void_p


def lib():
    return load_library()


def _ucheck(rc):
    if rc == _abi.OK:
        return rc
    msg = lib().slosh_unet_last_error()
    raise SloshError(rc, msg.decode() if msg else "")


def config_default():
    c = UnetConfig()
    lib().slosh_unet_config_default(C.byref(c))
    return c


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class WarmStartNet:
    """The U-Net on one GPU: parameters, training slots and the forward / backward / Adam steps."""

    def __init__(self, dim=(128, 128, 128), batch=1, seed=10000, learning_rate=1e-3, device=-1):
        self._lib = lib()
        cfg = config_default()
        cfg.dim[:] = list(dim)
        cfg.batch = batch
        cfg.seed = seed
        cfg.learning_rate = learning_rate
        self.dim, self.batch = tuple(dim), batch
        self._net = C.c_void_p()
        _ucheck(self._lib.slosh_unet_create(C.byref(cfg), int(device), C.byref(self._net)))
        self.num_params = int(self._lib.slosh_unet_num_params(self._net))

    def close(self):
        if self._net:
            self._lib.slosh_unet_destroy(self._net)
            self._net = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._net

    def params(self):
        p = np.empty(self.num_params, np.float32)
        _ucheck(self._lib.slosh_unet_get_params(self._net, _ptr(p), self.num_params))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _ucheck(self._lib.slosh_unet_set_params(self._net, _ptr(p), self.num_params))

    def set_sample(self, slot, input_bits, target=None):
        """input_bits: uint16 [D][H][W][16] BF16 bit patterns; target [D][H][W] float32 or None."""
        inp = np.ascontiguousarray(input_bits, np.uint16)
        tg = np.ascontiguousarray(target, np.float32) if target is not None else None
        fluid = int((((inp[..., 1].astype(np.uint32)) << 16).view(np.float32) > 0.5).sum())
        _ucheck(self._lib.slosh_unet_set_sample(self._net, slot, _ptr(inp), _ptr(tg), fluid))

    def capture(self, sim, slot):
        _ucheck(self._lib.slosh_unet_capture_sample(self._net, sim._ctx, slot))

    def forward(self, out=True):
        g = np.empty((self.batch, self.dim[2], self.dim[1], self.dim[0]), np.float32) if out else None
        _ucheck(self._lib.slosh_unet_forward(self._net, _ptr(g)))
        return g

    def backward(self, grads=True):
        loss = C.c_float()
        g = np.empty(self.num_params, np.float32) if grads else None
        _ucheck(self._lib.slosh_unet_backward(self._net, C.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step(self):
        loss = C.c_float()
        _ucheck(self._lib.slosh_unet_train_step(self._net, C.byref(loss)))
        return loss.value

    def launch_count(self):
        return int(self._lib.slosh_unet_launch_count(self._net))


def attach(sim, net):
    """Attaches net (or None) as sim's warm-start network."""
    return _check(lib().slosh_set_warm_start_network(sim._ctx, net.handle if net is not None else None))


def conv_test(x_bits, w, bias, dy_bits, dim, batch=1):
    """One convolution through the library's kernels; x_bits: list of 1-2 uint16 arrays
    [B][D][H][W][cin_k]; returns (y_bits, [dx_bits], dw, db)."""
    t = ConvTest()
    t.dim[:] = list(dim)
    t.batch = batch
    t.nblocks = len(x_bits)
    xs = [np.ascontiguousarray(x, np.uint16) for x in x_bits]
    for k, x in enumerate(xs):
        t.cin[k] = x.shape[-1]
        t.x[k] = x.ctypes.data
    n = w.shape[1]
    t.cout = n
    w = np.ascontiguousarray(w, np.float32)
    b = np.ascontiguousarray(bias, np.float32)
    dy = np.ascontiguousarray(dy_bits, np.uint16)
    t.w, t.bias, t.dy = w.ctypes.data, b.ctypes.data, dy.ctypes.data
    shape = xs[0].shape[:-1]
    y = np.zeros(shape + (n,), np.uint16)
    dxs = [np.zeros(x.shape, np.uint16) for x in xs]
    dw = np.zeros(w.shape, np.float32)
    db = np.zeros(n, np.float32)
    t.y = y.ctypes.data
    for k, d in enumerate(dxs):
        t.dx[k] = d.ctypes.data
    t.dw, t.db = dw.ctypes.data, db.ctypes.data
    _ucheck(lib().slosh_unet_conv_test(C.byref(t)))
    return y, dxs, dw, db


# ---- randomised training scenes -------------------------------------------------------------------
def random_scene(settings_default, seed, n=128):
    """A scene of the learned-warm-start set: 1-4 fluid boxes (sizes U[0.1, 0.4] of the domain, 8
    particles per cell by FillCells), each with a velocity ~ N(0, 0.5^2) m/s per component, and 0-3
    static solid spheres (radius U[0.05, 0.15]); h = 1/n, gravity -9.81 y, tolerance 1e-6, zero warm
    start. Returns (settings, emits, colliders)."""
    rng = np.random.default_rng(seed)
    s = settings_default()
    s.grid_dim[:] = [n, n, n]
    s.cell_size = 1.0 / n
    s.gravity[:] = [0.0, -9.81, 0.0]
    s.tolerance = 1e-6
    s.max_iterations = 200
    s.warm_start = _abi.WARM_START_ZERO
    s.sort_interval = 4
    boxes = int(rng.integers(1, 5))
    emits = []
    cells_total = 0
    for _ in range(boxes):
        size = rng.uniform(0.1, 0.4, 3)
        lo = rng.uniform(0.0, 1.0 - size)
        cmin = np.maximum((lo * n).astype(int), 1)
        cdim = np.maximum(np.minimum((size * n).astype(int), n - 1 - cmin), 1)
        e = EmitRequest()
        e.shape = _abi.EMIT_FILL_CELLS
        e.cell_min[:] = [int(v) for v in cmin]
        e.cell_dims[:] = [int(v) for v in cdim]
        e.velocity[:] = [float(v) for v in rng.normal(0.0, 0.5, 3)]
        e.rotation[:] = [0.0, 0.0, 0.0, 1.0]
        e.fill_jitter = 1.0
        emits.append(e)
        cells_total += int(np.prod(cdim))
    colliders = []
    for _ in range(int(rng.integers(0, 4))):
        c = Collider()
        c.type = _abi.COLLIDER_SPHERE
        r = float(rng.uniform(0.05, 0.15))
        c.center[:] = [float(v) for v in rng.uniform(0.15, 0.85, 3)]
        c.extent[:] = [r, r, r]
        c.rotation[:] = [0.0, 0.0, 0.0, 1.0]
        colliders.append(c)
    s.particle_capacity = max(8 * cells_total + 1024, 1 << 20)
    return s, emits, colliders
