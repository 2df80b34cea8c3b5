"""B200-native FLIP/APIC simulation substep of the Slosh liquid solver.

The compute path is libslosh_b200.so (hand-written sm_100a CUDA kernels and a C++ host driver behind
the C ABI in include/slosh_cuda.h). This module is a thin ctypes mirror of the plugin's proxy
interface (FSloshProxy, SloshDemo/Plugins/Slosh/Source/SloshCore/Public/SloshProxy.h:23-147):
`Simulation.step_frame` stands in for SubmitFrame_GameThread + Step_RenderThread, `results()` for
GetResults, `particles()` / `particle_device_ptr()` for GetParticleBuffer_RenderThread. There is no CPU
fallback: constructing a Simulation without the built library or without a CUDA device raises.
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (BUF, EmitRequest, FrameInput, Layout, Particle, PARTICLE_DTYPE, Results, Settings, SurfaceInfo,  # noqa: F401
                   SurfaceParams,
                   frame_input)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libslosh_b200.so")

# Every function the header declares, with its ctypes signature.
_VP = C.c_void_p
SIGNATURES = {
    "slosh_abi_version": ([], C.c_uint32),
    "slosh_settings_default": ([C.POINTER(Settings)], None),
    "slosh_last_error_string": ([], C.c_char_p),
    "slosh_create": ([C.POINTER(Settings), C.c_int32, C.POINTER(_VP)], C.c_int),
    "slosh_destroy": ([_VP], None),
    "slosh_set_stream": ([_VP, _VP], C.c_int),
    "slosh_synchronize": ([_VP], C.c_int),
    "slosh_step_frame": ([_VP, C.POINTER(FrameInput)], C.c_int),
    "slosh_begin_frame": ([_VP, C.POINTER(FrameInput), C.POINTER(C.c_int32), C.POINTER(C.c_float)], C.c_int),
    "slosh_substep": ([_VP, C.c_int32], C.c_int),
    "slosh_end_frame": ([_VP], C.c_int),
    "slosh_sort_particles": ([_VP], C.c_int),
    "slosh_sort_particles_static": ([_VP, _VP, C.c_uint32, C.POINTER(C.c_int32), C.c_float, _VP, _VP, _VP, _VP], C.c_int),
    "slosh_emit": ([_VP, C.POINTER(EmitRequest)], C.c_int),
    "slosh_set_emit_seed": ([_VP, C.c_uint32], C.c_int),
    "slosh_upload_particles": ([_VP, _VP, C.c_uint32], C.c_int),
    "slosh_download_particles": ([_VP, _VP, C.c_uint32, C.POINTER(C.c_uint32)], C.c_int),
    "slosh_particle_device_ptr": ([_VP, C.POINTER(_VP), C.POINTER(C.c_uint32)], C.c_int),
    "slosh_get_results": ([_VP, C.POINTER(Results)], C.c_int),
    "slosh_get_layout": ([_VP, C.POINTER(Layout)], C.c_int),
    "slosh_buffer_bytes": ([_VP, C.c_int32, C.POINTER(C.c_size_t)], C.c_int),
    "slosh_read_buffer": ([_VP, C.c_int32, _VP, C.c_size_t], C.c_int),
    "slosh_write_buffer": ([_VP, C.c_int32, _VP, C.c_size_t], C.c_int),
    "slosh_enable_phase_timing": ([_VP, C.c_int32], C.c_int),
    "slosh_get_phase_ms": ([_VP, C.POINTER(C.c_float), C.c_int32], C.c_int),
    "slosh_launch_count": ([_VP], C.c_uint64),
    "slosh_transfer_bytes": ([_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
    "slosh_step_frames": ([C.POINTER(_VP), C.POINTER(FrameInput), C.c_uint32, C.POINTER(C.c_int)], C.c_int),
    "slosh_surface_params_default": ([C.POINTER(SurfaceParams)], None),
    "slosh_build_surface": ([_VP, C.POINTER(SurfaceParams), C.POINTER(SurfaceInfo)], C.c_int),
    "slosh_surface_device_ptrs": ([_VP, C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP)], C.c_int),
    "slosh_autotune": ([_VP, C.POINTER(FrameInput), C.c_uint32, C.POINTER(_abi.AutotuneResult)], C.c_int),
    "slosh_set_ctas_per_sm": ([_VP, C.c_uint32], C.c_int),
    "slosh_set_mg_ctas_per_sm": ([_VP, C.c_uint32], C.c_int),
    "slosh_unet_config_default": ([C.POINTER(_abi.UnetConfig)], None),
    "slosh_unet_create": ([C.POINTER(_abi.UnetConfig), C.c_int32, C.POINTER(_VP)], C.c_int),
    "slosh_unet_destroy": ([_VP], None),
    "slosh_unet_last_error": ([], C.c_char_p),
    "slosh_unet_num_params": ([_VP], C.c_uint64),
    "slosh_unet_get_params": ([_VP, C.c_void_p, C.c_uint64], C.c_int),
    "slosh_unet_set_params": ([_VP, C.c_void_p, C.c_uint64], C.c_int),
    "slosh_unet_set_sample": ([_VP, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32], C.c_int),
    "slosh_unet_capture_sample": ([_VP, _VP, C.c_uint32], C.c_int),
    "slosh_unet_forward": ([_VP, C.c_void_p], C.c_int),
    "slosh_unet_backward": ([_VP, C.POINTER(C.c_float), C.c_void_p], C.c_int),
    "slosh_unet_train_step": ([_VP, C.POINTER(C.c_float)], C.c_int),
    "slosh_unet_launch_count": ([_VP], C.c_uint64),
    "slosh_set_warm_start_network": ([_VP, _VP], C.c_int),
    "slosh_unet_conv_test": ([C.POINTER(_abi.ConvTest)], C.c_int),
}
PHASES = ("sort", "pool", "p2g", "grid", "pressure", "project", "density", "extrapolate", "g2p")

_lib = None


class SloshError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"slosh status {status}: {message}")
        self.status = status


def load_library(path=None):
    """Loads libslosh_b200.so and binds the C ABI; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise SloshError(_abi.ERR_NO_DEVICE, f"{p} is missing: build it with `python -m slosh_b200.build`")
    lib = C.CDLL(p)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def step_frames(sims, inputs):
    """One frame of each Simulation in `sims` with the matching FrameInput, overlapped on the device
    (slosh_step_frames). Returns the per-simulation status codes."""
    n = len(sims)
    if n != len(inputs):
        raise ValueError("one frame input per simulation")
    ctxs = (_VP * max(n, 1))(*[s._ctx for s in sims])
    fis = (FrameInput * max(n, 1))(*inputs)
    st = (C.c_int * max(n, 1))()
    _check(load_library().slosh_step_frames(ctxs, fis, n, st))
    return list(st)[:n]


def surface_params_default():
    q = SurfaceParams()
    load_library().slosh_surface_params_default(C.byref(q))
    return q


def settings_default():
    s = Settings()
    load_library().slosh_settings_default(C.byref(s))
    return s


def _check(rc, allow_warnings=True):
    if rc == _abi.OK or (allow_warnings and rc in _abi.WARNINGS):
        return rc
    msg = load_library().slosh_last_error_string()
    raise SloshError(rc, msg.decode() if msg else "")


def sort_particles_static(particles_in, particles_out, count, grid_dim, cell_size, perm_out=0, key_offsets_out=0,
                          live_count_out=0, stream=0):
    """Allocation-free sort of caller-owned device particle records (slosh_sort_particles_static).

    Pointers are device addresses (ints) on the current device; the call is enqueued on `stream` (a
    cudaStream_t as int, 0 = default stream) and returns without waiting for it."""
    lib = load_library()
    dims = (C.c_int32 * 3)(*[int(v) for v in grid_dim])
    _check(lib.slosh_sort_particles_static(C.c_void_p(particles_in), C.c_void_p(particles_out), int(count), dims,
                                           float(cell_size), C.c_void_p(perm_out or None),
                                           C.c_void_p(key_offsets_out or None), C.c_void_p(live_count_out or None),
                                           C.c_void_p(stream or None)), allow_warnings=False)


class Simulation:
    """One liquid domain on one GPU (the C-ABI context)."""

    def __init__(self, settings, device=-1):
        self._lib = load_library()
        self._ctx = C.c_void_p()
        _check(self._lib.slosh_create(C.byref(settings), int(device), C.byref(self._ctx)), allow_warnings=False)
        self.settings = settings

    def close(self):
        if self._ctx:
            self._lib.slosh_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- frame ----
    def step_frame(self, fi):
        return _check(self._lib.slosh_step_frame(self._ctx, C.byref(fi)))

    def begin_frame(self, fi):
        n, dt = C.c_int32(), C.c_float()
        _check(self._lib.slosh_begin_frame(self._ctx, C.byref(fi), C.byref(n), C.byref(dt)))
        return n.value, dt.value

    def substep(self, i):
        return _check(self._lib.slosh_substep(self._ctx, int(i)))

    def end_frame(self):
        return _check(self._lib.slosh_end_frame(self._ctx))

    def sort_particles(self):
        _check(self._lib.slosh_sort_particles(self._ctx))

    def emit(self, req):
        _check(self._lib.slosh_emit(self._ctx, C.byref(req)))

    def set_emit_seed(self, seed):
        _check(self._lib.slosh_set_emit_seed(self._ctx, int(seed)))

    def set_stream(self, stream_handle):
        _check(self._lib.slosh_set_stream(self._ctx, C.c_void_p(stream_handle)))

    def synchronize(self):
        _check(self._lib.slosh_synchronize(self._ctx))

    # ---- particles ----
    def upload_particles(self, arr):
        arr = np.ascontiguousarray(arr, dtype=PARTICLE_DTYPE)
        _check(self._lib.slosh_upload_particles(self._ctx, arr.ctypes.data, len(arr)))

    def particles(self):
        n = C.c_uint32()
        _check(self._lib.slosh_download_particles(self._ctx, None, 0, C.byref(n)))
        out = np.empty(n.value, dtype=PARTICLE_DTYPE)
        _check(self._lib.slosh_download_particles(self._ctx, out.ctypes.data, n.value, C.byref(n)))
        return out

    def particle_device_ptr(self):
        p, n = C.c_void_p(), C.c_uint32()
        _check(self._lib.slosh_particle_device_ptr(self._ctx, C.byref(p), C.byref(n)))
        return p.value, n.value

    # ---- state ----
    def results(self):
        r = Results()
        _check(self._lib.slosh_get_results(self._ctx, C.byref(r)))
        return r

    def layout(self):
        L = Layout()
        _check(self._lib.slosh_get_layout(self._ctx, C.byref(L)))
        return L

    def read(self, name):
        bid = BUF[name]
        n = C.c_size_t()
        _check(self._lib.slosh_buffer_bytes(self._ctx, bid, C.byref(n)))
        dt = _abi.BUF_DTYPE[name] or PARTICLE_DTYPE
        out = np.empty(n.value // np.dtype(dt).itemsize, dtype=dt)
        _check(self._lib.slosh_read_buffer(self._ctx, bid, out.ctypes.data, n.value))
        return out

    def write(self, name, arr):
        arr = np.ascontiguousarray(arr)
        _check(self._lib.slosh_write_buffer(self._ctx, BUF[name], arr.ctypes.data, arr.nbytes))

    def enable_phase_timing(self, on=True):
        _check(self._lib.slosh_enable_phase_timing(self._ctx, 1 if on else 0))

    def phase_ms(self):
        out = (C.c_float * len(PHASES))()
        _check(self._lib.slosh_get_phase_ms(self._ctx, out, len(PHASES)))
        return dict(zip(PHASES, list(out)))

    # ---- headless surface ----
    def build_surface(self, params=None):
        """Density field and surface-nets mesh of the current particles (slosh_build_surface)."""
        q = params or surface_params_default()
        info = SurfaceInfo()
        _check(self._lib.slosh_build_surface(self._ctx, C.byref(q), C.byref(info)), allow_warnings=False)
        return info

    def launch_count(self):
        return int(self._lib.slosh_launch_count(self._ctx))

    # ---- launch-shape autotuner ----
    def autotune(self, fi, frames=2):
        """Times `frames` frames of fi per candidate CTAs-per-SM count of the brick passes and keeps the
        fastest (slosh_autotune); the simulation advances by those frames. Returns the result struct."""
        r = _abi.AutotuneResult()
        _check(self._lib.slosh_autotune(self._ctx, C.byref(fi), int(frames), C.byref(r)))
        return r

    def set_ctas_per_sm(self, n):
        _check(self._lib.slosh_set_ctas_per_sm(self._ctx, int(n)))

    def set_mg_ctas_per_sm(self, n):
        _check(self._lib.slosh_set_mg_ctas_per_sm(self._ctx, int(n)))

    def transfer_bytes(self):
        h2d, d2h = C.c_uint64(), C.c_uint64()
        _check(self._lib.slosh_transfer_bytes(self._ctx, C.byref(h2d), C.byref(d2h)))
        return int(h2d.value), int(d2h.value)
