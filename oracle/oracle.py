"""TEST INFRASTRUCTURE -- Python handle on the CPU oracle (liboracle.so, built from slosh_oracle.hpp).

Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py use this module: as the
reference the GPU results are compared with, or as the timed CPU baseline. Its calls mirror the product's C ABI so a parity test drives both sides the same way.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from slosh_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build(force=False):
    """Compiles liboracle.so with the committed Makefile."""
    if force or not os.path.exists(_LIB_PATH) or _stale():
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def _stale():
    lib_t = os.path.getmtime(_LIB_PATH)
    srcs = [os.path.join(_HERE, f) for f in ("slosh_oracle.hpp", "oracle_capi.cpp", "Makefile")]
    srcs.append(os.path.join(_HERE, "..", "include", "slosh_cuda.h"))
    return any(os.path.getmtime(s) > lib_t for s in srcs if os.path.exists(s))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp = C.c_void_p
        L.oracle_create.argtypes = [C.POINTER(A.Settings), C.c_int, C.POINTER(vp)]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_destroy.restype = None
        L.oracle_set_emit_seed.argtypes = [vp, C.c_uint32]
        L.oracle_begin_frame.argtypes = [vp, C.POINTER(A.FrameInput), C.POINTER(C.c_int32), C.POINTER(C.c_float)]
        L.oracle_substep.argtypes = [vp, C.c_int32]
        L.oracle_end_frame.argtypes = [vp]
        L.oracle_step_frame.argtypes = [vp, C.POINTER(A.FrameInput)]
        L.oracle_emit.argtypes = [vp, C.POINTER(A.EmitRequest)]
        L.oracle_sort_particles.argtypes = [vp]
        L.oracle_upload_particles.argtypes = [vp, C.c_void_p, C.c_uint32]
        L.oracle_get_layout.argtypes = [vp, C.POINTER(A.Layout)]
        L.oracle_get_results.argtypes = [vp, C.POINTER(A.Results)]
        L.oracle_buffer_bytes.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t)]
        L.oracle_read_buffer.argtypes = [vp, C.c_int, C.c_void_p, C.c_size_t]
        L.oracle_read_buffer_f64.argtypes = [vp, C.c_int, C.c_void_p, C.c_size_t]
        L.oracle_build_surface.argtypes = [vp, C.POINTER(A.SurfaceParams), C.POINTER(A.SurfaceInfo)]
        L.oracle_write_buffer.argtypes = [vp, C.c_int, C.c_void_p, C.c_size_t]
        L.oracle_copy_state.argtypes = [vp, vp]
        L.oracle_settings_default.argtypes = [C.POINTER(A.Settings)]
        L.oracle_settings_default.restype = None
        L.oracle_f32_to_f16.argtypes = [C.c_float]
        L.oracle_f32_to_f16.restype = C.c_uint16
        L.oracle_f32_to_bf16.argtypes = [C.c_float]
        L.oracle_f32_to_bf16.restype = C.c_uint16
        L.oracle_f16_to_f32.argtypes = [C.c_uint16]
        L.oracle_f16_to_f32.restype = C.c_float
        L.oracle_pcg_hash.argtypes = [C.c_uint32]
        L.oracle_pcg_hash.restype = C.c_uint32
        L.oracle_hash_to_unit.argtypes = [C.c_uint32]
        L.oracle_hash_to_unit.restype = C.c_float
        L.oracle_reduce_final.argtypes = [C.c_void_p, C.c_uint32]
        L.oracle_reduce_final.restype = C.c_double
        L.oracle_reduce_brick.argtypes = [C.c_void_p]
        L.oracle_reduce_brick.restype = C.c_double
        L.oracle_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def settings_default():
    s = A.Settings()
    lib().oracle_settings_default(C.byref(s))
    return s


def set_threads(n):
    return lib().oracle_set_threads(int(n))


def _check(rc, what):
    if rc not in (A.OK,) + A.WARNINGS:
        raise RuntimeError(f"oracle {what} failed with status {rc}")
    return rc


class Oracle:
    """One simulated domain on the CPU (FP32 canonical, or FP64 with fp64=True)."""

    def __init__(self, settings, fp64=False):
        self._h = C.c_void_p()
        self.fp64 = fp64
        _check(lib().oracle_create(C.byref(settings), 1 if fp64 else 0, C.byref(self._h)), "create")
        self.settings = settings

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_emit_seed(self, seed):
        _check(lib().oracle_set_emit_seed(self._h, seed), "set_emit_seed")

    def begin_frame(self, fi):
        n = C.c_int32()
        dt = C.c_float()
        _check(lib().oracle_begin_frame(self._h, C.byref(fi), C.byref(n), C.byref(dt)), "begin_frame")
        return n.value, dt.value

    def substep(self, i):
        _check(lib().oracle_substep(self._h, i), "substep")

    def end_frame(self):
        _check(lib().oracle_end_frame(self._h), "end_frame")

    def step_frame(self, fi):
        _check(lib().oracle_step_frame(self._h, C.byref(fi)), "step_frame")

    def emit(self, req):
        _check(lib().oracle_emit(self._h, C.byref(req)), "emit")

    def sort_particles(self):
        _check(lib().oracle_sort_particles(self._h), "sort")

    def upload_particles(self, arr):
        arr = np.ascontiguousarray(arr, dtype=A.PARTICLE_DTYPE)
        _check(lib().oracle_upload_particles(self._h, arr.ctypes.data, len(arr)), "upload")

    def layout(self):
        L = A.Layout()
        _check(lib().oracle_get_layout(self._h, C.byref(L)), "layout")
        return L

    def results(self):
        r = A.Results()
        _check(lib().oracle_get_results(self._h, C.byref(r)), "results")
        return r

    def build_surface(self, params):
        info = A.SurfaceInfo()
        _check(lib().oracle_build_surface(self._h, C.byref(params), C.byref(info)), "build_surface")
        return info

    def read(self, name):
        bid = A.BUF[name]
        n = C.c_size_t()
        _check(lib().oracle_buffer_bytes(self._h, bid, C.byref(n)), "buffer_bytes")
        dt = A.BUF_DTYPE[name] or A.PARTICLE_DTYPE
        out = np.empty(n.value // np.dtype(dt).itemsize, dtype=dt)
        _check(lib().oracle_read_buffer(self._h, bid, out.ctypes.data, n.value), "read_buffer")
        return out

    def read_f64(self, name):
        bid = A.BUF[name]
        n = C.c_size_t()
        _check(lib().oracle_buffer_bytes(self._h, bid, C.byref(n)), "buffer_bytes")
        out = np.empty(n.value // 4, dtype=np.float64)
        _check(lib().oracle_read_buffer_f64(self._h, bid, out.ctypes.data, out.size), "read_buffer_f64")
        return out

    def write(self, name, arr):
        arr = np.ascontiguousarray(arr)
        _check(lib().oracle_write_buffer(self._h, A.BUF[name], arr.ctypes.data, arr.nbytes), "write_buffer")

    def copy_state_from(self, other):
        _check(lib().oracle_copy_state(self._h, other._h), "copy_state")
