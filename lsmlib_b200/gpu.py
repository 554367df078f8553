"""ctypes binding of liblsmgpu.so (the CUDA library).

``load()`` opens the in-tree library and fails loudly when it is missing:
there is no CPU fallback.  ``toolbox()`` returns a
:class:`lsmlib_b200.toolbox.Toolbox` over the library's reference-compatible
symbols that raises :class:`LsmgpuError` when a call records an error.
"""
import ctypes
import os

import numpy as np

from .toolbox import Field, Toolbox

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblsmgpu.so")

_lib = None


class LsmgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("lsmgpu error %d: %s" % (code, msg))
        self.code = code


ERR_NAMES = {0: "SUCCESS", 1: "INVALID_BOX", 2: "NULL_POINTER", 3: "CUDA",
             4: "ALLOC", 5: "INVALID_VALUE", 6: "DEVICE"}

_EXT = {
    # name: (restype, argtypes)
    "lsmgpu_get_last_error": (ctypes.c_int, []),
    "lsmgpu_peek_last_error": (ctypes.c_int, []),
    "lsmgpu_get_last_error_string": (ctypes.c_char_p, []),
    "lsmgpu_set_device": (ctypes.c_int, [ctypes.c_int]),
    "lsmgpu_set_stream": (ctypes.c_int, [ctypes.c_void_p]),
    "lsmgpu_get_stream": (ctypes.c_void_p, []),
    "lsmgpu_set_sync": (ctypes.c_int, [ctypes.c_int]),
    "lsmgpu_set_fp_mode": (ctypes.c_int, [ctypes.c_int]),
    "lsmgpu_get_fp_mode": (ctypes.c_int, []),
    "lsmgpu_stream_synchronize": (ctypes.c_int, []),
    "lsmgpu_kernel_launch_count": (ctypes.c_ulonglong, []),
    "lsmgpu_malloc": (ctypes.c_void_p, [ctypes.c_size_t]),
    "lsmgpu_free": (ctypes.c_int, [ctypes.c_void_p]),
    "lsmgpu_host_alloc": (ctypes.c_void_p, [ctypes.c_size_t]),
    "lsmgpu_host_free": (ctypes.c_int, [ctypes.c_void_p]),
    "lsmgpu_release_scratch": (ctypes.c_int, []),
    "lsmgpu_memcpy_htod": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "lsmgpu_memcpy_dtoh": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "lsmgpu_memcpy_dtod": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]),
    "lsmgpu_event_create": (ctypes.c_void_p, []),
    "lsmgpu_event_record": (ctypes.c_int, [ctypes.c_void_p]),
    "lsmgpu_event_elapsed_ms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.POINTER(ctypes.c_float)]),
    "lsmgpu_event_destroy": (ctypes.c_int, [ctypes.c_void_p]),
}


def load(path=LIB_PATH):
    """Open liblsmgpu.so (once).  Raises if the library was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(
            "%s is missing: build it with `python -m lsmlib_b200.build` "
            "(there is no CPU fallback)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in _EXT.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _bind_extra(lib)
    _lib = lib
    return lib


def _bind_extra(lib):
    """Bind the fused-stepper / batched / adjoint entry points when present."""
    from . import ext_abi
    for name, (res, args) in ext_abi.SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is not None:
            fn.restype, fn.argtypes = res, args


def check(where="lsmgpu"):
    lib = load()
    code = lib.lsmgpu_peek_last_error()
    if code != 0:
        msg = lib.lsmgpu_get_last_error_string().decode()
        lib.lsmgpu_get_last_error()
        raise LsmgpuError(code, "%s: %s" % (where, msg))


def check_rc(rc, where):
    if rc != 0:
        check(where)
        raise LsmgpuError(rc, where)


def toolbox():
    """Reference-compatible routines of the GPU library."""
    return Toolbox(load(), prefix="", check=check)


class DeviceArray:
    """A device buffer holding a Fortran-ordered 3D array."""

    def __init__(self, shape, dtype=np.float64):
        self.shape = tuple(int(x) for x in shape)
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        lib = load()
        self.ptr = lib.lsmgpu_malloc(max(self.nbytes, 1))
        if not self.ptr:
            check("lsmgpu_malloc")
            raise MemoryError("lsmgpu_malloc(%d) failed" % self.nbytes)

    @classmethod
    def from_host(cls, arr):
        arr = np.asfortranarray(arr)
        d = cls(arr.shape, arr.dtype)
        d.upload(arr)
        return d

    def upload(self, arr):
        arr = np.asfortranarray(arr, dtype=self.dtype)
        assert arr.shape == self.shape
        check_rc(load().lsmgpu_memcpy_htod(self.ptr, arr.ctypes.data, self.nbytes),
                 "memcpy_htod")

    def download(self, out=None):
        if out is None:
            out = np.empty(self.shape, dtype=self.dtype, order="F")
        check_rc(load().lsmgpu_memcpy_dtoh(out.ctypes.data, self.ptr, self.nbytes),
                 "memcpy_dtoh")
        return out

    def free(self):
        if self.ptr:
            load().lsmgpu_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def device_field(field):
    """Copy a host :class:`Field` to the device (same lower bounds)."""
    return Field(DeviceArray.from_host(field.data), field.lo)


def host_field(dfield):
    return Field(dfield.data.download(), dfield.lo)


class Timer:
    """CUDA-event timer on the library's current stream."""

    def __init__(self):
        lib = load()
        self.a, self.b = lib.lsmgpu_event_create(), lib.lsmgpu_event_create()

    def start(self):
        load().lsmgpu_event_record(self.a)

    def stop(self):
        load().lsmgpu_event_record(self.b)

    def ms(self):
        v = ctypes.c_float()
        check_rc(load().lsmgpu_event_elapsed_ms(self.a, self.b, ctypes.byref(v)),
                 "event_elapsed")
        return v.value

    def __del__(self):
        try:
            lib = load()
            lib.lsmgpu_event_destroy(self.a)
            lib.lsmgpu_event_destroy(self.b)
        except Exception:
            pass
