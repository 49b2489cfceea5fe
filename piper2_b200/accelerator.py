"""Host mirror of the reference's Accelerator interface (Src/Interface/Infrastructure/Accelerator.hpp:130-161) over
the C ABI's pb2_acc_* calls (the CUDA accelerator, Src/Infrastructure/Accelerator/CUDA/CUDA.cpp:497-927).

    acc = Accelerator()
    x = acc.create_buffer(nbytes, 64, lambda view: view[:] = ...)      # createBuffer(size, alignment, fill)
    z = acc.create_tiled_output(nbytes, 64)                           # createTiledOutput
    lut = acc.create_resource_lut([x, y, z])                          # createResourceLUT
    kernel = acc.compile_kernel("convEntry")                          # compileKernel (registered native kernels)
    fut = acc.launch_kernel((height, 1, width), kernel, lut, np.uint32(w), np.uint32(h), np.uint32(k))
    z.mark_dirty(fut)
    data = z.download()                                               # Future<Binary> -> bytes

Arguments are packed as the reference's ArgumentPackage (Accelerator.hpp:95-118): each trivially copyable
argument (a numpy scalar, a ctypes value or structure, or bytes) appended to one byte string with its
(offset, size) pair.  Errors raise capi.PB2Error (the reference logs and aborts).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi


def _bytes(arg) -> bytes:
    if isinstance(arg, (bytes, bytearray)):
        return bytes(arg)
    if isinstance(arg, np.generic):
        return arg.tobytes()
    if isinstance(arg, (C._SimpleCData, C.Structure, C.Array)):
        return C.string_at(C.addressof(arg), C.sizeof(arg))
    raise TypeError(f"argument of type {type(arg).__name__} is not trivially copyable; pass a numpy scalar, a ctypes "
                    "value or bytes")


def pack_arguments(*args):
    """ArgumentPackage: (data bytes, flat (offset, size) array) of the arguments in order."""
    data = bytearray()
    desc = []
    for a in args:
        b = _bytes(a)
        desc += [len(data), len(b)]
        data += b
    return bytes(data), np.asarray(desc, dtype=np.uint32)


def pack_launch(handles, *args) -> bytes:
    """The launch buffer the library writes for these table handles and arguments (pb2_acc_pack_launch)."""
    data, desc = pack_arguments(*args)
    h = np.ascontiguousarray(handles, dtype=np.uint64)
    hp = h.ctypes.data_as(C.POINTER(C.c_uint64)) if h.size else None
    dp = desc.ctypes.data_as(C.POINTER(C.c_uint32)) if desc.size else None
    dbuf = C.create_string_buffer(data, max(len(data), 1))
    need = C.c_size_t()
    lib = capi.lib()
    capi.check(lib.pb2_acc_pack_launch(hp, h.size, dbuf, dp, len(desc) // 2, None, 0, C.byref(need)))
    out = C.create_string_buffer(need.value)
    capi.check(lib.pb2_acc_pack_launch(hp, h.size, dbuf, dp, len(desc) // 2, out, need.value, C.byref(need)))
    return out.raw[:need.value]


class Future:
    """Future<void> of a launch or upload."""

    def __init__(self, h):
        self.h = h

    def wait(self):
        capi.check(capi.lib().pb2_future_wait(self.h))

    def ready(self) -> bool:
        r = C.c_int()
        capi.check(capi.lib().pb2_future_ready(self.h, C.byref(r)))
        return bool(r.value)

    def release(self):
        if self.h:
            capi.lib().pb2_future_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Resource:
    def __init__(self, h, size=0):
        self.h = h
        self.size = size

    @property
    def handle(self) -> int:
        v = C.c_uint64()
        capi.check(capi.lib().pb2_resource_get_handle(self.h, C.byref(v)))
        return v.value

    def release(self):
        if self.h:
            capi.lib().pb2_resource_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class TiledOutput(Resource):
    def mark_dirty(self, future: Future):
        capi.check(capi.lib().pb2_tiled_output_mark_dirty(self.h, future.h))

    def download(self) -> bytes:
        buf = C.create_string_buffer(self.size)
        capi.check(capi.lib().pb2_tiled_output_download(self.h, buf, self.size))
        return buf.raw


class Kernel:
    def __init__(self, h, entry):
        self.h = h
        self.entry = entry

    def release(self):
        if self.h:
            capi.lib().pb2_kernel_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class Accelerator:
    """One device (the current one), `streams` CUDA streams (0 = the library's default)."""

    def __init__(self, streams: int = 0):
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_create(streams, C.byref(h)))
        self.h = h
        self._fills = []

    def get_native_platform(self) -> str:
        return capi.lib().pb2_acc_native_platform(self.h).decode()

    def info(self):
        d, s = C.c_int(), C.c_uint32()
        capi.check(capi.lib().pb2_acc_get_info(self.h, C.byref(d), C.byref(s)))
        return d.value, s.value

    def create_buffer(self, size: int, alignment: int, fill=None) -> Resource:
        """`fill(view)` writes the initial bytes into `view`, a writable numpy uint8 array of `size` bytes."""
        cb = None
        if fill is not None:
            def _fill(dst, n, _user):
                fill(np.ctypeslib.as_array(C.cast(dst, C.POINTER(C.c_uint8)), shape=(n,)))
            cb = capi.FILL_FN(_fill)
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_create_buffer(self.h, size, alignment, C.cast(cb, C.c_void_p) if cb else None,
                                                    None, C.byref(h)))
        return Resource(h, size)

    def create_tiled_output(self, size: int, alignment: int) -> TiledOutput:
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_create_tiled_output(self.h, size, alignment, C.byref(h)))
        return TiledOutput(h, size)

    def create_resource_lut(self, resources) -> Resource:
        arr = (C.c_void_p * max(len(resources), 1))(*[r.h for r in resources])
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_create_resource_lut(self.h, arr, len(resources), C.byref(h)))
        return Resource(h)

    def register_kernel(self, entry: str, cu_function: int):
        capi.check(capi.lib().pb2_acc_register_kernel(self.h, entry.encode(), C.c_void_p(cu_function)))

    def compile_kernel(self, entry: str) -> Kernel:
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_compile_kernel(self.h, entry.encode(), C.byref(h)))
        return Kernel(h, entry)

    def launch_kernel(self, dim, kernel: Kernel, root: Resource | None, *args) -> Future:
        data, desc = pack_arguments(*args)
        d = (C.c_uint32 * 3)(*dim)
        dbuf = C.create_string_buffer(data, max(len(data), 1))
        dp = desc.ctypes.data_as(C.POINTER(C.c_uint32)) if desc.size else None
        h = C.c_void_p()
        capi.check(capi.lib().pb2_acc_launch_kernel(self.h, d, kernel.h, root.h if root else None, dbuf, dp,
                                                    len(desc) // 2, C.byref(h)))
        return Future(h)

    def close(self):
        if self.h:
            capi.lib().pb2_acc_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
