"""The accelerator's host side without a GPU: the launch buffer it builds has the layout of the reference's
CUDAAccelerator::launchKernelImpl (Src/Infrastructure/Accelerator/CUDA/CUDA.cpp:826-850), the Python mirror packs
arguments as the reference's ArgumentPackage (Src/Interface/Infrastructure/Accelerator.hpp:95-118), and creating
an accelerator where there is no device fails with a status instead of aborting."""
import ctypes as C
import struct

import numpy as np
import pytest

from piper2_b200 import accelerator, capi


def _reference_layout(handles, args):
    """CUDA.cpp:826-850 restated: [handle bytes + 8][handle + offset bytes + 8][handles][offsets][data]."""
    data = b"".join(args)
    offsets, off = [], 0
    for a in args:
        offsets.append((off, len(a)))
        off += len(a)
    hb = 8 * len(handles)
    ob = 8 * len(offsets)
    out = struct.pack("<II", hb + 8, hb + ob + 8)
    out += b"".join(struct.pack("<Q", h) for h in handles)
    out += b"".join(struct.pack("<II", o, s) for o, s in offsets)
    return out + data


@pytest.mark.parametrize("handles,args", [
    ([], []),
    ([0x7f0000001000, 3, 0x7f0000002000], [np.uint32(8192).tobytes(), np.uint32(1024).tobytes(), np.uint32(63).tobytes()]),
    ([1], [np.uint64(0x0123456789ABCDEF).tobytes(), np.float32(0.5).tobytes(), b"\x01\x02\x03", np.uint16(7).tobytes()]),
])
def test_launch_buffer_layout(handles, args):
    got = accelerator.pack_launch(handles, *args)
    assert got == _reference_layout(handles, args)


def test_argument_package_order_and_sizes():
    class S(C.Structure):
        _fields_ = [("a", C.c_uint8), ("b", C.c_float)]

    data, desc = accelerator.pack_arguments(np.uint32(5), np.float64(2.5), S(7, 1.25), b"xyz")
    assert desc.tolist() == [0, 4, 4, 8, 12, C.sizeof(S), 12 + C.sizeof(S), 3]
    assert data[:4] == np.uint32(5).tobytes() and data[4:12] == np.float64(2.5).tobytes()
    assert data[-3:] == b"xyz"
    with pytest.raises(TypeError):
        accelerator.pack_arguments([1, 2])


def test_pack_launch_rejects_short_destination():
    lib = capi.lib()
    h = (C.c_uint64 * 2)(1, 2)
    need = C.c_size_t()
    assert lib.pb2_acc_pack_launch(h, 2, None, None, 0, None, 0, C.byref(need)) == capi.PB2_OK
    assert need.value == 8 + 16
    small = C.create_string_buffer(8)
    assert lib.pb2_acc_pack_launch(h, 2, None, None, 0, small, 8, C.byref(need)) == capi.PB2_ERR_INVALID_ARGUMENT


def test_create_without_device_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    out = C.c_void_p()
    rc = capi.lib().pb2_acc_create(0, C.byref(out))
    assert rc == capi.PB2_ERR_CUDA and not out.value
    assert capi.lib().pb2_acc_launch_kernel(None, None, None, None, None, None, 0, None) == capi.PB2_ERR_INVALID_ARGUMENT
