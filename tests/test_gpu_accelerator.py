"""The accelerator (Accelerator.hpp:130-161, CUDA.cpp:497-927) on the GPU: the reference's own accelerator test
(Src/Test/Accelerator-Test.cpp:31-96, a 2-D convolution through createBuffer / createTiledOutput /
createResourceLUT / compileKernel / launchKernel / markDirty / download) against the oracle's restatement of its
kernel, bit for bit; nested lookup tables, every argument kind and the task index mapping; futures and errors.
The kernels are native sm_100a code (tests/kernels/generic_kernels.cu) registered by entry name."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from piper2_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    from piper2_b200 import accelerator

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "kernels"))
    import build_kernels

    kl = C.CDLL(build_kernels.build())
    kl.pb2t_kernel_function.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
    a = accelerator.Accelerator(streams=3)
    for name in ("convEntry", "echoEntry"):
        f = C.c_void_p()
        assert kl.pb2t_kernel_function(name.encode(), C.byref(f)) == 0
        a.register_kernel(name, f.value)
    yield a
    a.close()


def _conv(acc, width, height, ksize, seed):
    import oracle_py

    rng = np.random.default_rng(seed)
    x = rng.uniform(0, 1, width * height).astype(np.float32)
    y = rng.uniform(0, 1, ksize * ksize).astype(np.float32)

    def filler(src):
        return lambda view: view.__setitem__(slice(None), src.view(np.uint8))

    dx = acc.create_buffer(x.nbytes, 64, filler(x))
    dy = acc.create_buffer(y.nbytes, 64, filler(y))
    dz = acc.create_tiled_output(x.nbytes, 64)
    kernel = acc.compile_kernel("convEntry")
    lut = acc.create_resource_lut([dx, dy, dz])
    fut = acc.launch_kernel((height, 1, width), kernel, lut, np.uint32(width), np.uint32(height), np.uint32(ksize))
    dz.mark_dirty(fut)
    z = np.frombuffer(dz.download(), dtype=np.float32)
    assert fut.ready()
    expect = oracle_py.conv(x, y, width, height, ksize)
    return z, expect


@pytest.mark.parametrize("width,height,ksize", [(1024, 256, 63), (1000, 37, 15), (7, 5, 3)])
def test_convolution_equals_oracle(acc, width, height, ksize):
    z, expect = _conv(acc, width, height, ksize, seed=width + ksize)
    assert np.array_equal(z.view(np.uint32), expect.view(np.uint32))


def test_nested_tables_arguments_and_task_indices(acc):
    nx, ny, nz = 3, 2, 700  # z spans three 256-thread blocks, the last one ragged
    n = nx * ny * nz
    base = np.arange(n, dtype=np.uint32) * 3
    t = acc.create_tiled_output(4 * n, 256)
    h = acc.create_tiled_output(8 * 16, 8)
    b0 = acc.create_buffer(4 * n, 4096, lambda v: v.__setitem__(slice(None), base.view(np.uint8)))
    b1 = acc.create_buffer(4, 4, lambda v: v.__setitem__(slice(None), np.array([1000], np.uint32).view(np.uint8)))
    b2 = acc.create_buffer(4, 4, lambda v: v.__setitem__(slice(None), np.array([20000], np.uint32).view(np.uint8)))
    n2 = acc.create_resource_lut([b2])
    n1 = acc.create_resource_lut([b1, n2])
    root = acc.create_resource_lut([t, h, n1, b0])
    assert b0.handle % 4096 == 0 and t.handle % 256 == 0
    kernel = acc.compile_kernel("echoEntry")
    magic = np.uint64(0xFEDCBA9876543210)
    fut = acc.launch_kernel((nx, ny, nz), kernel, root, np.uint32(nx), np.uint32(ny), np.uint32(nz), magic,
                            np.float32(-3.25), b"\x07\x08\x09")
    t.mark_dirty(fut)
    h.mark_dirty(fut)
    got = np.frombuffer(t.download(), dtype=np.uint32)
    assert np.array_equal(got, base + 21000)
    rec = np.frombuffer(h.download(), dtype=np.uint64)
    # flattened: root [t, h, ->4, b0], then n1 at 4: [b1, ->6], then n2 at 6: [b2]
    assert rec[0] == t.handle and rec[1] == h.handle and rec[2] == 4 and rec[3] == b0.handle
    assert rec[4] == b1.handle and rec[5] == 6 and rec[6] == b2.handle
    assert rec[7] == magic and rec[8] == np.float32(-3.25).view(np.uint32)
    assert rec[9] == 0x090807 and rec[10] == (nx << 40) | (ny << 20) | nz
    assert rec[11] == 3 and rec[12] == 256  # grid z = ceil(700 / 256), 256-thread blocks


def test_errors_and_futures(acc):
    from piper2_b200 import accelerator

    with pytest.raises(capi.PB2Error, match="noSuchEntry"):
        acc.compile_kernel("noSuchEntry")
    kernel = acc.compile_kernel("echoEntry")
    with pytest.raises(capi.PB2Error, match="Empty launch"):
        acc.launch_kernel((1, 0, 1), kernel, None)
    assert acc.get_native_platform() == "NVIDIA CUDA"
    import torch

    assert acc.info() == (torch.cuda.current_device(), 3)
    # many launches in a row reuse staging and complete in order on the download's wait
    x = np.ones(64 * 64, np.float32)
    dx = acc.create_buffer(x.nbytes, 64, lambda v: v.__setitem__(slice(None), x.view(np.uint8)))
    dy = acc.create_buffer(4 * 9, 64, lambda v: v.__setitem__(slice(None), np.ones(9, np.float32).view(np.uint8)))
    dz = acc.create_tiled_output(x.nbytes, 64)
    conv = acc.compile_kernel("convEntry")
    lut = acc.create_resource_lut([dx, dy, dz])
    futs = [acc.launch_kernel((64, 1, 64), conv, lut, np.uint32(64), np.uint32(64), np.uint32(3)) for _ in range(50)]
    dz.mark_dirty(futs[-1])
    z = np.frombuffer(dz.download(), dtype=np.float32).reshape(64, 64)
    assert z[10, 10] == 9.0 and z[0, 0] == 4.0 and z[0, 10] == 6.0
    for f in futs:
        f.wait()
        assert f.ready()
    # a zero-filled buffer when no fill is given
    zb = acc.create_buffer(4096, 16)
    assert isinstance(zb, accelerator.Resource) and zb.handle % 16 == 0
