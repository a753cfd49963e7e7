"""rt_ffa2_noalloc: the FFA transform for callers that cannot allocate device memory (their
memory is reserved by another framework's pool, or allocation is forbidden after start-up in
a real-time loop). It must agree with rt_ffa2 bit for bit, call after call, while using only
its fixed scratch array. This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(fn, x, out):
    import torch

    from riptide_b200 import _lib

    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return fn(ctypes.c_void_p(x.data_ptr()), x.shape[0], x.shape[1], ctypes.c_void_p(out.data_ptr()), st)


def test_noalloc_matches_ffa2_twice_in_a_row():
    import torch

    from riptide_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(2024)
    # two calls in a row through the C ABI: a multi-stage block (uses the scratch) then a
    # smaller one, each against rt_ffa2 on the same input
    for m, b in [(3900, 260), (1342, 251), (97, 240)]:
        x = torch.from_numpy(rng.standard_normal((m, b)).astype(np.float32)).cuda()
        ref = torch.empty_like(x)
        got = torch.full_like(x, float("nan"))
        _lib.check(_call(lib.rt_ffa2, x, ref))
        _lib.check(_call(lib.rt_ffa2_noalloc, x, got))
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (m, b)


def test_noalloc_takes_no_device_memory():
    # after a first call (which looks up the array's address), further calls leave the
    # device's free memory unchanged: no allocation by the library, the driver or torch
    import torch

    from riptide_b200 import _lib

    lib = _lib.load()
    x = torch.from_numpy(np.random.default_rng(7).standard_normal((3000, 256)).astype(np.float32)).cuda()
    out = torch.empty_like(x)
    _lib.check(_call(lib.rt_ffa2_noalloc, x, out))
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        _lib.check(_call(lib.rt_ffa2_noalloc, x, out))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_oversized_blocks():
    import torch

    from riptide_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(8)
    # too many values; too many columns within the value budget; too many rows. The sizes
    # are rejected on the host before anything is launched, so one-value buffers stand in.
    x = torch.zeros(1, dtype=torch.float32, device="cuda")
    out = torch.zeros_like(x)
    for shape in [(4100, 260), (200, 4097), (1 << 24, 1)]:
        rows, cols = shape
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        status = lib.rt_ffa2_noalloc(ctypes.c_void_p(x.data_ptr()), rows, cols,
                                     ctypes.c_void_p(out.data_ptr()), st)
        assert status == _lib.RT_EINVAL, shape
        assert b"fixed scratch" in lib.rt_last_error(), shape
        # a rejected call leaves nothing behind: the next valid call matches rt_ffa2
        y = torch.from_numpy(rng.standard_normal((1500, 250)).astype(np.float32)).cuda()
        ref = torch.empty_like(y)
        got = torch.full_like(y, float("nan"))
        _lib.check(_call(lib.rt_ffa2, y, ref))
        _lib.check(_call(lib.rt_ffa2_noalloc, y, got))
        torch.cuda.synchronize()
        assert torch.equal(got, ref), shape
