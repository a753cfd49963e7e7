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


def test_noalloc_rejects_oversized_blocks():
    import torch

    from riptide_b200 import _lib

    lib = _lib.load()
    x = torch.zeros((4100, 260), dtype=torch.float32, device="cuda")  # 1,066,000 values
    out = torch.zeros_like(x)
    status = _call(lib.rt_ffa2_noalloc, x, out)
    assert status == _lib.RT_EINVAL
    assert b"fixed scratch" in lib.rt_last_error()
