"""Error paths of the batched search, exercised without any GPU fault: a bounded wait inside
the persistent kernel that runs out (later-stage work items wait on a count that nothing
reaches, injected on the host), and a device allocation of the plan that fails (injected in
the plan's allocator). Each failure comes back as a status code; the same plan then searches
correctly. The reference has no device waits and no allocation of its own to fail; its
pipeline catches per-candidate exceptions (pipeline/pipeline.py:345-350)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rb():
    import riptide_b200

    return riptide_b200


def _series(n, seed):
    import torch

    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()


def test_stage_wait_times_out_and_the_plan_recovers(rb):
    import torch

    n = 1 << 22  # the first cycles' transforms are cut into several stages
    x = _series(n, 5)
    bs = rb.BatchedSearch([n], 64e-6, period_min=0.2, period_max=30.0)
    assert bs.stats["num_multistage"] > 0
    ref = [t.clone() for t in bs.run(x)]
    bs.set_wait_limit(20000)
    bs.inject_fault("stage_wait")
    for graph in (False, True):
        bs.enable_graph(graph)
        t0 = time.perf_counter()
        with pytest.raises(rb._lib.RiptideError, match="bounded wait"):
            bs.run(x)
        assert time.perf_counter() - t0 < 5.0
    bs.enable_graph(False)
    bs.inject_fault(None)
    out = bs.run(x)
    for a, b in zip(out, ref):
        assert torch.equal(a, b)
    with pytest.raises(ValueError):
        bs.set_wait_limit(0)
    bs.close()
    # another plan in the same process: the context is still usable
    bs2 = rb.BatchedSearch([n], 64e-6, period_min=0.2, period_max=30.0)
    for a, b in zip(bs2.run(x), ref):
        assert torch.equal(a, b)
    bs2.close()


def test_allocation_failure_is_reported_and_leaks_nothing(rb):
    import torch

    n = 1 << 22
    x = _series(n, 6)
    bs = rb.BatchedSearch([n], 64e-6, period_min=0.2, period_max=30.0)
    ref = [t.clone() for t in bs.run(x)]
    torch.cuda.synchronize()
    free_ready = torch.cuda.mem_get_info()[0]
    bs.inject_fault("alloc", 1)
    free_released = torch.cuda.mem_get_info()[0]
    # the plan's buffers (scratch ring, downsampled arena, dereddened series) are large
    assert free_released - free_ready > 64 << 20
    for k in (1, 4, 6, 9, 15):
        bs.inject_fault("alloc", k)
        with pytest.raises(MemoryError, match="injected"):
            bs.run(x)
        torch.cuda.synchronize()
        # whatever was allocated before the failing call has been released again
        assert abs(torch.cuda.mem_get_info()[0] - free_released) <= 2 << 20, k
    bs.inject_fault(None)
    out = bs.run(x)
    for a, b in zip(out, ref):
        assert torch.equal(a, b)
    bs.close()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] >= free_released - (2 << 20)
