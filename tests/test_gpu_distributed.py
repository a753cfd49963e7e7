"""The sharded search on the GPU: two ranks (spawned processes, gloo for the host-side gather,
both searching on cuda:0 with the package's own pipeline) each search their shard of the
trials; rank 0 gathers every periodogram, which must equal searching all trials in one
batch. No kernel of one rank waits on the other: the trials are independent and the only
exchange is the host-side gather."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KW = dict(period_min=0.2, period_max=3.0, bins_min=240, bins_max=260, rmed_width=1.0)
TSAMP = 5e-4


def _series():
    import riptide_b200 as rb

    rng = np.random.default_rng(91)
    lengths = [70001, 65536, 90000, 50000, 81234, 60000]
    return [rb.generate_signal(n, 0.9 / TSAMP + 7 * i, ducy=0.04, amplitude=12.0, rng=rng)
            .astype(np.float32) + 0.25 for i, n in enumerate(lengths)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist

    from riptide_b200 import distributed as D

    torch.cuda.set_device(0)
    try:
        w, r, _ = D.init_from_env(backend="gloo", timeout_s=120)
        series = _series()
        start, stop = D.shard_range([s.size for s in series], r, w)
        pgs = D.search_sharded(series, TSAMP, r, w, **KW)
        out = None if pgs is None else [(p.periods, p.foldbins, p.snrs) for p in pgs]
        D.barrier(w)
        results.put((r, start, stop, out, None))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent instead of a hung queue
        results.put((rank, -1, -1, None, repr(e)))


def test_sharded_search_two_ranks_on_the_gpu():
    import multiprocessing as mp

    import riptide_b200 as rb

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    try:
        for _ in range(2):
            rank, start, stop, out, err = q.get(timeout=300)
            assert err is None, err
            got[rank] = (start, stop, out)
    finally:
        for p in procs:
            p.join(timeout=120)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    series = _series()
    assert got[0][0] == 0 and got[0][1] == got[1][0] and got[1][1] == len(series)
    assert got[1][2] is None
    ref = rb.ffa_search_batched(series, TSAMP, **KW)
    assert len(got[0][2]) == len(series)
    for (p, fb, sn), one in zip(got[0][2], ref):
        assert np.array_equal(p, one.periods)
        assert np.array_equal(fb, one.foldbins)
        assert np.array_equal(sn, one.snrs)
