"""Multi-GPU path on the host, world size 2 with gloo (no GPU): trial sharding, the MAX-over-
ranks time reduction and the gather of periodograms, with the oracle standing in for the
per-rank search (the data path has no collective, so the GPU part is the single-GPU search
covered by the GPU tests)."""
import os
import socket

import numpy as np
import pytest

from riptide_b200 import distributed as D


def test_shard_bounds_cover_and_balance():
    rng = np.random.default_rng(5)
    lengths = rng.integers(int(0.9 * 2**22), 2**22, 512)
    for world in (1, 2, 3, 4, 8):
        b = D.shard_bounds(lengths, world)
        assert b[0] == 0 and b[-1] == lengths.size
        assert np.all(np.diff(b) >= 1)
        sizes = [lengths[b[r]:b[r + 1]].sum() for r in range(world)]
        # contiguous shards: within one trial of an equal split
        assert max(sizes) - min(sizes) <= 2 * lengths.max()
    # fewer trials than ranks: some shards empty, all trials covered once
    b = D.shard_bounds([10, 20], 4)
    assert b[0] == 0 and b[-1] == 2 and np.all(np.diff(b) >= 0)
    assert D.shard_bounds([], 3).tolist() == [0, 0, 0, 0]
    with pytest.raises(ValueError):
        D.shard_bounds([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_search(series, tsamp, **kw):
    from oracle import oracle as O

    out = []
    for x in series:
        z, widths, p, fb, sn = O.ffa_search(x, tsamp, **kw)
        out.append((p, fb, sn))
    return out


def _worker(rank, world, port, series, kw, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist

    w, r, _ = D.init_from_env(backend="gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    start, stop = D.shard_range([s.size for s in series], rank, world)
    t = D.max_over_ranks(10.0 + rank, world)
    pg = D.search_sharded(series, 1e-3, rank, world, search=_oracle_search, **kw)
    D.barrier(world)
    results.put((rank, start, stop, t, pg))
    dist.destroy_process_group()


def test_two_ranks_gloo():
    import multiprocessing as mp

    rng = np.random.default_rng(11)
    series = [rng.standard_normal(n).astype(np.float32) for n in (9000, 12000, 15000, 7000, 11000)]
    kw = dict(period_min=0.5, period_max=2.0, bins_min=100, bins_max=110, rmed_width=0.3)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, series, kw, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, start, stop, t, pg = q.get(timeout=120)
        got[rank] = (start, stop, t, pg)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # shards: disjoint, contiguous, covering every trial
    assert got[0][0] == 0 and got[0][1] == got[1][0] and got[1][1] == len(series)
    # the time of the job is the slowest rank's on every rank
    assert got[0][2] == got[1][2] == 11.0
    # rank 0 holds every periodogram, in trial order, equal to searching them all at once
    assert got[1][3] is None
    ref = _oracle_search(series, 1e-3, **kw)
    assert len(got[0][3]) == len(series)
    for (p, fb, sn), (rp, rfb, rsn) in zip(got[0][3], ref):
        assert np.array_equal(p, rp) and np.array_equal(fb, rfb) and np.array_equal(sn, rsn)
