"""Benchmark: batched FFA search of DM trials (ffa_search = deredden + normalise + periodogram)
on B200, against the reference's CPU implementation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 3]

One step = one search of the whole synthetic batch (default: 512 trials of
U[0.9, 1.0] * 2^22 samples, 64 us, P 0.2-30 s, bins 240-260). Prints one JSON line on rank 0.
Under torchrun each rank searches its own batch (weak scaling, no data-path collective).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = ("DM-trial searches/s (2^22 samp, 0.2–60 s) batched vs plain GPU at equal S/N; "
          "%HBM")
FALLBACK_HBM_GBS = 6650.0


# --------------------------------------------------------------------------------------
# CPU reference arm (runs in spawned worker processes)
# --------------------------------------------------------------------------------------
def _cpu_worker(args):
    data, tsamp, kw = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, HERE)
    from oracle import oracle as O

    ref = O.ref_libcpp()
    t0 = time.perf_counter()
    O.ffa_search(data, tsamp, libcpp=ref, **kw)
    return time.perf_counter() - t0


def _cpu_file_worker(args):
    """The reference's WorkerPool.process_fname for one PRESTO file and one range
    (worker_pool.py:47-68): read, deredden, normalise, search, find_peaks."""
    inf_path, tsamp, kw, fpkw = args
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, HERE)
    from oracle import oracle as O

    ref = O.ref_libcpp()
    t0 = time.perf_counter()
    data = np.fromfile(inf_path[:-4] + ".dat", dtype=np.float32)
    z, widths, periods, foldbins, snrs = O.ffa_search(data, tsamp, libcpp=ref, **kw)
    O.find_peaks(periods, foldbins, snrs, widths, data.size * tsamp, **fpkw)
    return time.perf_counter() - t0


def cpu_kind():
    from oracle import oracle as O

    return "reference" if O.ref_libcpp() is not None else "port"


def cpu_sample_trials(config_id, nsample, first_index=1_000_000):
    """Host copies of `nsample` synthetic trials (generated on the GPU, same generator)."""
    from riptide_b200 import synth

    cfg = synth.CONFIGS[config_id]
    lengths = synth.trial_lengths(config_id, nsample, first_index)
    out = []
    for k, n in enumerate(lengths):
        x, _ = synth.make_trial(config_id, first_index + k, n, cfg["tsamp"], "cuda")
        out.append(x.cpu().numpy())
    return out


def run_cpu_steps(pool, trials, tsamp, kw, steps):
    """Time `steps` rounds; each round searches every trial of the sample in parallel."""
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        list(pool.map(_cpu_worker, [(x, tsamp, kw) for x in trials]))
        times.append(time.perf_counter() - t0)
    return times


def cpu_pool(ncores):
    import multiprocessing as mp

    return mp.get_context("spawn").Pool(processes=ncores)


# --------------------------------------------------------------------------------------
# helpers
# --------------------------------------------------------------------------------------
class ClockSampler(object):
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while active."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_trial(config_id):
    """DRAM bytes per trial of the search kernel from the committed ncu summaries (the
    batched 2^22-sample workload and the large sweep), or None for other workloads."""
    try:
        with open(os.path.join(HERE, "profiles", "search_persistent_traffic.json")) as f:
            t = json.load(f)
        if config_id == 3:
            return float(t["dram_bytes_per_trial"])
        if config_id == 5:
            return float(t["large_sweep"]["dram_bytes_per_trial"])
    except (OSError, KeyError, ValueError):
        pass
    return None


def dist_setup():
    """One process per GPU (torchrun environment); NCCL process group for N > 1."""
    from riptide_b200 import distributed as D

    return D.init_from_env(backend="nccl", timeout_s=600)


def max_over_ranks(v, world):
    from riptide_b200 import distributed as D

    return D.max_over_ranks(v, world)


def barrier(world):
    from riptide_b200 import distributed as D

    D.barrier(world)


# --------------------------------------------------------------------------------------
def bench_reference(args):
    """--impl reference: the reference's CPU implementation on the host cores."""
    world, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return 0
    from riptide_b200 import synth

    cfg = synth.CONFIGS[args.config]
    ncores = os.cpu_count() or 1
    nsample = max(1, min(ncores, args.cpu_sample))
    trials = cpu_sample_trials(args.config, nsample)
    kw = dict(cfg["search"])
    pool = cpu_pool(ncores)
    try:
        run_cpu_steps(pool, trials, cfg["tsamp"], kw, args.warmup and 1)
        times = run_cpu_steps(pool, trials, cfg["tsamp"], kw, args.steps)
    finally:
        pool.close()
    step = float(np.mean(times))
    value = nsample / step
    kind = cpu_kind()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": cfg["name"], "trials_per_step": nsample},
        "cpu_baseline": {"value": value, "unit": "trials/s", "cores": ncores, "kind": kind,
                         "sample": f"{nsample} trials of the workload per step, one per process"},
        "e2e": {"value": value, "unit": "trials/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def bench_ours(args):
    world, rank, local = dist_setup()
    import torch

    import riptide_b200 as rb
    from riptide_b200 import synth

    torch.cuda.set_device(local)
    cfg = synth.CONFIGS[args.config]
    ntrials = args.trials
    # CPU baseline pool is spawned before any heavy GPU work of this process
    ncores = os.cpu_count() or 1
    do_cpu = (rank == 0 and world == 1 and not args.no_cpu)
    pool = cpu_pool(ncores) if do_cpu else None

    data, lengths, infos = synth.make_batch(args.config, ntrials, first_index=rank * ntrials)
    tuning = None
    if args.autotune:  # engine tile choices timed on a sample of this workload
        from riptide_b200 import tuning as TU

        tuning = TU.autotune(lengths, cfg["tsamp"], sample_trials=16, **cfg["search"])
    t0 = time.perf_counter()
    bs = rb.BatchedSearch(lengths, cfg["tsamp"], tuning=tuning, **cfg["search"])
    plan_ms = (time.perf_counter() - t0) * 1e3
    st = bs.stats
    nw = int(bs.widths.size)
    L = st["total_rows"]
    bytes_kernel = 4 * st["folded_samples"] + L * (4 * nw + 12)
    bytes_job = 4 * st["total_samples"] + 4 * st["downsampled_samples"] + bytes_kernel

    outs = bs.allocate_outputs()
    bs.run(data, outs, check=True)  # first run allocates the plan's device buffers
    # every step replays the whole search (its launches and memsets) as one CUDA graph
    bs.enable_graph(not args.no_graph)
    for _ in range(max(0, args.warmup - 1)):
        bs.run(data, outs, check=False)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            bs.run(data, outs, check=False)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    from riptide_b200 import _lib

    _lib.check(_lib.load().rt_search_check(bs._plan, _lib.ctypes.c_void_p(stream.cuda_stream)))
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, world)
    value = ntrials * world / (ms * 1e-3)
    # per-stage CUDA-event times and launch count: one more run, launched directly
    bs.enable_timing(True)
    bs.run(data, outs, check=False)
    s0, s1, s2, nl = bs.last_timing()
    bs.enable_timing(False)
    stage = np.array([s0, s1, s2]) * args.steps
    launches = nl * args.steps
    k_ms = stage[2] / args.steps
    peak, peak_kind = measured_peak()
    achieved = bytes_kernel / (k_ms * 1e-3) / 1e9
    tr = traffic_per_trial(args.config)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": (tr * ntrials if tr else None),
                "kernel": "k_search_persistent", "peak_source": peak_kind,
                "alg_bytes_per_launch": bytes_kernel}

    # ---- end to end through the public API with host buffers (rank 0 prints) ----
    # SearchPipeline (C ABI rt_search_pipeline_*): host series in, host periodograms out, in
    # chunks of trials whose copies overlap the search of the neighbouring chunks.
    e2e = None
    if not args.no_e2e:
        pipe = rb.SearchPipeline(lengths, cfg["tsamp"], chunk_trials=args.chunk_trials,
                                 **cfg["search"])
        host_in, host_out = pipe.allocate_host()
        host_in.copy_(data.cpu())
        h2d = host_in.numel() * 4
        d2h = sum(o.numel() * o.element_size() for o in host_out)
        pipe.run(host_in, host_out, check=True)
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(max(1, args.e2e_steps)):
            pipe.run(host_in, host_out, check=False)
        b.record(stream)
        torch.cuda.synchronize()
        pipe.check()
        ems = max_over_ranks(a.elapsed_time(b) / max(1, args.e2e_steps), world)
        e2e = {"value": ntrials * world / (ems * 1e-3), "unit": "trials/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": ems, "api": "SearchPipeline (rt_search_pipeline_run), "
               "page-locked host buffers, %d chunks of %d trials" % (pipe.num_chunks,
                                                                      args.chunk_trials)}
        pipe.close()
        del host_in, host_out

    # ---- peak detection on the step's periodograms (opt-in; outside the timed step) ----
    peaks_line = None
    if args.peaks and rank == 0:
        tobs = np.asarray(lengths, dtype=np.float64) * cfg["tsamp"]
        rb.find_peaks_batched(outs[0], outs[1], outs[2], bs.row_offsets, tobs, bs.widths)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        res = rb.find_peaks_batched(outs[0], outs[1], outs[2], bs.row_offsets, tobs, bs.widths)
        torch.cuda.synchronize()
        gpu_s = time.perf_counter() - t1
        # the reference's numpy find_peaks on host copies of a few periodograms
        from oracle import oracle as O

        nref = min(4, ntrials)
        P = outs[0][:int(bs.row_offsets[nref])].cpu().numpy()
        F = outs[1][:int(bs.row_offsets[nref])].cpu().numpy().view(np.uint32)
        S = outs[2][:int(bs.row_offsets[nref])].cpu().numpy()
        t1 = time.perf_counter()
        for t in range(nref):
            a, b = int(bs.row_offsets[t]), int(bs.row_offsets[t + 1])
            O.find_peaks(P[a:b], F[a:b], S[a:b], bs.widths, float(tobs[t]))
        cpu_s = (time.perf_counter() - t1) / nref
        peaks_line = {"trials": ntrials, "gpu_ms_all_trials": gpu_s * 1e3,
                      "cpu_ms_per_trial_1_core": cpu_s * 1e3,
                      "peaks_found": int(sum(len(r[0]) for r in res))}

    # ---- the pipeline's search stage from files (opt-in): WorkerPool vs the reference ----
    wp_line = None
    if args.workerpool > 0 and rank == 0:
        wp_line = bench_workerpool(args, cfg, data, lengths, pool if do_cpu else None)

    # ---- readers and candidate folding (opt-in) ----
    io_line = bench_ingest(args, cfg, data, lengths) if args.ingest > 0 and rank == 0 else None
    fold_line = bench_fold(args, cfg, data, lengths) if args.fold > 0 and rank == 0 else None

    # ---- plain per-trial GPU paths on a few trials, for the batching ratio ----
    plain = bench_plain(args, cfg, data, lengths) if rank == 0 and args.plain_trials > 0 else None
    # ---- the large-sweep workload and the differentiable search (rank 0, default on) ----
    sweep = bench_sweep(args) if rank == 0 and args.sweep_trials > 0 else None
    sweep_full = bench_sweep_full(args) if rank == 0 and args.sweep_full > 0 else None
    grad_line = None
    if rank == 0 and not args.no_grad:
        from riptide_b200.grad import benchmark_training_step

        grad_line = benchmark_training_step(64, steps=3, warmup=2)

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if do_cpu:
        nsample = max(1, min(ncores, args.cpu_sample))
        trials = cpu_sample_trials(args.config, nsample)
        run_cpu_steps(pool, trials[:1], cfg["tsamp"], dict(cfg["search"]), 1)
        times = run_cpu_steps(pool, trials, cfg["tsamp"], dict(cfg["search"]), 1)
        pool.close()
        cpu = {"value": nsample / times[0], "unit": "trials/s", "cores": ncores,
               "kind": cpu_kind(),
               "sample": f"{nsample} trials of the workload searched in parallel, one per process"}

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded white + 1/f noise + von Mises pulsars, generated on device)",
            "config": {"workload": cfg["name"], "trials_per_gpu": ntrials,
                       "period_range_s": [cfg["search"]["period_min"], cfg["search"]["period_max"]],
                       "bins": [cfg["search"]["bins_min"], cfg["search"]["bins_max"]],
                       "samples_per_gpu": int(sum(lengths)), "periodogram_rows_per_gpu": L,
                       "widths": nw, "l2": "inputs larger than L2 (%.1f GB per step)" %
                       (4 * sum(lengths) / 1e9),
                       "plan_ms": plan_ms, "tuning": tuning or "default", "stage_ms": {"deredden_normalise": stage[0] / args.steps,
                                                        "downsample": stage[1] / args.steps,
                                                        "ffa_snr": k_ms},
                       "alg_bytes_per_step": bytes_job,
                       "hbm_frac_whole_job": bytes_job / (ms * 1e-3) / 1e9 / peak,
                       "parallelism": "trials sharded across GPUs" if world > 1 else "1 GPU"},
            "roofline": roofline,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "plain_gpu": plain,
            "batched_vs_plain": (value / world / plain["engine_one_trial"]["trials_per_s"])
            if plain else None,
            "batched_vs_per_launch": (value / world / plain["per_launch"]["trials_per_s"])
            if plain and plain.get("per_launch") else None,
            "large_sweep": sweep,
            "large_sweep_full": sweep_full,
            "grad": grad_line,
            "find_peaks": peaks_line,
            "workerpool": wp_line,
            "ingest": io_line,
            "fold": fold_line,
        }
        print(json.dumps(line), flush=True)
    bs.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def _event_ms(fn, reps):
    """Mean CUDA-event time (ms) of fn() over reps calls on the current stream."""
    import torch

    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(st)
    for _ in range(reps):
        fn()
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def bench_plain(args, cfg, data, lengths):
    """The per-trial GPU paths the batched engine replaces, on the first `plain_trials`
    trials of the workload:
    * engine_one_trial: the fused engine searching one trial per run (BatchedSearch of one
      trial = rt_periodogram's path: deredden, normalise, downsampling, the persistent
      FFA + S/N kernel), plans built outside the timed region, CUDA events over 3 runs;
    * per_launch: rt_deredden + rt_normalise + rt_periodogram_plain (one launch per (cycle,
      bins) step), on 2 trials."""
    import torch

    import riptide_b200 as rb
    from riptide_b200 import _lib

    offs = np.concatenate([[0], np.cumsum(lengths)])
    n_eng = min(args.plain_trials, len(lengths))
    ms = []
    for i in range(n_eng):
        x = data[int(offs[i]):int(offs[i + 1])]
        one = rb.BatchedSearch([lengths[i]], cfg["tsamp"], **cfg["search"])
        outs = one.allocate_outputs()
        one.run(x, outs, check=True)
        ms.append(_event_ms(lambda: one.run(x, outs, check=False), 3))
        one.close()
        del outs
    eng = {"trials_per_s": 1e3 / float(np.mean(ms)), "ms_per_trial": float(np.mean(ms)),
           "sample_trials": n_eng,
           "api": "BatchedSearch of one trial per run (deredden, normalise, downsampling, "
                  "persistent FFA + S/N kernel), CUDA events"}
    per_launch = None
    n_pl = min(2, len(lengths))
    if n_pl:
        tms = []
        p = rb.libcpp
        for i in range(n_pl):
            x = data[int(offs[i]):int(offs[i + 1])]
            y = torch.empty_like(x)
            z = torch.empty_like(x)

            def run():
                _lib.check(_lib.load().rt_deredden(p._ptr(x), x.numel(), cfg["tsamp"],
                                                   cfg["search"]["rmed_width"],
                                                   cfg["search"]["rmed_minpts"], p._ptr(y),
                                                   p._stream()))
                _lib.check(_lib.load().rt_normalise(p._ptr(y), y.numel(), p._ptr(z), p._stream()))
                from riptide_b200.ffautils import generate_width_trials

                w = generate_width_trials(cfg["search"]["bins_min"])
                p.periodogram_plain(z, cfg["tsamp"], w, cfg["search"]["period_min"],
                                    cfg["search"]["period_max"], cfg["search"]["bins_min"],
                                    cfg["search"]["bins_max"])

            run()
            tms.append(_event_ms(run, 1))
        per_launch = {"trials_per_s": 1e3 / float(np.mean(tms)), "sample_trials": n_pl,
                      "api": "rt_deredden + rt_normalise + rt_periodogram_plain (one launch per "
                             "(cycle, bins) step)"}
    return {"engine_one_trial": eng, "per_launch": per_launch}


def bench_sweep(args):
    """The large batched sweep's workload (2^23-sample trials, 64 us, P 0.2-60 s, bins
    480-520, 12 widths) on `sweep_trials` trials in one batch: trials/s with inputs in HBM
    (graph replays, CUDA events) and the search kernel's HBM roofline fraction."""
    import torch

    import riptide_b200 as rb
    from riptide_b200 import _lib, synth

    cfg = synth.CONFIGS[5]
    data, lengths, _ = synth.make_batch(5, args.sweep_trials)
    bs = rb.BatchedSearch(lengths, cfg["tsamp"], **cfg["search"])
    st = bs.stats
    nw = int(bs.widths.size)
    bytes_kernel = 4 * st["folded_samples"] + st["total_rows"] * (4 * nw + 12)
    outs = bs.allocate_outputs()
    bs.run(data, outs, check=True)
    bs.enable_graph(True)
    bs.run(data, outs, check=False)
    steps = 3
    ms = _event_ms(lambda: bs.run(data, outs, check=False), steps)
    _lib.check(_lib.load().rt_search_check(bs._plan, rb.libcpp._stream()))
    bs.enable_timing(True)
    bs.run(data, outs, check=True)
    s0, s1, s2, _ = bs.last_timing()
    bs.close()
    peak, kind = measured_peak()
    achieved = bytes_kernel / (s2 * 1e-3) / 1e9
    tr = traffic_per_trial(5)
    del data, outs
    torch.cuda.empty_cache()
    return {"workload": cfg["name"], "trials": args.sweep_trials, "steps": steps,
            "value": args.sweep_trials / (ms * 1e-3), "unit": "trials/s", "ms_per_step": ms,
            "stage_ms": {"deredden_normalise": s0, "downsample": s1, "ffa_snr": s2},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "kernel": "k_search_persistent",
                         "peak_source": kind, "alg_bytes_per_launch": bytes_kernel,
                         "traffic": tr * args.sweep_trials if tr else None}}


def bench_sweep_full(args):
    """The whole large batched sweep (`sweep_full` trials of 2^23 samples, P 0.2-60 s, bins
    480-520), streamed through the GPU in batches of `sweep_trials`: each batch is generated
    on the device, searched and released before the next (all 1024 trials' periodograms,
    75 GB, and inputs, 32 GB, do not fit one GPU at once); the host builds the next batch's
    plan while the GPU searches the current one. Reports trials/s of the searches alone (CUDA
    events around each batch's run) and of plan + device set-up + search + release (host
    clock, synchronised; the synthetic data generation, which stands in for data arriving,
    is excluded)."""
    import time

    import torch

    import riptide_b200 as rb
    from riptide_b200 import _lib, synth

    cfg = synth.CONFIGS[5]
    chunk = max(1, args.sweep_trials or 64)
    starts = list(range(0, args.sweep_full, chunk))
    sizes = [min(chunk, args.sweep_full - a) for a in starts]
    search_ms, wall_s = 0.0, 0.0
    t0 = time.perf_counter()
    bs = rb.BatchedSearch(synth.trial_lengths(5, sizes[0], 0), cfg["tsamp"], **cfg["search"])
    wall_s += time.perf_counter() - t0
    for b, (first, n) in enumerate(zip(starts, sizes)):
        data, lengths, _ = synth.make_batch(5, n, first_index=first)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs = bs.allocate_outputs()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        bs.run(data, outs, check=False)
        e1.record()
        nxt = None
        if b + 1 < len(starts):  # host planning of the next batch overlaps this search
            nxt = rb.BatchedSearch(synth.trial_lengths(5, sizes[b + 1], starts[b + 1]),
                                   cfg["tsamp"], **cfg["search"])
        _lib.check(_lib.load().rt_search_check(bs._plan, rb.libcpp._stream()))
        torch.cuda.synchronize()
        search_ms += e0.elapsed_time(e1)
        bs.close()
        del outs
        wall_s += time.perf_counter() - t0
        del data
        torch.cuda.empty_cache()
        bs = nxt
    return {"workload": cfg["name"], "trials": args.sweep_full, "batch_trials": chunk,
            "batches": len(starts), "value": args.sweep_full / (search_ms * 1e-3),
            "unit": "trials/s", "search_ms": search_ms,
            "wall_trials_per_s": args.sweep_full / wall_s}


def bench_workerpool(args, cfg, data, lengths, pool):
    """Time WorkerPool.process_fname_list on `args.workerpool` PRESTO files of the workload
    (written to a temporary folder first, so they are read from the page cache) with one
    search range of the workload's parameters and find_peaks' defaults; and the reference's
    process_fname on a sample of the files on all host cores."""
    import shutil
    import tempfile

    import torch

    import riptide_b200 as rb
    from riptide_b200.reading.writers import write_presto

    n = min(int(args.workerpool), len(lengths))
    offs = np.concatenate([[0], np.cumsum(lengths)])
    kw = {k: v for k, v in cfg["search"].items() if k not in ("rmed_width", "rmed_minpts")}
    rng_conf = [{"ffa_search": kw, "find_peaks": {}}]
    dered = {"rmed_width": cfg["search"]["rmed_width"],
             "rmed_minpts": cfg["search"]["rmed_minpts"]}
    tmp = tempfile.mkdtemp(prefix="rt_wp_")
    try:
        fnames = []
        for i in range(n):
            base = os.path.join(tmp, f"trial{i:04d}")
            x = data[int(offs[i]):int(offs[i + 1])].cpu().numpy()
            write_presto(base, x, dict(
                basename=os.path.basename(base), telescope="Synthetic", instrument="none",
                source_name="synthetic", raj="00:00:00.0000", decj="00:00:00.0000",
                observer="none", mjd=60000.0, barycentered=False, nsamp=int(x.size),
                tsamp=cfg["tsamp"], breaks=False, em_band="Radio", fov_arcsec=1.0,
                dm=float(i), fbot=1200.0, bandwidth=400.0, nchan=1024, cbw=0.390625,
                analyst="none"))
            fnames.append(base + ".inf")
        wp = rb.WorkerPool(dered, rng_conf, fmt="presto", chunk_trials=args.chunk_trials)
        peaks = wp.process_fname_list(fnames)  # warm-up: plans, first touch
        torch.cuda.synchronize()
        times = []
        for _ in range(2):
            t0 = time.perf_counter()
            peaks = wp.process_fname_list(fnames)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        wp.close()
        gpu_s = min(times)
        line = {"files": n, "files_per_s": n / gpu_s, "s_per_call": gpu_s,
                "peaks_found": len(peaks),
                "api": "WorkerPool.process_fname_list (PRESTO .inf/.dat from the page cache, "
                       "one range, find_peaks defaults)"}
        if pool is not None:
            ncores = os.cpu_count() or 1
            sample = fnames[:max(1, min(ncores, n))]
            job = [(f, cfg["tsamp"], dict(cfg["search"]), {}) for f in sample]
            t0 = time.perf_counter()
            list(pool.map(_cpu_file_worker, job))
            cpu_s = time.perf_counter() - t0
            line["cpu_reference"] = {"files_per_s": len(sample) / cpu_s, "cores": ncores,
                                     "kind": cpu_kind(), "sample": f"{len(sample)} files, "
                                     "one per process (process_fname of the reference)"}
        return line
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def bench_ingest(args, cfg, data, lengths):
    """Time load_series_batch on `args.ingest` SIGPROC files of the workload, float32 and
    8-bit (written first, read from the page cache), against the reference's data path for
    the same files (np.fromfile + astype(np.float32) per file, one core, then one copy of
    the packed batch to the GPU)."""
    import shutil
    import tempfile

    import torch

    from riptide_b200.reading import describe, load_series_batch
    from riptide_b200.reading.writers import write_sigproc

    n = min(int(args.ingest), len(lengths))
    offs = np.concatenate([[0], np.cumsum(lengths)])
    tmp = tempfile.mkdtemp(prefix="rt_io_")
    out = {}
    try:
        for nbits in (32, 8):
            fnames = []
            for i in range(n):
                x = data[int(offs[i]):int(offs[i + 1])].cpu().numpy()
                if nbits == 8:
                    x = np.clip(np.round(x * 16.0), -128, 127)
                hdr = dict(source_name="synthetic", telescope_id=0, machine_id=0, data_type=2,
                           refdm=float(i), fch1=1400.0, nchans=1, nbits=nbits, tstart=60000.0,
                           tsamp=cfg["tsamp"], nifs=1, src_raj=0.0, src_dej=0.0)
                if nbits == 8:
                    hdr["signed"] = True
                fn = os.path.join(tmp, f"t{i:04d}_{nbits}.tim")
                write_sigproc(fn, x, hdr)
                fnames.append(fn)
            files = describe(fnames, "sigproc")
            load_series_batch(files)
            torch.cuda.synchronize()
            best = 1e30
            for _ in range(3):
                t0 = time.perf_counter()
                dev, _ = load_series_batch(files)
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
            t0 = time.perf_counter()
            host = [np.fromfile(f.path, dtype=(np.float32 if nbits == 32 else np.int8),
                                offset=f.offset).astype(np.float32) for f in files]
            torch.from_numpy(np.concatenate(host)).to("cuda")
            torch.cuda.synchronize()
            ref = time.perf_counter() - t0
            payload = sum(f.nsamp for f in files) * (4 if nbits == 32 else 1)
            out[f"nbits{nbits}"] = {"files": n, "s": best, "files_per_s": n / best,
                                    "payload_GB_per_s": payload / best / 1e9,
                                    "reference_path_files_per_s": n / ref}
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def bench_fold(args, cfg, data, lengths):
    """Fold trial 0 at `args.fold` candidate periods (log-uniform over the search range,
    256 bins, 32 sub-integrations with the candidate rule) in one fold_candidates call, against
    the reference's TimeSeries.fold arithmetic on the host (the oracle's restatement: numpy and
    the C restatement of downsample.hpp, one core) on a sample of 32 of them."""
    import torch

    import riptide_b200 as rb
    from oracle import oracle as O

    x = data[:int(lengths[0])].cpu().numpy()
    ts = rb.TimeSeries(x, cfg["tsamp"])
    rng = np.random.default_rng(5)
    lo, hi = np.log(cfg["search"]["period_min"]), np.log(cfg["search"]["period_max"])
    periods = np.exp(rng.uniform(lo, hi, int(args.fold)))
    rb.fold_candidates(ts, periods[:8], 256, 32)
    best = 1e30
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rb.fold_candidates(ts, periods, 256, 32)
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    sample = periods[:32]
    t0 = time.perf_counter()
    for p in sample:
        sub = rb.folding.candidate_subints(float(p), 32, ts.length)
        O.fold(x, cfg["tsamp"], float(p), 256, sub)
    cpu = (time.perf_counter() - t0) / len(sample)
    return {"candidates": int(args.fold), "s_all": best, "ms_per_candidate": best * 1e3 / args.fold,
            "cpu_ms_per_candidate_1_core": cpu * 1e3, "cpu_kind": "port",
            "api": "fold_candidates (rt_fold_batched, one launch), host series copied in"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 5])
    ap.add_argument("--trials", type=int, default=None)
    ap.add_argument("--cpu-sample", type=int, default=64)
    ap.add_argument("--plain-trials", type=int, default=8,
                    help="trials timed one at a time through the fused engine")
    ap.add_argument("--sweep-trials", type=int, default=64,
                    help="trials of the large-sweep workload timed beside the main line (0: skip)")
    ap.add_argument("--sweep-full", type=int, default=0,
                    help="also stream this many large-sweep trials through the GPU in batches "
                         "of --sweep-trials (1024: the whole sweep)")
    ap.add_argument("--no-grad", action="store_true",
                    help="skip the differentiable-search training step")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--chunk-trials", type=int, default=16,
                    help="trials per SearchPipeline chunk in the end-to-end leg")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--peaks", action="store_true")
    ap.add_argument("--workerpool", type=int, default=0,
                    help="also time WorkerPool.process_fname_list on this many files")
    ap.add_argument("--ingest", type=int, default=0,
                    help="also time load_series_batch on this many SIGPROC files")
    ap.add_argument("--fold", type=int, default=0,
                    help="also time fold_candidates at this many candidate periods")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.trials is None:
        args.trials = {1: 1, 2: 1, 3: 512, 5: 1024}[args.config]
    if args.impl == "reference":
        return bench_reference(args)
    return bench_ours(args)


if __name__ == "__main__":
    sys.exit(main())
