"""The drop-in from the reference's side. tests/golden/dropin_trace.npz holds every
riptide.libcpp call that the reference's own glue made -- ffa_search (search.py:11-93) with
TimeSeries.deredden / normalise and fast_running_median, libffa.ffa2 / boxcar_snr /
downsample and TimeSeries.downsample -- with its arguments and the reference libcpp's outputs
(tests/golden/make_golden.py, section dropin). The glue is deterministic given those outputs,
so riptide_b200.libcpp answering every recorded call the same way is what binding
riptide.libcpp to it (the one-line binding a maintainer adds) requires.

CPU part: every call names a function riptide_b200.libcpp exports, with a signature that
accepts the recorded arguments. GPU part: the calls replayed through the C ABI give the
recorded outputs (bit-exact where the reference's arithmetic is reproduced exactly; the
periodogram's S/N and the downsampled series within the tolerances of the parity tests)."""
import inspect
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _calls():
    g = np.load(os.path.join(HERE, "golden", "dropin_trace.npz"))
    out = []
    for k in range(int(g["n"])):
        args = []
        for j in range(int(g[f"c{k}_nargs"])):
            a, t = g[f"c{k}_a{j}"], str(g[f"c{k}_t{j}"])
            args.append(a if t == "array" else {"int": int, "float": float}[t](a))
        outs = [g[f"c{k}_o{j}"] for j in range(int(g[f"c{k}_nout"]))]
        out.append((str(g[f"c{k}_name"]), args, outs))
    return out


def test_trace_names_and_signatures():
    from riptide_b200 import libcpp

    calls = _calls()
    names = {c[0] for c in calls}
    assert {"running_median", "periodogram", "ffa2", "snr2", "downsample"} <= names
    for name, args, _ in calls:
        fn = getattr(libcpp, name)
        inspect.signature(fn).bind(*args)


@pytest.mark.gpu
def test_trace_replayed_through_the_c_abi():
    from riptide_b200 import libcpp

    for k, (name, args, outs) in enumerate(_calls()):
        got = getattr(libcpp, name)(*args)
        got = got if isinstance(got, tuple) else (got,)
        assert len(got) == len(outs), name
        if name == "periodogram":
            p, fb, s = got
            assert np.array_equal(p, outs[0]) and np.array_equal(fb, outs[1]), k
            assert s.shape == outs[2].shape
            assert np.allclose(s, outs[2], rtol=1e-5, atol=2e-5), k
        elif name == "downsample":
            f = args[1]
            assert got[0].shape == outs[0].shape
            assert np.allclose(got[0], outs[0], rtol=1e-5, atol=1e-6 * np.sqrt(f)), k
        else:
            assert got[0].dtype == outs[0].dtype and np.array_equal(got[0], outs[0]), (k, name)
