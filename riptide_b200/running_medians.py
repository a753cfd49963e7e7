"""Running medians (running_medians.py of the reference), computed on the GPU."""
import ctypes

import numpy as np

from . import _lib, libcpp


def running_median(x, width_samples):
    """Exact running median, odd width < size, edge padding (running_medians.py:5-37)."""
    return libcpp.running_median(np.ascontiguousarray(x), width_samples)


def fast_running_median(data, width_samples, min_points=101):
    """Approximate running median for large windows (running_medians.py:49-85): mean-scrunch,
    exact running median of width min_points, linear interpolation back (float64 output)."""
    if not (min_points % 2):
        raise ValueError("min_points must be an odd number")
    t, dev = libcpp._as_f32(np.ascontiguousarray(data) if not libcpp._is_cuda_tensor(data) else data, 1)
    torch = libcpp._t()
    out = torch.empty(t.shape, dtype=torch.float64, device=t.device)
    _lib.check(_lib.load().rt_fast_running_median(
        libcpp._ptr(t), t.numel(), int(width_samples), int(min_points), libcpp._ptr(out),
        libcpp._stream()))
    return libcpp._out(out, dev)
