"""Drop-in replacement of the reference's compiled module ``riptide.libcpp``
(cpp/python_bindings.cpp:225-279), running on a B200.

Same function names, argument meaning, output shapes/dtypes and ValueError messages as the
reference. Arguments may be numpy arrays (results come back as numpy arrays, with the
host<->device copies done here) or CUDA torch tensors (no copies; results are CUDA tensors
on the same device, computed on the current torch stream).

Input conversion follows pybind11's ``py::array_t<float>`` as the reference uses it: a
non-float32 array is cast to a new C-contiguous float32 array; a float32 array that is not
C-contiguous raises ValueError("Input numpy array must be contiguous in memory")
(python_bindings.cpp:33-41).
"""
import ctypes

import numpy as np

from . import _lib

__all__ = [
    "rollback", "fused_rollback_add", "circular_prefix_sum", "ffa2", "benchmark_ffa2",
    "snr1", "snr2", "downsample", "periodogram", "periodogram_plain", "running_median",
    "periodogram_length", "downsampled_size",
]

_torch = None


def _t():
    global _torch
    if _torch is None:
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("riptide_b200 needs a CUDA device (none is available)")
        _torch = torch
    return _torch


def _is_cuda_tensor(x):
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _as_f32(x, ndim=None):
    """(device tensor, was_device). Mirrors py::array_t<float> conversion + the contiguity
    check of python_bindings.cpp:33-41."""
    torch = _t()
    if _is_cuda_tensor(x):
        t = x
        if t.dtype != torch.float32:
            t = t.to(torch.float32).contiguous()
        elif not t.is_contiguous():
            raise ValueError("Input numpy array must be contiguous in memory")
        dev = True
    else:
        a = np.asarray(x)
        if a.dtype != np.float32:
            a = np.ascontiguousarray(a, dtype=np.float32)
        elif not a.flags.c_contiguous:
            raise ValueError("Input numpy array must be contiguous in memory")
        t = torch.from_numpy(a).to("cuda", non_blocking=False)
        dev = False
    if ndim is not None and t.dim() != ndim:
        raise ValueError(f"array has incorrect number of dimensions: {t.dim()}; expected {ndim}")
    return t, dev


def _out(t, dev):
    if dev:
        return t
    _t().cuda.current_stream().synchronize()
    return t.cpu().numpy()


def _stream():
    return ctypes.c_void_p(_t().cuda.current_stream().cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _empty(shape, dtype, like):
    torch = _t()
    return torch.empty(shape, dtype=dtype, device=like.device)


# --------------------------------------------------------------------------------------
def rollback(x, shift):
    """out = roll(x, -shift) (python_bindings.cpp:44-52)."""
    t, dev = _as_f32(x, 1)
    out = _empty(t.shape, t.dtype, t)
    _lib.check(_lib.load().rt_rollback(_ptr(t), t.numel(), int(shift), _ptr(out), _stream()))
    return _out(out, dev)


def fused_rollback_add(x, y, shift):
    """x + roll(y, -shift) (python_bindings.cpp:55-70)."""
    nx = x.numel() if _is_cuda_tensor(x) else np.size(x)
    ny = y.numel() if _is_cuda_tensor(y) else np.size(y)
    if nx != ny:
        raise ValueError("Arrays must have the same number of elements")
    tx, dev = _as_f32(x, 1)
    ty, _ = _as_f32(y, 1)
    out = _empty(tx.shape, tx.dtype, tx)
    _lib.check(_lib.load().rt_fused_rollback_add(_ptr(tx), _ptr(ty), tx.numel(), int(shift),
                                                 _ptr(out), _stream()))
    return _out(out, dev)


def circular_prefix_sum(x, nsum):
    """Circular prefix sum over nsum elements (python_bindings.cpp:73-81). Returns nsum
    values (the reference's output buffer is sized like the input, which overflows when
    nsum > size; here it always holds nsum values)."""
    t, dev = _as_f32(x, 1)
    out = _empty((int(nsum),), t.dtype, t)
    _lib.check(_lib.load().rt_circular_prefix_sum(_ptr(t), t.numel(), int(nsum), _ptr(out),
                                                  _stream()))
    return _out(out, dev)


def ffa2(arr):
    """FFA transform of a 2D (rows, cols) array, bit-identical to the reference
    (python_bindings.cpp:84-96)."""
    t, dev = _as_f32(arr, 2)
    out = _empty(t.shape, t.dtype, t)
    rows, cols = t.shape
    _lib.check(_lib.load().rt_ffa2(_ptr(t), rows, cols, _ptr(out), _stream()))
    return _out(out, dev)


def benchmark_ffa2(rows, cols, loops):
    """Seconds per FFA transform of a zero rows x cols block (python_bindings.cpp:99-118)."""
    _t()
    sec = ctypes.c_double(0.0)
    _lib.check(_lib.load().rt_benchmark_ffa2(int(rows), int(cols), int(loops), ctypes.byref(sec)))
    return sec.value


def _snr(t, dev, widths, stdnoise):
    w, wp = _lib.u64_array(widths)
    rows, cols = t.shape
    out = _empty((rows, w.size), t.dtype, t)
    _lib.check(_lib.load().rt_snr2(_ptr(t), rows, cols, wp, w.size, float(stdnoise), _ptr(out),
                                   _stream()))
    return out


def snr1(data, widths, stdnoise=1.0):
    """S/N of one profile for several boxcar widths (python_bindings.cpp:121-138)."""
    t, dev = _as_f32(data, 1)
    out = _snr(t.reshape(1, -1), dev, widths, stdnoise)
    return _out(out.reshape(-1), dev)


def snr2(data, widths, stdnoise=1.0):
    """S/N of (num_profiles, num_bins) profiles (python_bindings.cpp:141-160)."""
    t, dev = _as_f32(data, 2)
    return _out(_snr(t, dev, widths, stdnoise), dev)


def downsampled_size(size, f):
    return int(_lib.load().rt_downsampled_size(int(size), float(f)))


def downsample(data, factor):
    """Downsample by a real-valued factor (python_bindings.cpp:163-177)."""
    t, dev = _as_f32(data, 1)
    f = float(factor)
    if not ((f > 1.0) and (f <= t.numel())):
        raise ValueError("Downsampling factor must verify: 1 < f <= size")
    out = _empty((downsampled_size(t.numel(), f),), t.dtype, t)
    _lib.check(_lib.load().rt_downsample(_ptr(t), t.numel(), f, _ptr(out), _stream()))
    return _out(out, dev)


def running_median(data, width):
    """Exact running median, odd width < size, edge padding (python_bindings.cpp:212-222)."""
    t, dev = _as_f32(data, 1)
    out = _empty(t.shape, t.dtype, t)
    _lib.check(_lib.load().rt_running_median(_ptr(t), t.numel(), int(width), _ptr(out),
                                             _stream()))
    return _out(out, dev)


def periodogram_length(size, tsamp, period_min, period_max, bins_min, bins_max):
    L = ctypes.c_size_t(0)
    _lib.check(_lib.load().rt_periodogram_length(int(size), float(tsamp), float(period_min),
                                                 float(period_max), int(bins_min),
                                                 int(bins_max), ctypes.byref(L)))
    return L.value


def _periodogram(fn, data, tsamp, widths, period_min, period_max, bins_min, bins_max):
    torch = _t()
    t, dev = _as_f32(data, 1)
    w, wp = _lib.u64_array(widths)
    L = periodogram_length(t.numel(), tsamp, period_min, period_max, bins_min, bins_max)
    if L == 0:
        # the reference cannot return an empty periodogram: pybind11 raises on
        # mutable_data(0) of the zero-length output (python_bindings.cpp:196-205)
        raise IndexError("index 0 is out of bounds for axis 0 with size 0")
    periods = torch.empty((L,), dtype=torch.float64, device=t.device)
    foldbins = torch.empty((L,), dtype=torch.int32, device=t.device)
    snrs = torch.empty((L, w.size), dtype=torch.float32, device=t.device)
    _lib.check(fn(_ptr(t), t.numel(), float(tsamp), wp, w.size, float(period_min),
                  float(period_max), int(bins_min), int(bins_max), _ptr(periods),
                  _ptr(foldbins), _ptr(snrs), _stream()))
    if dev:
        return periods, foldbins, snrs
    torch.cuda.current_stream().synchronize()
    return (periods.cpu().numpy(), foldbins.cpu().numpy().view(np.uint32),
            snrs.cpu().numpy())


def periodogram(data, tsamp, widths, period_min, period_max, bins_min, bins_max):
    """Periodogram of a normalised series: (periods f64[L], foldbins u32[L], snrs f32[L, nw])
    (python_bindings.cpp:180-209). Runs the fused batched engine on one series. For CUDA
    tensor input, foldbins is an int32 tensor holding the uint32 values."""
    return _periodogram(_lib.load().rt_periodogram, data, tsamp, widths, period_min,
                        period_max, bins_min, bins_max)


def periodogram_plain(data, tsamp, widths, period_min, period_max, bins_min, bins_max):
    """Same result computed with one launch per step of the reference's loop nest
    (cpp/periodogram.hpp:153-200): the plain GPU path used as the batching baseline."""
    return _periodogram(_lib.load().rt_periodogram_plain, data, tsamp, widths, period_min,
                        period_max, bins_min, bins_max)
