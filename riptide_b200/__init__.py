"""riptide_b200: riptide's FFA search (v-morello/riptide) on NVIDIA B200 GPUs.

Hand-written sm_100a CUDA kernels behind a C ABI (include/riptide_b200.h), with the
reference's Python API on top. ``riptide_b200.libcpp`` replaces ``riptide.libcpp``.
"""
from . import libcpp
from .batched import BatchedSearch, SearchPipeline, ffa_search_batched
from .ffautils import generate_width_trials
from .folding import fold, fold_batched, fold_candidates
from .libffa import boxcar_snr, downsample, ffa1, ffa2, ffafreq, ffaprd, generate_signal
from .metadata import Metadata
from .peaks import Peak, find_peaks, find_peaks_batched
from .periodogram import Periodogram
from .running_medians import fast_running_median, running_median
from .search import ffa_search
from .time_series import TimeSeries
from .worker_pool import WorkerPool

__all__ = [
    "TimeSeries", "Periodogram", "ffa_search", "ffa_search_batched", "BatchedSearch", "SearchPipeline",
    "ffa1",
    "ffa2", "ffafreq", "ffaprd", "generate_signal", "downsample", "boxcar_snr",
    "running_median", "fast_running_median", "generate_width_trials", "libcpp",
    "find_peaks", "find_peaks_batched", "Peak", "fold", "fold_batched", "fold_candidates", "Metadata", "WorkerPool",
]
