"""mountainsort_b200: B200-native ms3.bandpass_filter and ms3.whiten.

The compute runs in libms3gpu.so (hand-written sm_100a CUDA behind a C ABI,
include/ms3gpu.h).  This package holds the Python binding, the file-level
processor mirror, .mda I/O and the seeded synthetic-recording generator.
"""
from . import mdaio  # noqa: F401
from .api import (apply_whitening_matrix, bandpass_filter, bandpass_opts, bandpass_whiten,  # noqa: F401
                  bandpass_whiten_batch, chunk_size, default_num_threads, release_cached_memory,
                  requirements, whiten,
                  whiten_blocks, whiten_covariance, whitening_matrix)
from ._lib import Ms3GpuError  # noqa: F401

__version__ = "0.1.0"
