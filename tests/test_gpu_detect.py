"""Event detection of mountainsortalg on the GPU (detect_events.cpp:69-135 over
the time chunks of p_mountainsort3.cpp:190-215) vs the oracle.  The chunk
statistics are formed in double in the reference's order, so the detected
times are identical (gate: exact equality per channel)."""
import numpy as np
import pytest

from mountainsort_b200 import _lib, api, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pre(gpu_lib):
    X = synth.generate_numpy(24, 400000, K=20, seed=21, sites=(3, 6))
    return api.bandpass_whiten(X, 30000, 300, 6000, num_threads=16)


@pytest.mark.parametrize("thr,interval,sign,chunk", [(3.0, 10.0, 0, 0), (4.0, 10.0, -1, 50000),
                                                      (3.5, 25.5, 1, 20000), (2.0, 3.0, 0, 123457),
                                                      (2.5, 300.0, 0, 70001)])
def test_detect_events_matches_oracle(gpu_lib, ref32, pre, thr, interval, sign, chunk):
    got = api.detect_events(pre, detect_threshold=thr, detect_interval=interval, detect_sign=sign, chunk_size=chunk)
    ref = ref32.detect_events(pre, detect_threshold=thr, detect_interval=interval, detect_sign=sign,
                              chunk_size=chunk or None)
    assert len(got) == pre.shape[1]
    for m in range(pre.shape[1]):
        np.testing.assert_array_equal(got[m], ref[m], err_msg=f"channel {m}")
    assert sum(len(t) for t in got) > 100


def test_detect_events_capacity(gpu_lib, pre):
    L = _lib.load()
    X = np.ascontiguousarray(pre[:100000])
    N, M = X.shape
    counts = np.zeros(M, np.int64)
    times = np.zeros(4, np.int64)
    rc = L.ms3gpu_detect_events(X.ctypes.data, M, N, 3.0, 10.0, 0, 0, counts.ctypes.data, times.ctypes.data, 4,
                                None)
    assert rc == _lib.ERR_INVALID and counts.sum() > 4 and "entries" in _lib.last_error()
