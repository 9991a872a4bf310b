"""The shared-atomic probe that bench.py rates the vote kernel against
(peaks/shared_atomic_peak.cu): its three address patterns must show the
bank-wavefront cost model the roofline uses.  Lanes on 32 distinct banks and
lanes on one word each take one wavefront; two distinct words per bank take
two, so they retire at half the rate."""
import pytest

import bench


@pytest.mark.gpu
def test_shared_atomic_probe_wavefront_model():
    peaks = bench.shared_atomic_peaks(0)
    assert peaks is not None, "libppf_peaks.so not built"
    one = peaks["1_wavefront"]
    assert 0.25 < one <= 1.05, peaks  # warp-wide atomics per SM cycle
    assert peaks["2_wavefronts"] == pytest.approx(one / 2, rel=0.15), peaks
    assert peaks["one_word"] == pytest.approx(one, rel=0.15), peaks
