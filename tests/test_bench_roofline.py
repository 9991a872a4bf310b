"""bench.py's shared-atomic roofline: the arithmetic that rates the vote
kernel against the probe's measured atomic rates, and the probe library's
export (no GPU call)."""
import ctypes

import pytest

import bench


def test_atomic_roofline_arithmetic():
    peaks = {"1_wavefront": 0.5, "2_wavefronts": 0.25, "one_word": 0.5}
    # 32 votes per warp-wide atomic; 148 SMs at 1000 MHz for 1 s
    votes = 32 * 0.2 * 148 * 1000e6
    r = bench.atomic_roofline(peaks, votes, 1.0, 1000.0, 148)
    assert r["achieved"] == pytest.approx(0.2)
    # cycles per atomic interpolate linearly in wavefronts: 2 + 0.82 * 2
    w = bench.VOTE_WAVEFRONTS_PER_ATOMIC
    assert r["ceiling_at_kernel_conflicts"] == pytest.approx(1.0 / (2.0 + (w - 1.0) * 2.0))
    assert r["frac"] == pytest.approx(0.2 * (2.0 + (w - 1.0) * 2.0))
    assert r["frac_of_conflict_free"] == pytest.approx(0.4)


def test_atomic_roofline_absent_inputs():
    assert bench.atomic_roofline(None, 1e12, 1.0, 1965.0, 148) is None
    assert bench.atomic_roofline({"1_wavefront": 0.5, "2_wavefronts": 0.25}, 1e12, 0.0, 1965.0, 148) is None
    assert bench.atomic_roofline({"1_wavefront": 0.5, "2_wavefronts": 0.25}, 1e12, 1.0, None, 148) is None


def test_probe_library_exports_its_entry_point():
    lib = bench.ROOT / "ppf-registration-spatial-hashing_b200" / "libppf_peaks.so"
    if not lib.exists():
        pytest.skip("probe library not built")
    assert hasattr(ctypes.CDLL(str(lib)), "ppf_peak_shared_atomics")
