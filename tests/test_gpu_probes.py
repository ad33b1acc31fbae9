"""GPU checks of the measurement probes (csrc/probes.cu) that bench.py reports."""
import pytest

pytestmark = pytest.mark.gpu


def test_fp64_step_stream_probe(cbf, gpu_ok):
    """The step-stream probe measures a plausible FP64 issue rate: below the pure
    FMA probe's rate (the same pipe with independent FMAs), above a fifth of it,
    and the divergence tracking does not make the stream faster."""
    fma_lane_rate = cbf.probe_fp64_peak(100.0) * 1e12 / 2  # FMAs per second
    tracked = cbf.probe_fp64_step(2, True, 6, 100.0)
    bare = cbf.probe_fp64_step(2, False, 6, 100.0)
    four = cbf.probe_fp64_step(4, True, 4, 100.0)
    for r in (tracked, bare, four):
        assert 0.2 * fma_lane_rate < r < 1.1 * fma_lane_rate, (r, fma_lane_rate)
    assert tracked < 1.05 * bare
    with pytest.raises(Exception):
        cbf.probe_fp64_step(3, True, 6, 10.0)
    with pytest.raises(Exception):
        cbf.probe_fp64_step(2, True, 17, 10.0)
