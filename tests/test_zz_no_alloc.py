"""The no-allocation DBSCAN entry point, through the C-ABI.

cbf_bifurcation2d_dbscan_noalloc exists for callers that cannot call cudaMalloc
(device memory owned by another allocator, or latency-critical loops that cannot
take an allocation's synchronisation or an out-of-memory failure mid-run): the
caller owns the output, and the kernel's scratch is a fixed array inside the
library.  Its maps must equal those of the regular entry point
(cbf_bifurcation2d_dbscan) exactly -- DBSCAN counts are integers, compared
bit-exactly like every integer output in this suite -- on consecutive calls, since
every call reuses the same scratch.

This file is named to be collected last and must pass both on its own in a fresh
process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LORENZ = dict(nPts=24, tMax=60.0, h=0.005, ic=[0.1, 0.1, 0.1], ranges=[5.0, 20.0, 20.0, 200.0],
              idx=[1, 2], wv=0, maxValue=1e4, maxPeaks=10000, transient=50.0,
              values=[0.5, 10.0, 28.0, 8.0 / 3.0], pre=1, eps=0.05)


def _arrays(p):
    return (np.ascontiguousarray(p["ic"], np.float64), np.ascontiguousarray(p["ranges"], np.float64),
            np.ascontiguousarray(p["idx"], np.int32), np.ascontiguousarray(p["values"], np.float64))


def _call_noalloc(cbf, p, d_out_ptr, stream_ptr):
    ic, rg, ix, v = _arrays(p)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    return cbf.lib().cbf_bifurcation2d_dbscan_noalloc(
        2, p["tMax"], p["nPts"], p["h"], 3, ic.ctypes.data_as(dp), rg.ctypes.data_as(dp),
        ix.ctypes.data_as(ip), p["wv"], p["maxValue"], p["maxPeaks"], p["transient"],
        v.ctypes.data_as(dp), 4, p["pre"], p["eps"], C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr))


def _regular(cbf, p):
    return cbf.bifurcation2DDBSCAN(p["tMax"], p["nPts"], p["h"], 3, p["ic"], p["ranges"], p["idx"],
                                   p["wv"], p["maxValue"], p["maxPeaks"], p["transient"],
                                   p["values"], 4, p["pre"], p["eps"], system="lorenz").ravel()


@pytest.mark.parametrize("eps", [0.05, 1e-3])
def test_noalloc_matches_regular_entry_point_twice(cbf, gpu_ok, eps):
    torch = pytest.importorskip("torch")
    p = dict(LORENZ, eps=eps)
    n = p["nPts"] ** 2
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()

    cbf.check(_call_noalloc(cbf, p, out.data_ptr(), s.cuda_stream))  # first call: set-up
    first = out.cpu().numpy().copy()
    out.fill_(-7)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    cbf.check(_call_noalloc(cbf, p, out.data_ptr(), s.cuda_stream))
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    second = out.cpu().numpy().copy()

    want = _regular(cbf, p)
    assert np.array_equal(first, want)
    assert np.array_equal(second, want)
    assert (want > 0).any()
    # No device memory was taken by the second call.
    assert free_after >= free_before


def test_noalloc_long_records_match_two_pass_entry_point(cbf, gpu_ok):
    """Peak lists longer than the regular entry point's 1024-slot first pass.

    h = 0.01 over 900 time units gives 985..2849 peaks per point; with
    maxAmountOfPeaks 2500 the regular call computes some points in its first
    pass, recomputes the 1025..2500-peak points in its second pass and returns
    only the count-based result for the rest, while the no-allocation call runs
    every point once at the full capacity of 2500.  The maps must be equal."""
    torch = pytest.importorskip("torch")
    p = dict(LORENZ, nPts=6, h=0.01, tMax=900.0, transient=20.0, maxPeaks=2500, eps=0.05)
    n = p["nPts"] ** 2
    out = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    for _ in range(2):
        out.fill_(-7)
        torch.cuda.synchronize()
        cbf.check(_call_noalloc(cbf, p, out.data_ptr(), s.cuda_stream))
        assert np.array_equal(out.cpu().numpy(), _regular(cbf, p))


def test_noalloc_rejects_maps_beyond_its_scratch(cbf, gpu_ok):
    torch = pytest.importorskip("torch")
    # record 200 000 samples, maxAmountOfPeaks 100 000 -> 100 000 peaks per point > 32 767
    p = dict(LORENZ, nPts=4, tMax=1000.0, maxPeaks=100000)
    out = torch.zeros(16, dtype=torch.int32, device="cuda")
    st = _call_noalloc(cbf, p, out.data_ptr(), 0)
    assert st == 1  # CBF_ERR_INVALID_ARG
    msg = cbf.lib().cbf_last_error().decode()
    assert "64 MiB" in msg and "32767" in msg
