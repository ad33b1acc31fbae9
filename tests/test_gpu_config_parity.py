"""GPU parity at the full lengths of the benchmarked configurations.

The parity suite (test_gpu_parity.py) runs short records so that the oracle
finishes every map in seconds.  Here the benchmark's own job parameters
(bench.py: WORKLOAD, SUR_WORKLOAD, SECONDARY) run at their full transient and
record lengths on samples of their grids, through the C-ABI, against the CPU
oracle:

* Chen 2048^2 LLE map (tMax 1000 after a 500-unit transient, 1.25e6 steps per
  point, seed chunk 200000): 256 seeded random grid points, LLE within 1e-9
  absolute from the device's seed vectors (cudaLibrary.cu:666-785);
* Chen 8192^2 LLE + regime map (exact grid, 50-unit window, DBSCAN eps 0.02,
  range below 1e-6 -> class 0, LLE above 0.05 -> class 15): 256 seeded random
  points, class bit-exact, LLE within 1e-9;
* Lorenz 1024^2 KDE maps, 256 fixed samples and 4 samples per peak (record 200,
  transient 500; cudaLibrary.cu:356-441): 48-point slices, bit-exact;
* the Rossler 1-D diagram on all 1000 points (transient 1000, record 500;
  cudaLibrary.cu:220-284): peak values and counts bit-exact;
* the fused tcgen05 grid prediction against the network's CPU restatement
  (oracle/mlp_oracle.py) on 37^2 and 256^2 grids.
"""
import ctypes as C
import sys
from pathlib import Path

import numpy as np
import pytest

import mlp_oracle as M
from test_gpu_parity import assert_lle_close

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
import bench  # noqa: E402  (the benchmarked job parameters)

pytestmark = pytest.mark.gpu


def _sample(n_total, count, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n_total, size=count, replace=False)).astype(np.int64)


def _job_kw(w, drop=()):
    return {k: v for k, v in w.items() if k not in drop}


def _run_list(cbf, torch, task, kw, idx, out_dtype, with_aux):
    """The job's points idx (a device point list) through cbf_run."""
    d_idx = torch.from_numpy(idx).cuda()
    m = len(idx)
    out = torch.empty(m, dtype=out_dtype, device="cuda")
    aux = torch.empty(m, dtype=torch.int32, device="cuda") if with_aux else None
    j = cbf.make_job(task=task, nPoints=m, pointIndex=d_idx.data_ptr(), **kw)
    cbf.run_device(j, out.data_ptr(), aux.data_ptr() if with_aux else 0)
    seeds = cbf.lle_seeds(j)
    torch.cuda.synchronize()
    return out.cpu().numpy(), (aux.cpu().numpy() if with_aux else None), seeds


def test_chen_lle2d_2048_full_length(cbf, orc, gpu_ok):
    torch = pytest.importorskip("torch")
    w = dict(bench.WORKLOAD)
    assert (w["nPts"], w["tMax"], w["transientTime"], w["seedChunk"]) == (2048, 1000.0, 500.0, 200000)
    idx = _sample(w["nPts"] ** 2, 256, 11)
    got, _, seeds = _run_list(cbf, torch, cbf.TASK_LLE, w, idx, torch.float64, False)
    want = orc.map_lle_list(orc.make_job(**w), idx, z=seeds)
    assert_lle_close(got, want)
    assert np.isfinite(want).all()
    assert (want > 0.05).any() and (want < 0).any()  # chaotic and periodic points both sampled


def test_chen_regime_8192_full_length(cbf, orc, gpu_ok):
    torch = pytest.importorskip("torch")
    w = dict(bench.SUR_WORKLOAD)
    assert w["nPts"] == 8192 and w["flags"] & cbf.FLAG_EXACT_GRID and w["regimeTime"] == 50.0
    idx = _sample(w["nPts"] ** 2, 256, 12)
    got_l, got_c, seeds = _run_list(cbf, torch, cbf.TASK_LLE_REGIME, w, idx, torch.float64, True)
    want_l, want_c = orc.map_lle_regime(orc.make_job(**w), idx, seeds)
    assert np.array_equal(got_c, want_c), np.nonzero(got_c != want_c)
    assert_lle_close(got_l, want_l)
    assert len(np.unique(want_c)) >= 3  # equilibria, periodic classes and chaos sampled


@pytest.mark.parametrize("first", [0, 400_000, 1_048_000])
def test_lorenz_kde256_1024_full_length(cbf, orc, gpu_ok, first):
    w = dict(bench.SECONDARY["lorenz-kde256-1024"])
    assert w["flags"] & cbf.FLAG_KDE_FIXED and w["kdeSampling"] == 256
    kw = _job_kw(w, ("task",))
    got, _ = cbf.run_host(cbf.make_job(task=cbf.TASK_KDE, firstPoint=first, nPoints=48, **kw))
    j = cbf.make_job(task=cbf.TASK_KDE, **kw)
    o = orc.make_job(**kw)
    peaks, _, counts = orc.map_peaks(o, first, 48, cbf.lib().cbf_peak_capacity(C.byref(j)))
    want = np.array([orc.kde_fixed(peaks[k, :counts[k]], w["maxAmountOfPeaks"], w["kdeSampling"],
                                   w["kdeI1"], w["kdeI2"], w["kdeH"]) for k in range(48)], np.int32)
    assert np.array_equal(got, want), np.nonzero(got != want)
    assert counts.max() > 100  # full-length records: hundreds of peaks


@pytest.mark.parametrize("first", [0, 600_000, 1_048_000])
def test_lorenz_kde_1024_full_length(cbf, orc, gpu_ok, first):
    w = dict(bench.SECONDARY["lorenz-kde-1024"])
    assert w["kdeSampling"] == 4 and not w.get("flags", 0)
    kw = _job_kw(w, ("task",))
    got, _ = cbf.run_host(cbf.make_job(task=cbf.TASK_KDE, firstPoint=first, nPoints=48, **kw))
    want = orc.map_kde(orc.make_job(**kw), first, 48)
    assert np.array_equal(got, want), np.nonzero(got != want)
    assert want.max() >= 1


def test_rossler_bif1d_1000_all_points(cbf, orc, gpu_ok):
    w = dict(bench.SECONDARY["rossler-bif1d-1000"])
    assert (w["nPts"], w["tMax"], w["transientTime"]) == (1000, 500.0, 1000.0)
    kw = _job_kw(w, ("task",))
    peaks, counts = cbf.run_host(cbf.make_job(task=cbf.TASK_PEAKS, **kw))
    cap = peaks.shape[1]
    wp, _, wc = orc.map_peaks(orc.make_job(**kw), 0, 1000, cap)
    assert np.array_equal(counts, wc), np.nonzero(counts != wc)
    for k in range(1000):
        assert np.array_equal(peaks[k, :counts[k]], wp[k, :wc[k]]), k
    # most points oscillate; past the range of a where the attractor exists they diverge
    assert counts.sum() > 10_000


CHEN_REGIME = dict(system="chen", ranges=[30.0, 45.0, 20.0, 30.0], idxMut=[1, 3], ic=[0.1, 0.1, 0.1],
                   values=[0.5, 35.0, 3.0, 28.0], h=0.002, NT=0.5, lleEps=1e-8, maxValue=1e4,
                   seedChunk=200000, maxAmountOfPeaks=512, dbscanEps=0.02, regimeMinAmp=1e-6,
                   regimeChaosLle=0.05, flags=1, tMax=1.0, transientTime=1.0, regimeTime=1.0)


@pytest.mark.parametrize("side,seed,scale", [(37, 3, 1.0), (256, 8, 1.0), (256, 9, 0.25)])
def test_mlp_grid_prediction_tcgen05_matches_oracle(cbf, orc, gpu_ok, side, seed, scale):
    """The fused tcgen05 kernel against the float64 restatement with the same
    BF16 rounding points.  The kernel accumulates in FP32, so outputs differ by
    accumulation error (~1e-6), and where a hidden pre-activation lands within
    that error of a BF16 rounding midpoint the unit rounds the other way (one BF16
    ulp, moving an output by ~1e-4): with 768 hidden units that touches about 1 %
    of the points; the encoded inputs (sines and cosines from sincospif, within
    about an FP32 ulp of the oracle's) flip a BF16 rounding now and then too.
    Bounds: median difference below 1e-5, at most 5 % of points above 1e-4, none
    above 1e-2 (a point where a few units flip together; the largest seen is
    5.2e-3).  Classes: wherever the oracle's top-two logit gap exceeds twice the
    bound the argmax cannot change, so the classes must be equal there (side 37:
    a ragged last 128-point tile; scale 1/4: the encoding at a lower frequency
    scale)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(seed)
    net = cbf.Mlp(512, seed=seed)
    p = M.init_params(seed)
    off = M.offsets()
    for b in ("b1", "b2", "b3", "b4"):
        o, shape = off[b]
        p[o:o + shape[0]] = rng.normal(scale=0.3, size=shape[0])
    p32 = p.astype(np.float32)
    net.set_params(p32)
    net.set_encoding_scale(scale)
    job = cbf.make_job(task=cbf.TASK_LLE_REGIME, nPts=side, **CHEN_REGIME)
    n = side * side
    mean, std = 0.25, 2.0
    got_l = torch.empty(n, dtype=torch.float64, device="cuda")
    got_c = torch.empty(n, dtype=torch.int32, device="cuda")
    got_f = torch.empty(n, dtype=torch.float32, device="cuda")
    net.predict_grid(job, mean, std, got_l.data_ptr(), got_c.data_ptr(), got_f.data_ptr())
    # the features the kernel generates, restated from the grid coordinates
    idx = torch.arange(n, dtype=torch.int64, device="cuda")
    X = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    cbf.grid_features(job, idx.data_ptr(), n, X.data_ptr())
    torch.cuda.synchronize()
    coords = cbf.grid_coordinates(job)
    x = M.grid_features(3, side, CHEN_REGIME["ranges"], CHEN_REGIME["idxMut"], CHEN_REGIME["values"], coords)
    assert np.array_equal(X.cpu().numpy(), x)
    wl, wc, wf, wout, margin = M.predict(p32.astype(np.float64), x, mean, std, scale=scale)
    gl, gc, gf = got_l.cpu().numpy(), got_c.cpu().numpy(), got_f.cpu().numpy()
    d_out0 = np.abs((gl - mean) / std - wout[:, 0])
    assert d_out0.max() < 1e-2, d_out0.max()
    assert np.median(d_out0) < 1e-5, np.median(d_out0)
    assert np.mean(d_out0 > 1e-4) < 0.05, np.mean(d_out0 > 1e-4)
    assert np.abs(gf - wf).max() < 1e-2
    # logit differences are bounded like out0's; the argmax is stable where the gap is wide
    safe = margin > 2 * 1e-2
    assert np.array_equal(gc[safe], wc[safe]), np.nonzero(gc[safe] != wc[safe])
    assert safe.mean() > 0.9  # the class comparison covers most points
    assert len(np.unique(wc)) > 1
    net.close()
