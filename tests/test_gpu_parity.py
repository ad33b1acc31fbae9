"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Bar: bit-exact for integer outputs (peak counts, KDE and DBSCAN counts), for
trajectories and for peak values/intervals; LLE within 1e-9 absolute.  The LLE
seed is FP32 `sinf` of an integer, whose last bit differs between CUDA and glibc
for some arguments, so the LLE comparisons start the oracle from the device's
seed vectors (cbf_lle_seeds) and a separate test bounds the seed difference;
what remains is CUDA vs glibc `log` in the sum.  Sizes are chosen so the oracle
finishes in seconds.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LLE_TOL = 1e-9

# Parameter sets (values[0] = s = 0.5, the reference's CD symmetry convention).
ROSSLER = dict(system="rossler", values=[0.5, 0.2, 0.2, 5.7], ic=[0.1, 0.1, 0.1])
LORENZ = dict(system="lorenz", values=[0.5, 10.0, 28.0, 8.0 / 3.0], ic=[0.1, 0.1, 0.1])
CHEN = dict(system="chen", values=[0.5, 35.0, 3.0, 28.0], ic=[0.1, 0.1, 0.1])
MEMRISTIVE = dict(system="memristive5", values=[8, 35, 15, 0.01, -1.6676, 0.0676, 0.3682, 0.5],
                  ic=[0.001, 0, 0, 0, 0])


def assert_lle_close(got, want, tol=LLE_TOL):
    """Same non-finite values (-inf when a trajectory lands exactly on a fixed
    point and log(0) enters the sum, NaN after inf-inf) at the same positions;
    finite values within tol."""
    got = np.asarray(got)
    want = np.asarray(want)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.array_equal(got[np.isinf(want)], want[np.isinf(want)])
    err = np.abs(got[fin] - want[fin])
    assert err.size == 0 or err.max() <= tol, (err.max(), np.argmax(err))


def both(cbf, orc, **kw):
    """The same job for the product (cbf.Job) and the oracle (orc.OrcJob)."""
    okw = {k: v for k, v in kw.items() if k not in ("task", "firstPoint", "nPoints", "flags",
                                                    "peakCapacity", "pointIndex")}
    return cbf.make_job(**kw), orc.make_job(**okw)


def test_expf_underflow_region_is_exactly_zero(cbf, gpu_ok):
    # The KDE epilogue skips terms whose FP32 exponent argument is <= -128.
    assert cbf.probe_expf_zero(-110.0) == 0
    assert cbf.probe_expf_zero(-100.0) > 0  # the probe does see nonzero results


@pytest.mark.parametrize("nPts,first,count", [(2048, 0, 4096), (2048, 4190000, 4304),
                                               (8192, 16777000, 6000), (8192, 67100000, 8864)])
def test_grid_coordinates_match_oracle(cbf, orc, gpu_ok, nPts, first, count):
    j = cbf.make_job(task=cbf.TASK_LLE, system="chen", nPts=nPts, ranges=[30, 45, 20, 30],
                     idxMut=[1, 3], ic=[0.1] * 3, values=[0.5, 35, 3, 28], h=0.002, tMax=1, NT=0.5,
                     firstPoint=first, nPoints=count)
    got = cbf.grid_coordinates(j)
    L = orc.lib()
    want0 = np.array([L.orc_get_value_by_idx(first + k, nPts, 30.0, 45.0, 0) for k in range(count)])
    want1 = np.array([L.orc_get_value_by_idx(first + k, nPts, 20.0, 30.0, 1) for k in range(count)])
    assert np.array_equal(got[:, 0], want0)
    assert np.array_equal(got[:, 1], want1)


@pytest.mark.parametrize("params,extra", [
    (ROSSLER, dict(ranges=[0.05, 0.35, 0.05, 0.35], idxMut=[1, 2], h=0.01, writableVar=0)),
    (LORENZ, dict(ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.005, writableVar=2)),
    (CHEN, dict(ranges=[30, 45, 20, 30], idxMut=[1, 3], h=0.002, writableVar=1)),
    # s = 0.3: the rescaled step's 9-instruction form, z (stored scaled) recorded
    (dict(CHEN, values=[0.3, 35.0, 3.0, 28.0]), dict(ranges=[30, 45, 20, 30], idxMut=[1, 3], h=0.002,
                                                    writableVar=2)),
    (MEMRISTIVE, dict(ranges=[-6, 6, -15, 15], idxMut=[4, 3], h=0.005, writableVar=4)),
])
@pytest.mark.parametrize("sweepIC", [False, True])
def test_trajectories_bit_exact(cbf, orc, gpu_ok, params, extra, sweepIC):
    kw = dict(params, **extra)
    if sweepIC:
        kw["idxMut"] = [0, 1]
        kw["ranges"] = [-2, 2, -3, 3]
    j, o = both(cbf, orc, task=cbf.TASK_TRAJECTORY, nPts=5, tMax=20 * kw["h"] * 100,
                transientTime=kw["h"] * 700, preScaller=2, maxValue=1e4, sweepIC=sweepIC, **kw)
    traj, div = cbf.run_host(j)
    rec = cbf.record_length(j)
    for g in range(25):
        want, wdiv = orc.trajectory(o, g)
        assert bool(div[g]) == wdiv, g
        got = traj[g, :rec]
        if wdiv:
            n_ok = np.argmax(~np.isfinite(got)) if not np.all(np.isfinite(got)) else rec
            assert np.array_equal(got[:n_ok], want[:n_ok]), g
        else:
            assert np.array_equal(got, want), g


def test_divergence_stops_trajectories_like_reference(cbf, orc, gpu_ok):
    # maxValue far inside the attractor: most points diverge during the record.
    j, o = both(cbf, orc, task=cbf.TASK_TRAJECTORY, nPts=6, tMax=5.0, transientTime=1.0,
                preScaller=1, maxValue=12.0, ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.005,
                writableVar=0, **LORENZ)
    traj, div = cbf.run_host(j)
    n_div = 0
    for g in range(36):
        want, wdiv = orc.trajectory(o, g)
        assert bool(div[g]) == wdiv
        n_div += wdiv
    assert n_div > 0


def test_bifurcation1d_rossler_bit_exact(cbf, orc, gpu_ok):
    # The 1-D diagram configuration (Rossler a in [0.05, 0.40], 1000 t.u. transient,
    # 500 t.u. record, h = 0.01) on 64 points.
    kw = dict(nPts=64, ranges=[0.05, 0.40], idxMut=[1], h=0.01, tMax=500.0, transientTime=1000.0,
              maxValue=1e4, writableVar=0, preScaller=1, **ROSSLER)
    j, o = both(cbf, orc, task=cbf.TASK_PEAKS, **kw)
    peaks, counts = cbf.run_host(j)
    cap = peaks.shape[1]
    wp, wt, wc = orc.map_peaks(o, 0, 64, cap)
    assert np.array_equal(counts, wc)
    for k in range(64):
        assert np.array_equal(peaks[k, :counts[k]], wp[k, :wc[k]]), k
    assert counts.sum() > 64


def test_bifurcation1d_reference_api_matches_job_api(cbf, gpu_ok):
    peaks, counts = cbf.bifurcation1D(100.0, 16, 0.01, 3, [0.1, 0.1, 0.1], [0.05, 0.35], [1], 0,
                                      1e4, 200.0, [0.5, 0.2, 0.2, 5.7], 4, 1, system="rossler")
    j = cbf.make_job(task=cbf.TASK_PEAKS, nPts=16, ranges=[0.05, 0.35], idxMut=[1], h=0.01,
                     tMax=100.0, transientTime=200.0, maxValue=1e4, **ROSSLER)
    p2, c2 = cbf.run_host(j)
    assert np.array_equal(counts, c2)
    for k in range(16):  # entries past the count are unspecified, as in the reference
        assert np.array_equal(peaks[k, :counts[k]], p2[k, :c2[k]])


LORENZ_MAP = dict(nPts=10, ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.005, tMax=60.0,
                  transientTime=50.0, maxValue=1e4, writableVar=0, preScaller=1, **LORENZ)


@pytest.mark.parametrize("maxPeaks,samp,i1,i2,hh,flags", [
    (10000, 10, -20.0, 60.0, 0.05, 0),
    (10000, 4, -30.0, 60.0, 0.5, 0),
    (40, 10, -20.0, 60.0, 0.05, 0),          # some points exceed maxAmountOfPeaks
    (10000, 256, -20.0, 60.0, 0.05, 2),      # fixed 256-sample extension
    (10000, 4, 60.0, -30.0, 0.5, 0),         # reversed interval: samples run downwards
    (10000, 10, -20.0, 60.0, 2.0, 0),        # wide kernel: most peaks reach most chunks
    (10000, 64, -20.0, 60.0, 0.005, 0),      # narrow kernel: most chunks see no peak
])
def test_kde_map_bit_exact(cbf, orc, gpu_ok, maxPeaks, samp, i1, i2, hh, flags):
    kw = dict(LORENZ_MAP, maxAmountOfPeaks=maxPeaks, kdeSampling=samp, kdeI1=i1, kdeI2=i2, kdeH=hh)
    j, o = both(cbf, orc, task=cbf.TASK_KDE, flags=flags, **kw)
    got, _ = cbf.run_host(j)
    n = kw["nPts"] ** 2
    if flags & cbf.FLAG_KDE_FIXED:
        # oracle: the same kde() with k1 = 256 fixed, i.e. kdeSampling = 256 / n per point
        peaks, _, counts = orc.map_peaks(o, 0, n, cbf.lib().cbf_peak_capacity(C.byref(j)))
        want = []
        for k in range(n):
            want.append(orc.kde_fixed(peaks[k, :counts[k]], maxPeaks, samp, i1, i2, hh))
        want = np.array(want, np.int32)
    else:
        want = orc.map_kde(o, 0, n)
    assert np.array_equal(got, want), np.nonzero(got != want)


@pytest.mark.parametrize("maxPeaks,eps", [(10000, 1e-3), (10000, 0.05), (10000, 2.0), (30, 0.05)])
def test_dbscan_map_bit_exact(cbf, orc, gpu_ok, maxPeaks, eps):
    kw = dict(LORENZ_MAP, maxAmountOfPeaks=maxPeaks, dbscanEps=eps)
    j, o = both(cbf, orc, task=cbf.TASK_DBSCAN, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_dbscan(o, 0, kw["nPts"] ** 2)
    assert np.array_equal(got, want), np.nonzero(got != want)


@pytest.mark.parametrize("tMax,eps", [(300.0, 1e-3), (300.0, 0.3), (300.0, 3.0), (500.0, 1e-3)])
def test_dbscan_long_records_bit_exact(cbf, orc, gpu_ok, tMax, eps):
    """Hundreds of peaks per point: about 400 (sorted-window scans, with small and
    large windows) and about 670 (more than a warp sorts: chunked scans)."""
    kw = dict(LORENZ_MAP, nPts=8, tMax=tMax, maxAmountOfPeaks=10000, dbscanEps=eps)
    j, o = both(cbf, orc, task=cbf.TASK_DBSCAN, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_dbscan(o, 0, 64)
    assert np.array_equal(got, want), np.nonzero(got != want)
    assert len(np.unique(want)) > 3


@pytest.mark.parametrize("first", [200_000, 530_000, 1_000_000])
def test_dbscan_full_workload_slices(cbf, orc, gpu_ok, first):
    """Slices of the 1024^2 Lorenz DBSCAN map (sigma in [5,20], rho in [20,200],
    transient 500, record 200, eps 1e-3), through the two-pass launch."""
    kw = dict(nPts=1024, ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.005, tMax=200.0, transientTime=500.0,
              maxValue=1e4, writableVar=0, preScaller=1, maxAmountOfPeaks=10000, dbscanEps=1e-3, **LORENZ)
    j, o = both(cbf, orc, task=cbf.TASK_DBSCAN, firstPoint=first, nPoints=48, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_dbscan(o, first, 48)
    assert np.array_equal(got, want), np.nonzero(got != want)


def test_kde_dbscan_ic_sweep_and_divergence(cbf, orc, gpu_ok):
    kw = dict(LORENZ_MAP, sweepIC=True, idxMut=[0, 1], ranges=[-16, 16, -16, 16], maxValue=30.0,
              maxAmountOfPeaks=10000)
    j, o = both(cbf, orc, task=cbf.TASK_DBSCAN, dbscanEps=0.05, **kw)
    got, _ = cbf.run_host(j)
    assert np.array_equal(got, orc.map_dbscan(o, 0, 100))
    j, o = both(cbf, orc, task=cbf.TASK_KDE, kdeSampling=10, kdeI1=-20.0, kdeI2=60.0, kdeH=0.05,
                **kw)
    got, _ = cbf.run_host(j)
    assert np.array_equal(got, orc.map_kde(o, 0, 100))


# Long records: 985..2849 peaks per point, so with maxAmountOfPeaks 2500 the
# map has points that fit the first pass (<= 1024 peaks), points recomputed in
# the second pass (1025..2500) and points that only need their count (> 2500).
SPLIT_MAP = dict(nPts=6, ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.01, tMax=900.0, transientTime=20.0,
                 maxValue=1e4, writableVar=0, preScaller=1, maxAmountOfPeaks=2500, **LORENZ)


@pytest.mark.parametrize("task", ["dbscan", "kde", "ostrovsky"])
def test_two_pass_maps_bit_exact(cbf, orc, gpu_ok, task):
    kw = dict(SPLIT_MAP)
    n = kw["nPts"] ** 2
    if task == "dbscan":
        j, o = both(cbf, orc, task=cbf.TASK_DBSCAN, dbscanEps=0.05, **kw)
        want = orc.map_dbscan(o, 0, n)
    elif task == "kde":
        j, o = both(cbf, orc, task=cbf.TASK_KDE, kdeSampling=2, kdeI1=-20.0, kdeI2=60.0, kdeH=0.5, **kw)
        want = orc.map_kde(o, 0, n)
    else:
        kw.update(sweepIC=True, idxMut=[0, 2], ranges=[-10.0, 10.0, 5.0, 40.0])
        j, o = both(cbf, orc, task=cbf.TASK_OSTROVSKY, dbscanEps=0.05, ostrovskyThreshold=12.0, **kw)
        want = orc.map_ostrovsky(o, 0, n)
    got, _ = cbf.run_host(j)
    assert np.array_equal(got, want), np.nonzero(got != want)
    if task == "ostrovsky":
        assert np.array_equal(np.signbit(got), np.signbit(want))


CHEN_LLE = dict(nPts=8, ranges=[30, 45, 20, 30], idxMut=[1, 3], h=0.002, NT=0.5, tMax=40.0,
                transientTime=10.0, lleEps=1e-8, maxValue=1e4, **CHEN)


@pytest.mark.parametrize("extra", [
    dict(),
    dict(seedChunk=37),                                     # chunk-local seed index
    dict(maxValue=20.0),                                    # early exits every interval
    dict(sweepIC=True, idxMut=[0, 2], ranges=[-16, 16, 5, 30]),
    dict(dims=1),
    dict(values=[0.3, 35.0, 3.0, 28.0]),                    # the rescaled step's 9-instruction form
])
def test_lle_map_matches_oracle(cbf, orc, gpu_ok, extra):
    kw = dict(CHEN_LLE)
    dims = extra.pop("dims", 2)
    kw.update(extra)
    if dims == 1:
        kw["idxMut"] = kw["idxMut"][:1]
        kw["ranges"] = kw["ranges"][:2]
        kw["nPts"] = 40
    j, o = both(cbf, orc, task=cbf.TASK_LLE, **kw)
    got, _ = cbf.run_host(j)
    n = kw["nPts"] ** dims
    want = orc.map_lle_seeded(o, 0, n, cbf.lle_seeds(j))
    assert_lle_close(got, want)
    assert np.isfinite(want).mean() > 0.9


@pytest.mark.parametrize("extra", [dict(), dict(maxValue=20.0), dict(sweepIC=True, idxMut=[0, 2],
                                                                    ranges=[-16, 16, 5, 30])])
def test_every_lle_kernel_shape_gives_the_same_map(cbf, orc, gpu_ok, extra):
    """Every shape the autotuner chooses from (points per thread, block size,
    register cap, step-loop unrolling) runs the same arithmetic: its map equals
    the oracle's, and shape 0's bit for bit; 37 points leave partial
    blocks and, with two points per thread, a half-used thread."""
    kw = dict(CHEN_LLE, nPts=37)
    kw.update(extra)
    j, o = both(cbf, orc, task=cbf.TASK_LLE, **kw)
    want = orc.map_lle_seeded(o, 0, 37 * 37, cbf.lle_seeds(j))
    maps = []
    try:
        for v in range(cbf.NUM_LLE_VARIANTS):
            cbf.set_lle_variant("chen", v)
            got, _ = cbf.run_host(j)
            assert_lle_close(got, want)
            maps.append(got)
    finally:
        cbf.set_lle_variant("chen", -1)
    for m in maps[1:]:
        assert np.array_equal(m, maps[0], equal_nan=True)


@pytest.mark.parametrize("params,extra", [
    (LORENZ, dict(ranges=[5, 20, 20, 200], idxMut=[1, 2], h=0.005)),
    (ROSSLER, dict(ranges=[0.05, 0.35, 0.05, 0.35], idxMut=[1, 2], h=0.01)),
    (MEMRISTIVE, dict(ranges=[-6, 6, -15, 15], idxMut=[4, 3], h=0.005, maxValue=1e7)),
])
def test_lle_other_systems(cbf, orc, gpu_ok, params, extra):
    kw = dict(nPts=6, NT=0.4, tMax=20.0, transientTime=5.0, lleEps=1e-6, maxValue=1e4)
    kw.update(params)
    kw.update(extra)
    j, o = both(cbf, orc, task=cbf.TASK_LLE, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_lle_seeded(o, 0, 36, cbf.lle_seeds(j))
    assert_lle_close(got, want)


def test_reference_named_lle2d(cbf, orc, gpu_ok):
    got = cbf.LLE2D(40.0, 0.5, 8, 0.002, 1e-8, [0.1, 0.1, 0.1], 3, [30, 45, 20, 30], [1, 3], 0,
                    1e4, 10.0, [0.5, 35, 3, 28], 4, system="chen")
    o = orc.make_job(nPts=8, ranges=[30, 45, 20, 30], idxMut=[1, 3], h=0.002, NT=0.5, tMax=40.0,
                     transientTime=10.0, lleEps=1e-8, maxValue=1e4, seedChunk=200000, **CHEN)
    j = cbf.make_job(task=cbf.TASK_LLE, seedChunk=200000, **CHEN_LLE)
    want = orc.map_lle_seeded(o, 0, 64, cbf.lle_seeds(j)).reshape(8, 8)
    assert_lle_close(got, want)


@pytest.mark.parametrize("sweepIC,chunk", [(False, 0), (False, 200000), (False, 37), (True, 0)])
def test_lle_seeds_match_glibc_within_ulps(cbf, orc, gpu_ok, sweepIC, chunk):
    """The seed is 0.5*sinf(int) normalised (cudaLibrary.cu:720-732, :843-855):
    CUDA's and glibc's sinf agree to a few float ulps, i.e. ~1e-7 relative."""
    kw = dict(CHEN_LLE, nPts=64, seedChunk=chunk)
    if sweepIC:
        kw.update(sweepIC=True, idxMut=[0, 2], ranges=[-16, 16, 5, 30])
    j, o = both(cbf, orc, task=cbf.TASK_LLE, **kw)
    dev = cbf.lle_seeds(j)
    host = orc.lle_seeds(o, 0, 64 * 64)
    assert np.all(np.abs(dev - host) <= 1e-6), np.abs(dev - host).max()
    assert np.allclose(np.linalg.norm(dev, axis=1), 1.0, atol=1e-15)
    frac_exact = np.mean(np.all(dev == host, axis=1))
    assert frac_exact > 0.3  # most seeds are bit-identical


def test_lle_long_run_seed_sensitivity_is_small(cbf, orc, gpu_ok):
    """With the oracle's own glibc seeds, the LLE still agrees once the
    perturbation has aligned (long record): the libm difference washes out."""
    kw = dict(CHEN_LLE, nPts=4, tMax=200.0, transientTime=20.0)
    j, o = both(cbf, orc, task=cbf.TASK_LLE, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_lle(o, 0, 16)
    assert_lle_close(got, want, 1e-5)


REGIME = dict(CHEN_LLE, nPts=10, tMax=40.0, transientTime=20.0, maxAmountOfPeaks=512,
              dbscanEps=0.05, regimeTime=20.0)


@pytest.mark.parametrize("extra", [dict(), dict(maxValue=20.0), dict(maxAmountOfPeaks=20),
                                   dict(regimeTime=60.0), dict(writableVar=2),
                                   dict(regimeMinAmp=1e-6), dict(regimeMinAmp=15.0),
                                   dict(regimeMinAmp=1e-6, regimeChaosLle=0.05, dbscanEps=0.02)])
def test_lle_regime_matches_oracle(cbf, orc, gpu_ok, extra):
    kw = dict(REGIME, **extra)
    j, o = both(cbf, orc, task=cbf.TASK_LLE_REGIME, **kw)
    lle, cls = cbf.run_host(j)
    n = kw["nPts"] ** 2
    want_lle, want_cls = orc.map_lle_regime(o, np.arange(n), cbf.lle_seeds(j))
    assert np.array_equal(cls, want_cls), np.nonzero(cls != want_cls)
    assert_lle_close(lle, want_lle)
    assert 0 <= cls.min() and cls.max() <= 15
    # the LLE of the fused kernel is the LLE kernel's, bit for bit
    plain = {k: v for k, v in kw.items() if k not in ("maxAmountOfPeaks", "dbscanEps", "regimeTime",
                                                      "regimeMinAmp", "regimeChaosLle")}
    lle2, _ = cbf.run_host(cbf.make_job(task=cbf.TASK_LLE, **plain))
    assert np.array_equal(lle, lle2, equal_nan=True)


@pytest.mark.parametrize("task", ["lle", "regime", "dbscan"])
def test_point_lists_equal_full_map_entries(cbf, gpu_ok, task):
    torch = pytest.importorskip("torch")
    if task == "dbscan":
        kw = dict(LORENZ_MAP, maxAmountOfPeaks=10000, dbscanEps=0.05)
        t = cbf.TASK_DBSCAN
    else:
        kw = dict(REGIME)
        t = cbf.TASK_LLE if task == "lle" else cbf.TASK_LLE_REGIME
        if task == "lle":
            kw = {k: v for k, v in kw.items() if k not in ("maxAmountOfPeaks", "dbscanEps",
                                                           "regimeTime")}
    full, full_aux = cbf.run_host(cbf.make_job(task=t, **kw))
    n = kw["nPts"] ** 2
    idx = torch.tensor(np.random.default_rng(3).permutation(n)[: n // 3], dtype=torch.int64,
                       device="cuda")
    m = idx.numel()
    out = torch.empty(m, dtype=torch.int32 if t == cbf.TASK_DBSCAN else torch.float64, device="cuda")
    aux = torch.empty(m, dtype=torch.int32, device="cuda")
    j = cbf.make_job(task=t, nPoints=m, pointIndex=idx.data_ptr(), **kw)
    cbf.run_device(j, out.data_ptr(), aux.data_ptr() if t == cbf.TASK_LLE_REGIME else 0)
    torch.cuda.synchronize()
    sel = idx.cpu().numpy()
    assert np.array_equal(out.cpu().numpy(), full[sel], equal_nan=True)
    if t == cbf.TASK_LLE_REGIME:
        assert np.array_equal(aux.cpu().numpy(), full_aux[sel])


def test_device_api_with_torch_stream(cbf, gpu_ok):
    torch = pytest.importorskip("torch")
    j = cbf.make_job(task=cbf.TASK_LLE, **CHEN_LLE)
    n = 64
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    before = cbf.kernel_launches()
    with torch.cuda.stream(s):
        cbf.run_device(j, out.data_ptr(), 0, s.cuda_stream)
    s.synchronize()
    assert cbf.kernel_launches() == before + 1
    host, _ = cbf.run_host(cbf.make_job(task=cbf.TASK_LLE, **CHEN_LLE))
    assert np.array_equal(out.cpu().numpy(), host, equal_nan=True)


def test_exact_grid_flag(cbf, orc, gpu_ok):
    j = cbf.make_job(task=cbf.TASK_LLE, system="chen", nPts=8192, ranges=[0, 8191, 0, 8191],
                     idxMut=[1, 3], ic=[0.1] * 3, values=[0.5, 35, 3, 28], h=0.002, tMax=1, NT=0.5,
                     firstPoint=16777216, nPoints=2048, flags=cbf.FLAG_EXACT_GRID)
    got = cbf.grid_coordinates(j)
    g = np.arange(16777216, 16777216 + 2048)
    assert np.array_equal(got[:, 0], (g % 8192).astype(float))
    assert np.array_equal(got[:, 1], (g // 8192).astype(float))


@pytest.mark.parametrize("task", ["lle", "traj"])
def test_fourteen_instruction_form_when_the_grid_holds_a_zero(cbf, orc, gpu_ok, task):
    """A Chen grid whose a-axis holds a = 0 runs the 14-instruction step (the
    rescaled form needs a != 0); results still equal the oracle's, which makes the
    same choice.  y (writableVar 1) is recorded in physical units either way."""
    kw = dict(CHEN, nPts=11, ranges=[-5.0, 5.0, 20.0, 30.0], idxMut=[1, 3], h=0.002, maxValue=1e4)
    j0 = cbf.make_job(task=cbf.TASK_LLE, NT=0.5, tMax=10.0, transientTime=2.0, lleEps=1e-8, **kw)
    import ctypes as C2
    cbf.lib().cbf_job_scaled_step.restype = C2.c_int32
    assert cbf.lib().cbf_job_scaled_step(C2.byref(j0)) == 0
    if task == "lle":
        j, o = both(cbf, orc, task=cbf.TASK_LLE, NT=0.5, tMax=10.0, transientTime=2.0, lleEps=1e-8, **kw)
        got, _ = cbf.run_host(j)
        assert_lle_close(got, orc.map_lle_seeded(o, 0, 121, cbf.lle_seeds(j)))
    else:
        j, o = both(cbf, orc, task=cbf.TASK_TRAJECTORY, tMax=2.0, transientTime=1.0, preScaller=1,
                    writableVar=1, **kw)
        traj, div = cbf.run_host(j)
        rec = cbf.record_length(j)
        for g in range(0, 121, 7):
            want, wdiv = orc.trajectory(o, g)
            assert bool(div[g]) == wdiv
            got = traj[g, :rec]
            # after a divergence the kernel writes NaN where the reference leaves memory unwritten
            n_ok = int(np.argmax(~np.isfinite(got))) if wdiv and not np.all(np.isfinite(got)) else rec
            assert np.array_equal(got[:n_ok], want[:n_ok], equal_nan=True), g
