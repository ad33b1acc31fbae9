"""GPU tests of the Ostrovsky periodicity map (calculationOfPeriodicityByOstrovsky,
hostLibrary.cu:748-925; flags cudaLibrary.cu:288-352, value :628-662).

The values come from a small set (0, +-0.5, +-1, +-cluster counts), so the map
is compared with the oracle bit for bit, the sign of zero included (the
reference can produce -0 through `-1 * 0`, and its CSV then prints "-0").
"""
import ctypes as C

import numpy as np
import pytest

from test_abi import _ref_map_csv
from test_gpu_parity import LORENZ, ROSSLER, both

pytestmark = pytest.mark.gpu


def _kw(system_kw, **extra):
    kw = dict(system_kw, nPts=14, sweepIC=True, idxMut=[0, 2], h=0.01, tMax=40.0, transientTime=20.0,
              writableVar=0, preScaller=1, maxAmountOfPeaks=400, dbscanEps=0.05)
    if system_kw is LORENZ:
        kw.update(ranges=[-10.0, 10.0, 5.0, 40.0], ostrovskyThreshold=12.0)
    else:
        kw.update(ranges=[-6.0, 6.0, -2.0, 4.0], ostrovskyThreshold=3.0)
    kw.update(extra)
    return kw


CASES = [
    ("lorenz-all-below", LORENZ, dict(ostrovskyThreshold=100.0)),        # -clusters
    ("lorenz-all-above", LORENZ, dict(ostrovskyThreshold=-100.0)),       # +clusters
    ("lorenz-both-sides", LORENZ, {}),                                   # 0
    ("lorenz-over-cap", LORENZ, dict(ostrovskyThreshold=100.0, maxAmountOfPeaks=3)),  # -0
    ("lorenz-short", LORENZ, dict(tMax=1.5, ostrovskyThreshold=10.0)),   # +-0.5, +-1
    ("lorenz-diverged", LORENZ, dict(maxValue=15.0)),                    # -1
    ("rossler", ROSSLER, dict(ostrovskyThreshold=5.0)),
    ("rossler-prescaller", ROSSLER, dict(preScaller=3, tMax=90.0, ostrovskyThreshold=5.0)),
    ("rossler-short", ROSSLER, dict(tMax=3.0, ostrovskyThreshold=1.0)),
]


@pytest.mark.parametrize("name,system_kw,extra", CASES)
def test_ostrovsky_matches_oracle(cbf, orc, gpu_ok, name, system_kw, extra):
    kw = _kw(system_kw, **extra)
    j, o = both(cbf, orc, task=cbf.TASK_OSTROVSKY, **kw)
    got, _ = cbf.run_host(j)
    want = orc.map_ostrovsky(o, 0, kw["nPts"] ** 2)
    assert np.array_equal(got, want), np.nonzero(got != want)
    assert np.array_equal(np.signbit(got), np.signbit(want))


def test_ostrovsky_values_cover_the_rules(cbf, gpu_ok):
    """The cases produce every outcome of the rules: negative and positive
    cluster counts, 0 and -0, +-0.5, +-1."""
    vals = np.concatenate([cbf.run_host(cbf.make_job(task=cbf.TASK_OSTROVSKY, **_kw(sk, **ex)))[0]
                           for _, sk, ex in CASES])
    assert (vals <= -2).any() and (vals >= 2).any()
    assert ((vals == 0) & np.signbit(vals)).any() and ((vals == 0) & ~np.signbit(vals)).any()
    assert {-1.0, -0.5, 0.5, 1.0} <= set(vals.tolist())


def test_facade_ostrovsky_csv(cbf, gpu_ok, tmp_path):
    L = cbf.lib()
    kw = _kw(LORENZ)
    L.cbf_facade_set_system(cbf.SYS_LORENZ)
    path = tmp_path / "ost.csv"
    try:
        L.cbf_facade_set_output_path(str(path).encode())
        f = getattr(L, "_Z35calculationOfPeriodicityByOstrovskydidiPKdS0_PKiididS0_iidd")
        f.restype = None
        f.argtypes = [C.c_double, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                      C.c_double, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]
        ic = np.ascontiguousarray(kw["ic"], np.float64)
        rg = np.ascontiguousarray(kw["ranges"], np.float64)
        ix = np.ascontiguousarray(kw["idxMut"], np.int32)
        vv = np.ascontiguousarray(kw["values"], np.float64)
        f(kw["tMax"], kw["nPts"], kw["h"], 3, ic.ctypes.data, rg.ctypes.data, ix.ctypes.data, 0, 0.0,
          kw["maxAmountOfPeaks"], kw["transientTime"], vv.ctypes.data, 4, 1, kw["dbscanEps"],
          kw["ostrovskyThreshold"])
        want = cbf.calculationOfPeriodicityByOstrovsky(
            kw["tMax"], kw["nPts"], kw["h"], 3, ic, rg, ix, 0, 0.0, kw["maxAmountOfPeaks"],
            kw["transientTime"], vv, 4, 1, kw["dbscanEps"], kw["ostrovskyThreshold"], system="lorenz")
        assert path.read_bytes() == _ref_map_csv(want.ravel().tolist(), kw["nPts"], list(rg), 6, True)
    finally:
        L.cbf_facade_set_output_path(None)
        L.cbf_facade_set_system(-1)
