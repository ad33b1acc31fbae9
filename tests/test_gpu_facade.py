"""The C++ drop-in facade, called through the reference's mangled C++ symbols.

Each of the ten hot-path entry points of Library/hostLibrary.cuh is called via
ctypes by its mangled name with the output file chosen by CBF_OUT_FILE_PATH (the
reference hard-codes OUT_FILE_PATH, hostLibrary.cu:3) and the system by
cbf_facade_set_system, and the file is compared byte for byte with the CPU
oracle's values written in the reference's ostream layout:

* 1-D diagrams: "param, peak\\n" per peak at precision 12 (hostLibrary.cu:125-138),
  param = getValueByIdx on the host;
* KDE maps: header "r0 r1\\nr2 r3\\n" at precision 12 (:474-480); the IC variant
  writes no header (:1004-1079);
* DBSCAN maps: header at the default precision 6 (:651-655), the IC variant too
  (:1172-1176);
* 1-D LLE: "param, lle\\n" at precision 6 (:1368-1378);
* LLE2D: header + map; LLE2DIC: map without header (:1732-1788).

Integer maps and peak values are bit-exact against the oracle.  LLE values are
compared after formatting to 6 significant digits, from the device's seed
vectors (FP32 sinf of the seed index; the oracle otherwise matches to ~1e-13,
far below the printed precision).  The LLE seed index is chunk-local in the
reference (LLE1D/LLE1DIC/LLE2DIC size the chunk from free device memory,
LLE2D uses 200000 points); these grids are smaller than any such chunk, so the
index is the point's own.
"""
import ctypes as C

import numpy as np
import pytest

from test_abi import _ref_map_csv

pytestmark = pytest.mark.gpu

D, I, P = C.c_double, C.c_int, C.c_void_p
BIF1D_ARGS = [D, I, D, I, P, P, P, I, D, D, P, I, I]
KDE_ARGS = [D, I, D, I, P, P, P, I, D, I, D, P, I, I, I, D, D, D]
DBSCAN_ARGS = [D, I, D, I, P, P, P, I, D, I, D, P, I, I, D]
LLE_ARGS = [D, D, I, D, D, P, I, P, P, I, D, D, P, I]

SYMBOLS = {
    "bifurcation1D": ("_Z13bifurcation1DdidiPKdS0_PKiiddS0_ii", BIF1D_ARGS),
    "bifurcation1DIC": ("_Z15bifurcation1DICdidiPKdS0_PKiiddS0_ii", BIF1D_ARGS),
    "bifurcation2DKDE": ("_Z16bifurcation2DKDEdidiPKdS0_PKiididS0_iiiddd", KDE_ARGS),
    "bifurcation2DKDEIC": ("_Z18bifurcation2DKDEICdidiPKdS0_PKiididS0_iiiddd", KDE_ARGS),
    "bifurcation2DDBSCAN": ("_Z19bifurcation2DDBSCANdidiPKdS0_PKiididS0_iid", DBSCAN_ARGS),
    "bifurcation2DDBSCANIC": ("_Z21bifurcation2DDBSCANICdidiPKdS0_PKiididS0_iid", DBSCAN_ARGS),
    "LLE1D": ("_Z5LLE1DddiddPKdiS0_PKiiddS0_i", LLE_ARGS),
    "LLE1DIC": ("_Z7LLE1DICddiddPKdiS0_PKiiddS0_i", LLE_ARGS),
    "LLE2D": ("_Z5LLE2DddiddPKdiS0_PKiiddS0_i", LLE_ARGS),
    "LLE2DIC": ("_Z7LLE2DICddiddPKdiS0_PKiiddS0_i", LLE_ARGS),
}

ROSSLER = dict(system="rossler", ic=[0.1, 0.1, 0.1], values=[0.5, 0.2, 0.2, 5.7])
LORENZ = dict(system="lorenz", ic=[0.1, 0.1, 0.1], values=[0.5, 10.0, 28.0, 8.0 / 3.0])
CHEN = dict(system="chen", ic=[0.1, 0.1, 0.1], values=[0.5, 35.0, 3.0, 28.0])


class Arrays:
    """Host arrays kept alive for the duration of a call."""

    def __init__(self, ic, ranges, idx, values):
        self.ic = np.ascontiguousarray(ic, np.float64)
        self.ranges = np.ascontiguousarray(ranges, np.float64)
        self.idx = np.ascontiguousarray(idx, np.int32)
        self.values = np.ascontiguousarray(values, np.float64)

    def ptrs(self):
        return (self.ic.ctypes.data, self.ranges.ctypes.data, self.idx.ctypes.data,
                self.values.ctypes.data)


@pytest.fixture
def facade(cbf, gpu_ok, tmp_path, monkeypatch):
    """call(name, system, *args) -> the bytes of the file the entry point wrote."""
    L = cbf.lib()
    counter = [0]

    def call(name, system, *args):
        sym, argtypes = SYMBOLS[name]
        f = getattr(L, sym)
        f.restype = None
        f.argtypes = argtypes
        counter[0] += 1
        path = tmp_path / f"{name}_{counter[0]}.csv"
        monkeypatch.setenv("CBF_OUT_FILE_PATH", str(path))
        L.cbf_facade_set_system(cbf.SYSTEMS[system])
        f(*args)
        return path.read_bytes()

    L.cbf_facade_set_output_path(None)  # the environment variable decides
    yield call
    L.cbf_facade_set_system(-1)


def _param(orc, k, nPts, r0, r1):
    return orc.lib().orc_get_value_by_idx(k, nPts, r0, r1, 0)


def _peak_rows(orc, o, nPts, r, cap):
    peaks, _, counts = orc.map_peaks(o, 0, nPts, cap)
    out = []
    for k in range(nPts):
        par = _param(orc, k, nPts, r[0], r[1])
        for j in range(counts[k]):
            out.append("%.12g, %.12g\n" % (par, peaks[k, j]))
    return "".join(out).encode(), counts


@pytest.mark.parametrize("name,ic_sweep", [("bifurcation1D", False), ("bifurcation1DIC", True)])
def test_facade_bifurcation1d(cbf, orc, facade, name, ic_sweep):
    nPts, tMax, h, tr, pre = 12, 60.0, 0.01, 100.0, 2
    if ic_sweep:
        ranges, idx = [-3.0, 3.0], [1]
    else:
        ranges, idx = [0.05, 0.40], [1]
    a = Arrays(ROSSLER["ic"], ranges, idx, ROSSLER["values"])
    ic, rg, ix, vv = a.ptrs()
    got = facade(name, "rossler", tMax, nPts, h, 3, ic, rg, ix, 0, 1e4, tr, vv, 4, pre)
    o = orc.make_job(system="rossler", nPts=nPts, ranges=ranges, idxMut=idx, ic=ROSSLER["ic"],
                     values=ROSSLER["values"], h=h, tMax=tMax, transientTime=tr, maxValue=1e4,
                     preScaller=pre, sweepIC=ic_sweep)
    cap = int(tMax / h / pre) // 2
    want, counts = _peak_rows(orc, o, nPts, ranges, cap)
    assert counts.sum() > nPts
    assert got == want


@pytest.mark.parametrize("name,ic_sweep,header", [("bifurcation2DKDE", False, True),
                                                  ("bifurcation2DKDEIC", True, False)])
def test_facade_kde_maps(cbf, orc, facade, name, ic_sweep, header):
    nPts, tMax, h, tr = 6, 40.0, 0.005, 20.0
    maxPeaks, samp, i1, i2, hh = 10000, 10, -20.0, 60.0, 0.05
    if ic_sweep:
        ranges, idx = [-16.0, 16.0, -16.0, 16.0], [0, 1]
    else:
        ranges, idx = [5.0, 20.0, 20.0, 200.0], [1, 2]
    a = Arrays(LORENZ["ic"], ranges, idx, LORENZ["values"])
    ic, rg, ix, vv = a.ptrs()
    got = facade(name, "lorenz", tMax, nPts, h, 3, ic, rg, ix, 0, 1e4, maxPeaks, tr, vv, 4, 1, samp, i1, i2, hh)
    o = orc.make_job(system="lorenz", nPts=nPts, ranges=ranges, idxMut=idx, ic=LORENZ["ic"],
                     values=LORENZ["values"], h=h, tMax=tMax, transientTime=tr, maxValue=1e4,
                     maxAmountOfPeaks=maxPeaks, kdeSampling=samp, kdeI1=i1, kdeI2=i2, kdeH=hh,
                     sweepIC=ic_sweep)
    vals = orc.map_kde(o, 0, nPts * nPts)
    assert got == _ref_map_csv(vals.tolist(), nPts, ranges if header else None, 12, False)
    assert len(np.unique(vals)) > 1


@pytest.mark.parametrize("name,ic_sweep", [("bifurcation2DDBSCAN", False), ("bifurcation2DDBSCANIC", True)])
def test_facade_dbscan_maps(cbf, orc, facade, name, ic_sweep):
    nPts, tMax, h, tr, eps = 6, 40.0, 0.005, 20.0, 0.05
    if ic_sweep:
        ranges, idx = [-16.0, 16.0, -16.0, 16.0], [0, 1]
    else:
        ranges, idx = [5.0, 20.0, 20.0, 200.0], [1, 2]
    a = Arrays(LORENZ["ic"], ranges, idx, LORENZ["values"])
    ic, rg, ix, vv = a.ptrs()
    got = facade(name, "lorenz", tMax, nPts, h, 3, ic, rg, ix, 0, 1e4, 10000, tr, vv, 4, 1, eps)
    o = orc.make_job(system="lorenz", nPts=nPts, ranges=ranges, idxMut=idx, ic=LORENZ["ic"],
                     values=LORENZ["values"], h=h, tMax=tMax, transientTime=tr, maxValue=1e4,
                     maxAmountOfPeaks=10000, dbscanEps=eps, sweepIC=ic_sweep)
    vals = orc.map_dbscan(o, 0, nPts * nPts)
    assert len(np.unique(vals)) > 1
    assert got == _ref_map_csv(vals.tolist(), nPts, ranges, 6, False)  # both write the header


def _lle_oracle(cbf, orc, dims, ic_sweep, nPts, ranges, idx, tMax, NT, h, eps, tr):
    kw = dict(system="chen", nPts=nPts, ranges=ranges, idxMut=idx, ic=CHEN["ic"], values=CHEN["values"],
              h=h, tMax=tMax, NT=NT, transientTime=tr, lleEps=eps, maxValue=1e4, sweepIC=ic_sweep)
    j = cbf.make_job(task=cbf.TASK_LLE, **kw)
    n = nPts ** dims
    return orc.map_lle_seeded(orc.make_job(**kw), 0, n, cbf.lle_seeds(j))


@pytest.mark.parametrize("name,ic_sweep", [("LLE1D", False), ("LLE1DIC", True)])
def test_facade_lle1d(cbf, orc, facade, name, ic_sweep):
    nPts, tMax, NT, h, eps, tr = 9, 20.0, 0.5, 0.002, 1e-8, 5.0
    if ic_sweep:
        ranges, idx = [-10.0, 10.0], [0]
    else:
        ranges, idx = [30.0, 45.0], [1]
    a = Arrays(CHEN["ic"], ranges, idx, CHEN["values"])
    ic, rg, ix, vv = a.ptrs()
    got = facade(name, "chen", tMax, NT, nPts, h, eps, ic, 3, rg, ix, 0, 1e4, tr, vv, 4)
    vals = _lle_oracle(cbf, orc, 1, ic_sweep, nPts, ranges, idx, tMax, NT, h, eps, tr)
    want = "".join("%.6g, %.6g\n" % (_param(orc, k, nPts, ranges[0], ranges[1]), vals[k])
                   for k in range(nPts)).encode()
    assert got == want


@pytest.mark.parametrize("name,ic_sweep,header", [("LLE2D", False, True), ("LLE2DIC", True, False)])
def test_facade_lle2d(cbf, orc, facade, name, ic_sweep, header):
    nPts, tMax, NT, h, eps, tr = 5, 20.0, 0.5, 0.002, 1e-8, 5.0
    if ic_sweep:
        ranges, idx = [-10.0, 10.0, 5.0, 30.0], [0, 2]
    else:
        ranges, idx = [30.0, 45.0, 20.0, 30.0], [1, 3]
    a = Arrays(CHEN["ic"], ranges, idx, CHEN["values"])
    ic, rg, ix, vv = a.ptrs()
    got = facade(name, "chen", tMax, NT, nPts, h, eps, ic, 3, rg, ix, 0, 1e4, tr, vv, 4)
    vals = _lle_oracle(cbf, orc, 2, ic_sweep, nPts, ranges, idx, tMax, NT, h, eps, tr)
    assert got == _ref_map_csv(vals.tolist(), nPts, ranges if header else None, 6, True)
