"""C-ABI library checks that need no GPU: load, exports, validation, host logic."""
import ctypes as C
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

# The reference's hot-path entry points (Library/hostLibrary.cuh:29-459) by their
# C++ mangled names: the facade must link in their place.
REFERENCE_ENTRY_POINTS = [
    "_Z13bifurcation1DdidiPKdS0_PKiiddS0_ii",
    "_Z15bifurcation1DICdidiPKdS0_PKiiddS0_ii",
    "_Z16bifurcation2DKDEdidiPKdS0_PKiididS0_iiiddd",
    "_Z18bifurcation2DKDEICdidiPKdS0_PKiididS0_iiiddd",
    "_Z19bifurcation2DDBSCANdidiPKdS0_PKiididS0_iid",
    "_Z21bifurcation2DDBSCANICdidiPKdS0_PKiididS0_iid",
    "_Z5LLE1DddiddPKdiS0_PKiiddS0_i",
    "_Z7LLE1DICddiddPKdiS0_PKiiddS0_i",
    "_Z5LLE2DddiddPKdiS0_PKiiddS0_i",
    "_Z7LLE2DICddiddPKdiS0_PKiiddS0_i",
    "_Z35calculationOfPeriodicityByOstrovskydidiPKdS0_PKiididS0_iidd",
    "_Z22modelingOneSystemDenisdddiPKdiS0_i",
    "_Z4LS1DddiddPKdiS0_PKiiddS0_i",
    "_Z4LS2DddiddPKdiS0_PKiiddS0_i",
]


def _exports():
    out = subprocess.run(["nm", "-D", "--defined-only", str(ROOT / "cudabifurcation3.0_b200" / "libcbf.so")],
                         capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def _declared_in_headers():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"\b(cbf_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_loads_and_exports_every_declared_symbol(cbf):
    L = cbf.lib()
    assert L.cbf_abi_version() == 1
    exported = _exports()
    declared = _declared_in_headers()
    assert declared, "no declarations found in include/*.h"
    missing = sorted(declared - exported)
    assert not missing, f"declared in include/*.h but not exported: {missing}"
    assert not sorted(set(cbf.EXPORTS) - exported)


def test_facade_links_as_the_reference_entry_points(cbf):
    exported = _exports()
    assert not [s for s in REFERENCE_ENTRY_POINTS if s not in exported]


def test_facade_names_match_reference_header_when_available(orc):
    root = orc.reference_dir()
    if root is None:
        pytest.skip("reference sources not present")
    ref = root / "Library" / "hostLibrary.cuh"
    text = ref.read_text()
    for name in ("bifurcation1D", "bifurcation1DIC", "bifurcation2DKDE", "bifurcation2DKDEIC",
                 "bifurcation2DDBSCAN", "bifurcation2DDBSCANIC", "LLE1D", "LLE1DIC", "LLE2D",
                 "LLE2DIC", "calculationOfPeriodicityByOstrovsky", "LS1D", "LS2D",
                 "modelingOneSystemDenis"):
        assert re.search(r"__host__ void " + name + r"\(", text), name


def _job(cbf, **kw):
    base = dict(task=cbf.TASK_LLE, system="chen", nPts=16, ranges=[30, 45, 20, 30], idxMut=[1, 3],
                ic=[0.1, 0.1, 0.1], values=[0.5, 35, 3, 28], h=0.002, tMax=10, NT=0.5,
                lleEps=1e-8, transientTime=1, maxValue=1e4)
    base.update(kw)
    return cbf.make_job(**base)


@pytest.mark.parametrize("bad,code", [
    (dict(system=9), 2),
    (dict(ic=[0.1, 0.1]), 1),                 # wrong number of state variables
    (dict(values=[0.5, 35, 3]), 1),           # too few parameters
    (dict(idxMut=[1, 7]), 1),                 # swept index out of range
    (dict(h=0.0), 1),
    (dict(NT=0.0), 1),
    (dict(task=9), 1),
    (dict(task=1, preScaller=0, maxAmountOfPeaks=10), 1),
    (dict(task=1, writableVar=5, maxAmountOfPeaks=10), 1),
    (dict(nPts=0), 1),
])
def test_validation_errors(cbf, bad, code):
    j = _job(cbf, **bad)
    st = cbf.lib().cbf_validate(C.byref(j))
    assert st == code
    assert cbf.lib().cbf_last_error()  # a message is set


def test_validation_accepts_reference_configs(cbf):
    assert cbf.lib().cbf_validate(C.byref(_job(cbf))) == 0
    # LLE ignores writableVar (the reference hard-codes x[0], cudaLibrary.cu:735)
    assert cbf.lib().cbf_validate(C.byref(_job(cbf, writableVar=17))) == 0


def test_derived_sizes_use_reference_truncations(cbf):
    j = _job(cbf, task=cbf.TASK_KDE, tMax=200, h=0.005, maxAmountOfPeaks=10)
    assert cbf.record_length(j) == int(200 / 0.005)
    j = _job(cbf)
    assert cbf.record_length(j) == int(10 / 0.5)
    j = _job(cbf, task=cbf.TASK_PEAKS, tMax=500, h=0.01, preScaller=3, idxMut=[1], ranges=[0, 1])
    assert cbf.record_length(j) == int(500 / 0.01 / 3)


def test_divergence_threshold_is_exact(cbf, orc):
    """fabs(x) >= T reproduces `fabsf(x) > maxValue` (cudaLibrary.cu:69-71) exactly."""
    L = orc.lib()
    rng = np.random.default_rng(3)
    maxima = [1e4, 10.0, 6.0, 1000000.0, 1e7, 0.1, 1e-30, 3.4028234663852886e38, 1e300,
              -1.0, 5e-45] + list(rng.uniform(0, 1e5, 60)) + list(10 ** rng.uniform(-40, 38, 60))
    for m in maxima:
        active, t = cbf.divergence_threshold(m)
        assert active
        probes = [t, np.nextafter(t, 0), np.nextafter(t, np.inf), m, -m, 0.0, np.inf, -np.inf,
                  np.nextafter(m, 0), np.nextafter(m, np.inf)]
        probes += list(t * (1 + rng.uniform(-1e-6, 1e-6, 20)))
        for x in probes:
            x = float(x)
            if not np.isfinite(t) and not np.isfinite(x):
                continue
            want = bool(L.orc_diverged(x, m))
            got = abs(x) >= t
            assert want == got, (m, x, t)
    assert cbf.divergence_threshold(0.0)[0] is False
    assert cbf.divergence_threshold(float("inf"))[0] is False
    assert cbf.divergence_threshold(float("nan"))[0] is False


def _ref_map_csv(values, nPts, header, precision, is_double):
    """The reference's ostream output (hostLibrary.cu:474-546), restated in Python.
    glibc prints a NaN with its sign bit set as "-nan"; Python's %g drops the sign."""
    def fmt_double(v):
        if math.isnan(v):
            return "-nan" if math.copysign(1.0, v) < 0 else "nan"
        return "%.*g" % (precision, v)

    fmt = fmt_double if is_double else (lambda v: "%d" % v)
    s = []
    if header is not None:
        g = lambda v: "%.*g" % (precision, v)  # noqa: E731
        s.append(f"{g(header[0])} {g(header[1])}\n{g(header[2])} {g(header[3])}\n")
    cnt = 0
    for v in values:
        if cnt != 0:
            s.append(", ")
        if cnt == nPts:
            s.append("\n")
            cnt = 0
        s.append(fmt(v))
        cnt += 1
    return "".join(s).encode()


@pytest.mark.parametrize("nPts,precision,header,is_double", [
    (4, 12, [0.05, 0.35, 0.05, 0.35], False),
    (3, 6, [5, 20, 20, 200], False),
    (5, 6, None, True),
    (2, 6, [30, 45, 20, 30], True),
])
def test_csv_map_layout_is_byte_compatible(cbf, tmp_path, nPts, precision, header, is_double):
    rng = np.random.default_rng(nPts)
    if is_double:
        vals = np.concatenate([rng.normal(size=nPts * nPts - 3) * 10.0 ** rng.integers(-8, 8, nPts * nPts - 3),
                               [0.0, -0.0, 1.0 / 3.0]])
        buf = np.ascontiguousarray(vals, np.float64)
    else:
        buf = np.ascontiguousarray(rng.integers(-1, 50, nPts * nPts), np.int32)
    path = tmp_path / "m.csv"
    hdr = None if header is None else np.array(header, np.float64)
    st = cbf.lib().cbf_csv_write_map(str(path).encode(), buf.ctypes.data_as(C.c_void_p),
                                     int(is_double), len(buf), nPts,
                                     None if hdr is None else hdr.ctypes.data_as(C.c_void_p),
                                     precision)
    assert st == 0
    assert path.read_bytes() == _ref_map_csv(buf.tolist(), nPts, header, precision, is_double)
    text = path.read_text().split("\n")
    if header is not None:
        text = text[2:]
    assert len(text) == nPts and all(r.endswith(", ") for r in text[:-1])


def test_csv_peak_rows_layout(cbf, orc, tmp_path):
    nPts, cap = 5, 4
    ranges = np.array([0.05, 0.40], np.float64)
    peaks = np.arange(nPts * cap, dtype=np.float64).reshape(nPts, cap) / 7.0
    counts = np.array([0, 2, 4, 1, 3], np.int32)
    path = tmp_path / "p.csv"
    lib = cbf.lib()
    lib.cbf_csv_write_peaks.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_int64, C.c_int64,
                                        C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
    assert lib.cbf_csv_write_peaks(str(path).encode(), nPts, ranges.ctypes.data, 0, nPts,
                                   peaks.ctypes.data, cap, counts.ctypes.data, 0) == 0
    want = []
    for k in range(nPts):
        par = orc.lib().orc_get_value_by_idx(k, nPts, 0.05, 0.40, 0)
        for j in range(counts[k]):
            want.append("%.12g, %.12g\n" % (par, peaks[k, j]))
    assert path.read_text() == "".join(want)


def test_csv_open_failure_is_reported(cbf, tmp_path):
    buf = np.zeros(4, np.int32)
    bad = tmp_path / "missing_dir" / "x.csv"
    st = cbf.lib().cbf_csv_write_map(str(bad).encode(), buf.ctypes.data_as(C.c_void_p), 0, 4, 2,
                                     None, 6)
    assert st == 6  # CBF_ERR_IO


def test_csv_rows_layout(cbf, orc, tmp_path):
    """LS1D rows "param, l1, ..., lN\\n" at the default ostream precision
    (hostLibrary.cu:1900-1910)."""
    nPts, cols = 6, 3
    ranges = np.array([0.05, 0.40], np.float64)
    vals = np.random.default_rng(2).normal(size=(nPts, cols)) * 10.0 ** np.arange(-3, 3).reshape(nPts, 1)
    vals = np.ascontiguousarray(vals)
    path = tmp_path / "r.csv"
    assert cbf.lib().cbf_csv_write_rows(str(path).encode(), nPts, ranges.ctypes.data, vals.ctypes.data,
                                        nPts, cols, 6) == 0
    want = []
    for k in range(nPts):
        par = orc.lib().orc_get_value_by_idx(k, nPts, 0.05, 0.40, 0)
        want.append("%.6g" % par + "".join(", %.6g" % v for v in vals[k]) + "\n")
    assert path.read_text() == "".join(want)


@pytest.mark.parametrize("is_double", [True, False])
def test_csv_map_parallel_formatter_is_byte_compatible(cbf, tmp_path, monkeypatch, is_double):
    """The threaded map formatter (several rounds of 2^18-value blocks, a ragged
    last block) writes the same bytes as the reference's serial ostream rule."""
    nPts = 1100
    rng = np.random.default_rng(5)
    n = nPts * nPts
    if is_double:
        buf = np.ascontiguousarray(rng.normal(size=n) * 10.0 ** rng.integers(-9, 9, n), np.float64)
        buf[::997] = 0.0
    else:
        buf = np.ascontiguousarray(rng.integers(-5, 16, n), np.int32)
    hdr = np.array([30.0, 45.0, 20.0, 30.0], np.float64)
    want = _ref_map_csv(buf.tolist(), nPts, list(hdr), 6, is_double)
    for threads in ("3", "1"):
        monkeypatch.setenv("CBF_CSV_THREADS", threads)
        path = tmp_path / f"p{threads}.csv"
        assert cbf.lib().cbf_csv_write_map(str(path).encode(), buf.ctypes.data_as(C.c_void_p),
                                           int(is_double), n, nPts, hdr.ctypes.data_as(C.c_void_p), 6) == 0
        assert path.read_bytes() == want


def test_npy_sidecar_and_writer(cbf, tmp_path, monkeypatch):
    L = cbf.lib()
    L.cbf_npy_write.argtypes = [C.c_char_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int64]
    a = np.ascontiguousarray(np.random.default_rng(1).normal(size=(7, 5)))
    p = tmp_path / "a.npy"
    assert L.cbf_npy_write(str(p).encode(), a.ctypes.data_as(C.c_void_p), 1, 7, 5) == 0
    assert np.array_equal(np.load(p), a)
    b = np.ascontiguousarray(np.arange(36, dtype=np.int32))
    monkeypatch.setenv("CBF_NPY_SIDECAR", "1")
    m = tmp_path / "m.csv"
    assert L.cbf_csv_write_map(str(m).encode(), b.ctypes.data_as(C.c_void_p), 0, 36, 6, None, 6) == 0
    got = np.load(str(m) + ".npy")
    assert got.dtype == np.int32 and got.shape == (6, 6) and np.array_equal(got.ravel(), b)
    assert m.read_bytes() == _ref_map_csv(b.tolist(), 6, None, 6, False)


def test_surrogate_config_defaults(cbf):
    """The defaults of cbf_surrogate_config_init (host code) are the measured
    operating point that include/cbf.h documents: 512^2 coarse labels plus 65 536
    random points, 1500 Adam steps on minibatches of 4096, confidence threshold
    0.4, 1 % audit, automatic expansion radius, 12 expanding rounds."""
    c = cbf.surrogate_config()
    assert (c.coarseSide, c.randomPoints, c.batch, c.trainSteps) == (512, 65536, 4096, 1500)
    assert c.confThreshold == pytest.approx(0.4) and c.auditFraction == pytest.approx(0.01)
    assert (c.boundaryRadius, c.expandRadius, c.maxWaves, c.refine) == (1, -1, 12, 1)
    assert (c.predictor, c.auditFill, c.idleRadius) == (0, 0, 0)
    with pytest.raises(AttributeError):
        cbf.surrogate_config(noSuchField=1)


@pytest.mark.parametrize("kw,want", [
    (dict(), 2),                                              # Chen a in [30, 45], s = 1/2: 8-instruction form
    (dict(system="lorenz", values=[0.5, 10, 28, 8 / 3], ranges=[5, 20, 20, 200], idxMut=[1, 2]), 2),
    (dict(values=[0.3, 35, 3, 28]), 1),                       # s != 1/2: the 9-instruction form
    (dict(values=[0.0, 35, 3, 28]), 0),                       # s = 0 (k = 0): 14-instruction form
    (dict(values=[1.0, 35, 3, 28]), 1),                       # s = 1 (h1 = 0)
    (dict(ranges=[-5, 5, 20, 30], nPts=11), 0),               # a = 0 on the grid: 14-instruction form
    (dict(ranges=[-5, 5, 20, 30], nPts=10), 2),               # a never exactly 0
    (dict(idxMut=[0, 3], ranges=[0.2, 0.8, 20, 30]), 0),      # s swept
    (dict(system="rossler", values=[0.5, 0.2, 0.2, 5.7], ranges=[0.05, 0.35, 0.05, 0.35], idxMut=[1, 2]), 0),
    (dict(sweepIC=True, idxMut=[0, 2], ranges=[-5, 5, -5, 5]), 2),
    (dict(values=[0.5, 0.0, 3, 28], sweepIC=True, idxMut=[0, 2], ranges=[-5, 5, -5, 5]), 0),
    (dict(values=[0.5, 35, 3, 1e30], idxMut=[1, 2], ranges=[30, 45, 1, 5]), 0),  # c beyond 2^64
])
def test_step_form_choice_matches_oracle(cbf, orc, kw, want):
    """The rescaled Chen/Lorenz step is chosen per job by the same rule in the
    library and the oracle (every value the grid holds is checked): 2 for its
    8-instruction form (s = 1/2), 1 for the 9-instruction form, 0 for the
    14-instruction form."""
    base = dict(system="chen", nPts=16, ranges=[30, 45, 20, 30], idxMut=[1, 3], ic=[0.1, 0.1, 0.1],
                values=[0.5, 35, 3, 28], h=0.002, tMax=10, NT=0.5, lleEps=1e-8, transientTime=1, maxValue=1e4)
    base.update(kw)
    j = cbf.make_job(task=cbf.TASK_LLE, **base)
    L = cbf.lib()
    L.cbf_job_scaled_step.restype = C.c_int32
    L.cbf_job_scaled_step.argtypes = [C.c_void_p]
    got = L.cbf_job_scaled_step(C.addressof(j))
    O = orc.lib()
    O.orc_scaled_step.restype = C.c_int
    O.orc_scaled_step.argtypes = [C.c_void_p]
    o = orc.make_job(**base)
    assert got == want
    assert O.orc_scaled_step(C.addressof(o)) == want


def test_bench_step_cost_tables():
    """The bench's flop accounting: the rescaled forms keyed by
    cbf_job_scaled_step (8 instructions / 14 flops at s = 1/2, 9 / 15 otherwise)
    and the unfused CD formula's count for Chen, applied per point and step."""
    import importlib.util
    from pathlib import Path
    spec = importlib.util.spec_from_file_location("bench_for_test", Path(__file__).resolve().parents[1] / "bench.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    assert b.SCALED_COST[2][:2] == (14, 8) and b.SCALED_COST[1][:2] == (15, 9)
    r = b.unfused_cd("chen", 1000, 2000, 1000.0, 1.0)
    assert r["unfused_cd_flops_per_step"] == 28
    assert r["unfused_cd_achieved"] == pytest.approx(1000 * 2000 * 28 / 1.0 / 1e12)
    assert b.unfused_cd("lorenz", 1, 1, 1.0, 1.0) == {}


def test_encoding_frequencies_match_the_oracle(cbf):
    """The network's Fourier-encoding table, built at compile time for the
    kernels' constant memory, equals the oracle's table bit for bit (host call,
    no GPU)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    import mlp_oracle as M
    out = np.zeros(124, np.float32)
    assert cbf.lib().cbf_mlp_encoding_frequencies(out.ctypes.data_as(C.POINTER(C.c_float)), 124) == 0
    assert np.array_equal(out.reshape(62, 2), M.fourier_freqs())
    assert cbf.lib().cbf_mlp_encoding_frequencies(out.ctypes.data_as(C.POINTER(C.c_float)), 10) != 0
