"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
to check (never to produce) the CUDA path's results.  ``liboracle.so`` is the
plain-C restatement in oracle.c; ``_ref/libcbf_ref.so`` (optional) is the
reference's own host-callable code compiled from its sources by ``make ref``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libcbf_ref.so"

SYSTEMS = {"memristive5": 0, "rossler": 1, "lorenz": 2, "chen": 3}


class OrcJob(C.Structure):
    _fields_ = [
        ("ranges", C.c_double * 4),
        ("ic", C.c_double * 8),
        ("values", C.c_double * 16),
        ("h", C.c_double),
        ("tMax", C.c_double),
        ("transientTime", C.c_double),
        ("maxValue", C.c_double),
        ("NT", C.c_double),
        ("lleEps", C.c_double),
        ("kdeI1", C.c_double),
        ("kdeI2", C.c_double),
        ("kdeH", C.c_double),
        ("dbscanEps", C.c_double),
        ("seedChunk", C.c_int64),
        ("system", C.c_int32),
        ("sweepIC", C.c_int32),
        ("dims", C.c_int32),
        ("nPts", C.c_int32),
        ("nIC", C.c_int32),
        ("nV", C.c_int32),
        ("idxMut", C.c_int32 * 2),
        ("writableVar", C.c_int32),
        ("preScaller", C.c_int32),
        ("maxAmountOfPeaks", C.c_int32),
        ("kdeSampling", C.c_int32),
        ("regimeTime", C.c_double),
        ("regimeMinAmp", C.c_double),
        ("regimeChaosLle", C.c_double),
        ("ostrovskyThreshold", C.c_double),
        ("exactGrid", C.c_int32),
    ]


def make_job(*, system, nPts, ranges, idxMut, ic, values, h, tMax=0.0, transientTime=0.0,
             maxValue=0.0, writableVar=0, preScaller=1, sweepIC=False, maxAmountOfPeaks=0,
             kdeSampling=0, kdeI1=0.0, kdeI2=0.0, kdeH=0.0, dbscanEps=0.0, NT=0.0,
             lleEps=0.0, seedChunk=0, regimeTime=0.0, regimeMinAmp=0.0,
             regimeChaosLle=0.0, ostrovskyThreshold=0.0, flags=0, exactGrid=False) -> OrcJob:
    """flags: the library's job flags; bit 0 (exact grid) selects integer grid
    cells, the other bits do not concern the per-point code."""
    j = OrcJob()
    dims = len(idxMut)
    j.system = SYSTEMS[system] if isinstance(system, str) else int(system)
    j.sweepIC = 1 if sweepIC else 0
    j.dims = dims
    j.nPts = nPts
    for i, r in enumerate(ranges[: 2 * dims]):
        j.ranges[i] = r
    for i, m in enumerate(idxMut):
        j.idxMut[i] = m
    j.nIC = len(ic)
    for i, v in enumerate(ic):
        j.ic[i] = v
    j.nV = len(values)
    for i, v in enumerate(values):
        j.values[i] = v
    j.h, j.tMax, j.transientTime, j.maxValue = h, tMax, transientTime, maxValue
    j.writableVar, j.preScaller = writableVar, preScaller
    j.maxAmountOfPeaks, j.kdeSampling = maxAmountOfPeaks, kdeSampling
    j.kdeI1, j.kdeI2, j.kdeH = kdeI1, kdeI2, kdeH
    j.dbscanEps = dbscanEps
    j.NT, j.lleEps, j.seedChunk = NT, lleEps, seedChunk
    j.regimeTime = regimeTime
    j.regimeMinAmp = regimeMinAmp
    j.regimeChaosLle = regimeChaosLle
    j.ostrovskyThreshold = ostrovskyThreshold
    j.exactGrid = 1 if (exactGrid or (int(flags) & 1)) else 0
    return j


def reference_dir() -> Path | None:
    """The reference checkout the Makefile's `ref` target compiles from (the
    Makefile is the one place that locates it; CBF_REFERENCE_DIR overrides it),
    or None when it is not present on this machine."""
    try:
        out = subprocess.run(["make", "-s", "-C", str(HERE), "ref-dir"], check=True,
                             capture_output=True, text=True).stdout.strip()
    except (OSError, subprocess.CalledProcessError):
        return None
    p = Path(out) if out else None
    return p if p is not None and (p / "Library" / "cudaLibrary.cu").exists() else None


def build(with_ref: bool | None = None) -> None:
    """Compile liboracle.so (and the reference shim when its sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if with_ref is None:
        with_ref = reference_dir() is not None
    if with_ref:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref"], check=True)


_lib = None
_ref = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build(with_ref=False)
        L = C.CDLL(str(LIB_PATH))
        L.orc_get_value_by_idx.restype = C.c_double
        L.orc_get_value_by_idx.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        L.orc_system_dim.restype = C.c_int
        L.orc_system_dim.argtypes = [C.c_int]
        L.orc_model_step.restype = None
        L.orc_model_step.argtypes = [C.c_int, _dp, _dp, C.c_double]
        L.orc_loop.restype = C.c_int
        L.orc_loop.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int,
                               C.c_double, C.c_void_p, C.c_int64, C.c_int]
        L.orc_peak_finder.restype = C.c_int
        L.orc_peak_finder.argtypes = [_dp, C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_double]
        L.orc_kde.restype = C.c_int
        L.orc_kde.argtypes = [_dp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                              C.c_double]
        L.orc_kde_k1.restype = C.c_int
        L.orc_kde_k1.argtypes = [_dp, C.c_int64, C.c_int, C.c_int, C.c_double, C.c_double,
                                 C.c_double]
        L.orc_distance.restype = C.c_double
        L.orc_distance.argtypes = [C.c_double] * 4
        L.orc_dbscan.restype = C.c_int
        L.orc_dbscan.argtypes = [_dp, _dp, _dp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double]
        L.orc_diverged.restype = C.c_int
        L.orc_diverged.argtypes = [C.c_double, C.c_double]
        L.orc_record_len.restype = C.c_int
        L.orc_record_len.argtypes = [C.POINTER(OrcJob)]
        L.orc_skip_len.restype = C.c_int
        L.orc_skip_len.argtypes = [C.POINTER(OrcJob)]
        L.orc_trajectory_point.restype = C.c_int
        L.orc_trajectory_point.argtypes = [C.POINTER(OrcJob), C.c_int64, _dp]
        L.orc_lle_point.restype = C.c_double
        L.orc_lle_point.argtypes = [C.POINTER(OrcJob), C.c_int64]
        L.orc_map_peaks.restype = C.c_int
        L.orc_map_peaks.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, C.c_void_p,
                                    C.c_void_p, _ip, C.c_int64, C.c_int]
        L.orc_map_kde.restype = C.c_int
        L.orc_map_kde.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, _ip, C.c_int]
        L.orc_map_dbscan.restype = C.c_int
        L.orc_map_dbscan.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, _ip, C.c_int]
        L.orc_map_lle.restype = C.c_int
        L.orc_map_lle.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, _dp, C.c_int]
        L.orc_lle_point_seeded.restype = C.c_double
        L.orc_lle_point_seeded.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_void_p]
        L.orc_lle_seed.restype = None
        L.orc_lle_seed.argtypes = [C.POINTER(OrcJob), C.c_int64, _dp]
        L.orc_map_lle_seeded.restype = C.c_int
        L.orc_map_lle_seeded.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, _dp, _dp, C.c_int]
        L.orc_modeling_one_system.restype = C.c_int
        L.orc_modeling_one_system.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, C.c_int,
                                              C.c_int, _dp, C.c_int, _dp, C.c_int64]
        L.orc_map_ostrovsky.restype = C.c_int
        L.orc_map_ostrovsky.argtypes = [C.POINTER(OrcJob), C.c_int64, C.c_int64, _dp, C.c_int]
        L.orc_map_ls_list.restype = C.c_int
        L.orc_map_ls_list.argtypes = [C.POINTER(OrcJob), _lp, C.c_int64, C.c_void_p, _dp, C.c_int]
        L.orc_ls_seed.restype = None
        L.orc_ls_seed.argtypes = [C.POINTER(OrcJob), C.c_int64, _dp]
        L.orc_gram_schmidt.restype = None
        L.orc_gram_schmidt.argtypes = [_dp, _dp, C.c_int, C.c_void_p]
        L.orc_projection.restype = None
        L.orc_projection.argtypes = [_dp, _dp, _dp, C.c_int]
        L.orc_map_lle_regime_list.restype = C.c_int
        L.orc_map_lle_regime_list.argtypes = [C.POINTER(OrcJob), _lp, C.c_int64, C.c_void_p, _dp,
                                              _ip, C.c_int]
        L.orc_map_lle_list.restype = C.c_int
        L.orc_map_lle_list.argtypes = [C.POINTER(OrcJob), _lp, C.c_int64, _dp, C.c_int]
        L.orc_map_lle_list_seeded.restype = C.c_int
        L.orc_map_lle_list_seeded.argtypes = [C.POINTER(OrcJob), _lp, C.c_int64, C.c_void_p, _dp, C.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return REF_PATH.exists()


def ref():
    """The reference's own host-compiled functions (None when not built)."""
    global _ref
    if _ref is None and REF_PATH.exists():
        R = C.CDLL(str(REF_PATH))
        R.ref_getValueByIdx.restype = C.c_double
        R.ref_getValueByIdx.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        R.ref_calculateDiscreteModel.restype = None
        R.ref_calculateDiscreteModel.argtypes = [_dp, _dp, C.c_double]
        R.ref_loopCalculateDiscreteModel.restype = C.c_int
        R.ref_loopCalculateDiscreteModel.argtypes = [_dp, _dp, C.c_double, C.c_int, C.c_int,
                                                     C.c_int, C.c_double, C.c_void_p, C.c_int,
                                                     C.c_int]
        R.ref_peakFinder.restype = C.c_int
        R.ref_peakFinder.argtypes = [_dp, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double]
        R.ref_kde.restype = C.c_int
        R.ref_kde.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                              C.c_double]
        R.ref_distance.restype = C.c_double
        R.ref_distance.argtypes = [C.c_double] * 4
        R.ref_dbscan.restype = C.c_int
        R.ref_dbscan.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double]
        if hasattr(R, "ref_gramSchmidtProcess"):
            R.ref_gramSchmidtProcess.restype = None
            R.ref_gramSchmidtProcess.argtypes = [_dp, _dp, C.c_int, C.c_void_p]
            R.ref_projectionOperator.restype = None
            R.ref_projectionOperator.argtypes = [_dp, _dp, _dp, C.c_int]
        _ref = R
    return _ref


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------
# numpy-level helpers

def peak_finder(data, h=0.01, want_times=True):
    d = np.ascontiguousarray(data, dtype=np.float64).copy()
    peaks = np.zeros(len(d), np.float64)
    times = np.zeros(len(d), np.float64) if want_times else None
    n = lib().orc_peak_finder(d, 0, len(d), _ptr(peaks), _ptr(times), h)
    return peaks[:n].copy(), (times[:n].copy() if want_times else None)


def kde(peaks, maxAmountOfPeaks, kdeSampling, i1, i2, smooth):
    p = np.ascontiguousarray(peaks, dtype=np.float64)
    if len(p) == 0:
        p = np.zeros(1)
        return lib().orc_kde(p, 0, 0, maxAmountOfPeaks, kdeSampling, i1, i2, smooth)
    return lib().orc_kde(p, 0, len(peaks), maxAmountOfPeaks, kdeSampling, i1, i2, smooth)


def kde_fixed(peaks, maxAmountOfPeaks, k1, i1, i2, smooth):
    """kde() with a fixed total sample count k1 (the library's fixed-sample mode)."""
    p = np.ascontiguousarray(peaks, dtype=np.float64)
    n = len(p)
    if n == 0:
        return 0
    if n in (1, 2):
        return 1
    if n > maxAmountOfPeaks:
        return maxAmountOfPeaks
    return lib().orc_kde_k1(p, 0, n, k1, i1, i2, smooth)


def dbscan(peaks, intervals, maxAmountOfPeaks, eps, size_of_helpful=None):
    p = np.ascontiguousarray(peaks, dtype=np.float64)
    t = np.ascontiguousarray(intervals, dtype=np.float64)
    n = len(p)
    size = size_of_helpful if size_of_helpful is not None else max(2 * n + 2, 1)
    helpful = np.zeros(size, np.float64)
    if n == 0:
        p = np.zeros(1)
        t = np.zeros(1)
    return lib().orc_dbscan(p, t, helpful, 0, n, size, maxAmountOfPeaks, eps)


def trajectory(job: OrcJob, g: int):
    rec = lib().orc_record_len(C.byref(job))
    data = np.zeros(max(rec, 1), np.float64)
    div = lib().orc_trajectory_point(C.byref(job), g, data)
    return data[:rec], bool(div)


def map_peaks(job: OrcJob, first: int, count: int, cap: int, threads: int = 0):
    peaks = np.zeros((count, cap), np.float64)
    times = np.zeros((count, cap), np.float64)
    counts = np.zeros(count, np.int32)
    rc = lib().orc_map_peaks(C.byref(job), first, count, _ptr(peaks), _ptr(times), counts, cap,
                             threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_peaks failed: {rc}")
    return peaks, times, counts


def map_kde(job: OrcJob, first: int, count: int, threads: int = 0):
    out = np.zeros(count, np.int32)
    rc = lib().orc_map_kde(C.byref(job), first, count, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_kde failed: {rc}")
    return out


def map_dbscan(job: OrcJob, first: int, count: int, threads: int = 0):
    out = np.zeros(count, np.int32)
    rc = lib().orc_map_dbscan(C.byref(job), first, count, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_dbscan failed: {rc}")
    return out


def map_lle(job: OrcJob, first: int, count: int, threads: int = 0):
    out = np.zeros(count, np.float64)
    rc = lib().orc_map_lle(C.byref(job), first, count, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_lle failed: {rc}")
    return out


def map_lle_seeded(job: OrcJob, first: int, count: int, z, threads: int = 0):
    """LLE map started from the given perturbations z[count, nIC]."""
    z = np.ascontiguousarray(z, dtype=np.float64)
    out = np.zeros(count, np.float64)
    rc = lib().orc_map_lle_seeded(C.byref(job), first, count, z, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_lle_seeded failed: {rc}")
    return out


def lle_seeds(job: OrcJob, first: int, count: int):
    out = np.zeros((count, job.nIC), np.float64)
    row = np.zeros(job.nIC, np.float64)
    for k in range(count):
        lib().orc_lle_seed(C.byref(job), first + k, row)
        out[k] = row
    return out


def modeling_one_system(system, tMax, h, hSpecial, ic, writableVar, values) -> np.ndarray:
    """The step-offset trajectory of modelingOneSystemDenis ((int)(tMax/h) samples)."""
    sysid = SYSTEMS[system] if isinstance(system, str) else int(system)
    ic = np.ascontiguousarray(ic, np.float64)
    values = np.ascontiguousarray(values, np.float64)
    n = int(tMax / h)
    out = np.zeros(max(n, 0), np.float64)
    rc = lib().orc_modeling_one_system(sysid, tMax, h, hSpecial, ic, len(ic), writableVar, values,
                                       len(values), out, n)
    if rc != 0:
        raise RuntimeError(f"orc_modeling_one_system failed: {rc}")
    return out


def map_ostrovsky(job: OrcJob, first: int, count: int, threads: int = 0) -> np.ndarray:
    """Ostrovsky periodicity values of points [first, first + count)."""
    out = np.zeros(count, np.float64)
    rc = lib().orc_map_ostrovsky(C.byref(job), first, count, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_ostrovsky failed: {rc}")
    return out


def map_ls(job: OrcJob, idx, z=None, threads: int = 0):
    """Lyapunov spectra (nIC exponents) at grid indices idx; z (optional, per point
    nIC x nIC seed rows) replaces the oracle's own seeds."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    n = job.nIC
    out = np.zeros((len(idx), n), np.float64)
    zp = None
    if z is not None:
        z = np.ascontiguousarray(z, dtype=np.float64)
        zp = z.ctypes.data_as(C.c_void_p)
    rc = lib().orc_map_ls_list(C.byref(job), idx, len(idx), zp, out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_ls_list failed: {rc}")
    return out


def ls_seeds(job: OrcJob, idx):
    """The oracle's seed rows (glibc sinf) for grid indices idx: (len, nIC, nIC)."""
    n = job.nIC
    out = np.zeros((len(idx), n, n), np.float64)
    for k, g in enumerate(idx):
        row = np.zeros(n * n, np.float64)
        lib().orc_ls_seed(C.byref(job), int(g), row)
        out[k] = row.reshape(n, n)
    return out


def gram_schmidt(a, with_den: bool = True):
    """orc_gram_schmidt on an (n, n) array: (b, den)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    b = np.zeros_like(a)
    den = np.zeros(n, np.float64)
    lib().orc_gram_schmidt(a, b, n, den.ctypes.data_as(C.c_void_p) if with_den else None)
    return b, den


def map_lle_regime(job: OrcJob, idx, z=None, threads: int = 0):
    """LLE and regime class at grid indices idx (optionally from given seeds z)."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    lle = np.zeros(len(idx), np.float64)
    cls = np.zeros(len(idx), np.int32)
    zp = None
    if z is not None:
        z = np.ascontiguousarray(z, dtype=np.float64)
        zp = z.ctypes.data_as(C.c_void_p)
    rc = lib().orc_map_lle_regime_list(C.byref(job), idx, len(idx), zp, lle, cls, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_lle_regime_list failed: {rc}")
    return lle, cls


def map_lle_list(job: OrcJob, idx, threads: int = 0, z=None):
    """LLE at grid indices idx; z (optional, nIC per point) replaces the seeds."""
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.zeros(len(idx), np.float64)
    if z is not None:
        z = np.ascontiguousarray(z, dtype=np.float64)
        rc = lib().orc_map_lle_list_seeded(C.byref(job), idx, len(idx), z.ctypes.data_as(C.c_void_p),
                                           out, threads)
    else:
        rc = lib().orc_map_lle_list(C.byref(job), idx, len(idx), out, threads)
    if rc != 0:
        raise RuntimeError(f"orc_map_lle_list failed: {rc}")
    return out


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
