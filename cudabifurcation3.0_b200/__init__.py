"""B200 bifurcation engine -- Python host mirror of the C-ABI in include/cbf.h.

The product is ``libcbf.so`` (CUDA kernels for sm_100a + the C-ABI + the C++
drop-in facade with the reference's hostLibrary signatures).  This module only
binds it with ctypes for Python callers, tests and the benchmark: every compute
call runs on the GPU through that library.  There is no CPU fallback; if the
library or a GPU is missing the calls raise.

The function names and argument lists mirror the reference's host entry points
(Library/hostLibrary.cuh): ``bifurcation1D``, ``bifurcation1DIC``,
``bifurcation2DKDE``, ``bifurcation2DKDEIC``, ``bifurcation2DDBSCAN``,
``bifurcation2DDBSCANIC``, ``LLE1D``, ``LLE1DIC``, ``LLE2D``, ``LLE2DIC``, with a
``system=`` keyword (the reference compiles one ODE per build) and the results
returned as numpy arrays instead of written to a CSV file.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libcbf.so"

SYS_MEMRISTIVE5, SYS_ROSSLER, SYS_LORENZ, SYS_CHEN = 0, 1, 2, 3
SYSTEMS = {"memristive5": 0, "rossler": 1, "lorenz": 2, "chen": 3}
TASK_PEAKS, TASK_KDE, TASK_DBSCAN, TASK_LLE, TASK_TRAJECTORY, TASK_LLE_REGIME, TASK_LS = 0, 1, 2, 3, 4, 5, 6
TASK_OSTROVSKY = 7
FLAG_EXACT_GRID, FLAG_KDE_FIXED = 1, 2
STATUS = {0: "ok", 1: "invalid argument", 2: "unknown system", 3: "CUDA error",
          4: "out of device memory", 5: "no CUDA device", 6: "I/O error",
          7: "device wait timed out", 8: "internal consistency check failed"}

# Every symbol include/cbf.h declares (checked by the CPU test suite).
EXPORTS = [
    "cbf_abi_version", "cbf_status_string", "cbf_last_error", "cbf_kernel_launches",
    "cbf_device_count", "cbf_set_device", "cbf_job_init", "cbf_record_length",
    "cbf_peak_capacity", "cbf_job_points", "cbf_validate", "cbf_run",
    "cbf_bifurcation1d", "cbf_bifurcation1d_ic", "cbf_bifurcation2d_kde",
    "cbf_bifurcation2d_kde_ic", "cbf_bifurcation2d_dbscan", "cbf_bifurcation2d_dbscan_ic",
    "cbf_lle1d", "cbf_lle1d_ic", "cbf_lle2d", "cbf_lle2d_ic", "cbf_run_host",
    "cbf_grid_coordinates", "cbf_probe_fp64_peak", "cbf_probe_fp64_step", "cbf_probe_expf_zero",
    "cbf_divergence_threshold", "cbf_lle_seeds", "cbf_autotune", "cbf_set_lle_variant",
    "cbf_get_lle_variant", "cbf_batch_create", "cbf_batch_destroy", "cbf_batch_points",
    "cbf_batch_blocks_per_sm", "cbf_batch_run", "cbf_batch_capture", "cbf_batch_launch",
    "cbf_batch_run_sequential", "cbf_batch_check", "cbf_batch_autotune", "cbf_bifurcation2d_dbscan_noalloc",
    "cbf_csv_write_map", "cbf_csv_write_peaks", "cbf_csv_write_pairs",
    "cbf_mlp_num_params", "cbf_mlp_create", "cbf_mlp_destroy", "cbf_mlp_get_params",
    "cbf_mlp_set_params", "cbf_mlp_set_encoding_scale", "cbf_mlp_encoding_frequencies",
    "cbf_mlp_forward_backward", "cbf_mlp_train",
    "cbf_mlp_predict",
    "cbf_mlp_predict_grid", "cbf_mlp_grid_features",
    "cbf_surrogate_config_init", "cbf_lle_map_surrogate", "cbf_surrogate_release", "cbf_ls1d", "cbf_ls2d",
    "cbf_regime_rules_init", "cbf_lle2d_surrogate", "cbf_facade_set_system", "cbf_facade_set_output_path",
    "cbf_facade_set_surrogate", "cbf_job_scaled_step",
    "cbf_csv_write_rows", "cbf_npy_write", "cbf_ostrovsky2d", "cbf_modeling_one_system",
]


class CbfError(RuntimeError):
    def __init__(self, status: int, detail: str):
        super().__init__(f"{STATUS.get(status, status)}: {detail}")
        self.status = status
        self.detail = detail


class Job(C.Structure):
    """Mirror of ``cbf_job`` (include/cbf.h)."""
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
        ("firstPoint", C.c_int64),
        ("nPoints", C.c_int64),
        ("task", C.c_int32),
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
        ("flags", C.c_uint32),
        ("peakCapacity", C.c_int32),
        ("regimeTime", C.c_double),
        ("pointIndex", C.c_void_p),
        ("regimeMinAmp", C.c_double),
        ("regimeChaosLle", C.c_double),
        ("ostrovskyThreshold", C.c_double),
    ]


class SurrogateConfig(C.Structure):
    """Mirror of ``cbf_surrogate_config`` (include/cbf.h)."""
    _fields_ = [
        ("coarseSide", C.c_int32),
        ("randomPoints", C.c_int32),
        ("batch", C.c_int32),
        ("trainSteps", C.c_int32),
        ("lr", C.c_float),
        ("wLle", C.c_float),
        ("confThreshold", C.c_float),
        ("auditFraction", C.c_float),
        ("boundaryRadius", C.c_int32),
        ("refine", C.c_int32),
        ("seed", C.c_uint64),
        ("expandRadius", C.c_int32),
        ("maxWaves", C.c_int32),
        ("predictor", C.c_int32),
        ("auditFill", C.c_int32),
        ("idleRadius", C.c_int32),
    ]


class SurrogateReport(C.Structure):
    """Mirror of ``cbf_surrogate_report`` (include/cbf.h)."""
    _fields_ = [
        ("points", C.c_int64),
        ("labelled", C.c_int64),
        ("refined", C.c_int64),
        ("boundary", C.c_int64),
        ("lowConfidence", C.c_int64),
        ("audit", C.c_int64),
        ("auditOnly", C.c_int64),
        ("auditOnlyAgree", C.c_int64),
        ("refinedChanged", C.c_int64),
        ("auditOnlyLleMeanAbsErr", C.c_double),
        ("auditOnlyLleMaxAbsErr", C.c_double),
        ("lleMean", C.c_double),
        ("lleStd", C.c_double),
        ("finalLoss", C.c_float),
        ("msLabel", C.c_double),
        ("msTrain", C.c_double),
        ("msPredict", C.c_double),
        ("msMask", C.c_double),
        ("msRefine", C.c_double),
        ("msTotal", C.c_double),
        ("expanded", C.c_int64),
        ("waves", C.c_int32),
        ("refineTiles", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def lib():
    """Load libcbf.so (build it first: ``python cudabifurcation3.0_b200/build.py``)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build the CUDA library first")
        L = C.CDLL(str(LIB_PATH))
        L.cbf_abi_version.restype = C.c_int32
        L.cbf_status_string.restype = C.c_char_p
        L.cbf_status_string.argtypes = [C.c_int32]
        L.cbf_last_error.restype = C.c_char_p
        L.cbf_kernel_launches.restype = C.c_uint64
        L.cbf_device_count.argtypes = [_ip]
        L.cbf_set_device.argtypes = [C.c_int32]
        L.cbf_job_init.restype = None
        L.cbf_job_init.argtypes = [C.POINTER(Job)]
        for f in ("cbf_record_length", "cbf_peak_capacity"):
            getattr(L, f).restype = C.c_int32
            getattr(L, f).argtypes = [C.POINTER(Job)]
        L.cbf_job_points.restype = C.c_int64
        L.cbf_job_points.argtypes = [C.POINTER(Job)]
        L.cbf_validate.argtypes = [C.POINTER(Job)]
        L.cbf_run.argtypes = [C.POINTER(Job), C.c_void_p, C.c_void_p, C.c_void_p]
        L.cbf_run_host.argtypes = [C.POINTER(Job), C.c_void_p, C.c_void_p]
        L.cbf_grid_coordinates.argtypes = [C.POINTER(Job), _dp]
        L.cbf_autotune.argtypes = [C.POINTER(Job), _ip, _dp]
        L.cbf_autotune.restype = C.c_int32
        L.cbf_set_lle_variant.argtypes = [C.c_int32, C.c_int32]
        L.cbf_set_lle_variant.restype = C.c_int32
        L.cbf_get_lle_variant.argtypes = [C.c_int32]
        L.cbf_get_lle_variant.restype = C.c_int32
        L.cbf_batch_create.argtypes = [C.POINTER(Job), C.c_int32, C.POINTER(C.c_void_p),
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        L.cbf_batch_create.restype = C.c_int32
        L.cbf_batch_destroy.argtypes = [C.c_void_p]
        L.cbf_batch_destroy.restype = None
        L.cbf_batch_points.argtypes = [C.c_void_p]
        L.cbf_batch_points.restype = C.c_int64
        L.cbf_batch_blocks_per_sm.argtypes = [C.c_void_p]
        L.cbf_batch_blocks_per_sm.restype = C.c_int32
        for f in ("cbf_batch_run", "cbf_batch_capture", "cbf_batch_launch", "cbf_batch_run_sequential"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_void_p]
            getattr(L, f).restype = C.c_int32
        L.cbf_batch_check.argtypes = [C.c_void_p]
        L.cbf_batch_check.restype = C.c_int32
        L.cbf_batch_autotune.argtypes = [C.c_void_p, C.c_void_p, _ip, _dp]
        L.cbf_batch_autotune.restype = C.c_int32
        L.cbf_lle_seeds.argtypes = [C.POINTER(Job), _dp]
        L.cbf_lle_seeds.restype = C.c_int32
        L.cbf_probe_fp64_peak.argtypes = [C.c_double, _dp]
        L.cbf_probe_fp64_step.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_double, _dp]
        L.cbf_probe_expf_zero.argtypes = [C.c_float, C.POINTER(C.c_uint64)]
        L.cbf_divergence_threshold.argtypes = [C.c_double, _ip, _dp]
        bif1d = [C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_int32, _dp, _dp, _ip,
                 C.c_int32, C.c_double, C.c_double, _dp, C.c_int32, C.c_int32, _dp, C.c_int32, _ip]
        L.cbf_bifurcation1d.argtypes = bif1d
        L.cbf_bifurcation1d_ic.argtypes = bif1d
        kde = [C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_int32, _dp, _dp, _ip, C.c_int32,
               C.c_double, C.c_int32, C.c_double, _dp, C.c_int32, C.c_int32, C.c_int32, C.c_double,
               C.c_double, C.c_double, _ip]
        L.cbf_bifurcation2d_kde.argtypes = kde
        L.cbf_bifurcation2d_kde_ic.argtypes = kde
        db = [C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_int32, _dp, _dp, _ip, C.c_int32,
              C.c_double, C.c_int32, C.c_double, _dp, C.c_int32, C.c_int32, C.c_double, _ip]
        L.cbf_bifurcation2d_dbscan.argtypes = db
        L.cbf_bifurcation2d_dbscan_ic.argtypes = db
        L.cbf_bifurcation2d_dbscan_noalloc.argtypes = db[:-1] + [C.c_void_p, C.c_void_p]
        L.cbf_bifurcation2d_dbscan_noalloc.restype = C.c_int32
        lle = [C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_double, _dp, C.c_int32,
               _dp, _ip, C.c_int32, C.c_double, C.c_double, _dp, C.c_int32, C.c_int64, _dp]
        for f in ("cbf_lle1d", "cbf_lle1d_ic", "cbf_lle2d", "cbf_lle2d_ic", "cbf_ls1d", "cbf_ls2d"):
            getattr(L, f).argtypes = lle
        for f in ("cbf_device_count", "cbf_set_device", "cbf_validate", "cbf_run", "cbf_run_host",
                  "cbf_grid_coordinates", "cbf_probe_fp64_peak", "cbf_probe_fp64_step", "cbf_probe_expf_zero",
                  "cbf_divergence_threshold", "cbf_bifurcation1d", "cbf_bifurcation1d_ic",
                  "cbf_bifurcation2d_kde", "cbf_bifurcation2d_kde_ic", "cbf_bifurcation2d_dbscan",
                  "cbf_bifurcation2d_dbscan_ic", "cbf_lle1d", "cbf_lle1d_ic", "cbf_lle2d",
                  "cbf_lle2d_ic", "cbf_ls1d", "cbf_ls2d"):
            getattr(L, f).restype = C.c_int32
        L.cbf_csv_write_map.restype = C.c_int32
        L.cbf_csv_write_map.argtypes = [C.c_char_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32,
                                        C.c_void_p, C.c_int32]
        L.cbf_csv_write_peaks.restype = C.c_int32
        L.cbf_csv_write_peaks.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_int64, C.c_int64,
                                          C.c_void_p, C.c_int32, C.c_void_p, C.c_int32]
        L.cbf_csv_write_rows.restype = C.c_int32
        L.cbf_csv_write_rows.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                         C.c_int32, C.c_int32]
        L.cbf_csv_write_pairs.restype = C.c_int32
        L.cbf_csv_write_pairs.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64,
                                          C.c_int32]
        _fp = C.POINTER(C.c_float)
        L.cbf_mlp_num_params.restype = C.c_int64
        L.cbf_mlp_create.argtypes = [C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]
        L.cbf_mlp_create.restype = C.c_int32
        L.cbf_mlp_destroy.argtypes = [C.c_void_p]
        L.cbf_mlp_destroy.restype = None
        for f in ("cbf_mlp_get_params", "cbf_mlp_set_params"):
            getattr(L, f).argtypes = [C.c_void_p, _fp, C.c_int64]
            getattr(L, f).restype = C.c_int32
        L.cbf_mlp_set_encoding_scale.argtypes = [C.c_void_p, C.c_float]
        L.cbf_mlp_encoding_frequencies.argtypes = [_fp, C.c_int32]
        L.cbf_mlp_encoding_frequencies.restype = C.c_int32
        L.cbf_mlp_set_encoding_scale.restype = C.c_int32
        L.cbf_mlp_forward_backward.argtypes = [C.c_void_p, _fp, _fp, _ip, C.c_int32, C.c_float, _fp,
                                               _fp, _fp]
        L.cbf_mlp_forward_backward.restype = C.c_int32
        L.cbf_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                    C.c_int32, C.c_float, C.c_int32, C.c_float, _fp, C.c_void_p]
        L.cbf_mlp_train.restype = C.c_int32
        L.cbf_mlp_predict.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.cbf_mlp_predict.restype = C.c_int32
        L.cbf_mlp_predict_grid.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]
        L.cbf_mlp_predict_grid.restype = C.c_int32
        L.cbf_mlp_grid_features.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.cbf_mlp_grid_features.restype = C.c_int32
        L.cbf_surrogate_config_init.argtypes = [C.POINTER(SurrogateConfig)]
        L.cbf_surrogate_config_init.restype = None
        L.cbf_lle_map_surrogate.argtypes = [C.POINTER(Job), C.POINTER(SurrogateConfig), C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.POINTER(SurrogateReport), C.c_void_p]
        L.cbf_lle_map_surrogate.restype = C.c_int32
        L.cbf_facade_set_system.argtypes = [C.c_int32]
        L.cbf_facade_set_output_path.argtypes = [C.c_char_p]
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != 0:
        raise CbfError(status, lib().cbf_last_error().decode(errors="replace"))


def _sys(system) -> int:
    return SYSTEMS[system] if isinstance(system, str) else int(system)


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def make_job(*, task, system, nPts, ranges, idxMut, ic, values, h, tMax=0.0, transientTime=0.0,
             maxValue=0.0, writableVar=0, preScaller=1, sweepIC=False, maxAmountOfPeaks=0,
             kdeSampling=0, kdeI1=0.0, kdeI2=0.0, kdeH=0.0, dbscanEps=0.0, NT=0.0, lleEps=0.0,
             seedChunk=0, firstPoint=0, nPoints=0, flags=0, peakCapacity=0, regimeTime=0.0,
             pointIndex=0, regimeMinAmp=0.0, regimeChaosLle=0.0, ostrovskyThreshold=0.0) -> Job:
    j = Job()
    lib().cbf_job_init(C.byref(j))
    dims = len(idxMut)
    j.task, j.system, j.sweepIC, j.dims, j.nPts = task, _sys(system), int(bool(sweepIC)), dims, nPts
    for i, r in enumerate(list(ranges)[: 2 * dims]):
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
    j.kdeI1, j.kdeI2, j.kdeH, j.dbscanEps = kdeI1, kdeI2, kdeH, dbscanEps
    j.NT, j.lleEps, j.seedChunk = NT, lleEps, seedChunk
    j.firstPoint, j.nPoints, j.flags, j.peakCapacity = firstPoint, nPoints, flags, peakCapacity
    j.regimeTime = regimeTime
    j.pointIndex = pointIndex or None
    j.regimeMinAmp = regimeMinAmp
    j.regimeChaosLle = regimeChaosLle
    j.ostrovskyThreshold = ostrovskyThreshold
    return j


def run_host(job: Job):
    """Run a job through the C-ABI with host buffers; returns (out, aux)."""
    L = lib()
    check(L.cbf_validate(C.byref(job)))
    n = L.cbf_job_points(C.byref(job))
    aux = None
    if job.task == TASK_LLE:
        out = np.zeros(n, np.float64)
    elif job.task == TASK_LLE_REGIME:
        out = np.zeros(n, np.float64)
        aux = np.zeros(n, np.int32)
    elif job.task == TASK_LS:
        out = np.zeros((n, job.nIC), np.float64)
    elif job.task == TASK_OSTROVSKY:
        out = np.zeros(n, np.float64)
    elif job.task in (TASK_KDE, TASK_DBSCAN):
        out = np.zeros(n, np.int32)
    else:
        if job.task == TASK_PEAKS:
            cap = job.peakCapacity or L.cbf_peak_capacity(C.byref(job))
        else:
            cap = job.peakCapacity or L.cbf_record_length(C.byref(job))
        job.peakCapacity = cap
        out = np.zeros((n, cap), np.float64)
        aux = np.zeros(n, np.int32)
    check(L.cbf_run_host(C.byref(job), out.ctypes.data_as(C.c_void_p),
                         None if aux is None else aux.ctypes.data_as(C.c_void_p)))
    return out, aux


def grid_features(job: Job, d_idx: int, n: int, d_x: int, stream: int = 0) -> None:
    """The surrogate network's input features of grid points d_idx[0..n) (FP32, 4 per point)."""
    check(lib().cbf_mlp_grid_features(C.byref(job), C.c_void_p(d_idx), n, C.c_void_p(d_x),
                                      C.c_void_p(stream or None)))


def run_device(job: Job, d_out: int, d_aux: int = 0, stream: int = 0) -> None:
    """Run a job on device buffers (raw pointers, e.g. torch tensor.data_ptr())."""
    check(lib().cbf_run(C.byref(job), C.c_void_p(d_out), C.c_void_p(d_aux or None),
                        C.c_void_p(stream or None)))


def kernel_launches() -> int:
    return int(lib().cbf_kernel_launches())


def grid_coordinates(job: Job) -> np.ndarray:
    n = lib().cbf_job_points(C.byref(job))
    out = np.zeros((n, 2), np.float64)
    check(lib().cbf_grid_coordinates(C.byref(job), out.ctypes.data_as(_dp)))
    return out


NUM_LLE_VARIANTS = 8


def autotune(job: Job):
    """Time every LLE kernel shape on a short copy of `job`; returns (chosen, ms[])."""
    chosen = C.c_int32(0)
    ms = np.zeros(NUM_LLE_VARIANTS, np.float64)
    check(lib().cbf_autotune(C.byref(job), C.byref(chosen), ms.ctypes.data_as(_dp)))
    return int(chosen.value), ms


class Batch:
    """Many jobs in one persistent launch (cbf_batch_*); outputs are device pointers."""

    def __init__(self, jobs, d_outs, d_auxs=None):
        n = len(jobs)
        arr = (Job * n)(*jobs)
        outs = (C.c_void_p * n)(*[C.c_void_p(p) for p in d_outs])
        auxs = None
        if d_auxs is not None:
            auxs = (C.c_void_p * n)(*[C.c_void_p(p or None) for p in d_auxs])
        h = C.c_void_p()
        check(lib().cbf_batch_create(arr, n, outs, auxs, C.byref(h)))
        self.handle = h

    def points(self) -> int:
        return int(lib().cbf_batch_points(self.handle))

    def blocks_per_sm(self) -> int:
        return int(lib().cbf_batch_blocks_per_sm(self.handle))

    def run(self, stream: int = 0):
        check(lib().cbf_batch_run(self.handle, C.c_void_p(stream or None)))

    def capture(self, stream: int = 0):
        check(lib().cbf_batch_capture(self.handle, C.c_void_p(stream or None)))

    def launch(self, stream: int = 0):
        check(lib().cbf_batch_launch(self.handle, C.c_void_p(stream or None)))

    def run_sequential(self, stream: int = 0):
        check(lib().cbf_batch_run_sequential(self.handle, C.c_void_p(stream or None)))

    def check(self):
        check(lib().cbf_batch_check(self.handle))

    def autotune(self, stream: int = 0):
        chosen = C.c_int32(0)
        ms = np.zeros(8, np.float64)
        check(lib().cbf_batch_autotune(self.handle, C.c_void_p(stream or None), C.byref(chosen),
                                       ms.ctypes.data_as(_dp)))
        return int(chosen.value), ms

    def close(self):
        if self.handle:
            lib().cbf_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """The surrogate network (cbf_mlp_*): 4 -> 256 x3 (SiLU) -> 17, BF16 tensor-core
    kernels with FP32 accumulation.  Device arrays are raw pointers."""

    def __init__(self, batch: int, seed: int = 0):
        h = C.c_void_p()
        check(lib().cbf_mlp_create(batch, seed, C.byref(h)))
        self.handle = h
        self.batch = batch

    @staticmethod
    def num_params() -> int:
        return int(lib().cbf_mlp_num_params())

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), np.float32)
        check(lib().cbf_mlp_get_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(lib().cbf_mlp_set_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def set_encoding_scale(self, scale: float) -> None:
        """Frequency scale of the input encoding (a power of two in [2^-8, 16])."""
        check(lib().cbf_mlp_set_encoding_scale(self.handle, scale))

    def forward_backward(self, x, y_lle, y_cls, w_lle: float = 1.0):
        """One pass on host rows; returns (loss, grads, out[n, 17])."""
        fp = C.POINTER(C.c_float)
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 4)
        yl = np.ascontiguousarray(y_lle, np.float32)
        yc = np.ascontiguousarray(y_cls, np.int32)
        n = x.shape[0]
        loss = C.c_float(0.0)
        g = np.zeros(self.num_params(), np.float32)
        out = np.zeros((n, 17), np.float32)
        check(lib().cbf_mlp_forward_backward(self.handle, x.ctypes.data_as(fp), yl.ctypes.data_as(fp),
                                             yc.ctypes.data_as(_ip), n, w_lle, C.byref(loss),
                                             g.ctypes.data_as(fp), out.ctypes.data_as(fp)))
        return float(loss.value), g, out

    def train(self, d_x: int, d_yl: int, d_yc: int, n: int, steps: int, lr: float,
              horizon: int = 0, w_lle: float = 1.0, stream: int = 0, losses: bool = False):
        buf = np.zeros(max(steps, 1), np.float32) if losses else None
        check(lib().cbf_mlp_train(self.handle, C.c_void_p(d_x), C.c_void_p(d_yl), C.c_void_p(d_yc), n,
                                  steps, lr, horizon, w_lle,
                                  None if buf is None else buf.ctypes.data_as(C.POINTER(C.c_float)),
                                  C.c_void_p(stream or None)))
        return buf[:steps] if buf is not None else None

    def predict(self, d_x: int, n: int, lle_mean: float, lle_std: float, d_lle: int = 0, d_cls: int = 0,
                d_conf: int = 0, stream: int = 0) -> None:
        check(lib().cbf_mlp_predict(self.handle, C.c_void_p(d_x), n, lle_mean, lle_std,
                                    C.c_void_p(d_lle or None), C.c_void_p(d_cls or None),
                                    C.c_void_p(d_conf or None), C.c_void_p(stream or None)))

    def predict_grid(self, job: "Job", lle_mean: float, lle_std: float, d_lle: int, d_cls: int, d_conf: int,
                     stream: int = 0) -> None:
        """Predictions for every point of the job's 2-D grid (tcgen05 kernel)."""
        check(lib().cbf_mlp_predict_grid(self.handle, C.byref(job), lle_mean, lle_std, C.c_void_p(d_lle),
                                         C.c_void_p(d_cls), C.c_void_p(d_conf), C.c_void_p(stream or None)))

    def close(self):
        if self.handle:
            lib().cbf_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def surrogate_config(**kw) -> SurrogateConfig:
    """Defaults of cbf_surrogate_config_init, overridden by keyword."""
    c = SurrogateConfig()
    lib().cbf_surrogate_config_init(C.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise AttributeError(k)
        setattr(c, k, v)
    return c


def lle_map_surrogate(job: Job, cfg: SurrogateConfig, d_lle: int, d_cls: int, d_src: int = 0,
                      stream: int = 0, d_conf: int = 0, d_pred: int = 0) -> SurrogateReport:
    """Surrogate-refined LLE + regime map into device buffers; returns the report."""
    rep = SurrogateReport()
    check(lib().cbf_lle_map_surrogate(C.byref(job), C.byref(cfg), C.c_void_p(d_lle), C.c_void_p(d_cls),
                                      C.c_void_p(d_src or None), C.c_void_p(d_conf or None),
                                      C.c_void_p(d_pred or None), C.byref(rep),
                                      C.c_void_p(stream or None)))
    return rep


class RegimeRules(C.Structure):
    """Mirror of ``cbf_regime_rules`` (include/cbf.h)."""
    _fields_ = [
        ("regimeTime", C.c_double),
        ("maxAmountOfPeaks", C.c_int32),
        ("dbscanEps", C.c_double),
        ("regimeMinAmp", C.c_double),
        ("regimeChaosLle", C.c_double),
        ("flags", C.c_uint32),
    ]


def regime_rules(**kw) -> RegimeRules:
    """Defaults of cbf_regime_rules_init, overridden by keyword."""
    r = RegimeRules()
    L = lib()
    L.cbf_regime_rules_init.argtypes = [C.POINTER(RegimeRules)]
    L.cbf_regime_rules_init.restype = None
    L.cbf_regime_rules_init(C.byref(r))
    for k, v in kw.items():
        if not hasattr(r, k):
            raise AttributeError(k)
        setattr(r, k, v)
    return r


def LLE2D_surrogate(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
                    indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
                    system="memristive5", seedChunk=None, rules=None, config=None, out_lle=None,
                    out_cls=None):
    """LLE2D's arguments, surrogate-refined (cbf_lle2d_surrogate): returns (lle[nPts, nPts],
    class[nPts, nPts], report).  seedChunk defaults to LLE2D's min(points, 200000);
    out_lle / out_cls (optional, float64 / int32 with nPts^2 elements) receive the maps."""
    ic, icp = _d(initialConditions)
    r, rp = _d(ranges)
    ix, ixp = _i(indicesOfMutVars)
    v, vp = _d(values)
    n = nPts * nPts
    lle = out_lle if out_lle is not None else np.empty(n, np.float64)
    cls = out_cls if out_cls is not None else np.empty(n, np.int32)
    assert lle.dtype == np.float64 and lle.size == n and lle.flags.c_contiguous
    assert cls.dtype == np.int32 and cls.size == n and cls.flags.c_contiguous
    chunk = min(n, 200000) if seedChunk is None else seedChunk
    rep = SurrogateReport()
    L = lib()
    L.cbf_lle2d_surrogate.restype = C.c_int32
    L.cbf_lle2d_surrogate.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_double,
                                      _dp, C.c_int32, _dp, _ip, C.c_int32, C.c_double, C.c_double, _dp,
                                      C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    check(L.cbf_lle2d_surrogate(_sys(system), tMax, NT, nPts, h, eps, icp, amountOfInitialConditions, rp,
                                ixp, writableVar, maxValue, transientTime, vp, amountOfValues, chunk,
                                C.byref(rules) if rules is not None else None,
                                C.byref(config) if config is not None else None,
                                lle.ctypes.data, cls.ctypes.data, C.byref(rep)))
    return lle.reshape(nPts, nPts), cls.reshape(nPts, nPts), rep


def set_lle_variant(system, variant: int) -> None:
    check(lib().cbf_set_lle_variant(_sys(system), variant))


def lle_seeds(job: Job) -> np.ndarray:
    """Device-computed perturbation vectors: LLE jobs (points, nIC); LS jobs the
    seed rows (points, nIC, nIC)."""
    n = lib().cbf_job_points(C.byref(job))
    shape = (n, job.nIC, job.nIC) if job.task == TASK_LS else (n, job.nIC)
    out = np.zeros(shape, np.float64)
    check(lib().cbf_lle_seeds(C.byref(job), out.ctypes.data_as(_dp)))
    return out


def probe_fp64_peak(ms: float = 200.0) -> float:
    t = C.c_double(0.0)
    check(lib().cbf_probe_fp64_peak(ms, C.byref(t)))
    return t.value


def probe_fp64_step(chains: int = 2, tracking: bool = True, blocks_per_sm: int = 6, ms: float = 200.0) -> float:
    """FP64 lane instructions per second of the map kernels' step stream alone."""
    r = C.c_double(0.0)
    check(lib().cbf_probe_fp64_step(chains, 1 if tracking else 0, blocks_per_sm, ms, C.byref(r)))
    return r.value


def probe_expf_zero(threshold: float) -> int:
    c = C.c_uint64(0)
    check(lib().cbf_probe_expf_zero(threshold, C.byref(c)))
    return int(c.value)


def divergence_threshold(max_value: float):
    a = C.c_int32(0)
    t = C.c_double(0.0)
    check(lib().cbf_divergence_threshold(max_value, C.byref(a), C.byref(t)))
    return bool(a.value), t.value


def record_length(job: Job) -> int:
    return int(lib().cbf_record_length(C.byref(job)))


# ---------------------------------------------------------------------------
# Reference-named entry points (hostLibrary.cuh), results as numpy arrays.

def _bif1d(fn, system, tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
           indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues,
           preScaller):
    ic, icp = _d(initialConditions)
    r, rp = _d(ranges)
    ix, ixp = _i(indicesOfMutVars)
    v, vp = _d(values)
    rec = int(tMax / h / preScaller)
    cap = max(rec // 2, 1)
    peaks = np.zeros((nPts, cap), np.float64)
    counts = np.zeros(nPts, np.int32)
    check(fn(_sys(system), tMax, nPts, h, amountOfInitialConditions, icp, rp, ixp, writableVar,
             maxValue, transientTime, vp, amountOfValues, preScaller,
             peaks.ctypes.data_as(_dp), cap, counts.ctypes.data_as(_ip)))
    return peaks, counts


def bifurcation1D(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                  indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues,
                  preScaller, *, system="memristive5"):
    """hostLibrary.cuh:29-42.  Returns (peaks[nPts, cap], counts[nPts])."""
    return _bif1d(lib().cbf_bifurcation1d, system, tMax, nPts, h, amountOfInitialConditions,
                  initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                  transientTime, values, amountOfValues, preScaller)


def bifurcation1DIC(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                    indicesOfMutVars, writableVar, maxValue, transientTime, values,
                    amountOfValues, preScaller, *, system="memristive5"):
    """hostLibrary.cuh:89-102."""
    return _bif1d(lib().cbf_bifurcation1d_ic, system, tMax, nPts, h, amountOfInitialConditions,
                  initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                  transientTime, values, amountOfValues, preScaller)


def _kde(fn, system, tMax, nPts, h, nIC, icv, ranges, idx, wv, maxValue, maxPeaks, transient,
         values, nV, preScaller, kdeSampling, i1, i2, smooth):
    ic, icp = _d(icv)
    r, rp = _d(ranges)
    ix, ixp = _i(idx)
    v, vp = _d(values)
    out = np.zeros(nPts * nPts, np.int32)
    check(fn(_sys(system), tMax, nPts, h, nIC, icp, rp, ixp, wv, maxValue, maxPeaks, transient,
             vp, nV, preScaller, kdeSampling, i1, i2, smooth, out.ctypes.data_as(_ip)))
    return out.reshape(nPts, nPts)


def bifurcation2DKDE(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                     indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks, transientTime,
                     values, amountOfValues, preScaller, in_kdeSampling, in_kdeSamplesInterval1,
                     in_kdeSamplesInterval2, in_kdeSamplesSmooth, *, system="memristive5"):
    """hostLibrary.cuh:129-147.  Returns the int32 map [row=axis1, col=axis0]."""
    return _kde(lib().cbf_bifurcation2d_kde, system, tMax, nPts, h, amountOfInitialConditions,
                initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                maxAmountOfPeaks, transientTime, values, amountOfValues, preScaller,
                in_kdeSampling, in_kdeSamplesInterval1, in_kdeSamplesInterval2,
                in_kdeSamplesSmooth)


def bifurcation2DKDEIC(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                       indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks, transientTime,
                       values, amountOfValues, preScaller, in_kdeSampling, in_kdeSamplesInterval1,
                       in_kdeSamplesInterval2, in_kdeSamplesSmooth, *, system="memristive5"):
    """hostLibrary.cuh:254-272."""
    return _kde(lib().cbf_bifurcation2d_kde_ic, system, tMax, nPts, h, amountOfInitialConditions,
                initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                maxAmountOfPeaks, transientTime, values, amountOfValues, preScaller,
                in_kdeSampling, in_kdeSamplesInterval1, in_kdeSamplesInterval2,
                in_kdeSamplesSmooth)


def _db(fn, system, tMax, nPts, h, nIC, icv, ranges, idx, wv, maxValue, maxPeaks, transient,
        values, nV, preScaller, eps):
    ic, icp = _d(icv)
    r, rp = _d(ranges)
    ix, ixp = _i(idx)
    v, vp = _d(values)
    out = np.zeros(nPts * nPts, np.int32)
    check(fn(_sys(system), tMax, nPts, h, nIC, icp, rp, ixp, wv, maxValue, maxPeaks, transient,
             vp, nV, preScaller, eps, out.ctypes.data_as(_ip)))
    return out.reshape(nPts, nPts)


def bifurcation2DDBSCAN(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                        indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks, transientTime,
                        values, amountOfValues, preScaller, eps, *, system="memristive5"):
    """hostLibrary.cuh:171-186."""
    return _db(lib().cbf_bifurcation2d_dbscan, system, tMax, nPts, h, amountOfInitialConditions,
               initialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
               maxAmountOfPeaks, transientTime, values, amountOfValues, preScaller, eps)


def bifurcation2DDBSCANIC(tMax, nPts, h, amountOfInitialConditions, initialConditions, ranges,
                          indicesOfMutVars, writableVar, maxValue, maxAmountOfPeaks,
                          transientTime, values, amountOfValues, preScaller, eps, *,
                          system="memristive5"):
    """hostLibrary.cuh:296-311."""
    return _db(lib().cbf_bifurcation2d_dbscan_ic, system, tMax, nPts, h,
               amountOfInitialConditions, initialConditions, ranges, indicesOfMutVars,
               writableVar, maxValue, maxAmountOfPeaks, transientTime, values, amountOfValues,
               preScaller, eps)


def _lle(fn, dims, system, tMax, NT, nPts, h, eps, icv, nIC, ranges, idx, wv, maxValue,
         transient, values, nV, seedChunk):
    ic, icp = _d(icv)
    r, rp = _d(ranges)
    ix, ixp = _i(idx)
    v, vp = _d(values)
    n = nPts ** dims
    out = np.zeros(n, np.float64)
    check(fn(_sys(system), tMax, NT, nPts, h, eps, icp, nIC, rp, ixp, wv, maxValue, transient, vp,
             nV, seedChunk, out.ctypes.data_as(_dp)))
    return out.reshape((nPts, nPts) if dims == 2 else (nPts,))


def modelingOneSystemDenis(tMax, h, hSpecial, amountOfInitialConditions, initialConditions, writableVar,
                           values, amountOfValues, *, system="memristive5"):
    """hostLibrary.cuh:59-67: the step-offset series, (int)(tMax/h) samples."""
    ic, icp = _d(initialConditions)
    v, vp = _d(values)
    n = int(tMax / h)
    out = np.zeros(max(n, 0), np.float64)
    L = lib()
    L.cbf_modeling_one_system.restype = C.c_int32
    L.cbf_modeling_one_system.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, _dp,
                                          C.c_int32, _dp, C.c_int32, _dp, C.c_int64]
    check(L.cbf_modeling_one_system(_sys(system), tMax, h, hSpecial, amountOfInitialConditions, icp,
                                    writableVar, vp, amountOfValues, out.ctypes.data_as(_dp), len(out)))
    return out


def calculationOfPeriodicityByOstrovsky(tMax, nPts, h, amountOfInitialConditions, initialConditions,
                                        ranges, indicesOfMutVars, writableVar, maxValue,
                                        maxAmountOfPeaks, transientTime, values, amountOfValues,
                                        preScaller, eps, ostrovskyThreshold, *, system="memristive5"):
    """hostLibrary.cuh:211-227: the periodicity map, shape (nPts, nPts) (row = axis 1)."""
    ic, icp = _d(initialConditions)
    r, rp = _d(ranges)
    ix, ixp = _i(indicesOfMutVars)
    v, vp = _d(values)
    out = np.zeros(nPts * nPts, np.float64)
    L = lib()
    L.cbf_ostrovsky2d.restype = C.c_int32
    L.cbf_ostrovsky2d.argtypes = [C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_int32, _dp, _dp, _ip,
                                  C.c_int32, C.c_double, C.c_int32, C.c_double, _dp, C.c_int32,
                                  C.c_int32, C.c_double, C.c_double, _dp]
    check(L.cbf_ostrovsky2d(_sys(system), tMax, nPts, h, amountOfInitialConditions, icp, rp, ixp,
                            writableVar, maxValue, maxAmountOfPeaks, transientTime, vp, amountOfValues,
                            preScaller, eps, ostrovskyThreshold, out.ctypes.data_as(_dp)))
    return out.reshape(nPts, nPts)


def _ls(fn, dims, system, tMax, NT, nPts, h, eps, icv, nIC, ranges, idx, wv, maxValue, transient,
        values, nV, seedChunk):
    ic, icp = _d(icv)
    r, rp = _d(ranges)
    ix, ixp = _i(idx)
    v, vp = _d(values)
    n = nPts ** dims
    out = np.zeros((n, nIC), np.float64)
    check(fn(_sys(system), tMax, NT, nPts, h, eps, icp, nIC, rp, ixp, wv, maxValue, transient, vp,
             nV, seedChunk, out.ctypes.data_as(_dp)))
    return out.reshape((nPts, nPts, nIC) if dims == 2 else (nPts, nIC))


def LS1D(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
         indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
         system="memristive5", seedChunk=0):
    """hostLibrary.cuh:482-496: the Lyapunov spectrum per point, shape (nPts, nIC)."""
    return _ls(lib().cbf_ls1d, 1, system, tMax, NT, nPts, h, eps, initialConditions,
               amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
               transientTime, values, amountOfValues, seedChunk)


def LS2D(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
         indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
         system="memristive5", seedChunk=0):
    """hostLibrary.cuh:520-534: the spectrum per grid point, shape (nPts, nPts, nIC)
    (row = axis 1)."""
    return _ls(lib().cbf_ls2d, 2, system, tMax, NT, nPts, h, eps, initialConditions,
               amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
               transientTime, values, amountOfValues, seedChunk)


def LLE1D(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
          indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
          system="memristive5", seedChunk=0):
    """hostLibrary.cuh:334-348."""
    return _lle(lib().cbf_lle1d, 1, system, tMax, NT, nPts, h, eps, initialConditions,
                amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                transientTime, values, amountOfValues, seedChunk)


def LLE1DIC(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
            indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
            system="memristive5", seedChunk=0):
    """hostLibrary.cuh:371-385."""
    return _lle(lib().cbf_lle1d_ic, 1, system, tMax, NT, nPts, h, eps, initialConditions,
                amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                transientTime, values, amountOfValues, seedChunk)


def LLE2D(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
          indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
          system="memristive5", seedChunk=200000):
    """hostLibrary.cuh:408-422 (seedChunk 200000: the reference's fixed chunk, :1552)."""
    return _lle(lib().cbf_lle2d, 2, system, tMax, NT, nPts, h, eps, initialConditions,
                amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                transientTime, values, amountOfValues, seedChunk)


def LLE2DIC(tMax, NT, nPts, h, eps, initialConditions, amountOfInitialConditions, ranges,
            indicesOfMutVars, writableVar, maxValue, transientTime, values, amountOfValues, *,
            system="memristive5", seedChunk=0):
    """hostLibrary.cuh:445-459."""
    return _lle(lib().cbf_lle2d_ic, 2, system, tMax, NT, nPts, h, eps, initialConditions,
                amountOfInitialConditions, ranges, indicesOfMutVars, writableVar, maxValue,
                transientTime, values, amountOfValues, seedChunk)
