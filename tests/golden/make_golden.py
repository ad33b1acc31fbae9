"""Generate tests/golden/reference_vectors.npz from the reference's own code.

The reference (CUDABifurcation3.0) ships no tests or golden vectors.  Its
__host__ __device__ functions compile for the host unmodified, so
``make -C oracle ref`` builds them from the reference sources into
oracle/_ref/libcbf_ref.so; this script feeds them seeded inputs and records the
outputs.  The fixtures let the CPU test suite pin the oracle where the reference
sources are not available (e.g. on the GPU box).

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "reference_vectors.npz"
SEED = 20240101


def vp(a):
    return a.ctypes.data_as(C.c_void_p)


def peak_sequences(rng, count):
    seqs = []
    for _ in range(count):
        n = int(rng.integers(0, 64))
        kind = rng.integers(0, 3)
        if kind == 0:     # heavy plateaus
            s = rng.integers(0, 4, n).astype(np.float64)
        elif kind == 1:   # smooth oscillation with rounding ties
            t = np.arange(n)
            s = np.round(np.sin(t * rng.uniform(0.2, 1.5)) * rng.choice([2, 4, 8])) / 4
        else:             # continuous values
            s = rng.normal(size=n)
        seqs.append(np.ascontiguousarray(s, dtype=np.float64))
    return seqs


def main() -> int:
    R = O.ref()
    if R is None:
        print("oracle/_ref/libcbf_ref.so is missing: run `make -C oracle ref` first", file=sys.stderr)
        return 1
    rng = np.random.default_rng(SEED)
    out = {}

    # getValueByIdx (cudaLibrary.cu:210-216), including the 8192^2 float-index region.
    n = 4000
    g_idx = np.concatenate([rng.integers(0, 2048 * 2048, n // 4), rng.integers(0, 8192 * 8192, n // 2),
                            rng.integers(16777200, 16777300, n // 4)]).astype(np.int64)
    g_npts = np.where(np.arange(n) < n // 4, 2048, 8192).astype(np.int32)
    g_axis = (np.arange(n) % 2).astype(np.int32)
    g_lo = rng.uniform(-50, 50, n)
    g_hi = g_lo + rng.uniform(0.1, 100, n)
    g_val = np.array([R.ref_getValueByIdx(int(i), int(p), float(a), float(b), int(v))
                      for i, p, a, b, v in zip(g_idx, g_npts, g_lo, g_hi, g_axis)])
    out.update(grid_idx=g_idx, grid_npts=g_npts, grid_axis=g_axis, grid_lo=g_lo, grid_hi=g_hi,
               grid_val=g_val)

    # peakFinder (cudaLibrary.cu:220-266), with and without intervals.
    seqs = peak_sequences(rng, 600)
    offs = np.cumsum([0] + [len(s) for s in seqs]).astype(np.int64)
    flat = np.concatenate(seqs) if seqs else np.zeros(0)
    counts, peaks, times = [], [], []
    for s in seqs:
        d = s.copy() if len(s) else np.zeros(1)
        p = np.zeros(max(len(s), 1))
        t = np.zeros(max(len(s), 1))
        c = R.ref_peakFinder(d, 0, len(s), vp(p), vp(t), 0.01)
        counts.append(c)
        peaks.append(p[:c])
        times.append(t[:c])
    out.update(pf_flat=flat, pf_offs=offs, pf_counts=np.array(counts, np.int32),
               pf_peaks=np.concatenate(peaks) if peaks else np.zeros(0),
               pf_times=np.concatenate(times) if times else np.zeros(0))

    # kde (cudaLibrary.cu:356-422).
    kde_lists, kde_params, kde_res = [], [], []
    for i in range(400):
        n = int(rng.integers(0, 40))
        centers = rng.normal(size=int(rng.integers(1, 5))) * 3
        p = np.round(rng.choice(centers, n) + rng.normal(size=n) * rng.choice([0.0, 0.02, 0.3]), 3)
        maxp = int(rng.choice([5, 30, 100]))
        samp = int(rng.integers(1, 12))
        i1, i2 = -8.0, float(rng.choice([6.0, 8.0, 12.0]))
        hh = float(rng.choice([0.01, 0.05, 0.2, 0.5]))
        pp = p.copy() if n else np.zeros(1)
        kde_res.append(R.ref_kde(pp, 0, n, maxp, samp, i1, i2, hh))
        kde_lists.append(p)
        kde_params.append([maxp, samp, i1, i2, hh])
    koffs = np.cumsum([0] + [len(s) for s in kde_lists]).astype(np.int64)
    out.update(kde_flat=np.concatenate(kde_lists), kde_offs=koffs,
               kde_params=np.array(kde_params, np.float64), kde_res=np.array(kde_res, np.int32))

    # distance (cudaLibrary.cu:445-453) and dbscan (:457-529).
    a = rng.normal(size=(2000, 4))
    a[::7, 2:] = a[::7, :2]
    a[::11] *= 1e-4
    out["dist_in"] = a
    out["dist_out"] = np.array([R.ref_distance(*map(float, r)) for r in a])

    db_p, db_t, db_params, db_res = [], [], [], []
    for i in range(400):
        n = int(rng.integers(0, 48))
        k = int(rng.integers(1, 6))
        cp = rng.normal(size=k) * 2
        ct = rng.integers(1, 6, k) * 0.01 * rng.integers(2, 40)
        which = rng.integers(0, k, n)
        jitter = rng.choice([0.0, 1e-4, 5e-4, 3e-3])
        p = np.round(cp[which] + rng.normal(size=n) * jitter, 6)
        t = ct[which]
        maxp = int(rng.choice([10, 40, 100]))
        eps = float(rng.choice([1e-3, 5e-3, 0.05]))
        helpful = np.zeros(max(2 * n + 2, 1))
        pp = p.copy() if n else np.zeros(1)
        tt = t.copy() if n else np.zeros(1)
        db_res.append(R.ref_dbscan(pp, tt, helpful, 0, n, len(helpful), maxp, eps))
        db_p.append(p)
        db_t.append(t)
        db_params.append([maxp, eps])
    doffs = np.cumsum([0] + [len(s) for s in db_p]).astype(np.int64)
    out.update(db_p=np.concatenate(db_p), db_t=np.concatenate(db_t), db_offs=doffs,
               db_params=np.array(db_params, np.float64), db_res=np.array(db_res, np.int32))

    # The shipped 5-D model through loopCalculateDiscreteModel (cudaLibrary.cu:2-74).
    vals = np.array([8, 35, 15, 0.01, -1.6676, 0.0676, 0.3682, 0.5], np.float64)
    runs = 40
    x0 = rng.normal(size=(runs, 5)) * 0.5
    pre = rng.integers(1, 4, runs).astype(np.int32)
    wv = rng.integers(0, 5, runs).astype(np.int32)
    mv = rng.choice([0.0, 1.0, 1e7], runs)
    steps = 400
    xs, datas, oks = [], [], []
    for r in range(runs):
        x = x0[r].copy()
        d = np.zeros(steps)
        ok = R.ref_loopCalculateDiscreteModel(x, vals, 0.005, steps, int(pre[r]), int(wv[r]),
                                              float(mv[r]), vp(d), 0, 1)
        xs.append(x)
        datas.append(d)
        oks.append(ok)
    out.update(m5_vals=vals, m5_x0=x0, m5_pre=pre, m5_wv=wv, m5_max=mv, m5_steps=np.int32(steps),
               m5_x=np.array(xs), m5_data=np.array(datas), m5_ok=np.array(oks, np.int32))

    # projectionOperator / gramSchmidtProcess (cudaLibrary.cu:913-956) of the
    # Lyapunov-spectrum kernel, n = 3 and 5, including rank-deficient inputs (a
    # zero row, a repeated row) and scales from 1e-9 to 10.
    gs_n, gs_a, gs_b, gs_d = [], [], [], []
    pj_a, pj_b, pj_m, pj_out = [], [], [], []
    for r in range(60):
        n = 3 if r % 2 == 0 else 5
        a = rng.normal(size=(n, n)) * 10.0 ** float(rng.integers(-9, 2))
        if r % 10 == 3:
            a[1] = 0.0
        if r % 10 == 7:
            a[2] = a[0]
        a = np.ascontiguousarray(a)
        b = np.zeros((n, n))
        d = np.zeros(n)
        R.ref_gramSchmidtProcess(a.copy(), b, n, d.ctypes.data_as(C.c_void_p))
        pad = lambda m: np.pad(m, ((0, 5 - n), (0, 5 - n)))
        gs_n.append(n)
        gs_a.append(pad(a))
        gs_b.append(pad(b))
        gs_d.append(np.pad(d, (0, 5 - n)))
        m = rng.normal(size=n)
        if r % 10 == 5:
            a[1] = 0.0
        mm = m.copy()
        R.ref_projectionOperator(np.ascontiguousarray(a[0]), np.ascontiguousarray(a[1]), mm, n)
        pj_a.append(np.pad(a[0], (0, 5 - n)))
        pj_b.append(np.pad(a[1], (0, 5 - n)))
        pj_m.append(np.pad(m, (0, 5 - n)))
        pj_out.append(np.pad(mm, (0, 5 - n)))
    out.update(gs_n=np.array(gs_n, np.int32), gs_a=np.array(gs_a), gs_b=np.array(gs_b),
               gs_d=np.array(gs_d), pj_a=np.array(pj_a), pj_b=np.array(pj_b), pj_m=np.array(pj_m),
               pj_out=np.array(pj_out))

    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
