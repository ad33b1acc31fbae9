"""Ragged batches (cbf_batch_*): one persistent launch equals the same jobs run
one by one through the per-job kernels, bit for bit (GPU)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SYS = {
    "rossler": dict(values=[0.5, 0.2, 0.2, 5.7], idxMut=[1, 2], ranges=[0.05, 0.35, 0.05, 0.35],
                    ic=[0.1, 0.1, 0.1]),
    "lorenz": dict(values=[0.5, 10.0, 28.0, 8.0 / 3.0], idxMut=[1, 2], ranges=[5, 20, 20, 200],
                   ic=[0.1, 0.1, 0.1]),
    "chen": dict(values=[0.5, 35.0, 3.0, 28.0], idxMut=[1, 3], ranges=[30, 45, 20, 30],
                 ic=[0.1, 0.1, 0.1]),
    "memristive5": dict(values=[8, 35, 15, 0.01, -1.6676, 0.0676, 0.3682, 0.5], idxMut=[4, 3],
                        ranges=[-6, 6, -15, 15], ic=[0.001, 0, 0, 0, 0]),
}


def _jobs(cbf, with_m5=False):
    rng = np.random.default_rng(11)
    systems = ["rossler", "lorenz", "chen"] + (["memristive5"] if with_m5 else [])
    jobs, kinds = [], []
    for i in range(10):
        name = systems[i % len(systems)]
        task = [cbf.TASK_LLE, cbf.TASK_KDE, cbf.TASK_DBSCAN, cbf.TASK_PEAKS][i % 4]
        side = int(rng.integers(3, 20))
        h = float(rng.uniform(0.002, 0.01))
        kw = dict(system=name, nPts=side, h=h, tMax=float(rng.uniform(8, 30)), transientTime=5.0,
                  maxValue=1e4 if i % 3 else 30.0, **SYS[name])
        if task == cbf.TASK_PEAKS:
            kw["idxMut"] = kw["idxMut"][:1]
            kw["ranges"] = kw["ranges"][:2]
        if task == cbf.TASK_LLE:
            kw.update(NT=0.4, lleEps=1e-8)
        elif task == cbf.TASK_KDE:
            kw.update(maxAmountOfPeaks=300, kdeSampling=4, kdeI1=-60.0, kdeI2=60.0, kdeH=0.5)
        elif task == cbf.TASK_DBSCAN:
            kw.update(maxAmountOfPeaks=300, dbscanEps=0.05)
        jobs.append(cbf.make_job(task=task, **kw))
        kinds.append(task)
    return jobs, kinds


def _buffers(cbf, torch, jobs, kinds):
    outs, auxs = [], []
    for j, t in zip(jobs, kinds):
        n = cbf.lib().cbf_job_points(__import__("ctypes").byref(j))
        if t == cbf.TASK_PEAKS:
            cap = cbf.lib().cbf_peak_capacity(__import__("ctypes").byref(j))
            j.peakCapacity = cap
            outs.append(torch.zeros(n * cap, dtype=torch.float64, device="cuda"))
            auxs.append(torch.zeros(n, dtype=torch.int32, device="cuda"))
        else:
            dt = torch.float64 if t == cbf.TASK_LLE else torch.int32
            outs.append(torch.zeros(n, dtype=dt, device="cuda"))
            auxs.append(None)
    return outs, auxs


def _snapshot(outs, auxs, jobs, kinds, cbf):
    res = []
    for o, a, j, t in zip(outs, auxs, jobs, kinds):
        if t == cbf.TASK_PEAKS:
            cnt = a.cpu().numpy()
            pk = o.cpu().numpy().reshape(len(cnt), -1)
            res.append((cnt.copy(), [pk[k, :cnt[k]].copy() for k in range(len(cnt))]))
        else:
            res.append(o.cpu().numpy().copy())
    return res


def _same(a, b):
    if isinstance(a, tuple):
        return np.array_equal(a[0], b[0]) and all(np.array_equal(x, y) for x, y in zip(a[1], b[1]))
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("with_m5", [False, True])
def test_batch_equals_one_by_one(cbf, gpu_ok, with_m5):
    torch = pytest.importorskip("torch")
    jobs, kinds = _jobs(cbf, with_m5)
    outs, auxs = _buffers(cbf, torch, jobs, kinds)
    b = cbf.Batch(jobs, [o.data_ptr() for o in outs],
                  [a.data_ptr() if a is not None else 0 for a in auxs])
    s = torch.cuda.Stream()
    b.run(s.cuda_stream)
    s.synchronize()
    b.check()
    batched = _snapshot(outs, auxs, jobs, kinds, cbf)
    for o in outs:
        o.zero_()
    b.run_sequential(s.cuda_stream)
    s.synchronize()
    single = _snapshot(outs, auxs, jobs, kinds, cbf)
    assert all(_same(x, y) for x, y in zip(batched, single))
    # graph capture and replay, after autotuning the grid
    bps, ms = b.autotune(s.cuda_stream)
    assert 1 <= bps <= 16 and (ms > 0).any()
    b.capture(s.cuda_stream)
    for o in outs:
        o.zero_()
    b.launch(s.cuda_stream)
    b.launch(s.cuda_stream)
    s.synchronize()
    b.check()
    replayed = _snapshot(outs, auxs, jobs, kinds, cbf)
    assert all(_same(x, y) for x, y in zip(replayed, single))
    b.close()


def test_batch_rejects_bad_jobs(cbf, gpu_ok):
    torch = pytest.importorskip("torch")
    jobs, kinds = _jobs(cbf)
    outs, _ = _buffers(cbf, torch, jobs[:1], kinds[:1])
    bad = cbf.make_job(task=cbf.TASK_LLE, system="chen", nPts=4, h=0.0, tMax=1, NT=0.5,
                       **SYS["chen"])
    with pytest.raises(cbf.CbfError):
        cbf.Batch([bad], [outs[0].data_ptr()])
    # tasks the persistent kernel does not run are refused, not silently skipped
    for task, extra in ((cbf.TASK_LS, dict(NT=0.5)), (cbf.TASK_LLE_REGIME, dict(NT=0.5, regimeTime=1.0)),
                        (cbf.TASK_OSTROVSKY, dict(maxAmountOfPeaks=10)), (cbf.TASK_TRAJECTORY, {})):
        job = cbf.make_job(task=task, system="chen", nPts=4, h=0.01, tMax=1.0, **extra, **SYS["chen"])
        with pytest.raises(cbf.CbfError, match="batched"):
            cbf.Batch([job], [outs[0].data_ptr()], [outs[0].data_ptr()])


def test_seeded_64_job_mix_matches_the_oracle(cbf, orc, gpu_ok):
    """The benchmark's seeded 64-job batch (bench.batch_specs: systems, tasks, grid
    sides, record lengths and step sizes drawn from seed 20240101), with every grid
    cut to a few points per axis and every record and transient cut 100x / 20x so
    that the oracle finishes in seconds, in one persistent launch: each job
    against the CPU oracle directly -- KDE and DBSCAN counts bit-exact, LLE within
    1e-9 from the device's seeds."""
    torch = pytest.importorskip("torch")
    import sys
    from pathlib import Path
    root = str(Path(__file__).resolve().parents[1])
    if root not in sys.path:
        sys.path.insert(0, root)
    import bench
    from test_gpu_parity import assert_lle_close
    specs = bench.batch_specs()
    assert len(specs) == 64
    jobs, kinds, okw = [], [], []
    for sp in specs:
        sp = dict(sp)
        task = sp.pop("task")
        sp.update(nPts=max(3, sp["nPts"] // 128), tMax=sp["tMax"] / 100.0, transientTime=sp["transientTime"] / 20.0)
        jobs.append(cbf.make_job(task=task, **sp))
        kinds.append(task)
        okw.append(sp)
    outs, auxs = _buffers(cbf, torch, jobs, kinds)
    b = cbf.Batch(jobs, [o.data_ptr() for o in outs])
    b.run()
    torch.cuda.synchronize()
    b.check()
    assert {cbf.TASK_LLE, cbf.TASK_KDE, cbf.TASK_DBSCAN} <= set(kinds)
    for j, t, kw, o in zip(jobs, kinds, okw, outs):
        got = o.cpu().numpy()
        oj = orc.make_job(**kw)
        n = kw["nPts"] ** 2
        if t == cbf.TASK_LLE:
            assert_lle_close(got, orc.map_lle_seeded(oj, 0, n, cbf.lle_seeds(j)))
        elif t == cbf.TASK_KDE:
            assert np.array_equal(got, orc.map_kde(oj, 0, n)), kw
        else:
            assert np.array_equal(got, orc.map_dbscan(oj, 0, n)), kw
    b.close()
