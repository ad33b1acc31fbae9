"""Pin the CPU oracle to the reference's own code (CPU only).

tests/golden/reference_vectors.npz holds outputs of the reference's
getValueByIdx, peakFinder, kde, distance, dbscan and its shipped model through
loopCalculateDiscreteModel, computed by compiling those functions from the
reference sources (tests/golden/make_golden.py).  The oracle must reproduce all
of them bit for bit.  When oracle/_ref/libcbf_ref.so is present the same
checks also run live on fresh random inputs.
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_vectors.npz"


@pytest.fixture(scope="module")
def G():
    return np.load(GOLDEN)


def test_grid_index_matches_reference(G, orc):
    L = orc.lib()
    got = np.array([L.orc_get_value_by_idx(int(i), int(p), float(a), float(b), int(v))
                    for i, p, a, b, v in zip(G["grid_idx"], G["grid_npts"], G["grid_lo"],
                                             G["grid_hi"], G["grid_axis"])])
    assert np.array_equal(got.view(np.int64), G["grid_val"].view(np.int64))


def test_grid_index_float_quirk_is_real(orc):
    # 8192^2 grid: the float division rounds the index above 2^24 (cudaLibrary.cu:214).
    L = orc.lib()
    idx = 16777217  # 2^24 + 1 -> (float) rounds to 2^24
    quirk = L.orc_get_value_by_idx(idx, 8192, 0.0, 8191.0, 0)
    assert quirk == float((idx - 1) % 8192)


def test_peak_finder_matches_reference(G, orc):
    flat, offs = G["pf_flat"], G["pf_offs"]
    want_n = G["pf_counts"]
    pk_off = np.concatenate([[0], np.cumsum(want_n)])
    for i in range(len(want_n)):
        seq = flat[offs[i]:offs[i + 1]]
        p, t = orc.peak_finder(seq) if len(seq) else (np.zeros(0), np.zeros(0))
        assert len(p) == want_n[i], i
        assert np.array_equal(p, G["pf_peaks"][pk_off[i]:pk_off[i + 1]]), i
        assert np.array_equal(t, G["pf_times"][pk_off[i]:pk_off[i + 1]]), i


def test_peak_finder_quirks(orc):
    # rising plateau: the sample after the plateau is skipped (cudaLibrary.cu:231-234)
    d = [0, 2, 2, 3, 1, 0, 5, 0, 4, 0]
    p, t = orc.peak_finder(d)
    # detected peaks at 6 and 8 (3 at index 3 is skipped); first one is dropped
    assert list(p) == [4.0] and np.allclose(t, [0.02])
    # fewer than two detected peaks -> zero
    assert len(orc.peak_finder([0, 1, 0])[0]) == 0


def test_kde_matches_reference(G, orc):
    offs = G["kde_offs"]
    for i, (maxp, samp, i1, i2, hh) in enumerate(G["kde_params"]):
        p = G["kde_flat"][offs[i]:offs[i + 1]]
        got = orc.kde(p, int(maxp), int(samp), i1, i2, hh)
        assert got == G["kde_res"][i], i


def test_kde_special_cases(orc):
    assert orc.kde([], 10, 5, -1, 1, 0.1) == 0
    assert orc.kde([1.0], 10, 5, -1, 1, 0.1) == 1
    assert orc.kde([1.0, 2.0], 10, 5, -1, 1, 0.1) == 1
    assert orc.kde([1.0, 2.0, 3.0, 4.0], 3, 5, -1, 1, 0.1) == 3  # > max -> max


def test_distance_matches_reference(G, orc):
    L = orc.lib()
    got = np.array([L.orc_distance(*map(float, r)) for r in G["dist_in"]])
    assert np.array_equal(got, G["dist_out"])


def test_dbscan_matches_reference(G, orc):
    offs = G["db_offs"]
    for i, (maxp, eps) in enumerate(G["db_params"]):
        p = G["db_p"][offs[i]:offs[i + 1]]
        t = G["db_t"][offs[i]:offs[i + 1]]
        assert orc.dbscan(p, t, int(maxp), eps) == G["db_res"][i], i


def test_dbscan_special_cases(orc):
    assert orc.dbscan([], [], 10, 0.1) == 0
    assert orc.dbscan([1.0], [0.1], 10, 0.1) == 1
    assert orc.dbscan([1.0, 2.0, 3.0], [0.1] * 3, 2, 0.1) == 0  # > max -> 0
    # the last peak is never anyone's neighbour and the result is cluster-1
    assert orc.dbscan([1.0, 1.0, 1.0], [0.1] * 3, 10, 0.5) == 1


def test_shipped_model_matches_reference(G, orc):
    L = orc.lib()
    vals = G["m5_vals"]
    steps = int(G["m5_steps"])
    for r in range(len(G["m5_x0"])):
        x = G["m5_x0"][r].copy()
        d = np.zeros(steps)
        ok = L.orc_loop(0, x, vals, 0.005, steps, int(G["m5_pre"][r]), int(G["m5_wv"][r]),
                        float(G["m5_max"][r]), d.ctypes.data, 0, 1)
        assert ok == G["m5_ok"][r], r
        assert np.array_equal(x, G["m5_x"][r]), r
        assert np.array_equal(d, G["m5_data"][r]), r


@pytest.mark.skipif(not (Path(__file__).resolve().parents[1] / "oracle" / "_ref" /
                         "libcbf_ref.so").exists(), reason="reference shim not built")
def test_live_random_against_reference(orc):
    R = orc.ref()
    L = orc.lib()
    rng = np.random.default_rng(7)
    for _ in range(300):
        n = int(rng.integers(3, 50))
        s = rng.integers(0, 3, n).astype(float)
        a, b = s.copy(), s.copy()
        pa, ta, pb, tb = (np.zeros(n) for _ in range(4))
        ca = R.ref_peakFinder(a, 0, n, pa.ctypes.data, ta.ctypes.data, 0.01)
        cb = L.orc_peak_finder(b, 0, n, pb.ctypes.data, tb.ctypes.data, 0.01)
        assert ca == cb and np.array_equal(pa[:ca], pb[:cb]) and np.array_equal(ta[:ca], tb[:cb])
        p = np.round(rng.normal(size=n), 2)
        t = rng.integers(1, 3, n) * 0.01
        ha, hb = np.zeros(2 * n + 2), np.zeros(2 * n + 2)
        assert R.ref_dbscan(p.copy(), t.copy(), ha, 0, n, len(ha), 60, 0.05) == \
            L.orc_dbscan(p.copy(), t.copy(), hb, 0, n, len(hb), 60, 0.05)
        assert R.ref_kde(p.copy(), 0, n, 60, 4, -3.0, 3.0, 0.1) == \
            L.orc_kde(p.copy(), 0, n, 60, 4, -3.0, 3.0, 0.1)


def test_regime_amplitude_rule_on_oracle(orc):
    """The regime class of the plain labelling method: equilibria (negative LLE,
    no oscillation left after the transient) are class 0 once the window range
    rule is on, whatever ulp-level wobble the FP64 state shows; limit cycles keep
    their cluster count."""
    side = 2048
    kw = dict(system="chen", nPts=side, ranges=[30.0, 45.0, 20.0, 30.0], idxMut=[1, 3],
              ic=[0.1, 0.1, 0.1], values=[0.5, 35.0, 3.0, 28.0], h=0.002, NT=0.5, tMax=100.0,
              transientTime=500.0, lleEps=1e-8, maxValue=1e4, seedChunk=200000,
              maxAmountOfPeaks=512, dbscanEps=0.05, regimeTime=50.0)

    def idx(a, c):  # exact-grid index of the point nearest (a, c)
        i0 = int(round((a - 30.0) / 15.0 * (side - 1)))
        i1 = int(round((c - 20.0) / 10.0 * (side - 1)))
        return i1 * side + i0

    stable = [idx(a, c) for a in (38.5, 39.0, 39.7, 40.3) for c in (20.2, 20.5)]
    cycle = [idx(a, c) for a in (30.6, 31.2) for c in (27.2, 27.8)]
    on = orc.make_job(regimeMinAmp=1e-6, **kw)
    lle, cls = orc.map_lle_regime(on, stable)
    assert np.all(lle < -0.05), lle
    assert np.all(cls == 0), cls
    lle, cls = orc.map_lle_regime(on, cycle)
    assert np.all(np.abs(lle) < 0.05), lle
    assert np.all(cls >= 1), cls
    # the rule only ever lowers a class to 0
    off = orc.make_job(**kw)
    _, raw = orc.map_lle_regime(off, stable + cycle)
    _, ruled = orc.map_lle_regime(on, stable + cycle)
    assert np.all((ruled == raw) | (ruled == 0))


def test_gram_schmidt_matches_reference(G, orc):
    """projectionOperator and gramSchmidtProcess of the Lyapunov-spectrum kernel,
    bit for bit against the reference's own functions (zero and repeated rows
    included)."""
    L = orc.lib()
    for k, n in enumerate(G["gs_n"]):
        n = int(n)
        a = np.ascontiguousarray(G["gs_a"][k][:n, :n])
        b, d = orc.gram_schmidt(a)
        assert np.array_equal(b.view(np.int64), np.ascontiguousarray(G["gs_b"][k][:n, :n]).view(np.int64)), k
        assert np.array_equal(d.view(np.int64), np.ascontiguousarray(G["gs_d"][k][:n]).view(np.int64)), k
        m = np.ascontiguousarray(G["pj_m"][k][:n]).copy()
        L.orc_projection(np.ascontiguousarray(G["pj_a"][k][:n]), np.ascontiguousarray(G["pj_b"][k][:n]), m, n)
        assert np.array_equal(m.view(np.int64), np.ascontiguousarray(G["pj_out"][k][:n]).view(np.int64)), k


def test_gram_schmidt_live_against_reference(orc):
    R = orc.ref()
    if R is None or not hasattr(R, "ref_gramSchmidtProcess"):
        pytest.skip("reference shim not built")
    import ctypes as C
    rng = np.random.default_rng(11)
    for _ in range(200):
        n = int(rng.integers(2, 6))
        a = np.ascontiguousarray(rng.normal(size=(n, n)) * 10.0 ** float(rng.integers(-6, 3)))
        want_b, want_d = np.zeros((n, n)), np.zeros(n)
        R.ref_gramSchmidtProcess(a.copy(), want_b, n, want_d.ctypes.data_as(C.c_void_p))
        b, d = orc.gram_schmidt(a)
        assert np.array_equal(b, want_b) and np.array_equal(d, want_d)


def test_lyapunov_spectrum_oracle_is_physical(orc):
    """Lorenz (10, 28, 8/3): one positive, one ~zero exponent, and the sum close
    to the trace of the Jacobian, -(sigma + 1 + beta), as for any flow."""
    job = orc.make_job(system="lorenz", nPts=2, ranges=[28.0, 29.0], idxMut=[2], ic=[0.1, 0.1, 0.1],
                       values=[0.5, 10.0, 28.0, 8.0 / 3.0], h=0.005, NT=0.5, tMax=200.0,
                       transientTime=50.0, lleEps=1e-8, maxValue=0.0)
    ls = orc.map_ls(job, [0])[0]
    assert 0.75 < ls[0] < 1.1, ls
    assert abs(ls[1]) < 0.05, ls
    assert abs(ls.sum() + (10.0 + 1.0 + 8.0 / 3.0)) < 0.05, ls
    assert ls[0] >= ls[1] >= ls[2]
    # seeds: unit rows
    z = orc.ls_seeds(job, [0, 5, 12345])
    assert np.allclose(np.linalg.norm(z, axis=2), 1.0, atol=1e-15)


@pytest.mark.parametrize("system", ["chen", "lorenz"])
@pytest.mark.parametrize("s", [0.5, 0.3])
def test_rescaled_step_is_the_cd_step(orc, system, s):
    """The rescaled Chen/Lorenz step (state (x, sy*y, sz*z)) is the same CD step
    as the 14-instruction form: from the same physical states, ten steps of each
    agree to rounding error in physical units.  The GPU tests compare the kernels
    with the oracle form by form; this pins the algebra of the rescaled form
    itself.  sy = r1 A h cy, sz = (1 - kB) sy / k as the library defines them."""
    L = orc.lib()
    sid = orc.SYSTEMS[system]
    h = 0.002 if system == "chen" else 0.005
    rng = np.random.default_rng(11)
    lorenz = system == "lorenz"
    for _ in range(20):
        if lorenz:
            v = np.array([s, rng.uniform(5, 20), rng.uniform(20, 200), 8.0 / 3.0])
            A, B, cy = v[1], v[3], 1.0 - h * s
        else:
            v = np.array([s, rng.uniform(30, 45), 3.0, rng.uniform(20, 30)])
            A, B, cy = v[1], v[2], 1.0 + h * s * v[3]
        k, h1 = h * s, h * (1.0 - s)
        r1 = 1.0 / (1.0 + h1 * A)
        sy = (r1 * A) * h * cy
        sz = ((1.0 - k * B) * sy) / k
        x = rng.uniform(-20, 20, 3)
        a = x.copy()
        b = np.array([x[0], x[1] * sy, x[2] * sz])
        vv = np.ascontiguousarray(v)
        for _ in range(10):
            L.orc_model_step(sid, a, vv, h)
            L.orc_model_step(sid | 0x100, b, vv, h)
        phys = np.array([b[0], b[1] / sy, b[2] / sz])
        assert np.allclose(phys, a, rtol=1e-13, atol=1e-13), (system, s, v, a, phys)
