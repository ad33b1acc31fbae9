"""GPU tests of the step-offset single-system mode (modelingOneSystemDenis,
hostLibrary.cu:162-239; calculateDiscreteModelDenisCUDA, cudaLibrary.cu:121-161):
the series bit for bit against the oracle (the FP64 state is computed by the
same operations), including the reference's int truncations of hSpecial/h and
tMax/hSpecial that leave entries unwritten (NaN here), and the facade's rows."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_parity import CHEN, LORENZ, MEMRISTIVE, ROSSLER

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("system_kw,tMax,h,hSpecial,wv", [
    (LORENZ, 5.0, 0.001, 0.01, 0),        # T = 10, I = 500: every entry written
    (CHEN, 2.0, 0.002, 0.02, 2),
    (ROSSLER, 1.0, 0.01, 0.03, 1),        # T = 3, I = 33: the last of 100 entries unwritten
    (ROSSLER, 1.05, 0.1, 0.3, 0),         # 0.3/0.1 = 2.99.. -> T = 2; n = 10, I = 3: 4 NaN
    (MEMRISTIVE, 0.5, 0.001, 0.004, 3),
])
def test_offset_trajectory_matches_oracle(cbf, orc, gpu_ok, system_kw, tMax, h, hSpecial, wv):
    got = cbf.modelingOneSystemDenis(tMax, h, hSpecial, len(system_kw["ic"]), system_kw["ic"], wv,
                                     system_kw["values"], len(system_kw["values"]),
                                     system=system_kw["system"])
    want = orc.modeling_one_system(system_kw["system"], tMax, h, hSpecial, system_kw["ic"], wv,
                                   system_kw["values"])
    assert got.shape == want.shape == (int(tMax / h),)
    assert np.array_equal(got, want, equal_nan=True)
    T, I = int(hSpecial / h), int(tMax / hSpecial)
    assert np.isnan(got).sum() == max(0, len(got) - T * I)
    assert got[0] == system_kw["ic"][wv]


def test_facade_offset_trajectory_rows(cbf, gpu_ok, tmp_path):
    L = cbf.lib()
    L.cbf_facade_set_system(cbf.SYS_ROSSLER)
    path = tmp_path / "denis.csv"
    ic = np.ascontiguousarray(ROSSLER["ic"], np.float64)
    vals = np.ascontiguousarray(ROSSLER["values"], np.float64)
    try:
        L.cbf_facade_set_output_path(str(path).encode())
        f = getattr(L, "_Z22modelingOneSystemDenisdddiPKdiS0_i")
        f.restype = None
        f.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
        f(1.0, 0.01, 0.03, 3, ic.ctypes.data, 1, vals.ctypes.data, 4)
        series = cbf.modelingOneSystemDenis(1.0, 0.01, 0.03, 3, ic, 1, vals, 4, system="rossler")
        want = "".join("%.12g, %.12g\n" % (0.01 * j, v) for j, v in enumerate(series))
        assert path.read_text() == want
    finally:
        L.cbf_facade_set_output_path(None)
        L.cbf_facade_set_system(-1)
