"""PNLINT (src/oprop.f90:1564-1806) without a GPU: the oracle's restatement
against known answers, and the library's host-side point count against the
oracle's."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, gpu

CASES = [
    # v1, v2, dv, dvout
    (600.0, 700.0, 0.01, 0.0025),
    (600.0, 700.0, 0.01, 0.005),
    (600.0, 700.0, 0.01, 0.0037),
    (500.0, 1500.0, 0.0123, 0.0041),
    (999.5, 1000.5, 0.002, 0.00099),
    (10.0, 11.0, 0.01, 0.01),
    (700.0, 701.7, 0.0011, 0.00109999),
]


@pytest.mark.parametrize("v1,v2,dv,dvout", CASES)
def test_point_count_matches_oracle(v1, v2, dv, dvout):
    run = abi.make_run(v1=v1, v2=v2)
    n_in = O.npts(run, dv)
    out = O.pnlint(run, dv, dvout, np.zeros(n_in))
    assert gpu.pnlint_npts(run, dv, dvout) == len(out)
    # the grid ends at the first point at or beyond V2
    assert v1 + (len(out) - 1) * dvout >= v2 - 1e-9 * v2
    assert v1 + (len(out) - 2) * dvout < v2


def test_equal_spacing_passes_through():
    run = abi.make_run(v1=600.0, v2=700.0)
    od = np.random.default_rng(1).uniform(0, 3, O.npts(run, 0.01))
    for dvout in (0.01, 0.01 + 5e-9):
        out = O.pnlint(run, 0.01, dvout, od)
        assert np.array_equal(out, od)
    assert gpu.pnlint_npts(run, 0.01, 0.01 + 5e-9) == len(od)


def test_half_spacing_keeps_input_points():
    run = abi.make_run(v1=600.0, v2=700.0)
    od = np.random.default_rng(2).uniform(0, 3, O.npts(run, 0.01))
    out = O.pnlint(run, 0.01, 0.005, od)
    n = min(len(od), (len(out) + 1) // 2)
    assert np.array_equal(out[0:2 * n:2], od[:n])


def test_cubic_reproduced_at_quarter_spacing():
    """Four-point Lagrange weights are exact for cubics when the output
    points fall on the 1/100 weight table (here at quarters of DV)."""
    run = abi.make_run(v1=600.0, v2=700.0)
    dv, dvout = 0.01, 0.0025
    v = 600.0 + dv * np.arange(O.npts(run, dv))
    f = lambda x: 1.0 + 0.3 * (x - 650) / 50 - 0.2 * ((x - 650) / 50) ** 2 + 0.1 * ((x - 650) / 50) ** 3
    out = O.pnlint(run, dv, dvout, f(v))
    w = 600.0 + dvout * np.arange(len(out))
    inner = slice(8, len(out) - 16)
    np.testing.assert_allclose(out[inner], f(w[inner]), rtol=0, atol=1e-12)


def test_rejects_coarser_output():
    run = abi.make_run(v1=600.0, v2=700.0)
    assert gpu.load().lbl_pnlint_npts(C.byref(run), 0.01, 0.02) == -1  # -LBL_E_ARG
    with pytest.raises(RuntimeError):
        O.pnlint(run, 0.01, 0.02, np.zeros(O.npts(run, 0.01)))
