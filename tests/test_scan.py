"""SCANFN (src/postsub.f90:25-560) without a GPU: the oracle's scanning
functions against known answers, and the library's output grid against the
oracle's."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, gpu

JFNS = (1, 2, 3, 4)


@pytest.mark.parametrize("jfn", JFNS)
def test_constant_spectrum_scans_to_itself(jfn):
    """The tabulated functions are normalised (SHAPET/SHAPEG/SINCSQ/SINC sum
    to one over their extent), so a constant spectrum comes back constant."""
    v1, dv = 600.0, 0.002
    spec = np.full(200000, 0.37)
    sc = abi.make_scan(hwhm=0.5, v1=650.0, v2=750.0, jfn=jfn)
    out, dvo = O.scan(sc, spec, v1, dv)
    tol = {1: 1e-6, 2: 1e-3, 3: 2e-2, 4: 5e-2}[jfn]
    np.testing.assert_allclose(out, 0.37, rtol=tol)


def test_single_line_gives_the_gaussian():
    """A narrow line scanned by the Gaussian (JFN=2) takes its shape: HWHM
    0.5 cm-1, maximum at the line, half of it 0.5 cm-1 away (to the 0.04
    cm-1 of SHRKSC's compressed grid, which moves the line to the centre of
    its group of 40 points)."""
    v1, dv = 600.0, 0.001
    v = v1 + dv * np.arange(200000)
    spec = np.where(np.abs(v - 700.0) < 0.5 * dv, 1.0, 0.0)
    sc = abi.make_scan(hwhm=0.5, v1=690.0, v2=710.0, jfn=2, sampl=20.0)
    out, dvo = O.scan(sc, spec, v1, dv)
    w = 690.0 + dvo * np.arange(len(out))
    k = int(np.argmax(out))
    assert abs(w[k] - 700.0) <= dvo
    half = out[np.argmin(np.abs(w - 700.5))] / out[k]
    assert abs(half - 0.5) < 0.04


def test_linear_spectrum_kept_by_symmetric_functions():
    v1, dv = 600.0, 0.002
    v = v1 + dv * np.arange(200000)
    spec = 1.0 + 0.01 * (v - 700.0)
    sc = abi.make_scan(hwhm=0.4, v1=660.0, v2=740.0, jfn=1)
    out, dvo = O.scan(sc, spec, v1, dv)
    w = 660.0 + dvo * np.arange(len(out))
    # (the window edges, rounded per input point, leave a bias of ~DVI/2)
    np.testing.assert_allclose(out, 1.0 + 0.01 * (w - 700.0), rtol=5e-5)


@pytest.mark.parametrize("jfn,sampl", [(1, 0.0), (2, 4.0), (3, -0.05), (-4, 0.0)])
def test_output_grid_matches_oracle(jfn, sampl):
    sc = abi.make_scan(hwhm=0.6, v1=650.0, v2=751.3, jfn=jfn, sampl=sampl)
    n, dvo = gpu.scan_npts(sc, 0.004)
    _, dvo_o = O.scan(sc, np.zeros(10), 600.0, 0.004)
    assert dvo == dvo_o
    # PANLSC's last point: the one nearest V2 (NNHI = (V2-VFT)/DV + 1.5)
    assert abs(650.0 + (n - 1) * dvo - 751.3) <= 0.5 * dvo + 1e-9


def test_rejections():
    sc = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=2)
    assert gpu.load().lbl_scan_npts(C.byref(sc), 0.06, None) == -7   # DV > HWHM/12
    bad = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=-2)
    assert gpu.load().lbl_scan_npts(C.byref(bad), 0.001, None) == -1
