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


def _box_means(spec, v1, dv, centres, hwhm):
    """Mean of the nearest-point (step) reconstruction of spec over each box
    [c - hwhm, c + hwhm]: every point weighted by the length of its interval
    [v_i - dv/2, v_i + dv/2] inside the box."""
    v = v1 + dv * np.arange(len(spec))
    out = []
    for c in centres:
        lo = np.maximum(v - dv / 2, c - hwhm)
        hi = np.minimum(v + dv / 2, c + hwhm)
        w = np.clip(hi - lo, 0.0, None)
        out.append(np.dot(w, spec) / w.sum())
    return np.array(out)


@pytest.mark.parametrize("hwhm,sampl,jabs", [(0.5, 0.0, 0), (0.3, -0.07, 1), (1.25, 3.0, 0)])
def test_rectangle_is_the_box_mean(hwhm, sampl, jabs):
    """CNVRCT (JFN=0): each output point is the mean of the spectrum over a
    box of half width HWHM, the end points weighted by the fraction of their
    interval inside the box; DVOUT a whole number of input steps."""
    v1, dv = 600.0, 0.0013
    rng = np.random.default_rng(7)
    spec = np.exp(-rng.exponential(1.0, 150000))
    sc = abi.make_scan(hwhm=hwhm, v1=640.0, v2=760.0, jfn=0, sampl=sampl, jabs=jabs)
    out, dvo = O.scan(sc, spec, v1, dv)
    sample = sampl if sampl > 0 else (hwhm / -sampl if sampl < 0 else 0.5)
    assert dvo == round(hwhm / sample / dv) * dv
    n, dvo_lib = gpu.scan_npts(sc, dv)
    assert (n, dvo_lib) == (len(out), dvo)
    centres = 640.0 + dvo * np.arange(len(out))
    assert centres[-1] <= 760.0 < centres[-1] + dvo
    ref = _box_means(1.0 - spec if jabs else spec, v1, dv, centres, hwhm)
    np.testing.assert_allclose(out, ref, rtol=1e-11)
    const, _ = O.scan(sc, np.full(150000, 0.37), v1, dv)
    np.testing.assert_allclose(const, 0.63 if jabs else 0.37, rtol=1e-13)


def test_rejections():
    sc = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=2)
    # DV > HWHM/12: scanned on HWHM/12 after SCNINT, the same output grid
    assert gpu.load().lbl_scan_npts(C.byref(sc), 0.06, None) == \
        gpu.load().lbl_scan_npts(C.byref(sc), 0.05, None) > 0
    bad = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=-2)
    assert gpu.load().lbl_scan_npts(C.byref(bad), 0.001, None) == -1
    # rectangle: DVOUT under two input steps (IRATIO < 2)
    rect = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=0, sampl=-0.004)
    assert gpu.load().lbl_scan_npts(C.byref(rect), 0.004, None) == -7
    with pytest.raises(RuntimeError, match="IRATIO"):
        O.scan(rect, np.zeros(100000), 600.0, 0.004)
    # the boxes must lie inside the spectrum
    rect = abi.make_scan(hwhm=0.6, v1=650.0, v2=750.0, jfn=0)
    with pytest.raises(RuntimeError, match="inside the spectrum"):
        O.scan(rect, np.zeros(30000), 600.0, 0.004)


@pytest.mark.parametrize("jfn,angle,sampl,jabs", [(5, 2.0, -0.1, 0), (6, 1.5, -0.25, 1),
                                                  (5, 3.0, 0.0, 0)])
def test_field_of_view_boxes_are_box_means(jfn, angle, sampl, jabs):
    """CNVVRC (JFN 5) and CNVVRL (JFN 6): boxes whose width grows with
    wavenumber, V B^2/2 for a field-of-view half angle B (HWHM in degrees):
    centred at V1 + j DVOUT from VCNT (1 - B^2/4) to VCNT (1 + B^2/4), or
    starting there and reaching VLFT (1 + B^2/2); each output the weighted
    box mean of CNVRCT; DVOUT = HWHM/SAMPLE (SAMPLE 0.5 by default)."""
    v1, dv = 600.0, 0.0013
    rng = np.random.default_rng(8)
    spec = np.exp(-rng.exponential(1.0, 300000))
    sc = abi.make_scan(hwhm=angle, v1=640.0, v2=900.0, jfn=jfn, sampl=sampl, jabs=jabs)
    out, dvo = O.scan(sc, spec, v1, dv)
    sample = sampl if sampl > 0 else (angle / -sampl if sampl < 0 else 0.5)
    assert dvo == angle / sample
    n, dvo_lib = gpu.scan_npts(sc, dv)
    assert (n, dvo_lib) == (len(out), dvo)
    b = angle * 3.141592654 / 180.0
    v0 = 640.0 + dvo * np.arange(len(out))
    assert v0[-1] <= 900.0 < v0[-1] + dvo
    lo = v0 * (1 - b * b / 4) if jfn == 5 else v0
    hi = v0 * (1 + b * b / 4) if jfn == 5 else v0 * (1 + b * b / 2)
    s = 1.0 - spec if jabs else spec
    v = v1 + dv * np.arange(len(s))
    ref = []
    for a, c in zip(lo, hi):
        w = np.clip(np.minimum(v + dv / 2, c) - np.maximum(v - dv / 2, a), 0.0, None)
        ref.append(np.dot(w, s) / w.sum())
    np.testing.assert_allclose(out, np.array(ref), rtol=1e-11)


def test_field_of_view_dvint():
    """DVINT for JFN 5/6 is a twelfth of the first box (V1 B^2/24); a coarser
    input is interpolated onto it (SCNINT) and gives the same output grid."""
    sc = abi.make_scan(hwhm=1.0, v1=640.0, v2=700.0, jfn=5, sampl=-0.1)
    dvint = 640.0 * (1.0 * 3.141592654 / 180.0) ** 2 / 24
    n = gpu.load().lbl_scan_npts(C.byref(sc), dvint * 0.99, None)
    assert n > 0
    assert gpu.load().lbl_scan_npts(C.byref(sc), dvint * 1.5, None) == n
    bad = abi.make_scan(hwhm=1.0, v1=640.0, v2=700.0, jfn=-5)
    assert gpu.load().lbl_scan_npts(C.byref(bad), 0.001, None) == -1


def test_scnint_reproduces_constants_and_lines():
    """SCNINT/INTERP (postsub.f90:824-1035, 2940-3215): the 4-point cubic
    (weights summing to one, tabulated at P = (IP-1)/200) keeps a constant
    to rounding and a straight line to within its slope times DVI/200 (the
    tabulation step of P); the output runs from V1 in steps of DVO up to the
    input's last point."""
    v1, dv, n = 600.0, 0.05, 6000
    v = v1 + dv * np.arange(n)
    dvo = 0.0117
    const = O.scnint(np.full(n, 0.37), v1, dv, dvo)
    assert abs(len(const) - ((n - 1) * dv / dvo + 1)) <= 1.5
    np.testing.assert_allclose(const, 0.37, rtol=1e-15)
    line = O.scnint(1.0 + 0.01 * (v - 600.0), v1, dv, dvo)
    vo = v1 + dvo * np.arange(len(line))
    assert np.max(np.abs(line - (1.0 + 0.01 * (vo - 600.0)))) <= 0.01 * dv / 200 * (1 + 1e-6)


def test_coarse_spectrum_scanned_after_interpolation():
    """A spectrum coarser than DVINT is scanned as the reference does: SCNINT
    onto DVINT, then the scan of the interpolated spectrum (SCANFN
    :322-345); for a smooth spectrum the result is within 1e-5 of the scan
    of the same function sampled exactly on DVINT (the interpolation's own
    error, 6e-5 at most here, smoothed by the scanning function)."""
    v1, dv = 600.0, 0.07
    v = v1 + dv * np.arange(5000)
    f = lambda x: 1.0 + 0.3 * np.sin(x / 3.0) + 0.1 * np.cos(x / 1.7)  # noqa: E731
    sc = abi.make_scan(hwhm=0.5, v1=640.0, v2=900.0, jfn=2)
    dvint = 0.5 / 12
    got, dvo = O.scan(sc, f(v), v1, dv)
    fine = O.scnint(f(v), v1, dv, dvint)
    ref, dvo2 = O.scan(sc, fine, v1, dvint)
    assert dvo == dvo2 and np.array_equal(got, ref)
    vf = v1 + dvint * np.arange(len(fine))
    assert np.max(np.abs(fine - f(vf))) < 6e-5
    direct, _ = O.scan(sc, f(vf), v1, dvint)
    assert len(direct) == len(got)
    np.testing.assert_allclose(got, direct, atol=1e-5)
