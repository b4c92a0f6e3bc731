"""Known-answer tests that pin the FP64 oracle to the reference's own
arithmetic (no reference outputs exist to compare with)."""
import math

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs

RADCN1, RADCN2 = 1.191042722E-12, 1.4387752


def test_shapel_subfunctions_sum_to_lorentz_minus_q3():
    # F1+F2+F3 = (1/pi)[1/(1+x^2) - Q3(x^2)] on the F1 grid (SHAPEL :1822-1911)
    f1, f2, f3 = (O.shape_table(k) for k in range(3))
    a3 = (1 + 2 * 64.0 ** 2) / (1 + 64.0 ** 2) ** 2
    b3 = -1 / (1 + 64.0 ** 2) ** 2
    for i in (0, 7, 250, 999, 1500):            # x = i*0.002 within HWF1
        x = i * 0.002
        j2, j3 = int(round(x / 0.008)), int(round(x / 0.032))
        if abs(j2 * 0.008 - x) > 1e-12 or abs(j3 * 0.032 - x) > 1e-12:
            continue
        s = f1[i] + f2[j2] + f3[j3]
        want = (1 / (1 + x * x) - (a3 + b3 * x * x)) / math.pi
        assert abs(s - want) < 1e-12


def test_shapel_normalisation_total():
    # TOTAL of SHAPEL: integral of L - Q3 over [-64, 64] alpha_V
    f1, f2, f3 = (O.shape_table(k) for k in range(3))
    tot = 0.0
    for f, dx in ((f1, 0.002), (f2, 0.008), (f3, 0.032)):
        tot += (f[0] + 2 * f[1:2001].sum()) * dx
    a3 = (1 + 2 * 64.0 ** 2) / (1 + 64.0 ** 2) ** 2
    b3 = -1 / (1 + 64.0 ** 2) ** 2
    exact = (2 * math.atan(64.0) - 2 * (a3 * 64.0 + b3 * 64.0 ** 3 / 3)) / math.pi
    assert abs(tot - exact) < 2e-4


def test_shapeg_norm():
    fg = O.shape_table(3)
    s = (fg[0] + 2 * fg[1:2001].sum()) * 0.002
    assert abs(s - math.erf(4 * math.sqrt(math.log(2)))) < 1e-5


def test_tips_identity_and_scaling():
    for mol in (1, 2, 3, 6):
        assert abs(O.tips_scor(mol, 1, 296.0) - 1.0) < 1e-12
    # rotational partition sums grow ~T^1.5 (non-linear) / ~T (linear CO2)
    assert 1.6 < O.tips_scor(1, 1, 200.0) < 2.0
    assert 1.3 < O.tips_scor(2, 1, 200.0) < 1.9


def test_planck_and_radfn():
    for v, t in ((500.0, 290.0), (1500.0, 217.0), (10.0, 300.0)):
        x = v * RADCN2 / t
        b = RADCN1 * v ** 3 / math.expm1(x)
        assert abs(lib_planck(v, t) - b) / b < 1e-12
        assert abs(O.lib().orc_radfn(v, t) - v * math.tanh(x / 2)) / v < 1e-12


def lib_planck(v, t):
    return O.lib().orc_planck(v, t)


def test_dv_rule_config0_and_config1():
    cfg = configs.config0()
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    dv, it = O.dv_rule(run, lays)
    assert dv[0] == pytest.approx(0.0102, abs=1e-15)
    cfg = configs.config1()
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    dv, it = O.dv_rule(run, lays)
    assert it[0] == 99 and set(it[1:]) <= {0, 1, 2, 4, 5}
    ratio = dv[:-1] / dv[1:]
    assert np.all((ratio > 0.999) & (ratio < 2.0001))


def test_config0_matches_exact_voigt_sum():
    """The approximate-Voigt decomposition follows an exact Voigt sum (with
    the same 25 cm-1 bound subtraction) to its documented accuracy."""
    from scipy.special import wofz
    cfg = configs.config0()
    run = abi.make_run(**cfg["run"], dptmin=0.0, dptfac=0.0)
    lays = abi.make_layers(cfg["profile"])
    O.dv_rule(run, lays)
    lh = abi.LinesHandle(cfg["lines"])
    od, _ = O.layer_od(run, lays[0], lh)
    dv = lays[0].dv
    v = 600.0 + dv * np.arange(len(od))
    xkt = 296.0 / RADCN2
    fad = math.log(2.0) * 2.0 * 6.02214199E+23 * 1.3806503E-16 / 2.99792458E+10 ** 2
    alfd1 = math.sqrt(fad * 296.0 / 18.01)
    L = cfg["lines"]
    tot = np.zeros_like(v)
    sel = np.arange(0, len(v), 7)
    vs = v[sel]
    for i in range(len(L["vnu"])):
        nu, S, aL = L["vnu"][i], float(L["sp"][i]), float(L["alfa"][i])
        sig = nu * alfd1 / math.sqrt(2 * math.log(2))
        m = np.abs(vs - nu) < 25
        V = lambda x: np.real(wofz((x + 1j * aL) / (sig * math.sqrt(2)))) / (sig * math.sqrt(2 * math.pi))  # noqa: E731
        tot[sel[m]] += S * 1e22 * (1 + math.exp(-nu / xkt)) * (V(vs[m] - nu) - V(25.0))
    rad = vs * np.tanh(vs / xkt / 2)
    r = od[sel] / (tot[sel] * rad) - 1
    assert np.median(np.abs(r)) < 1e-3
    assert np.max(np.abs(r)) < 2e-2


def _one_layer(amount, t=250.0):
    prof = {"pave": np.array([500.0]), "tave": np.array([t]), "pzl": np.array([550.0]),
            "pzu": np.array([450.0]), "tzl": np.array([t]), "tzu": np.array([t]),
            "wk": np.zeros((1, 60)), "wbroad": np.array([1e24]), "nmol": 7}
    prof["wk"][0, 0] = amount
    return abi.make_layers(prof)


def test_isothermal_opaque_layer_emits_planck():
    lines = configs.gen_lines(400, 690.0, 710.0, seed=5)
    lines["sp"][:] = 1e-17
    t = 250.0
    run = abi.make_run(v1=695.0, v2=705.0, iemit=1, tmpbnd=t, bndemi=1.0, dptmin=0., dptfac=0.)
    lays = _one_layer(1e24, t)
    lh = abi.LinesHandle(lines)
    rad, tr = O.forward(run, lays, lh)
    dv = lays[0].dv
    v = 695.0 + dv * np.arange(len(rad))
    bt = RADCN2 * v / np.log(RADCN1 * v ** 3 / rad + 1)
    assert np.max(np.abs(bt - t)) < 1e-6


def test_transparent_layer_keeps_radiance():
    lines = configs.gen_lines(300, 690.0, 710.0, seed=6)
    run = abi.make_run(v1=695.0, v2=705.0, iemit=1, tmpbnd=280.0, bndemi=0.9)
    lays = _one_layer(1e20, 260.0)
    O.dv_rule(run, lays)
    lh = abi.LinesHandle(lines)
    od, _ = O.layer_od(run, lays[0], lh)
    rad0, tr0 = O.merge_layer(run, lays[0], True, 0.0, None, None, od)
    # a second layer with zero optical depth on the same grid
    rad1, tr1 = O.merge_layer(run, lays[0], False, lays[0].dv, rad0, tr0, np.zeros_like(od))
    assert np.max(np.abs(rad1 - rad0) / rad0) < 1e-15
    assert np.max(np.abs(tr1 - tr0)) < 1e-15


def test_merge_regrid_exact_for_cubics():
    """RADNN's 4-point Lagrange regrid reproduces a cubic in the interior."""
    run = abi.make_run(v1=500.0, v2=540.0, iemit=1, tmpbnd=0.0)
    lays = _one_layer(0.0)
    lays[0].dv = 0.006
    n_old = O.npts(run, 0.006)
    v_old = 500.0 + 0.006 * np.arange(n_old)
    cub = lambda x: 1.0 + 0.3 * (x - 520) + 0.01 * (x - 520) ** 2 - 1e-4 * (x - 520) ** 3  # noqa: E731
    rad_in = cub(v_old)
    tr_in = np.ones(n_old)
    for itype in (1, 2, 4, 5):
        dvn = 0.006 * itype / (itype + 1)
        lays[0].dv = dvn
        n_new = O.npts(run, dvn)
        rad, tr = O.merge_layer(run, lays[0], False, 0.006, rad_in, tr_in, np.zeros(n_new))
        v_new = 500.0 + dvn * np.arange(n_new)
        inner = slice(10, n_new - 10)
        assert np.max(np.abs(rad[inner] - cub(v_new[inner]))) < 1e-9


def test_testmm_fixture_pins_tape3_format(tmp_path):
    """The TESTMM line list of the reference (src/testmm.f90, 0-80 cm-1) as a
    TAPE3: write, read back, and compute a layer with it."""
    import os
    from lblrtm_b200 import tape3
    fx = os.path.join(os.path.dirname(__file__), "golden", "testmm_lines.npz")
    L = dict(np.load(fx))
    p = tmp_path / "TAPE3"
    tape3.write(p, L)
    R = tape3.read(p)
    for k in ("vnu", "sp", "alfa", "epp", "mol", "hwhms", "tmpalf", "pshift", "iflg"):
        assert np.array_equal(R[k], L[k])
    assert R["block_start"][-1] == len(L["vnu"])
    # a layer at 40-60 cm-1 through the oracle: finite, positive
    run = abi.make_run(v1=40.0, v2=60.0, iemit=0)
    lays = _one_layer(5e21, 250.0)
    for m in (3, 4, 7):
        lays[0].wk[m - 1] = 1e19
    O.dv_rule(run, lays)
    od, _ = O.layer_od(run, lays[0], abi.LinesHandle(R))
    assert np.all(np.isfinite(od)) and od.min() > 0


def _rayleigh_only(v1, v2, xrayl):
    """Oracle optical depth of one layer whose only absorber is the Rayleigh
    term of CONTNM: a zero H2O continuum table and lines far outside the band."""
    lines = configs.gen_lines(250, 6000.0, 6010.0, seed=3)
    lh = abi.LinesHandle(lines)
    zero = configs.mtckd_table(1)
    zero["self_absco_ref"] = np.zeros_like(zero["self_absco_ref"])
    zero["for_absco_ref"] = np.zeros_like(zero["for_absco_ref"])
    ck = abi.MtckdHandle(zero)
    run = abi.make_run(v1=v1, v2=v2, icntnm=1, ilblf4=1, xrayl=xrayl, xco2c=0.0)
    lay = abi.make_layers(configs.atmosphere(20, ptop=300.0))
    O.dv_rule(run, lay)
    od, _ = O.layer_od(run, lay[0], lh, ck)
    wtot = lay[0].wbroad + sum(lay[0].wk[m] for m in range(lay[0].nmol))
    v = v1 + lay[0].dv * np.arange(len(od))
    return od, v, wtot


def test_rayleigh_extinction_closed_form():
    """contnm.f90:955-976: xv^4/(9.38076e2 - 10.8426 xv^2) * WTOT * XRAYL *
    1e-20/(2.68675e-1 * 1e5), xv = v/1e4, with the radiation term (xv) put
    back by PANEL's RADFNI, reproduced to the accuracy of the 1 cm-1 grid
    interpolation and the piecewise-linear radiation term."""
    od, v, wtot = _rayleigh_only(1500.0, 1520.0, 1.0)
    xv = v / 1e4
    expect = xv ** 4 / (9.38076e2 - 10.8426 * xv ** 2) * wtot * 1e-20 / (2.68675e-1 * 1e5)
    np.testing.assert_allclose(od, expect, rtol=2e-4)
    od2, _, _ = _rayleigh_only(1500.0, 1520.0, 2.0)
    np.testing.assert_allclose(od2, 2.0 * od, rtol=1e-12)


def test_rayleigh_only_above_820():
    od, _, _ = _rayleigh_only(700.0, 719.0, 1.0)
    assert np.all(od == 0.0)
    od, _, _ = _rayleigh_only(1500.0, 1520.0, 0.0)
    assert np.all(od == 0.0)


def _planck(v, t):
    return RADCN1 * v ** 3 / np.expm1(RADCN2 * v / t)


def _two_layers(t1, t2):
    prof = {"pave": np.array([500.0, 400.0]), "tave": np.array([t1, t2]),
            "pzl": np.array([550.0, 450.0]), "pzu": np.array([450.0, 350.0]),
            "tzl": np.array([t1, t2]), "tzu": np.array([t1, t2]),
            "wk": np.zeros((2, 60)), "wbroad": np.array([1e24, 1e24]), "nmol": 7}
    prof["wk"][:, 0] = 1e20
    return abi.make_layers(prof)


def test_downwelling_order_of_layers():
    """RADNN IPATH=3 (xmerge.f90:3007-3013) looking up from layer 1, against
    IPATH=1 looking down onto it, for two isothermal layers of constant
    optical depth on one grid (EMIN's linear-in-tau term vanishes):
    down R = B1 (1-T1) + T1 B2 (1-T2), up R = B2 (1-T2) + T2 B1 (1-T1)."""
    t1, t2, tau1, tau2 = 280.0, 230.0, 0.7, 1.3
    lays = _two_layers(t1, t2)
    for l in lays:
        l.dv = 0.01
    out = {}
    for ipathl in (1, 3):
        run = abi.make_run(v1=700.0, v2=710.0, iemit=1, ipathl=ipathl, tmpbnd=0.0)
        n = O.npts(run, 0.01)
        od1, od2 = np.full(n, tau1), np.full(n, tau2)
        r1, x1 = O.merge_layer(run, lays[0], 1, 0.0, None, None, od1)
        out[ipathl] = O.merge_layer(run, lays[1], 2, 0.01, r1, x1, od2)
    v = 700.0 + 0.01 * np.arange(n)
    b1, b2 = _planck(v, t1), _planck(v, t2)
    e1, e2 = np.exp(-tau1), np.exp(-tau2)
    np.testing.assert_allclose(out[3][0], b1 * (1 - e1) + e1 * b2 * (1 - e2), rtol=1e-12)
    np.testing.assert_allclose(out[1][0], b2 * (1 - e2) + e2 * b1 * (1 - e1), rtol=1e-12)
    np.testing.assert_allclose(out[3][1], e1 * e2, rtol=1e-14)


def test_downwelling_boundary_beyond_last_layer():
    """Looking up, TMPBND/BNDEMI lie beyond the last layer (EMBND,
    xmerge.f90:3652-3733, applied by XMERGE at the last layer): through two
    transparent layers the radiance is BNDEMI B(TMPBND); a single layer
    (EMINIT) has no boundary term."""
    lays = _two_layers(250.0, 250.0)
    for l in lays:
        l.dv = 0.01
    run = abi.make_run(v1=700.0, v2=710.0, iemit=1, ipathl=3, tmpbnd=5800.0, bndemi=0.3)
    n = O.npts(run, 0.01)
    z = np.zeros(n)
    r1, x1 = O.merge_layer(run, lays[0], 3, 0.0, None, None, z)
    assert np.all(r1 == 0.0)
    r1, x1 = O.merge_layer(run, lays[0], 1, 0.0, None, None, z)
    r2, x2 = O.merge_layer(run, lays[1], 2, 0.01, r1, x1, z)
    v = 700.0 + 0.01 * np.arange(n)
    np.testing.assert_allclose(r2, 0.3 * _planck(v, 5800.0), rtol=1e-12)


def test_tangent_path_crosses_each_layer_twice():
    """IPATHL=2, the symmetric tangent path (EMINIT :2442-2447, RADNN
    IPATH=2 :2997-3005): the tangent layer is crossed twice, R1 = B1 (1 -
    T1^2), and each outer layer adds its near crossing and its far crossing
    seen through the inner path: R = T2 R1 + B2 (1-T2) + B2 (1-T2) T2 T1^2,
    T = T2^2 T1^2 (isothermal layers of constant optical depth on one grid,
    where EMIN's linear-in-tau term vanishes)."""
    t1, t2, tau1, tau2 = 280.0, 230.0, 0.7, 1.3
    lays = _two_layers(t1, t2)
    for l in lays:
        l.dv = 0.01
    run = abi.make_run(v1=700.0, v2=710.0, iemit=1, ipathl=2, tmpbnd=290.0)
    n = O.npts(run, 0.01)
    r1, x1 = O.merge_layer(run, lays[0], 1, 0.0, None, None, np.full(n, tau1))
    r2, x2 = O.merge_layer(run, lays[1], 2, 0.01, r1, x1, np.full(n, tau2))
    v = 700.0 + 0.01 * np.arange(n)
    b1, b2 = _planck(v, t1), _planck(v, t2)
    e1, e2 = np.exp(-tau1), np.exp(-tau2)
    np.testing.assert_allclose(r1, b1 * (1 - e1 * e1), rtol=1e-12)
    np.testing.assert_allclose(x1, e1 * e1, rtol=1e-14)
    np.testing.assert_allclose(r2, e2 * r1 + b2 * (1 - e2) * (1 + e2 * e1 * e1), rtol=1e-12)
    np.testing.assert_allclose(x2, e2 * e2 * e1 * e1, rtol=1e-14)
    # one temperature: the path's emission is B (1 - T_path)
    lays = _two_layers(250.0, 250.0)
    for l in lays:
        l.dv = 0.01
    r1, x1 = O.merge_layer(run, lays[0], 1, 0.0, None, None, np.full(n, tau1))
    r2, x2 = O.merge_layer(run, lays[1], 2, 0.01, r1, x1, np.full(n, tau2))
    np.testing.assert_allclose(r2, _planck(v, 250.0) * (1 - x2), rtol=1e-12)


def _cont_macro(name):
    """An initializer list of cont_tables.h (the continuum DATA of CONTNM)."""
    import os
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                        "lblrtm_b200", "data", "cont_tables.h")
    txt = open(path).read()
    m = re.search(r"#define LBL_%s \\\n(.*?)(\n#define|\n#endif)" % name, txt, re.S)
    if m:
        body = m.group(1)
    else:
        body = re.search(r"#define LBL_%s (\S+)" % name, txt).group(1)
    return np.array([float(x) for x in body.replace("\\", " ").replace(",", " ").split()])


def _fco2_table():
    """The CO2 continuum table of cont_tables.h (BLOCK DATA BFCO2)."""
    vals = _cont_macro("FCO2_VALUES")
    assert len(vals) == 5003
    return -4.0 + 2.0 * np.arange(5003), vals


def _co2_continuum_only(v1, v2, xco2c, jrad=None, **scales):
    """Oracle optical depth of one layer whose only absorbers are CONTNM's
    CO2, O2 and N2 continua: zero H2O continuum table, no Rayleigh, lines
    far away."""
    lines = configs.gen_lines(250, 6000.0, 6010.0, seed=3)
    lh = abi.LinesHandle(lines)
    zero = configs.mtckd_table(1)
    zero["self_absco_ref"] = np.zeros_like(zero["self_absco_ref"])
    zero["for_absco_ref"] = np.zeros_like(zero["for_absco_ref"])
    ck = abi.MtckdHandle(zero)
    run = abi.make_run(v1=v1, v2=v2, icntnm=1, ilblf4=1, xrayl=0.0, xco2c=xco2c, **scales)
    lay = abi.make_layers(configs.atmosphere(20, ptop=300.0))
    O.dv_rule(run, lay)
    od, j = O.layer_od(run, lay[0], lh, ck, jrad=jrad)
    v = v1 + lay[0].dv * np.arange(len(od))
    return od, v, lay[0], j


def _radfn(v, t):
    x = v * RADCN2 / t
    e = np.exp(-np.minimum(x, 10.0))
    return np.where(x <= 0.01, 0.5 * x * v, np.where(x <= 10.0, v * (1 - e) / (1 + e), v))


def _xint_points(v1a, dva, a, vi):
    """XINT's 4-point interpolation (src/oprop.f90:2201-2234) of the values
    a (a[0] is point 1 at v1a, spacing dva) at the wavenumbers vi."""
    ap = np.concatenate([[0.0], a, [0.0, 0.0]])          # 1-based with pads
    j = ((vi - v1a) / dva + 1.0 + 1e-5).astype(int)     # J = (VI-V1A)/DVA + ONEPL
    p = (vi - (v1a + dva * (j - 1))) / dva
    c = (3 - 2 * p) * p * p
    b = 0.5 * p * (1 - p)
    b1, b2 = b * (1 - p), b * p
    return -ap[j - 1] * b1 + ap[j] * (1 - c + b2) + ap[j + 1] * (c + b1) - ap[j + 2] * b2


def test_co2_continuum_follows_its_table():
    """contnm.f90:326-378 with FRNCO2: between 600 and 640 cm-1 the layer's
    optical depth is WCO2 = WK(2) RHOAVE 1e-20 XCO2C times the 2 cm-1 table,
    put on the 1 cm-1 continuum grid by XINT, carried to the layer grid by
    the finer interpolations (XINT onto R3, PANEL onto R2 and R1) and
    multiplied by the radiation term (PANEL's RADFNI for JRAD=0, on the
    2 cm-1 grid for JRAD=1): within 1e-3 of XINT onto the 1 cm-1 grid
    followed by a cubic spline (the later 4-point stages differ from the
    spline by a few 1e-4).  Linear in XCO2C."""
    from scipy.interpolate import CubicSpline
    vt, st = _fco2_table()
    for jrad in (0, 1):
        od, v, lay, j = _co2_continuum_only(600.0, 640.0, 1.0, jrad=jrad)
        wco2 = lay.wk[1] * (lay.pave / 1013.0) * (296.0 / lay.tave) * 1e-20
        va = 597.0 + np.arange(47.0)                    # V1ABS = INT(V1)-3, DVABS = 1
        c = st * wco2
        if j == 1:
            c = c * _radfn(vt, lay.tave)
        cabs = _xint_points(vt[0], 2.0, c, va)
        expect = CubicSpline(va, cabs)(v)
        if j != 1:
            expect = expect * _radfn(v, lay.tave)
        np.testing.assert_allclose(od, expect, rtol=1e-3)
    od2, _, _, _ = _co2_continuum_only(600.0, 640.0, 2.0, jrad=0)
    od1, _, _, _ = _co2_continuum_only(600.0, 640.0, 1.0, jrad=0)
    np.testing.assert_allclose(od2, 2.0 * od1, rtol=1e-12)
    od0, _, _, _ = _co2_continuum_only(600.0, 640.0, 0.0, jrad=0)
    assert np.all(od0 == 0.0)


def test_o2_and_n2_collision_induced_bands_follow_their_tables():
    """The O2 fundamental (contnm.f90:491-540, o2_ver_1 :7254-7318) at
    1500-1540 cm-1 and the N2 fundamental (:811-858, n2_ver_1 :2668-2754) at
    2300-2340 cm-1, the N2 first overtone (:860-906) and the O2 1.27 um band
    (:543-584) as the layer's only absorbers: the coefficients formed on
    their own grids from the two tables (O2: exp(XO2T (1/296 - 1/T)); N2:
    log-interpolation in 1/T between 272 K and 228 K, the O2 and H2O
    broadening efficiencies), XINT onto the 1 cm-1 grid restated here, then
    a cubic spline and the radiation term: within 1e-3.  Linear in the
    scale factors; no CO2 or N2/O2 term where the scale is 0."""
    from scipy.interpolate import CubicSpline
    lay0 = abi.make_layers(configs.atmosphere(20, ptop=300.0))[0]
    wtot = lay0.wbroad + sum(lay0.wk[m] for m in range(lay0.nmol))
    x_h2o, x_o2 = lay0.wk[0] / wtot, lay0.wk[6] / wtot
    x_n2 = 1 - x_h2o - x_o2
    t = lay0.tave
    amagat = (lay0.pave / 1013.0) * (273.0 / t)
    # O2: 5 cm-1 grid from 1340
    vo = 1340.0 + 5.0 * np.arange(103)
    co = (1e20 / 2.68675e19) * _cont_macro("O2F_XO2_VALUES") * np.exp(
        _cont_macro("O2F_XO2T_VALUES") * (1 / 296.0 - 1 / t)) / vo
    co = co * lay0.wk[6] * 1e-20 * amagat
    # N2 fundamental: 228 points from 1997.784896 every 3.981461525
    dvn = 3.981461525
    vn = 1997.784896 + dvn * np.arange(228)
    a, b = _cont_macro("N2F_X272_VALUES"), _cont_macro("N2F_X228_VALUES")
    xtfac = (1 / t - 1 / 272.0) / (1 / 228.0 - 1 / 272.0)
    pos = (a > 0) & (b > 0)
    c0 = np.where(pos, a * (np.where(pos, b, 1) / np.where(pos, a, 1)) ** xtfac,
                  a + (b - a) * (t - 272.0) / (228.0 - 272.0)) / vn
    a_o2 = 1.294 - 0.4545 * t / 296.0
    cn = (x_n2 * c0 + x_o2 * a_o2 * c0 + x_h2o * (9.0 / 7.0) * _cont_macro("N2F_AH2O_VALUES") * c0)
    cn = cn * (x_n2 * wtot / 2.68675e19) * amagat
    # N2 first overtone: 4340-4910 every 3 cm-1; O2 1.27 um: 7536-8500 every 2
    vo1 = 4340.0 + 3.0 * np.arange(191)
    co1 = _cont_macro("N2O1_X_VALUES") / vo1 * (x_n2 * wtot / 2.68675e19) * amagat * (
        x_n2 + x_o2 + x_h2o)
    vo2 = 7536.0 + 2.0 * np.arange(483)
    co2 = _cont_macro("O2I1_X_VALUES") / vo2 * (lay0.wk[6] / 2.68675e19) * amagat * (
        x_o2 / 0.446 + 0.3 / 0.446 * x_n2 + x_h2o)
    for (v1, v2), (vt, ct, dvt) in (((1500.0, 1540.0), (vo, co, 5.0)),
                                    ((2300.0, 2340.0), (vn, cn, dvn)),
                                    ((4500.0, 4540.0), (vo1, co1, 3.0)),
                                    ((7800.0, 7840.0), (vo2, co2, 2.0))):
        od, v, lay, j = _co2_continuum_only(v1, v2, 0.0, jrad=0)
        assert j == 0
        va = (int(v1) - 3.0) + np.arange(int(v2 + 3.5) - (int(v1) - 3.0) + 1)
        cabs = _xint_points(vt[0], dvt, ct, va)
        expect = CubicSpline(va, cabs)(v) * _radfn(v, t)
        np.testing.assert_allclose(od, expect, rtol=1e-3)
        od2, _, _, _ = _co2_continuum_only(v1, v2, 0.0, jrad=0, xo2cn=2.0, xn2cn=2.0)
        np.testing.assert_allclose(od2, 2.0 * od, rtol=1e-12)
        od0, _, _, _ = _co2_continuum_only(v1, v2, 0.0, jrad=0, xo2cn=0.0, xn2cn=0.0)
        assert np.all(od0 == 0.0)


def test_reflected_atmosphere_specular():
    """IPATHL=1 with BNDRFL(1) > 0 is the reflected atmosphere (IPATHL=-1,
    specular; EMINIT :2486-2540, RADNN IPATH=-10 :3051-3066): each layer's
    downward emission reaches the surface through the layers below, is
    reflected and comes back up: with surface temperature Ts, emissivity e
    and reflectivity r, R1 = B1(1-T1)(1 + r T1) + T1 e B(Ts), and the next
    layer adds B2(1-T2)(1 + r T1^2 T2) over T2 R1 (isothermal layers of
    constant optical depth on one grid)."""
    t1, t2, tau1, tau2, ts, emis, refl = 280.0, 230.0, 0.7, 1.3, 295.0, 0.9, 0.1
    lays = _two_layers(t1, t2)
    for l in lays:
        l.dv = 0.01
    run = abi.make_run(v1=700.0, v2=710.0, iemit=1, ipathl=1, tmpbnd=ts, bndemi=emis,
                       bndrfl=refl)
    n = O.npts(run, 0.01)
    r1, x1 = O.merge_layer(run, lays[0], 1, 0.0, None, None, np.full(n, tau1))
    r2, x2 = O.merge_layer(run, lays[1], 0, 0.01, r1, x1, np.full(n, tau2))
    v = 700.0 + 0.01 * np.arange(n)
    b1, b2, bs = _planck(v, t1), _planck(v, t2), _planck(v, ts)
    e1, e2 = np.exp(-tau1), np.exp(-tau2)
    np.testing.assert_allclose(r1, b1 * (1 - e1) * (1 + refl * e1) + e1 * emis * bs, rtol=1e-12)
    np.testing.assert_allclose(x1, e1, rtol=1e-14)
    np.testing.assert_allclose(r2, e2 * r1 + b2 * (1 - e2) * (1 + refl * e1 * e1 * e2), rtol=1e-12)
    np.testing.assert_allclose(x2, e1 * e2, rtol=1e-14)
    # no reflectivity: the plain upwelling merge
    run0 = abi.make_run(v1=700.0, v2=710.0, iemit=1, ipathl=1, tmpbnd=ts, bndemi=emis)
    q1, _ = O.merge_layer(run0, lays[0], 1, 0.0, None, None, np.full(n, tau1))
    np.testing.assert_allclose(q1, b1 * (1 - e1) + e1 * emis * bs, rtol=1e-12)
