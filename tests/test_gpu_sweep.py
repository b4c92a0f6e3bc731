"""Parity of the CUDA path with the FP64 oracle on the inputs config 1 does
not reach, each through the C ABI against the oracle on the same inputs.

* Config 2 (the precision sweep: the config-1 atmosphere, 400,000 lines over
  10-3000 cm-1 with strengths 1e-28..1e-18, seeded MT_CKD-layout continuum),
  run as 25 cm-1 slices of its two reference-legal sub-runs, all 60 layers:
    - 20-45 cm-1: DV down to 8.5e-6 cm-1 at the top layers, continuum, the
      Van Vleck-Weisskopf image of far-wing lines below 25 cm-1, JRAD=0
      (radiation term applied per panel, RADFNI);
    - 700-725 cm-1: the mid band;
    - 2500-2525 cm-1: V1/XKT > 5 in every layer, so JRAD stays 1 and the
      radiation term multiplies the line strengths in LNCOR1
      (src/oprop.f90:1030) and the far wing in LBLF4 (:3733-3758).
  FP64 layer optical depths, the FP64 and FP32/FP64-split forwards, with the
  maximum and RMS error of optical depth, transmittance and brightness
  temperature printed.
* RSYM (negative-wavenumber folding, src/oprop.f90:2145-2200): runs starting
  below 32 DV, on the reference's TESTMM line list and on synthetic lines.
* IEMIT=0 (ABINIT/ABSMRG, src/xmerge.f90:270-682) over a 70-layer profile,
  end-of-data averaging included.
* The reference's own MT_CKD 4.3 coefficient table (tests/golden/mtckd_h2o.npz).

Bars: FP64 optical depth within 1e-9 relative above OD_FLOOR at all but a
few points per million (FMA and table-index ties, which may move a point to
the neighbouring table entry) and within 1e-4 everywhere (the drop-in bar);
split optical depth within 1e-4 relative above OD_FLOOR; brightness
temperature within 0.01 K.
"""
import os

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

RTOL_OD = 1e-4      # the drop-in bar (relative optical depth)
RTOL_FP64 = 1e-9    # FP64 against FP64 away from ties
TIE_FRAC = 5e-6     # points allowed between RTOL_FP64 and RTOL_OD
OD_FLOOR = 1e-9     # below this the value is radiatively zero (T within 1e-9 of 1)
BT_TOL = 0.01
HERE = os.path.dirname(os.path.abspath(__file__))


def floored_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), OD_FLOOR)


def check_fp64(od, ref, what):
    e = floored_err(od, ref)
    assert e.max() < RTOL_OD, (what, e.max(), int(e.argmax()))
    assert np.mean(e > RTOL_FP64) <= TIE_FRAC, (what, int(np.sum(e > RTOL_FP64)), len(e))


def real_mtckd():
    d = np.load(os.path.join(HERE, "golden", "mtckd_h2o.npz"))
    wn = d["wavenumbers"]
    return {"v0": float(wn[0]), "dv": float(wn[1] - wn[0]),
            "self_absco_ref": d["self_absco_ref"], "for_absco_ref": d["for_absco_ref"],
            "self_texp": d["self_texp"], "ref_press": float(d["ref_press"]),
            "ref_temp": float(d["ref_temp"])}


@pytest.fixture(scope="module")
def c2():
    return configs.config2()


SLICES = {"low": (20.0, 45.0), "mid": (700.0, 725.0), "jrad1": (2500.0, 2525.0)}


@pytest.fixture(scope="module", params=list(SLICES), ids=list(SLICES))
def c2slice(request, c2, gpu_ctx):
    v1, v2 = SLICES[request.param]
    run = abi.make_run(**c2["run"], v1=v1, v2=v2)
    lays = abi.make_layers(c2["profile"])
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(configs.subset_lines(c2["lines"], v1, v2, margin=30.0))
    ck = abi.MtckdHandle(c2["mtckd"])
    # oracle optical depths of every layer with the forward's JRAD chain
    ref, jr = [], []
    j = run.jrad
    for L in lays:
        jr.append(j)
        od, j = O.layer_od(run, L, lh, ck, jrad=j)
        ref.append(od)
    rad_ref, tr_ref = O.forward(run, abi.make_layers_like(lays), lh, ck)
    return request.param, run, lays, lh, ck, ref, jr, rad_ref, tr_ref


def load(ctx, lh, ck):
    ctx.upload_lines(lh)
    ctx.upload_mtckd(ck)


def test_config2_slice_jrad_chain(c2slice):
    name, run, lays, *_ , jr, _, _ = c2slice
    if name == "jrad1":
        assert all(j == 1 for j in jr)
    else:
        assert jr[1:] == [0] * (len(jr) - 1)


def test_config2_slice_layers_fp64(gpu_ctx, c2slice):
    name, run, lays, lh, ck, ref, jr, _, _ = c2slice
    load(gpu_ctx, lh, ck)
    for l, L in enumerate(lays):
        od, j = gpu_ctx.layer_od(run, L, jrad=jr[l])
        check_fp64(od, ref[l], (name, l))


def test_config2_slice_layers_split(gpu_ctx, c2slice):
    name, run, lays, lh, ck, ref, jr, _, _ = c2slice
    load(gpu_ctx, lh, ck)
    worst = (0.0, -1)
    for l, L in enumerate(lays):
        od, _ = gpu_ctx.layer_od(run, L, jrad=jr[l], precision=abi.PREC_SPLIT)
        e = floored_err(od, ref[l]).max()
        worst = max(worst, (e, l))
    assert worst[0] < RTOL_OD, (name, worst)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_SPLIT], ids=["fp64", "split"])
def test_config2_slice_forward(gpu_ctx, c2slice, prec):
    name, run, lays, lh, ck, _, _, rad_ref, tr_ref = c2slice
    load(gpu_ctx, lh, ck)
    rad, tr = gpu_ctx.forward(run, abi.make_layers_like(lays), precision=prec)
    dv = lays[len(lays) - 1].dv
    b = gpu.brightness_temperature(rad, run.v1, dv)
    b_ref = gpu.brightness_temperature(rad_ref, run.v1, dv)
    e_bt = np.abs(b - b_ref)
    e_tr = np.abs(tr - tr_ref)
    e_rad = np.abs(rad - rad_ref) / np.abs(rad_ref)
    print(f"\nconfig2 {name} prec={prec}: BT max {e_bt.max():.3e} rms "
          f"{np.sqrt(np.mean(e_bt ** 2)):.3e} K; T max {e_tr.max():.3e}; "
          f"rad rel max {e_rad.max():.3e}")
    assert e_bt.max() < BT_TOL
    assert e_rad.max() < (1e-8 if prec == abi.PREC_FP64 else RTOL_OD)


# ---- RSYM -------------------------------------------------------------------

def load_testmm_lines():
    return dict(np.load(os.path.join(HERE, "golden", "testmm_lines.npz")))


def lowband_case(lines, v1, v2, nlay=6, ptop=300.0, scale=1.0, icntnm=1):
    prof = configs.atmosphere(nlay, ptop=ptop)
    prof["wk"] = prof["wk"] * scale
    run = abi.make_run(v1=v1, v2=v2, iemit=1, ilblf4=1, icntnm=icntnm, tmpbnd=290.0,
                       bndemi=0.98)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    return run, lays, abi.LinesHandle(lines)


@pytest.mark.parametrize("src", ["testmm", "synthetic"])
def test_rsym_first_panel_below_zero(gpu_ctx, src):
    """V1 < 32 DV: the first panel's origin lies below zero wavenumber and
    the grids are folded (RSYM) before PANEL."""
    if src == "testmm":
        lines = load_testmm_lines()
        run, lays, lh = lowband_case(lines, 0.1, 60.0)
    else:
        lines = configs.gen_lines(3000, 0.01, 70.0, seed=21, mols=configs.MOLS)
        run, lays, lh = lowband_case(lines, 0.05, 50.0)
    ck = abi.MtckdHandle(real_mtckd())
    load(gpu_ctx, lh, ck)
    assert run.v1 - 32 * lays[0].dv < 0
    j = run.jrad
    for l, L in enumerate(lays):
        ref, jn = O.layer_od(run, L, lh, ck, jrad=j)
        od, _ = gpu_ctx.layer_od(run, L, jrad=j)
        check_fp64(od, ref, (src, l))
        j = jn
    rad_ref, _ = O.forward(run, abi.make_layers_like(lays), lh, ck)
    rad, _ = gpu_ctx.forward(run, abi.make_layers_like(lays))
    assert np.max(np.abs(rad - rad_ref) / np.abs(rad_ref)) < 1e-8


def test_rsym_changes_the_first_points(gpu_ctx):
    """The fold matters: the lowest points differ from the unfolded sum by
    far more than the parity bar (the oracle with RSYM switched off stands
    for the unfolded sum)."""
    lines = configs.gen_lines(3000, 0.01, 70.0, seed=21, mols=configs.MOLS)
    run, lays, lh = lowband_case(lines, 0.05, 50.0, icntnm=0)
    gpu_ctx.upload_lines(lh)
    od, _ = gpu_ctx.layer_od(run, lays[0], jrad=run.jrad)
    folded, _ = O.layer_od(run, lays[0], lh, jrad=run.jrad)
    L = O.lib()
    L.orc_set_rsym(0)
    try:
        plain, _ = O.layer_od(run, lays[0], lh, jrad=run.jrad)
    finally:
        L.orc_set_rsym(1)
    assert np.max(floored_err(od, folded)) < RTOL_OD
    assert np.max(floored_err(plain, folded)[:64]) > 100 * RTOL_OD


def test_testmm_layer_40_60(gpu_ctx):
    """The reference's TESTMM line list (0-80 cm-1, molecules 1, 3, 4, 7)
    through the GPU path against the oracle, one layer at 40-60 cm-1."""
    lines = load_testmm_lines()
    prof = {"pave": np.array([500.0]), "tave": np.array([250.0]), "pzl": np.array([550.0]),
            "pzu": np.array([450.0]), "tzl": np.array([250.0]), "tzu": np.array([250.0]),
            "wk": np.zeros((1, 60)), "wbroad": np.array([1e24]), "nmol": 7}
    prof["wk"][0, 0] = 5e21
    for m in (3, 4, 7):
        prof["wk"][0, m - 1] = 1e19
    run = abi.make_run(v1=40.0, v2=60.0, iemit=0)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(lines)
    gpu_ctx.upload_lines(lh)
    ref, _ = O.layer_od(run, lays[0], lh)
    od, _ = gpu_ctx.layer_od(run, lays[0])
    check_fp64(od, ref, "testmm")


# ---- IEMIT=0 ----------------------------------------------------------------

@pytest.mark.parametrize("nlay,ptop", [(70, 0.01), (12, 100.0)])
def test_absmrg_forward_against_oracle(gpu_ctx, nlay, ptop):
    """Accumulated optical depth (IEMIT=0) against the oracle's ABSINIT/ABSMRG,
    the 4-point regrid and its end-of-data averaging included."""
    cfg = configs.config1(nlines=3000)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    run = abi.make_run(v1=600.0, v2=700.0, iemit=0, ilblf4=1)
    lays = abi.make_layers(configs.atmosphere(nlay, ptop=ptop))
    od, _ = gpu_ctx.forward(run, abi.make_layers_like(lays))
    ref, _ = O.forward(run, abi.make_layers_like(lays), lh)
    assert len(od) == len(ref)
    check_fp64(od, ref, ("absmrg", nlay))
    # the last points, where ABSMRG averages the old field's last two points
    assert np.max(floored_err(od[-50:], ref[-50:])) < 1e-12


# ---- the reference's MT_CKD table ---------------------------------------------

def test_real_mtckd_continuum_layers(gpu_ctx):
    """H2O self and foreign continuum from the reference's MT_CKD 4.3 file
    (mt_ckd_h2o_module.f90:68-174, contnm.f90:279-311) in the window region,
    continuum only (no lines), every layer of a 12-layer profile, and with
    lines."""
    tab = abi.MtckdHandle(real_mtckd())
    prof = configs.atmosphere(12, ptop=100.0)
    run = abi.make_run(v1=780.0, v2=980.0, iemit=1, ilblf4=1, icntnm=1, tmpbnd=290.0,
                       bndemi=0.98)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    none = configs.gen_lines(8, 5000.0, 5001.0, seed=3)
    for lines in (none, configs.gen_lines(4000, 750.0, 1010.0, seed=23, mols=configs.MOLS)):
        lh = abi.LinesHandle(lines)
        load(gpu_ctx, lh, tab)
        j = run.jrad
        for l, L in enumerate(lays):
            ref, jn = O.layer_od(run, L, lh, tab, jrad=j)
            od, _ = gpu_ctx.layer_od(run, L, jrad=j)
            assert ref.min() > 0
            check_fp64(od, ref, ("mtckd", l))
            j = jn
