"""GPU parity of the paths config 1 does not reach.

* The H2O continuum (CONTNM -> mt_ckd_h2o_absco onto the 1 cm-1 ABSRB grid,
  XINT into R3) and the Van Vleck-Weisskopf image of far-wing lines below
  25 cm-1 (CONVF4 :4014-4024): a 10-250 cm-1 run with 6,000 lines from
  5 cm-1 and a seeded MT_CKD-layout table, every layer against the oracle.
* The many-profile entry point (lbl_forward_batch): profiles of different
  layer counts in one call against one lbl_forward per profile.
"""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-9   # FP64 path against the FP64 oracle, above OD_FLOOR
OD_FLOOR = 1e-9
BT_TOL = 0.01


def floored_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), OD_FLOOR)


@pytest.fixture(scope="module")
def lowband(gpu_ctx):
    lines = configs.gen_lines(6000, 5.0, 260.0, seed=7, mols=configs.MOLS)
    prof = configs.atmosphere(6, ptop=300.0)
    run = abi.make_run(v1=10.0, v2=250.0, iemit=1, ilblf4=1, icntnm=1, tmpbnd=290.0,
                       bndemi=0.98)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(lines)
    ck = abi.MtckdHandle(configs.mtckd_table(2))
    gpu_ctx.upload_lines(lh)
    gpu_ctx.upload_mtckd(ck)
    return run, lays, lh, ck


@pytest.mark.parametrize("layer", range(6))
def test_continuum_and_image_lines_layer_fp64(gpu_ctx, lowband, layer):
    run, lays, lh, ck = lowband
    ref, _ = O.layer_od(run, lays[layer], lh, ck, jrad=0)
    od, _ = gpu_ctx.layer_od(run, lays[layer], jrad=0)
    e = floored_err(od, ref)
    assert e.max() < RTOL_FP64, (layer, e.max(), int(e.argmax()))


def test_continuum_and_image_lines_forward(gpu_ctx, lowband):
    run, lays, lh, ck = lowband
    rad, _ = gpu_ctx.forward(run, lays)
    ref, _ = O.forward(run, lays, lh, ck)
    dv = lays[len(lays) - 1].dv
    dbt = np.abs(gpu.brightness_temperature(rad, run.v1, dv)
                 - gpu.brightness_temperature(ref, run.v1, dv))
    assert dbt.max() < BT_TOL
    assert np.max(np.abs(rad - ref) / np.abs(ref)) < 1e-8


def test_forward_batch_matches_single_profiles(gpu_ctx):
    cfg = configs.config1(nlines=3000)
    gpu_ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    profiles = [abi.make_layers(configs.atmosphere(n, ptop=p))
                for n, p in ((4, 500.0), (6, 300.0), (5, 400.0))]
    out = gpu_ctx.forward_batch(run, profiles)
    for p, (rad, tr) in zip(profiles, out):
        ref, tref = gpu_ctx.forward(run, abi.make_layers_like(p))
        assert len(rad) == len(ref)
        assert np.array_equal(rad, ref)
        assert np.array_equal(tr, tref)


@pytest.mark.parametrize("iemit", [1, 0])
def test_forward_merge_runs_match_layer_by_layer(gpu_ctx, iemit):
    """lbl_forward merges consecutive layers on one grid in one launch; on
    this 70-layer profile the top 39 layers share a grid, so that run is
    split into launches of 32 and 7.  The result must be lbl_merge_layer
    applied layer by layer (optical depths from lbl_layer_od with the JRAD
    chain the forward uses)."""
    cfg = configs.config1(nlines=3000)
    gpu_ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    run = abi.make_run(v1=600.0, v2=700.0, iemit=iemit, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(configs.atmosphere(70))
    dv, _ = gpu.dv_rule(run, lays)
    assert max(sum(1 for d in dv if d == x) for x in set(dv)) > 32
    rad = tr = None
    dv_old = 0.0
    j = run.jrad
    for l in range(len(lays)):
        od, j = gpu_ctx.layer_od(run, lays[l], jrad=j)
        rad, tr = gpu_ctx.merge_layer(run, lays[l], l == 0, dv_old, rad, tr, od)
        dv_old = lays[l].dv
    frad, ftr = gpu_ctx.forward(run, abi.make_layers_like(lays))
    assert len(frad) == len(rad)
    assert np.max(np.abs(frad - rad) / np.abs(rad)) < 1e-12
    assert np.max(np.abs(ftr - tr)) < 1e-12


def coupled_lines(n, v1, v2, seed, frac=0.05):
    """Synthetic lines where a fraction carry line coupling: IFLG=1 (Y, G) or
    IFLG=3 (width coefficients), each followed by its coefficient record
    (IFLG=-1; the four-temperature values packed into the record's fields as
    the reference reads them, LNCOR1 :1039-1061).  Block boundaries never
    split a line from its record."""
    base = configs.gen_lines(n, v1, v2, seed=seed, mols=configs.MOLS)
    rng = np.random.default_rng(seed + 100)
    pick = rng.random(n) < frac
    kind = np.where(rng.random(n) < 0.5, 1, 3)
    recs = {k: [] for k in base}
    for i in range(n):
        for k in base:
            recs[k].append(base[k][i])
        if not pick[i]:
            continue
        recs["iflg"][-1] = int(kind[i])
        amp = 0.05 if kind[i] == 1 else 0.02
        a = rng.uniform(-amp, amp, 4)
        b = rng.uniform(-amp / 10, amp / 10, 4)
        recs["vnu"].append(a[0])
        recs["sp"].append(b[0])
        recs["alfa"].append(a[1])
        recs["epp"].append(b[1])
        recs["mol"].append(np.frombuffer(np.float32(a[2]).tobytes(), dtype=np.int32)[0])
        recs["hwhms"].append(b[2])
        recs["tmpalf"].append(a[3])
        recs["pshift"].append(b[3])
        recs["iflg"].append(-1)
    lines = {k: np.asarray(v, dtype=base[k].dtype) for k, v in recs.items()}
    nrec = len(lines["vnu"])
    bs = [0]
    while bs[-1] < nrec:
        b = min(bs[-1] + 250, nrec)
        if b < nrec and lines["iflg"][b] < 0:
            b -= 1
        bs.append(b)
    lines["block_start"] = np.asarray(bs, dtype=np.int64)
    return lines


@pytest.fixture(scope="module")
def coupled(gpu_ctx):
    lines = coupled_lines(4000, 600.0, 700.0, seed=11)
    prof = configs.atmosphere(6, ptop=300.0)
    run = abi.make_run(v1=610.0, v2=690.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(lines)
    gpu_ctx.upload_lines(lh)
    return run, lays, lh


@pytest.mark.parametrize("layer", range(6))
def test_line_coupling_layer_fp64(gpu_ctx, coupled, layer):
    run, lays, lh = coupled
    ref, _ = O.layer_od(run, lays[layer], lh, jrad=0)
    od, _ = gpu_ctx.layer_od(run, lays[layer], jrad=0)
    e = floored_err(od, ref)
    assert e.max() < RTOL_FP64, (layer, e.max(), int(e.argmax()))


def test_line_coupling_changes_the_spectrum(gpu_ctx, coupled):
    run, lays, lh = coupled
    plain = dict(lh.a)
    keep = plain["iflg"] >= 0
    plain = {k: (v[keep] if k != "block_start" else None) for k, v in plain.items()}
    plain.pop("block_start")
    plain["iflg"] = np.zeros(int(keep.sum()), np.int32)
    gpu_ctx.upload_lines(abi.LinesHandle(plain))
    od0, _ = gpu_ctx.layer_od(run, lays[0], jrad=0)
    gpu_ctx.upload_lines(lh)
    od1, _ = gpu_ctx.layer_od(run, lays[0], jrad=0)
    assert np.max(np.abs(od1 - od0) / np.abs(od0)) > 1e-4


def test_coupling_record_without_line_is_rejected(gpu_ctx):
    bad = configs.gen_lines(600, 600.0, 700.0, seed=12)
    bad["iflg"][10] = -1
    with pytest.raises(gpu.LblError):
        gpu_ctx.upload_lines(abi.LinesHandle(bad))


def test_rayleigh_continuum_matches_oracle():
    """CONTNM's Rayleigh extinction (contnm.f90:955-976) with the H2O table
    zeroed, on both JRAD branches (850 cm-1: V1/XKT < 5, JRAD=0, the
    radiation term applied by RADFNI; 3000 cm-1: JRAD=1), against the oracle."""
    ctx = gpu.Context(0)
    try:
        lines = configs.gen_lines(500, 800.0, 3100.0, seed=11)
        lh = abi.LinesHandle(lines)
        zero = configs.mtckd_table(1)
        zero["self_absco_ref"] = np.zeros_like(zero["self_absco_ref"])
        zero["for_absco_ref"] = np.zeros_like(zero["for_absco_ref"])
        ck = abi.MtckdHandle(zero)
        ctx.upload_lines(lh)
        ctx.upload_mtckd(ck)
        for v1, v2 in ((850.0, 880.0), (3000.0, 3030.0)):
            run = abi.make_run(v1=v1, v2=v2, icntnm=1, ilblf4=1)
            lays = abi.make_layers(configs.atmosphere(20, ptop=300.0))
            gpu.dv_rule(run, lays)
            for l in (0, 10):
                got, jg = ctx.layer_od(run, lays[l])
                ref, jo = O.layer_od(run, lays[l], lh, ck)
                assert jg == jo
                assert np.max(floored_err(got, ref)) <= RTOL_FP64
    finally:
        ctx.close()


def test_downwelling_forward_matches_oracle_and_layer_steps(gpu_ctx):
    """Looking up (IPATHL=3: RADNN IPATH=3, EMIN with the lower level's
    temperature, TMPBND beyond the last layer) on a 40-layer profile: the
    whole-profile forward (merge runs) against the oracle, and against
    lbl_merge_layer applied layer by layer with the last-layer flag."""
    cfg = configs.config1(nlines=4000)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ipathl=3, ilblf4=1, tmpbnd=5800.0,
                       bndemi=1e-5)
    lays = abi.make_layers(configs.atmosphere(40))
    rad_ref, tr_ref = O.forward(run, abi.make_layers_like(lays), lh)
    frad, ftr = gpu_ctx.forward(run, lays)
    assert len(frad) == len(rad_ref)
    assert np.max(floored_err(frad, rad_ref)) <= 1e-7
    assert np.max(np.abs(ftr - tr_ref)) <= 1e-9
    rad = tr = None
    dv_old = 0.0
    j = run.jrad
    for l in range(len(lays)):
        od, j = gpu_ctx.layer_od(run, lays[l], jrad=j)
        flag = (1 if l == 0 else 0) | (2 if l == len(lays) - 1 else 0)
        rad, tr = gpu_ctx.merge_layer(run, lays[l], flag, dv_old, rad, tr, od)
        dv_old = lays[l].dv
    assert np.max(np.abs(frad - rad) / np.abs(rad)) < 1e-12
    assert np.max(np.abs(ftr - tr)) < 1e-12


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_SPLIT])
@pytest.mark.parametrize("path", ["tangent", "reflected"])
def test_tangent_and_reflected_forward_match_oracle_and_layer_steps(gpu_ctx, precision, path):
    """The symmetric tangent path (IPATHL=2, IANT=0: EMINIT crosses the
    tangent layer twice, RADNN IPATH=2 adds each outer layer's near crossing
    and its far crossing at TZL seen through the inner path) and the
    reflected atmosphere (IPATHL=1 with BNDRFL: the reference's IPATHL=-1,
    RADNN IPATH=-10, each layer's downward emission reflected at the
    surface) on a 40-layer profile: the whole-profile forward against the
    oracle (FP64: 1e-8 relative radiance; split: 0.01 K brightness
    temperature), and the FP64 forward against lbl_merge_layer applied
    layer by layer."""
    cfg = configs.config1(nlines=4000)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    if path == "tangent":
        run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ipathl=2, ilblf4=1, tmpbnd=290.0,
                           bndemi=0.98)
    else:
        run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ipathl=1, ilblf4=1, tmpbnd=290.0,
                           bndemi=0.9, bndrfl=0.1)
    lays = abi.make_layers(configs.atmosphere(40))
    rad_ref, tr_ref = O.forward(run, abi.make_layers_like(lays), lh)
    frad, ftr = gpu_ctx.forward(run, lays, precision=precision)
    assert len(frad) == len(rad_ref)
    if precision == abi.PREC_FP64:
        assert np.max(floored_err(frad, rad_ref)) <= 1e-8
        assert np.max(np.abs(ftr - tr_ref)) <= 1e-12
    else:
        dv = lays[len(lays) - 1].dv
        b = gpu.brightness_temperature(frad, run.v1, dv)
        b_ref = gpu.brightness_temperature(rad_ref, run.v1, dv)
        assert np.max(np.abs(b - b_ref)) < 0.01
        return
    rad = tr = None
    dv_old = 0.0
    j = run.jrad
    for l in range(len(lays)):
        od, j = gpu_ctx.layer_od(run, lays[l], jrad=j)
        rad, tr = gpu_ctx.merge_layer(run, lays[l], 1 if l == 0 else 0, dv_old, rad, tr, od)
        dv_old = lays[l].dv
    assert np.max(np.abs(frad - rad) / np.abs(rad)) < 1e-12
    assert np.max(np.abs(ftr - tr)) < 1e-12


def test_co2_o2_n2_continua_match_oracle(gpu_ctx):
    """CONTNM's CO2 continuum (contnm.f90:326-378, FRNCO2 :1295-1349) and
    the O2 and N2 collision-induced bands (:491-584, :745-906) with the H2O
    table zeroed and Rayleigh off: the 667 cm-1 CO2 band, the 2386-2434
    cm-1 band head (temperature-dependent coefficients), the mt_ckd_2.5
    factors above 2000 cm-1, the O2 fundamental, the N2 fundamental and
    rotational band, in JRAD=0 and JRAD=1 layers, against the oracle;
    and with the scales at 0."""
    lines = configs.gen_lines(500, 80.0, 2600.0, seed=12)
    lh = abi.LinesHandle(lines)
    zero = configs.mtckd_table(1)
    zero["self_absco_ref"] = np.zeros_like(zero["self_absco_ref"])
    zero["for_absco_ref"] = np.zeros_like(zero["for_absco_ref"])
    ck = abi.MtckdHandle(zero)
    gpu_ctx.upload_lines(lh)
    gpu_ctx.upload_mtckd(ck)
    # 4300-4400 and 7800-7880: no line within reach (every layer's near and
    # far line ranges empty), the continuum alone
    for v1, v2 in ((640.0, 700.0), (2370.0, 2450.0), (1990.0, 2030.0), (1480.0, 1560.0),
                   (2280.0, 2360.0), (100.0, 160.0), (4300.0, 4400.0), (7800.0, 7880.0)):
        run = abi.make_run(v1=v1, v2=v2, icntnm=1, ilblf4=1, xrayl=0.0)
        lays = abi.make_layers(configs.atmosphere(20, ptop=300.0))
        gpu.dv_rule(run, lays)
        for l in (0, 12, 19):
            for jrad in (0, 1):
                got, jg = gpu_ctx.layer_od(run, lays[l], jrad=jrad)
                ref, jo = O.layer_od(run, lays[l], lh, ck, jrad=jrad)
                assert jg == jo
                assert np.max(floored_err(got, ref)) <= RTOL_FP64, (v1, l, jrad)
    run = abi.make_run(v1=1480.0, v2=1560.0, icntnm=1, ilblf4=0, xrayl=0.0, xco2c=0.0,
                       xo2cn=0.5, xn2cn=0.0)
    lays = abi.make_layers(configs.atmosphere(20, ptop=300.0))
    gpu.dv_rule(run, lays)
    got, _ = gpu_ctx.layer_od(run, lays[5])
    ref, _ = O.layer_od(run, lays[5], lh, ck)
    assert np.max(floored_err(got, ref)) <= RTOL_FP64


def test_near_infrared_continua_match_oracle(gpu_ctx):
    """The N2 collision-induced first overtone (contnm.f90:860-906) and the
    O2 1.27 um band (:543-584) with the H2O table zeroed and Rayleigh off,
    lines present around both ranges, JRAD=0 and JRAD=1 layers, against the
    oracle."""
    lines = configs.gen_lines(800, 4200.0, 8000.0, seed=13)
    lh = abi.LinesHandle(lines)
    zero = configs.mtckd_table(1)
    zero["self_absco_ref"] = np.zeros_like(zero["self_absco_ref"])
    zero["for_absco_ref"] = np.zeros_like(zero["for_absco_ref"])
    ck = abi.MtckdHandle(zero)
    gpu_ctx.upload_lines(lh)
    gpu_ctx.upload_mtckd(ck)
    for v1, v2 in ((4400.0, 4480.0), (7800.0, 7880.0)):
        run = abi.make_run(v1=v1, v2=v2, icntnm=1, ilblf4=1, xrayl=0.0)
        lays = abi.make_layers(configs.atmosphere(20, ptop=300.0))
        gpu.dv_rule(run, lays)
        for l in (0, 19):
            for jrad in (0, 1):
                got, jg = gpu_ctx.layer_od(run, lays[l], jrad=jrad)
                ref, jo = O.layer_od(run, lays[l], lh, ck, jrad=jrad)
                assert jg == jo
                assert np.max(floored_err(got, ref)) <= RTOL_FP64, (v1, l, jrad)
