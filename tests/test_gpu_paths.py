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
