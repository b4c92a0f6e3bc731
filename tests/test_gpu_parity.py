"""Parity of the CUDA path with the FP64 oracle (through the C ABI).

Tolerances: optical depth relative error <= 1e-4 (the drop-in bar) and
brightness temperature within 0.01 K; the FP64 path is expected to agree far
more tightly and is also checked at 1e-9 relative where the arithmetic is
the same.
"""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

RTOL_OD = 1e-4
BT_TOL = 0.01


def rel_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


def bt(rad, v1, dv):
    return gpu.brightness_temperature(rad, v1, dv)


@pytest.fixture(scope="module")
def c0(gpu_ctx):
    cfg = configs.config0()
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    return cfg, run, lays, lh


def test_config0_layer_od_fp64(gpu_ctx, c0):
    cfg, run, lays, lh = c0
    od_ref, j_ref = O.layer_od(run, lays[0], lh)
    od, j = gpu_ctx.layer_od(run, lays[0])
    assert j == j_ref
    e = rel_err(od, od_ref)
    assert e.max() < 1e-9, (e.max(), int(e.argmax()))


@pytest.mark.parametrize("dptmin,dptfac", [(0.0, 0.0), (2e-4, 1e-3), (2e-2, 1e-1)])
def test_config0_rejection_thresholds(gpu_ctx, c0, dptmin, dptfac):
    cfg, _, lays, lh = c0
    run = abi.make_run(**cfg["run"], dptmin=dptmin, dptfac=dptfac)
    od_ref, _ = O.layer_od(run, lays[0], lh)
    od, _ = gpu_ctx.layer_od(run, lays[0])
    assert rel_err(od, od_ref).max() < RTOL_OD


def test_config0_no_far_wing(gpu_ctx, c0):
    cfg, _, lays, lh = c0
    run = abi.make_run(**dict(cfg["run"], ilblf4=0))
    od_ref, _ = O.layer_od(run, lays[0], lh)
    od, _ = gpu_ctx.layer_od(run, lays[0])
    assert rel_err(od, od_ref).max() < RTOL_OD


@pytest.fixture(scope="module")
def c1(gpu_ctx):
    cfg = configs.config1(nlines=8000)
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    return cfg, run, lays, lh


@pytest.mark.parametrize("layer", [0, 7, 23, 41, 59])
def test_config1_layers_fp64(gpu_ctx, c1, layer):
    cfg, run, lays, lh = c1
    jrad = 0  # every config-1 layer has V1/XKT < 5
    od_ref, _ = O.layer_od(run, lays[layer], lh, jrad=jrad)
    od, _ = gpu_ctx.layer_od(run, lays[layer], jrad=jrad)
    e = rel_err(od, od_ref)
    assert e.max() < RTOL_OD, (layer, e.max(), int(e.argmax()))


def test_config1_forward_fp64(gpu_ctx, c1):
    cfg, run, lays, lh = c1
    rad_ref, tr_ref = O.forward(run, lays, lh)
    rad, tr = gpu_ctx.forward(run, lays)
    dv = lays[len(lays) - 1].dv
    b_ref, b = bt(rad_ref, run.v1, dv), bt(rad, run.v1, dv)
    assert np.abs(b - b_ref).max() < BT_TOL
    assert rel_err(rad, rad_ref).max() < RTOL_OD
    assert np.abs(tr - tr_ref).max() < 1e-6
