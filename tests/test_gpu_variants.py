"""Every variant of the fused panel kernel (records staged 32 or 64 at a
time, four or five CTAs per SM) and of the far-wing kernel (adders per
window, deciding warps) writes the same optical depths: the same line
shapes summed in the same order at every grid point.  LBL_PANEL_VARIANT /
LBL_FAR_VARIANT fix the autotuner's choice for a new context; the whole
60-layer forward (70,000 panels, above the tuning threshold) is compared bit
for bit, and against the oracle."""
import os

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    cfg = configs.config1(nlines=8000)
    lh = abi.LinesHandle(cfg["lines"])
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    gpu.dv_rule(run, lays)
    return cfg, lh, run, lays


def _forward(case, variant, precision, far=0):
    """Forward and one layer with the panel variant fixed (and the far-wing
    variant, so that nothing else depends on the autotuner's timing)."""
    cfg, lh, run, lays = case
    keys = {"LBL_PANEL_VARIANT": str(variant), "LBL_FAR_VARIANT": str(far)}
    old = {k: os.environ.get(k) for k in keys}
    os.environ.update(keys)
    ctx = gpu.Context(0)
    try:
        ctx.upload_lines(lh)
        rad, tr = ctx.forward(run, abi.make_layers_like(lays), precision=precision)
        od, _ = ctx.layer_od(run, lays[0], jrad=0, precision=precision)
    finally:
        ctx.close()
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    return rad, tr, od


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_SPLIT])
def test_panel_variants_identical(case, precision):
    ref = _forward(case, 0, precision)
    for v in (1, 2):
        got = _forward(case, v, precision)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), (v, precision)
    if precision == abi.PREC_FP64:
        cfg, lh, run, lays = case
        od_ref, _ = O.layer_od(run, lays[0], lh, jrad=0)
        assert np.max(np.abs(ref[2] - od_ref) / np.abs(od_ref)) < 1e-9


def test_far_wing_variants_fp64_identical(case):
    """The far-wing variants (adders per window and deciding warps) sum every
    window point line by line in the same order in FP64."""
    ref = _forward(case, 0, abi.PREC_FP64, far=0)
    for f in (1, 2):
        got = _forward(case, 0, abi.PREC_FP64, far=f)
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), f


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_SPLIT])
def test_repeated_forward_identical(case, precision):
    """A context's first forward (which runs the autotuner on its batch) and
    its later forwards give the same result bit for bit, in both forms: the
    far wing's batch keeps the chosen variant's result, and the merge pairs
    its points at absolute positions whatever the launch's range."""
    cfg, lh, run, lays = case
    for k in ("LBL_PANEL_VARIANT", "LBL_FAR_VARIANT"):
        assert k not in os.environ
    ctx = gpu.Context(0)
    try:
        ctx.upload_lines(lh)
        outs = [ctx.forward(run, abi.make_layers_like(lays), precision=precision)
                for _ in range(3)]
    finally:
        ctx.close()
    for rad, tr in outs[1:]:
        assert np.array_equal(rad, outs[0][0])
        assert np.array_equal(tr, outs[0][1])
