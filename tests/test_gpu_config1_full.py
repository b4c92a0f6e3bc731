"""The benchmarked workload itself against the FP64 oracle: the 60-layer
atmosphere with its 50,000 lines over 500-1500 cm-1 (1.69e8 layer points),
every layer's optical depth and the upwelling TOA forward, in plain FP64 and
in the FP32/FP64-split form, through the C ABI.

Bars: FP64 layer optical depth within 1e-9 relative of the oracle (the same
arithmetic in the same order; what is left is the order of the far-wing
and near-wing sums inside a point), FP64 radiance within 1e-9 relative;
the split form within the drop-in bar, 1e-4 relative optical depth (depths
below 1e-9 compared in absolute terms) and 0.01 K brightness temperature.
The max and RMS errors are printed for the record (pytest -s)."""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-9
RTOL_OD = 1e-4
OD_FLOOR = 1e-9
BT_TOL = 0.01


@pytest.fixture(scope="module")
def full(gpu_ctx):
    cfg = configs.config1()
    assert len(cfg["lines"]["vnu"]) == 50000
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    rad_ref, tr_ref = O.forward(run, lays, lh)
    return run, lays, lh, rad_ref, tr_ref


def _layer_errors(gpu_ctx, run, lays, lh, precision):
    worst, sq, n = (0.0, -1, -1), 0.0, 0
    for layer in range(len(lays)):
        # every layer of this atmosphere has V1/XKT < 5: JRAD = 0 throughout
        od_ref, _ = O.layer_od(run, lays[layer], lh, jrad=0)
        od, _ = gpu_ctx.layer_od(run, lays[layer], jrad=0, precision=precision)
        floor = OD_FLOOR if precision == abi.PREC_SPLIT else 1e-300
        e = np.abs(od - od_ref) / np.maximum(np.abs(od_ref), floor)
        if e.max() > worst[0]:
            worst = (float(e.max()), layer, int(e.argmax()))
        sq += float(np.sum(e * e))
        n += e.size
    return worst, (sq / n) ** 0.5


def test_every_layer_fp64(gpu_ctx, full):
    run, lays, lh, _, _ = full
    worst, rms = _layer_errors(gpu_ctx, run, lays, lh, abi.PREC_FP64)
    print(f"config-1 50k FP64 layer OD rel: max {worst[0]:.3e} (layer {worst[1]}), rms {rms:.3e}")
    assert worst[0] < RTOL_FP64, worst


def test_every_layer_split(gpu_ctx, full):
    run, lays, lh, _, _ = full
    worst, rms = _layer_errors(gpu_ctx, run, lays, lh, abi.PREC_SPLIT)
    print(f"config-1 50k split layer OD rel: max {worst[0]:.3e} (layer {worst[1]}), rms {rms:.3e}")
    assert worst[0] < RTOL_OD, worst


@pytest.mark.parametrize("precision", [abi.PREC_FP64, abi.PREC_SPLIT])
def test_forward(gpu_ctx, full, precision):
    run, lays, lh, rad_ref, tr_ref = full
    rad, tr = gpu_ctx.forward(run, abi.make_layers_like(lays), precision=precision)
    dv = lays[len(lays) - 1].dv
    b_ref = gpu.brightness_temperature(rad_ref, run.v1, dv)
    b = gpu.brightness_temperature(rad, run.v1, dv)
    db = np.abs(b - b_ref)
    erad = np.abs(rad - rad_ref) / np.abs(rad_ref)
    etr = np.abs(tr - tr_ref)
    print(f"config-1 50k forward prec={precision}: BT max {db.max():.3e} K rms "
          f"{np.sqrt(np.mean(db * db)):.3e} K, rad rel max {erad.max():.3e}, "
          f"tr abs max {etr.max():.3e}")
    assert db.max() < BT_TOL
    assert etr.max() < 1e-6
    if precision == abi.PREC_FP64:
        assert erad.max() < RTOL_FP64
