"""Radiance Jacobians (lbl_jacobian) against plain finite differences.

The finite differences perturb one layer's temperature (+-0.1 K) or one
molecule's column amount (+-1 %) and rerun the forward model on fixed layer
grids (lbl_layer_od per layer, then lbl_merge_layer up the profile), which
is the derivative the reference's analytic-Jacobian path defines (layer
optical-depth differences, src/xmerge.f90 TDERIVup/QDERIVup :5786-6144).
lbl_jacobian gets the optical-depth derivatives the same way but carries
them to the top of the atmosphere by hand-written derivatives of the merge,
so the two differ only by the higher-order terms of the finite difference
of the merge itself (third derivative times the squared optical-depth step,
up to a few 1e-4 of a row where a 0.1 K step changes a thick layer's depth
by several percent).

Bar: every Jacobian row within 1e-3 of the largest value of its finite-
difference row (rows of layers hidden below opaque ones: within 1e-6 of the
largest value of any row), and the brightness-temperature change the
Jacobian predicts for the perturbation within 0.01 K of the finite-
difference one.

Two profiles: the 6-layer 1013-300 mb profile as generated (optically thick
near the surface; its two top layers share one grid, so a layer's row is
carried to the top by the transmittance product) and the same with 1 % of
the absorber amounts (every layer visible; the grid changes at every layer,
so every row is carried through the interpolation between grids).
"""
import math

import numpy as np
import pytest

from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

RTOL_ROW = 1e-3
BT_TOL = 0.01
DT = 0.1
DQ = 0.01
MOLS = (1, 3)  # H2O, O3


def fixed_grid_forward(ctx, run, lays, precision=abi.PREC_FP64):
    """TOA radiance with the layers' grids held fixed (no DV rule)."""
    rad = tr = None
    dv_old = 0.0
    for l, L in enumerate(lays):
        od, _ = ctx.layer_od(run, L, precision=precision)
        rad, tr = ctx.merge_layer(run, L, l == 0, dv_old, rad, tr, od)
        dv_old = L.dv
    return rad


@pytest.fixture(scope="module", params=[1.0, 0.01], ids=["thick", "thin"])
def case(gpu_ctx, request):
    cfg = configs.config1(nlines=3000)
    prof = configs.atmosphere(6, ptop=300.0)
    prof["wk"] = prof["wk"] * request.param
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    rad, jac = gpu_ctx.jacobian(run, lays, MOLS, precision=abi.PREC_FP64)
    return run, lays, rad, jac, lh


def perturbed(lays, l, k, sign):
    out = abi.make_layers_like(lays)
    if k == 0:
        out[l].tave += sign * DT
    else:
        out[l].wk[MOLS[k - 1] - 1] *= 1.0 + sign * DQ
    return out


def test_jacobian_forward_matches(gpu_ctx, case):
    run, lays, rad, jac, _ = case
    ref, _ = gpu_ctx.forward(run, lays)
    assert np.max(np.abs(rad - ref) / np.abs(ref)) < 1e-12


@pytest.mark.parametrize("k", [0, 1, 2])
def test_jacobian_vs_fd(gpu_ctx, case, k):
    run, lays, rad, jac, _ = case
    h = 2 * DT if k == 0 else math.log(1 + DQ) - math.log(1 - DQ)
    fds = []
    for l in range(len(lays)):
        rp = fixed_grid_forward(gpu_ctx, run, perturbed(lays, l, k, +1))
        rm = fixed_grid_forward(gpu_ctx, run, perturbed(lays, l, k, -1))
        fds.append(((rp - rm) / h, rp))
    top = max(np.max(np.abs(fd)) for fd, _ in fds)
    assert top > 0
    for l, (fd, rp) in enumerate(fds):
        row = jac[k, l]
        scale = np.max(np.abs(fd))
        if scale > 1e-6 * top:
            err = np.max(np.abs(row - fd)) / scale
            assert err < RTOL_ROW, (k, l, err)
        else:
            assert np.max(np.abs(row)) <= 1e-6 * top, (k, l)
        # brightness-temperature change for the +perturbation, predicted vs actual
        step = DT if k == 0 else math.log(1 + DQ)
        bt0 = gpu.brightness_temperature(rad, run.v1, lays[len(lays) - 1].dv)
        bt_lin = gpu.brightness_temperature(rad + row * step, run.v1, lays[len(lays) - 1].dv)
        bt_act = gpu.brightness_temperature(rp, run.v1, lays[len(lays) - 1].dv)
        assert np.max(np.abs((bt_lin - bt0) - (bt_act - bt0))) < BT_TOL, (k, l)


def test_jacobian_rejects_bad_arguments(gpu_ctx, case):
    run, lays, _, _, _ = case
    down = abi.make_run(v1=600.0, v2=700.0, iemit=0, ilblf4=1)
    with pytest.raises(gpu.LblError):
        gpu_ctx.jacobian(down, lays, MOLS, precision=abi.PREC_FP64)
    with pytest.raises(gpu.LblError):
        gpu_ctx.jacobian(run, lays, (99,), precision=abi.PREC_FP64)
