"""GPU parity of PNLINT (src/oprop.f90:1564-1806): the layer optical depth
re-gridded to DVOUT through lbl_pnlint, bit for bit against the oracle's
restatement of the reference's streaming loop on the same input.

The kernel and the oracle both round every product and sum of label 30
separately, so the results are compared exactly (tolerance 0): a different
interpolation coordinate, JP bin or panel assignment would show as a
mismatch.  Inputs: seeded random spectra over multi-panel layers at ratios
that put output panel ends at every offset inside the input panels, host and
device buffers, and a real layer optical depth from lbl_layer_od re-gridded
to the finest layer's DV (the IOD=3 common grid)."""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

CASES = [
    # v1, v2, dv, dvout
    (600.0, 700.0, 0.01, 0.0025),
    (600.0, 700.0, 0.01, 0.0037),
    (600.0, 700.0, 0.01, 0.00999),
    (500.0, 1500.0, 0.0123, 0.0041),
    (500.0, 1500.0, 0.00251, 0.000250977),
    (999.5, 1000.5, 0.002, 0.00099),
    (10.0, 11.0, 0.01, 0.01),
    (700.0, 701.7, 0.0011, 0.00109999),
    (650.0, 2500.0, 0.0513, 0.00731),
]


@pytest.mark.parametrize("v1,v2,dv,dvout", CASES)
def test_pnlint_bit_exact(gpu_ctx, v1, v2, dv, dvout):
    run = abi.make_run(v1=v1, v2=v2)
    n = gpu.layer_npts(run, dv)
    rng = np.random.default_rng(int(dv * 1e6) % 1000)
    od = np.exp(rng.normal(0.0, 2.0, n))
    ref = O.pnlint(run, dv, dvout, od)
    got = gpu_ctx.pnlint(run, dv, dvout, od)
    assert len(got) == len(ref)
    assert np.array_equal(got, ref), np.flatnonzero(got != ref)[:10]


def test_pnlint_device_buffers(gpu_ctx):
    import torch
    run = abi.make_run(v1=600.0, v2=700.0)
    dv, dvout = 0.01, 0.0037
    n = gpu.layer_npts(run, dv)
    od = np.random.default_rng(3).uniform(0.0, 5.0, n)
    ref = O.pnlint(run, dv, dvout, od)
    d_in = torch.from_numpy(od).cuda()
    d_out = torch.zeros(len(ref), dtype=torch.float64, device="cuda")
    gpu_ctx.pnlint(run, dv, dvout, d_in, out=d_out)
    assert np.array_equal(d_out.cpu().numpy(), ref)


def test_pnlint_layer_od_to_common_grid(gpu_ctx):
    cfg = configs.config1(nlines=8000)
    gpu_ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(cfg["profile"])
    dvs, _ = gpu.dv_rule(run, lays)
    dvout = dvs[-1]
    for l in (0, 20, 45):
        od, _ = gpu_ctx.layer_od(run, lays[l])
        ref = O.pnlint(run, dvs[l], dvout, od)
        got = gpu_ctx.pnlint(run, dvs[l], dvout, od)
        assert np.array_equal(got, ref)


def test_pnlint_rejects_bad_sizes(gpu_ctx):
    run = abi.make_run(v1=600.0, v2=700.0)
    n = gpu.layer_npts(run, 0.01)
    with pytest.raises(gpu.LblError):
        gpu_ctx.pnlint(run, 0.01, 0.005, np.zeros(n - 1))
    with pytest.raises(gpu.LblError):
        gpu_ctx.pnlint(run, 0.01, 0.02, np.zeros(n))
