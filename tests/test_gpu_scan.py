"""GPU parity of the SCANFN convolution (lbl_scan_spectrum) with the oracle's
restatement: the same compression, the same inputs summed in the same order
for each output point, every product and sum rounded separately, so the
results are compared exactly.  Inputs: a seeded synthetic radiance spectrum
and the TOA radiance of a short forward, host and device buffers, all four
functions, the rectangle and the field-of-view boxes (JFN 5, 6; HWHM the
half angle in degrees), SAMPL given as points per HWHM and as an output
spacing."""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

CASES = [
    (1, 0.25, 0.0, 0),
    (2, 0.5, 6.0, 0),
    (3, 0.3, -0.04, 1),
    (4, 0.8, 0.0, 0),
    (-3, 1.2, 0.0, 0),
    (0, 0.3, 0.0, 0),
    (0, 0.5, -0.07, 1),
    (5, 2.0, -0.1, 0),
    (6, 1.5, 0.0, 1),
]


@pytest.mark.parametrize("jfn,hwhm,sampl,jabs", CASES)
def test_scan_bit_exact(gpu_ctx, jfn, hwhm, sampl, jabs):
    v1, dv = 600.0, 0.0013
    rng = np.random.default_rng(abs(jfn))
    spec = np.exp(-rng.exponential(1.0, 300000))
    sc = abi.make_scan(hwhm=hwhm, v1=640.0, v2=900.0, jfn=jfn, sampl=sampl, jabs=jabs)
    ref, _ = O.scan(sc, spec, v1, dv)
    got = gpu_ctx.scan_spectrum(sc, spec, v1, dv)
    assert len(got) == len(ref)
    assert np.array_equal(got, ref), np.flatnonzero(got != ref)[:10]


def test_scan_device_buffers_and_forward(gpu_ctx):
    import torch
    cfg = configs.config1(nlines=4000)
    gpu_ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(configs.atmosphere(20))
    rad, _ = gpu_ctx.forward(run, lays)
    dv = lays[len(lays) - 1].dv
    sc = abi.make_scan(hwhm=0.25, v1=610.0, v2=690.0, jfn=2)
    ref, _ = O.scan(sc, rad, 600.0, dv)
    d_in = torch.from_numpy(rad).cuda()
    n, _ = gpu.scan_npts(sc, dv)
    d_out = torch.zeros(n, dtype=torch.float64, device="cuda")
    gpu_ctx.scan_spectrum(sc, d_in, 600.0, dv, out=d_out)
    assert np.array_equal(d_out.cpu().numpy(), ref)


@pytest.mark.parametrize("jfn,hwhm,sampl,dv", [(2, 0.5, 0.0, 0.07), (0, 0.6, -0.2, 0.09),
                                              (5, 2.0, -0.1, 0.05), (4, 0.8, 0.0, 0.1)])
def test_scan_coarse_input_bit_exact(gpu_ctx, jfn, hwhm, sampl, dv):
    """A spectrum coarser than DVINT: SCNINT/INTERP onto DVINT (host replay of
    the chunk structure, one GPU thread per chunk carrying P from point to
    point), then the scan, against the oracle's restatement of both."""
    v1 = 600.0
    rng = np.random.default_rng(jfn + 10)
    n = int(400.0 / dv)
    spec = np.exp(-rng.exponential(1.0, n))
    sc = abi.make_scan(hwhm=hwhm, v1=640.0, v2=900.0, jfn=jfn, sampl=sampl)
    ref, _ = O.scan(sc, spec, v1, dv)
    got = gpu_ctx.scan_spectrum(sc, spec, v1, dv)
    assert len(got) == len(ref)
    assert np.array_equal(got, ref), np.flatnonzero(got != ref)[:10]
