"""lbl_merge_layer_noalloc: the merge step for callers that cannot allocate
device memory (a caching allocator owns the device, or the caller may only
use buffers it already holds).  It must give the same radiance and
transmittance as lbl_merge_layer, which stages its own buffers.

Collected last on purpose (file name), so a run that stops at the first
failure has already run every other test; it also passes alone.
"""
import ctypes as C

import numpy as np
import pytest

from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu


def test_noalloc_merge_matches_merge_layer(gpu_ctx):
    import torch

    cfg = configs.config1(nlines=2000)
    prof = configs.atmosphere(3, ptop=500.0)
    run = abi.make_run(**cfg["run"])
    lays = abi.make_layers(prof)
    gpu.dv_rule(run, lays)
    gpu_ctx.upload_lines(cfg["lines"])
    lib = gpu.load()
    jrad = run.jrad
    ods = []
    for l in range(2):
        od, jrad = gpu_ctx.layer_od(run, lays[l], jrad=jrad)
        ods.append(od)
    # reference entry point (stages its own buffers), two merge steps
    r0, t0 = gpu_ctx.merge_layer(run, lays[0], True, 0.0, None, None, ods[0])
    r1, t1 = gpu_ctx.merge_layer(run, lays[1], False, lays[0].dv, r0, t0, ods[1])
    # allocation-free entry point on device buffers, same two steps in a row
    dev = [torch.from_numpy(o).cuda() for o in ods]
    n0, n1 = len(ods[0]), len(ods[1])
    rad0 = torch.empty(n0, dtype=torch.float64, device="cuda")
    tr0 = torch.empty(n0, dtype=torch.float64, device="cuda")
    rad1 = torch.empty(n1, dtype=torch.float64, device="cuda")
    tr1 = torch.empty(n1, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lays[0]), 1, 0.0, None, None, 0,
                                     P(dev[0]), P(rad0), P(tr0), n0, None)
    assert rc == 0, abi.STATUS.get(rc, rc)
    rc = lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lays[1]), 0, lays[0].dv, P(rad0),
                                     P(tr0), n0, P(dev[1]), P(rad1), P(tr1), n1, None)
    assert rc == 0, abi.STATUS.get(rc, rc)
    for got, want in ((rad0, r0), (tr0, t0), (rad1, r1), (tr1, t1)):
        g = got.cpu().numpy()
        assert np.max(np.abs(g - want) / np.maximum(np.abs(want), 1e-300)) < 1e-12


def test_noalloc_rejects_host_buffers_and_long_layers():
    lib = gpu.load()
    run = abi.make_run(v1=500.0, v2=1500.0, iemit=1, tmpbnd=290.0)
    lay = abi.Layer()
    lay.tave = 250.0
    lay.dv = 1e-5  # 1e8 points: beyond LBL_NOALLOC_MAX_PANELS * 2400
    host = [np.zeros(16) for _ in range(3)]
    H = [C.c_void_p(h.ctypes.data) for h in host]
    assert lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lay), 1, 0.0, None, None, 0,
                                       H[0], H[1], H[2], 16, None) == 1  # LBL_E_ARG: host memory
    import torch
    d = [torch.zeros(16, dtype=torch.float64, device="cuda") for _ in range(3)]
    D = [C.c_void_p(t.data_ptr()) for t in d]
    assert lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lay), 1, 0.0, None, None, 0,
                                       D[0], D[1], D[2], 16, None) == 7  # LBL_E_RANGE: too long


def test_noalloc_rejects_aliased_outputs_and_restores_device(gpu_ctx):
    """Outputs that overlap an input the kernel reads at neighbouring points
    (or each other) are refused before any device work; the caller's current
    device is left as it was."""
    import torch

    lib = gpu.load()
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, tmpbnd=290.0)
    lays = abi.make_layers(configs.atmosphere(2, ptop=500.0))
    gpu.dv_rule(run, lays)
    n0 = gpu.layer_npts(run, lays[0].dv)
    n1 = gpu.layer_npts(run, lays[1].dv)
    big = torch.zeros(4 * (n0 + n1), dtype=torch.float64, device="cuda")
    od = torch.ones(n1, dtype=torch.float64, device="cuda")
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rad_in, tr_in = big[:n0], big[n0:2 * n0]
    before = torch.cuda.current_device()
    # rad_out starting inside rad_in
    rc = lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lays[1]), 0, lays[0].dv,
                                     P(rad_in), P(tr_in), n0, P(od), P(big[n0 // 2:]),
                                     P(big[2 * n0 + 2 * n1:]), n1, None)
    assert rc == 1
    # rad_out and tr_out overlapping
    out = big[2 * n0:]
    rc = lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lays[1]), 0, lays[0].dv,
                                     P(rad_in), P(tr_in), n0, P(od), P(out), P(out[1:]), n1,
                                     None)
    assert rc == 1
    assert torch.cuda.current_device() == before
