"""Batched forward and Jacobians (lbl_forward_batch, lbl_adjoint_batch)
through the C ABI.

* The batched forward gathers profiles into groups that fit the device
  budget; with a small lbl_set_memory_limit cap the same profiles run in
  several groups and must give bit-identical spectra, equal to one
  lbl_forward per profile.
* The batched Jacobians against the oracle's restatement of the reference's
  analytic-Jacobian path (EMDT + TDERIVup/QDERIVup rows carried to the top,
  src/xmerge.f90:4406-6144; layer optical-depth derivatives from extra
  OPDPTH runs, src/lblrtm.f90:2855-3067), in both modes, on profiles of
  different layer counts; LBL_JAC_CENTRAL also against lbl_jacobian.
* Channel averaging equals the mean of the full-resolution rows.
* A cap below a profile's need returns LBL_E_NOMEM and leaves the context
  usable; a cap that fits one parameter at a time (recomputing the nominal
  optical depths per chunk) gives the same Jacobians.
"""
import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

MOLS = (1, 3)
RTOL_ROW = 1e-8   # FP64 GPU rows against the FP64 oracle, relative to the row maximum


def profiles_small():
    return [abi.make_layers(configs.atmosphere(n, ptop=p))
            for n, p in ((4, 500.0), (6, 300.0), (3, 600.0))]


@pytest.fixture(scope="module")
def lines3k(gpu_ctx):
    cfg = configs.config1(nlines=3000)
    lh = abi.LinesHandle(cfg["lines"])
    gpu_ctx.upload_lines(lh)
    return lh


def test_forward_batch_groups_identical(gpu_ctx, lines3k):
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    profs = profiles_small() * 3
    gpu_ctx.upload_lines(lines3k)
    one = [gpu_ctx.forward(run, abi.make_layers_like(p)) for p in profs]
    whole = gpu_ctx.forward_batch(run, profs)
    # the work buffers of one profile's forward set the scale of the cap
    gpu_ctx.set_memory_limit(1 << 50)
    gpu_ctx.forward(run, abi.make_layers_like(profs[1]))
    one_profile = gpu_ctx.memory_used()
    gpu_ctx.set_memory_limit(1 << 50)
    bare = gpu_ctx.memory_used()
    gpu_ctx.set_memory_limit(bare + 2 * (one_profile - bare))  # two or three profiles a group
    try:
        split = gpu_ctx.forward_batch(run, profs)
    finally:
        gpu_ctx.set_memory_limit(0)
    for (r1, t1), (rw, tw), (rs, ts) in zip(one, whole, split):
        assert np.array_equal(r1, rw) and np.array_equal(t1, tw)
        assert np.array_equal(r1, rs) and np.array_equal(t1, ts)


def test_forward_batch_device_and_split_precision(gpu_ctx, lines3k):
    import torch
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    profs = profiles_small()
    gpu_ctx.upload_lines(lines3k)
    host = gpu_ctx.forward_batch(run, profs, precision=abi.PREC_SPLIT)
    for p, (rad, _) in zip(profs, host):
        ref, _ = O.forward(run, abi.make_layers_like(p), lines3k)
        dv = p[len(p) - 1].dv
        dbt = np.abs(gpu.brightness_temperature(rad, run.v1, dv)
                     - gpu.brightness_temperature(ref, run.v1, dv))
        assert dbt.max() < 0.01
    assert torch.cuda.is_available()


@pytest.fixture(scope="module", params=[abi.JAC_REFERENCE, abi.JAC_CENTRAL],
                ids=["reference", "central"])
def adj(request, gpu_ctx, lines3k):
    mode = request.param
    run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    profs = [abi.make_layers(configs.atmosphere(n, ptop=p)) for n, p in ((4, 400.0), (3, 600.0))]
    gpu_ctx.upload_lines(lines3k)
    out = gpu_ctx.adjoint_batch(run, profs, MOLS, mode=mode)
    return mode, run, profs, out


def test_adjoint_batch_against_oracle(adj, lines3k):
    mode, run, profs, out = adj
    for p, (rad, jac) in zip(profs, out):
        rref, jref = O.jacobian(run, abi.make_layers_like(p), lines3k, MOLS, mode)
        assert np.max(np.abs(rad - rref) / np.abs(rref)) < 1e-12
        top = np.max(np.abs(jref))
        for k in range(jref.shape[0]):
            for l in range(jref.shape[1]):
                scale = max(np.max(np.abs(jref[k, l])), 1e-12 * top)
                err = np.max(np.abs(jac[k, l] - jref[k, l])) / scale
                assert err < RTOL_ROW, (mode, k, l, err)


def test_adjoint_batch_central_matches_lbl_jacobian(gpu_ctx, adj, lines3k):
    mode, run, profs, out = adj
    if mode != abi.JAC_CENTRAL:
        pytest.skip("central mode only")
    for p, (rad, jac) in zip(profs, out):
        r1, j1 = gpu_ctx.jacobian(run, abi.make_layers_like(p), MOLS)
        assert np.array_equal(rad, r1)
        assert np.array_equal(jac, j1)


def test_adjoint_batch_channel_means(gpu_ctx, adj, lines3k):
    mode, run, profs, out = adj
    gpu_ctx.upload_lines(lines3k)
    dvc = 0.5
    ch = gpu_ctx.adjoint_batch(run, profs, MOLS, mode=mode, dv_chan=dvc)
    for p, (rad, jac), (crad, cjac) in zip(profs, out, ch):
        q = abi.make_layers_like(p)
        dv, _ = gpu.dv_rule(run, q)
        v = run.v1 + dv[-1] * np.arange(len(rad))
        c = np.floor((v - run.v1) / dvc + 1e-12).astype(int)
        n = cjac.shape[2]
        assert n == int((run.v2 - run.v1) / dvc)
        # channels with a grid point within 1e-9 cm-1 of an edge are skipped
        # (the library places points by its panel origins, here by V1 + i DV)
        edge = np.abs((v - run.v1) / dvc - np.round((v - run.v1) / dvc)) * dvc < 1e-9
        for i in range(0, n, 7):
            m = c == i
            if np.any(edge[m]) or np.any(edge[c == i + 1]):
                continue
            assert abs(crad[i] - rad[m].mean()) <= 1e-12 * abs(rad[m].mean())
            want = jac[:, :, m].mean(axis=2)
            assert np.allclose(cjac[:, :, i], want, rtol=1e-12, atol=1e-30)


def test_memory_cap_nomem_then_usable(gpu_ctx, lines3k):
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(configs.atmosphere(6, ptop=300.0))
    gpu_ctx.upload_lines(lines3k)
    ref, _ = gpu_ctx.forward(run, abi.make_layers_like(lays))
    gpu_ctx.set_memory_limit(1 << 50)
    gpu_ctx.set_memory_limit(gpu_ctx.memory_used() + (1 << 20))
    try:
        with pytest.raises(gpu.LblError) as ei:
            gpu_ctx.adjoint_batch(run, [lays], MOLS, mode=abi.JAC_CENTRAL)
        assert ei.value.code == 6  # LBL_E_NOMEM
    finally:
        gpu_ctx.set_memory_limit(0)
    again, _ = gpu_ctx.forward(run, abi.make_layers_like(lays))
    assert np.array_equal(again, ref)


def jac_bytes(nk, nlay, ntot, npts, a):
    """Work space of nk parameters' rows (the library's sizing rule)."""
    rows, low = nk * nlay * npts, nk * max(a, 1) * npts
    return 8 * (nk * ntot + ntot + rows + 2 * low + 4 * npts + nlay) + 16 * 256


def test_jacobian_recompute_per_parameter(gpu_ctx, lines3k):
    """A cap that holds the work space of one parameter but not of two: the
    nominal optical depths are recomputed for each parameter and the rows
    are unchanged."""
    run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    lays = abi.make_layers(configs.atmosphere(4, ptop=400.0))
    gpu_ctx.upload_lines(lines3k)
    full = gpu_ctx.adjoint_batch(run, [lays], MOLS, mode=abi.JAC_REFERENCE)[0]
    dv, _ = gpu.dv_rule(run, abi.make_layers_like(lays))
    ntot = sum(gpu.layer_npts(run, d) for d in dv)
    npts = gpu.layer_npts(run, dv[-1])
    a = max([l for l in range(1, len(dv)) if dv[l] != dv[l - 1]], default=0)
    arena = ntot * 16 + len(dv) * 3000 * 200 + (64 << 20)
    b1 = jac_bytes(1, len(dv), ntot, npts, a)
    b2 = jac_bytes(2, len(dv), ntot, npts, a)
    gpu_ctx.set_memory_limit(1 << 50)
    base = gpu_ctx.memory_used()
    gpu_ctx.set_memory_limit(base + arena + (b1 + b2) // 2)
    try:
        part = gpu_ctx.adjoint_batch(run, [lays], MOLS, mode=abi.JAC_REFERENCE)[0]
    finally:
        gpu_ctx.set_memory_limit(0)
    assert np.array_equal(part[0], full[0])
    assert np.array_equal(part[1], full[1])


def test_forward_batch_graphs_and_direct_launches_agree(gpu_ctx, lines3k, monkeypatch):
    """Each group's device work runs as one captured CUDA graph (default) or
    as direct launches (LBL_BATCH_GRAPHS=0); the spectra are identical, and
    a second call with the same topology reuses the executable graph."""
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    profs = profiles_small() * 2
    gpu_ctx.upload_lines(lines3k)
    gpu_ctx.profile_read()
    g1 = gpu_ctx.forward_batch(run, profs)
    g2 = gpu_ctx.forward_batch(run, profs, precision=abi.PREC_SPLIT)
    stats = gpu_ctx.profile_read()
    assert stats.get("graph_groups", (0, 0, 0))[1] >= 2
    monkeypatch.setenv("LBL_BATCH_GRAPHS", "0")
    d1 = gpu_ctx.forward_batch(run, profs)
    d2 = gpu_ctx.forward_batch(run, profs, precision=abi.PREC_SPLIT)
    for (a, b), (c, d) in zip(g1 + g2, d1 + d2):
        assert np.array_equal(a, c) and np.array_equal(b, d)
