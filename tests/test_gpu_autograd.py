"""The adjoint wrapped as a torch.autograd.Function (test harness only).

TOARadiance's forward is the fixed-grid forward model through the C ABI
(lbl_layer_od per layer, then lbl_merge_layer up the profile) as a function
of every layer's temperature and the log column amounts of H2O and O3; its
backward applies the Jacobian rows of lbl_jacobian (LBL_JAC_CENTRAL, the
derivative of that same forward).  The gradient of a random linear
functional of the TOA spectrum, obtained by loss.backward(), is checked
against central finite differences of the functional (0.1 K, 1 % amount
steps, as in the reference's analytic-Jacobian checks): every component
within 1e-3 of the largest component.
"""
import math

import numpy as np
import pytest

from lblrtm_b200 import abi, configs, gpu

pytestmark = pytest.mark.gpu

MOLS = (1, 3)
DT, DQ = 0.1, 0.01


def fixed_grid_forward(ctx, run, lays):
    rad = tr = None
    dv_old = 0.0
    for l in range(len(lays)):
        od, _ = ctx.layer_od(run, lays[l])
        rad, tr = ctx.merge_layer(run, lays[l], l == 0, dv_old, rad, tr, od)
        dv_old = lays[l].dv
    return rad


def with_params(base, t, lnq):
    out = abi.make_layers_like(base)
    for l in range(len(out)):
        out[l].tave = float(t[l])
        for k, m in enumerate(MOLS):
            out[l].wk[m - 1] = float(math.exp(lnq[l, k]))
    return out


def make_function(ctx, run, base):
    import torch

    class TOARadiance(torch.autograd.Function):
        @staticmethod
        def forward(fctx, t, lnq):
            lays = with_params(base, t.detach().cpu().numpy(), lnq.detach().cpu().numpy())
            rad, jac = ctx.jacobian(run, lays, MOLS)
            fctx.save_for_backward(torch.from_numpy(jac))
            return torch.from_numpy(fixed_grid_forward(ctx, run, lays))

        @staticmethod
        def backward(fctx, grad):
            (jac,) = fctx.saved_tensors
            g = torch.einsum("kli,i->kl", jac, grad.to(jac.dtype))
            return g[0], g[1:].T.contiguous()

    return TOARadiance.apply


def test_autograd_gradient_against_central_differences(gpu_ctx):
    import torch

    cfg = configs.config1(nlines=3000)
    gpu_ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    run = abi.make_run(v1=600.0, v2=700.0, iemit=1, ilblf4=1, tmpbnd=290.0, bndemi=0.98)
    base = abi.make_layers(configs.atmosphere(5, ptop=350.0))
    gpu.dv_rule(run, base)  # the grids stay fixed from here on
    t0 = np.array([base[l].tave for l in range(len(base))])
    q0 = np.array([[math.log(base[l].wk[m - 1]) for m in MOLS] for l in range(len(base))])
    f = make_function(gpu_ctx, run, base)
    t = torch.tensor(t0, dtype=torch.float64, requires_grad=True)
    lnq = torch.tensor(q0, dtype=torch.float64, requires_grad=True)
    rad = f(t, lnq)
    w = torch.from_numpy(np.random.default_rng(5).uniform(0.5, 1.5, rad.numel()))
    loss = (w * rad).sum() / rad.numel()
    loss.backward()
    wn = w.numpy()

    def functional(tt, qq):
        return float(np.dot(wn, fixed_grid_forward(gpu_ctx, run, with_params(base, tt, qq))) /
                     rad.numel())

    fd_t = np.zeros(len(t0))
    for l in range(len(t0)):
        tp, tm = t0.copy(), t0.copy()
        tp[l] += DT
        tm[l] -= DT
        fd_t[l] = (functional(tp, q0) - functional(tm, q0)) / (2 * DT)
    h = math.log(1 + DQ) - math.log(1 - DQ)
    fd_q = np.zeros_like(q0)
    for l in range(len(t0)):
        for k in range(len(MOLS)):
            qp, qm = q0.copy(), q0.copy()
            qp[l, k] += math.log(1 + DQ)
            qm[l, k] += math.log(1 - DQ)
            fd_q[l, k] = (functional(t0, qp) - functional(t0, qm)) / h
    gt, gq = t.grad.numpy(), lnq.grad.numpy()
    st, sq = np.max(np.abs(fd_t)), np.max(np.abs(fd_q))
    assert st > 0 and sq > 0
    assert np.max(np.abs(gt - fd_t)) <= 1e-3 * st, (gt, fd_t)
    assert np.max(np.abs(gq - fd_q)) <= 1e-3 * sq, (gq, fd_q)
