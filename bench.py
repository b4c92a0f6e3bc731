#!/usr/bin/env python
"""Benchmark: layer-points/s of the LBLRTM layer optical-depth + merge path.

Workload (one "step"): the 60-layer upwelling forward of the config-1
atmosphere -- 50,000 seeded synthetic lines of H2O/CO2/O3/CH4 over
500-1500 cm-1, DV rule, per-layer optical depth (line shapes, far wing,
panel combination, radiation term) and the bottom-up radiance merge to the
top-of-atmosphere spectrum.  value = layer points processed per second
(sum over layers of the points on each layer's own grid), whole job.

Arms:
  default           the CUDA library through its C ABI (lblrtm_b200.gpu)
  --impl reference  the reference algorithm's CPU restatement (FP64 oracle,
                    the Fortran reference cannot be built here), one forward
                    per host core in parallel

Multi-GPU (torchrun): each rank runs its own replica of the workload (the
path shards by profile; there is no data-path collective); time is the max
over ranks.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lblrtm_b200 import abi, configs  # noqa: E402

METRIC = "layer-pts/s fwd; Jacobians/s adjoint vs plain FD, 1 B200, <=0.01 K BT err"
UNIT = "layer-points/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# nominal vector pipes of a B200 (148 SMs, 128 FP32 / 64 FP64 lanes per SM)
N_SM, FP32_LANES, FP64_LANES = 148, 128, 64
F4_FLOPS = 8      # algorithmic flops per far-wing line-point evaluation
NEAR_FLOPS = 13   # per near-wing point triple (R1+R2+R3)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "split"])
    p.add_argument("--nlines", type=int, default=50000)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-workers", type=int, default=0)
    p.add_argument("--no-jacobian", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-precision", action="store_true")
    p.add_argument("--batch-profiles", type=int, default=256)
    return p.parse_args()


WORKLOAD = ("config1: 60 layers, 4 absorbers (H2O, CO2, O3, CH4), {nlines:,} lines, "
            "500-1500 cm-1, upwelling TOA radiance")


def workload(nlines):
    cfg = configs.config1(nlines=nlines)
    run = abi.make_run(**cfg["run"])
    layers = abi.make_layers(cfg["profile"])
    return cfg, run, layers


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def layer_points(run, layers, npts_fn):
    return sum(npts_fn(run, layers[i].dv) for i in range(len(layers)))


# ---------------------------------------------------------------------------
# CPU arm: the oracle (restated reference), one forward per worker process
# ---------------------------------------------------------------------------

def _cpu_worker(args):
    nlines, variant = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    cfg, run, layers = workload(nlines)
    lh = abi.LinesHandle(cfg["lines"])
    t = time.perf_counter()
    O.forward(run, layers, lh, variant=variant)
    dt = time.perf_counter() - t
    pts = layer_points(run, layers, O.npts)
    return pts, dt


def cpu_run(nlines, workers, reps=1):
    """Wall time of `workers` concurrent oracle forwards (spawned processes)."""
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    O.build()
    ctx = mp.get_context("spawn")
    out = []
    with ctx.Pool(workers) as pool:
        for _ in range(reps):
            t = time.perf_counter()
            res = pool.map(_cpu_worker, [(nlines, "_opt")] * workers)
            wall = time.perf_counter() - t
            pts = sum(r[0] for r in res)
            out.append((pts, wall, max(r[1] for r in res)))
    return out


def default_workers():
    n = os.cpu_count() or 1
    return max(1, min(n, 32))


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    workers = a.cpu_workers or default_workers()
    # every step is one config-1 forward per worker, run concurrently (about
    # 6-7 s of wall time on 16 cores); warm-up and timed steps as asked
    steps = max(1, a.steps)
    warm = max(0, a.warmup)
    res = cpu_run(a.nlines, workers, reps=warm + steps)
    timed = res[-steps:]
    pts = timed[0][0]
    wall = sum(r[1] for r in timed) / steps
    value = pts / wall
    cfgd = {"workload": WORKLOAD.format(nlines=a.nlines), "nlines": a.nlines, "layers": 60,
            "precision": "fp64"}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": wall * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": cfgd,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                         "cpu": cpu_model(),
                         "sample": f"{workers} concurrent config-1 forwards per step "
                                   "(restated reference, C++ FP64 oracle, one process per "
                                   "core)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while timing."""

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for ln in out.strip().splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) >= 9:
                self.rows.append(f)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def merge_bytes_per_step(run, layers, run_max=32):
    """Algorithmic bytes of one forward's merge launches (see the roofline)."""
    from lblrtm_b200 import gpu
    q = abi.make_layers_like(layers)
    dv, _ = gpu.dv_rule(run, q)
    total, l = 0, 0
    while l < len(dv):
        e = l + 1
        while e < len(dv) and e - l < run_max and dv[e] == dv[l]:
            e += 1
        n = gpu.layer_npts(run, dv[l])
        total += 8 * n * (e - l) + 32 * n
        l = e
    return float(total)


def jacobian_leg(ctx, prec, torch):
    """Config 3: temperature, H2O and O3 Jacobians of the TOA radiance for all
    60 layers (3 x 60 rows over 650-2500 cm-1, 200,000 lines), by the
    adjoint-style path (lbl_jacobian) against the plain central-difference
    cost, (2 x 3 x 60 + 1) fixed-grid forwards, timed from one forward."""
    from lblrtm_b200 import gpu
    cfg = configs.config3()
    run = abi.make_run(**cfg["run"])
    layers = abi.make_layers(cfg["profile"])
    mols = list(cfg["jac_mols"])
    ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    dv, _ = gpu.dv_rule(run, layers)
    n = gpu.layer_npts(run, dv[-1])
    rad = torch.empty(n, dtype=torch.float64, device="cuda")
    tr = torch.empty_like(rad)
    jac = torch.empty((1 + len(mols), len(layers), n), dtype=torch.float64, device="cuda")
    # forward (warm, then timed with events)
    ctx.forward(run, layers, precision=prec, rad=rad, tr=tr)
    fwd = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.forward(run, layers, precision=prec, rad=rad, tr=tr)
        e1.record()
        e1.synchronize()
        fwd.append(e0.elapsed_time(e1))
    fwd_ms = sum(fwd) / len(fwd)
    ctx.jacobian(run, layers, mols, precision=prec, rad=rad, jac=jac)
    jt = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.jacobian(run, layers, mols, precision=prec, rad=rad, jac=jac)
        torch.cuda.synchronize()
        jt.append(1e3 * (time.perf_counter() - t0))
    jac_ms = sum(jt) / len(jt)
    # the reference's analytic-Jacobian definitions (one pass at T + 1 K and
    # one per molecule alone) through the batched entry point, full grid
    njr = (1 + len(mols)) * len(layers) * n
    jref = torch.empty(njr, dtype=torch.float64, device="cuda")
    ctx.adjoint_batch(run, [layers], mols, mode=abi.JAC_REFERENCE, precision=prec, rad=rad,
                      jac=jref)
    jr = []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.adjoint_batch(run, [layers], mols, mode=abi.JAC_REFERENCE, precision=prec, rad=rad,
                          jac=jref)
        torch.cuda.synchronize()
        jr.append(1e3 * (time.perf_counter() - t0))
    del jref
    jac_ref_ms = sum(jr) / len(jr)
    nfd = 2 * len(mols) * len(layers) + 2 * len(layers) + 1
    rows = (1 + len(mols)) * len(layers)
    del jac
    return {"config": "config3: 60 layers, 650-2500 cm-1, 200,000 lines; d/dT and d/dln q "
                      "(H2O, O3) per layer", "rows": rows, "npts_top": int(n),
            "ms_per_jacobian_set": jac_ms, "jacobian_sets_per_s": 1e3 / jac_ms,
            "forward_ms": fwd_ms, "fd_forwards": nfd, "fd_ms_estimate": fwd_ms * nfd,
            "speedup_vs_fd": fwd_ms * nfd / jac_ms,
            "ms_per_jacobian_set_reference_mode": jac_ref_ms,
            "speedup_vs_fd_reference_mode": fwd_ms * nfd / jac_ref_ms,
            "timing": "wall clock around the synchronous call (host planning included)"}


C2_SLICES = {"20-45 cm-1 (DV to 8.5e-6, continuum, image lines)": (20.0, 45.0),
             "700-725 cm-1": (700.0, 725.0),
             "2500-2525 cm-1 (JRAD=1 in every layer)": (2500.0, 2525.0)}


def precision_leg(ctx):
    """Config 2, the precision sweep: FP32/FP64-split against plain FP64 on
    25 cm-1 slices of both sub-runs (all 60 layers, 400,000 lines over
    10-3000 cm-1, seeded MT_CKD-layout continuum); max and RMS error of
    every layer's optical depth (relative, above 1e-9), of its
    transmittance, of the total transmittance and of the TOA brightness
    temperature.  The FP64 path agrees with the FP64 oracle to 1e-9 on these
    slices (tests/test_gpu_sweep.py)."""
    from lblrtm_b200 import gpu
    cfg = configs.config2()
    ck = abi.MtckdHandle(cfg["mtckd"])
    ctx.upload_mtckd(ck)
    od_max = od_ss = t_max = t_ss = 0.0
    od_n = t_n = 0
    bt_max = bt_ss = tt_max = 0.0
    bt_n = 0
    per = {}
    for name, (v1, v2) in C2_SLICES.items():
        run = abi.make_run(**cfg["run"], v1=v1, v2=v2)
        lays = abi.make_layers(cfg["profile"])
        gpu.dv_rule(run, lays)
        ctx.upload_lines(abi.LinesHandle(configs.subset_lines(cfg["lines"], v1, v2, margin=30.0)))
        j = run.jrad
        smax = 0.0
        for l in range(len(lays)):
            o64, jn = ctx.layer_od(run, lays[l], jrad=j)
            o32, _ = ctx.layer_od(run, lays[l], jrad=j, precision=abi.PREC_SPLIT)
            j = jn
            e = np.abs(o32 - o64) / np.maximum(np.abs(o64), 1e-9)
            te = np.abs(np.exp(-o32) - np.exp(-o64))
            od_max = max(od_max, float(e.max()))
            smax = max(smax, float(e.max()))
            od_ss += float(np.sum(e * e))
            od_n += e.size
            t_max = max(t_max, float(te.max()))
            t_ss += float(np.sum(te * te))
            t_n += te.size
        r64, tr64 = ctx.forward(run, abi.make_layers_like(lays))
        r32, tr32 = ctx.forward(run, abi.make_layers_like(lays), precision=abi.PREC_SPLIT)
        dv = lays[len(lays) - 1].dv
        be = np.abs(gpu.brightness_temperature(r32, v1, dv) - gpu.brightness_temperature(r64, v1, dv))
        bt_max = max(bt_max, float(be.max()))
        bt_ss += float(np.sum(be * be))
        bt_n += be.size
        tt_max = max(tt_max, float(np.abs(tr32 - tr64).max()))
        per[name] = {"od_rel_max": smax, "bt_max_K": float(be.max()),
                     "dv_top": float(dv), "npts_top": int(len(r64))}
    return {"config": "config2: 400,000 lines 10-3000 cm-1 (strengths 1e-28..1e-18), 60 layers, "
                      "MT_CKD-layout continuum; 25 cm-1 slices of both sub-runs",
            "compared": "FP32/FP64-split against plain FP64 (the FP64 path matches the FP64 "
                        "oracle to 1e-9 on the same slices)",
            "layer_od_rel_max": od_max, "layer_od_rel_rms": (od_ss / od_n) ** 0.5,
            "layer_transmittance_max": t_max, "layer_transmittance_rms": (t_ss / t_n) ** 0.5,
            "total_transmittance_max": tt_max,
            "bt_max_K": bt_max, "bt_rms_K": (bt_ss / bt_n) ** 0.5, "slices": per}


def config2_leg(ctx, torch):
    """Config 2 at full size: both reference-legal sub-runs (10-1505 and
    1505-3000 cm-1) with all 400,000 lines, FP64 and split, timed with CUDA
    events on device buffers."""
    from lblrtm_b200 import gpu
    cfg = configs.config2()
    ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    ctx.upload_mtckd(abi.MtckdHandle(cfg["mtckd"]))
    out = {}
    for prec, pname in ((abi.PREC_FP64, "fp64"), (abi.PREC_SPLIT, "split")):
        pts = 0
        ms = 0.0
        for v1, v2 in cfg["subruns"]:
            run = abi.make_run(**cfg["run"], v1=v1, v2=v2)
            lays = abi.make_layers(cfg["profile"])
            dv, _ = gpu.dv_rule(run, lays)
            n = gpu.layer_npts(run, dv[-1])
            rad = torch.empty(n, dtype=torch.float64, device="cuda")
            tr = torch.empty_like(rad)
            ctx.forward(run, lays, precision=prec, rad=rad, tr=tr)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(2):
                ctx.forward(run, lays, precision=prec, rad=rad, tr=tr)
            e1.record()
            e1.synchronize()
            ms += e0.elapsed_time(e1) / 2
            pts += sum(gpu.layer_npts(run, d) for d in dv)
        out[pname] = {"ms": ms, "layer_points": pts, "layer_points_per_s": pts / (ms / 1e3)}
    out["config"] = "config2: 60 layers, 400,000 lines, sub-runs 10-1505 and 1505-3000 cm-1"
    return out


def batch_leg(ctx, torch, dist, world, rank, nprof=256):
    """Config 4: 256 perturbed profiles of 30-90 layers, 200,000 lines over
    600-2500 cm-1, FP32/FP64-split.  The batched forward (lbl_forward_batch)
    and the batched forward + Jacobians (lbl_adjoint_batch, the reference's
    analytic-Jacobian definitions: d/dT and d/d ln q for H2O and O3 at every
    layer, averaged over 1 cm-1 channels) of this rank's shard of the
    profiles (greedy by layer points, no data-path collective), timed with
    CUDA events, max over ranks.  The plain-FD baseline is the FP64 forward
    per profile times (2 x 3 x layers + 1) forwards, the forward timed on a
    sample of profiles and scaled by layer points; the brightness-
    temperature error is split against FP64 on the same sample."""
    from lblrtm_b200 import dist as shard_mod
    from lblrtm_b200 import gpu
    cfg = configs.config4(nprof=nprof)
    run = abi.make_run(**cfg["run"])
    profs = [abi.make_layers(p) for p in cfg["profiles"]]
    lp = []
    for p in profs:
        dv, _ = gpu.dv_rule(run, abi.make_layers_like(p))
        lp.append(sum(gpu.layer_npts(run, d) for d in dv))
    mine = shard_mod.shard(lp, rank, world)
    sub = [profs[i] for i in mine]
    ctx.upload_lines(abi.LinesHandle(cfg["lines"]))
    mols = list(cfg["jac_mols"])
    npf = sum(gpu.layer_npts(run, gpu.dv_rule(run, abi.make_layers_like(p))[0][-1]) for p in sub)
    rad = torch.empty(npf, dtype=torch.float64, device="cuda")
    tr = torch.empty_like(rad)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def maxr(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # warm-up on a few profiles, then the whole shard once
    ctx.forward_batch(run, sub[:4], precision=abi.PREC_SPLIT)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ctx.forward_batch(run, sub, precision=abi.PREC_SPLIT, rad=rad, tr=tr)
    e1.record()
    e1.synchronize()
    fwd_ms = maxr(e0.elapsed_time(e1))
    barrier()
    nchan = int((run.v2 - run.v1) / 1.0)
    njac = sum((1 + len(mols)) * len(p) * nchan for p in sub)
    crad = torch.empty(len(sub) * nchan, dtype=torch.float64, device="cuda")
    cjac = torch.empty(njac, dtype=torch.float64, device="cuda")
    ctx.adjoint_batch(run, sub[:2], mols, mode=abi.JAC_REFERENCE, dv_chan=1.0,
                      precision=abi.PREC_SPLIT)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ctx.adjoint_batch(run, sub, mols, mode=abi.JAC_REFERENCE, dv_chan=1.0,
                      precision=abi.PREC_SPLIT, rad=crad, jac=cjac)
    e1.record()
    e1.synchronize()
    adj_ms = maxr(e0.elapsed_time(e1))
    barrier()
    # plain FP64 forward on a sample (FD baseline) and the split error there
    sample = list(range(0, nprof, max(1, nprof // 8)))[:8]
    f64_ms, f64_pts, bt_err = 0.0, 0, 0.0
    for i in sample:
        p = profs[i]
        r64, _ = ctx.forward(run, abi.make_layers_like(p))
        n64 = len(r64)
        d64 = torch.empty(n64, dtype=torch.float64, device="cuda")
        t64 = torch.empty_like(d64)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.forward(run, abi.make_layers_like(p), rad=d64, tr=t64)
        e1.record()
        e1.synchronize()
        f64_ms += e0.elapsed_time(e1)
        f64_pts += lp[i]
        r32 = ctx.forward_batch(run, [p], precision=abi.PREC_SPLIT)[0][0]
        dv = gpu.dv_rule(run, abi.make_layers_like(p))[0][-1]
        bt_err = max(bt_err, float(np.abs(gpu.brightness_temperature(r32, run.v1, dv)
                                          - gpu.brightness_temperature(r64, run.v1, dv)).max()))
    ms_per_pt = f64_ms / f64_pts
    np_ = 1 + len(mols)
    fd_ms = sum((2 * np_ * len(profs[i]) + 1) * lp[i] * ms_per_pt for i in range(nprof))
    total_pts = sum(lp)
    return {
        "config": "config4: 256 profiles, 30-90 layers (seeded T and H2O perturbations), "
                  "200,000 lines 600-2500 cm-1, fp32/fp64-split",
        "profiles": nprof, "layers_total": sum(len(p) for p in profs),
        "layer_points_total": int(total_pts),
        "shard": f"{len(mine)} profiles on rank 0 of {world} (greedy by layer points)",
        "forward_ms": fwd_ms, "forward_layer_points_per_s": total_pts / (fwd_ms / 1e3),
        "adjoint_ms": adj_ms, "jacobian_sets_per_s": nprof / (adj_ms / 1e3),
        "jacobian_rows": np_ * sum(len(p) for p in profs),
        "adjoint_mode": "LBL_JAC_REFERENCE (T + 1 K pass, one pass per molecule alone; "
                        "TDERIVup/QDERIVup rows), 1 cm-1 channel means",
        "fd_forwards_per_profile": f"2 x {np_} x layers + 1",
        "fd_ms_estimate": fd_ms, "speedup_vs_fd": fd_ms / adj_ms,
        "fd_basis": f"plain FP64 lbl_forward timed on {len(sample)} profiles, "
                    f"{ms_per_pt * 1e6:.3f} ms per 1e6 layer points",
        "bt_err_split_vs_fp64_max_K": bt_err,
        "timing": "CUDA events around one call over the shard (host planning included), "
                  "max over ranks",
    }


def gpu_arm(a):
    import torch
    from lblrtm_b200 import gpu

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    prec = abi.PREC_FP64 if a.precision == "fp64" else abi.PREC_SPLIT
    cfg, run, layers = workload(a.nlines)
    ctx = gpu.Context(local)
    lines_h = abi.LinesHandle(cfg["lines"])
    ctx.upload_lines(lines_h)
    dv, _ = gpu.dv_rule(run, layers)
    npts_top = gpu.layer_npts(run, dv[-1])
    pts = layer_points(run, layers, gpu.layer_npts)
    rad_d = torch.empty(npts_top, dtype=torch.float64, device="cuda")
    tr_d = torch.empty(npts_top, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(a.warmup):
        ctx.forward(run, layers, precision=prec, rad=rad_d, tr=tr_d)
    warm = ctx.profile_read()
    tuning = {k: {"ms": v[0], "chosen": bool(v[2])} for k, v in warm.items()
              if k.startswith("tune_")}
    ctx.profile(True)
    ctx.profile_read()
    barrier()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1.0)  # evict L2 between steps (outside the timed events)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            ctx.forward(run, layers, precision=prec, rad=rad_d, tr=tr_d)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
    stats = ctx.profile_read()
    ctx.profile(False)
    step_ms = sum(times) / len(times)
    if dist is not None:
        t = torch.tensor([step_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms = float(t.item())
    value = world * pts / (step_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in cfg["lines"].items()}
    pin_np = {k: v.numpy() for k, v in pin.items()}
    rad_h = torch.empty(npts_top, dtype=torch.float64).pin_memory()
    tr_h = torch.empty(npts_top, dtype=torch.float64).pin_memory()
    h2d = sum(v.nbytes for v in pin_np.values()) + C.sizeof(abi.Layer) * len(layers)
    d2h = rad_h.numel() * 8 + tr_h.numel() * 8
    e2e_times = []
    barrier()
    for k in range(a.steps + 1):
        t0 = time.perf_counter()
        ctx.upload_lines(abi.LinesHandle(pin_np))
        ctx.forward(run, layers, precision=prec, rad=rad_h, tr=tr_h)
        torch.cuda.synchronize()
        if k > 0:
            e2e_times.append(time.perf_counter() - t0)
    barrier()
    print("e2e step ms:", [round(1e3 * t, 2) for t in e2e_times], file=sys.stderr)
    e2e_s = sum(e2e_times) / len(e2e_times)
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * pts / e2e_s

    # ---- rooflines ----
    nstep = a.steps
    peaks = json.load(open(PEAKS_FILE)) if os.path.exists(PEAKS_FILE) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    traffic_file = os.path.join(ROOT, "profiles", "traffic_config1.json")
    try:
        traffic_db = json.load(open(traffic_file))
    except (OSError, ValueError):
        traffic_db = {}
    # dominant kernel: the fused near-wing/PANEL kernel, one launch per step;
    # algorithmic bytes = the optical depth it must write (8 B per layer point)
    pn = stats.get("panels", (0.0, 0, 0.0))
    pn_ms = pn[0] / max(pn[1], 1)
    pn_bytes = 8.0 * pts
    pn_gbs = pn_bytes / (pn_ms / 1e3) / 1e9 if pn_ms > 0 else None
    roofline = {
        "bound": "hbm", "kernel": "k_panel_od (CNVFNV sums + XINT + PANEL + RADFNI)",
        "achieved": pn_gbs, "peak": hbm_peak, "unit": "GB/s",
        "frac": (pn_gbs / hbm_peak) if pn_gbs else None,
        "traffic": traffic_db.get("k_panel_od"),
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                          "from an earlier capture recorded in profiles/traffic_config1.json "
                          "(not measured in this run)",
        "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650",
        "work": f"{pn_bytes:.4g} B of optical depth written per launch (8 B x layer points)",
        "launch_ms": pn_ms,
    }
    # far wing: FP pipe roofline (line-point evaluations x 8 flops)
    fw = stats.get("far_wing", (0.0, 0, 0.0))
    fw_ms = fw[0] / max(fw[1], 1)
    evals = fw[2] / nstep
    fw_flops = evals * F4_FLOPS
    lanes = FP64_LANES if prec == abi.PREC_FP64 else FP32_LANES
    peak_tf = N_SM * lanes * 2 * 1965e6 / 1e12
    achieved_tf = fw_flops / (fw_ms / 1e3) / 1e12 if fw_ms > 0 else None
    roof_fw = {
        "bound": "fp64" if prec == abi.PREC_FP64 else "fp32",
        "kernel": "k_far_wing (LBLF4/CONVF4 far wing)",
        "achieved": achieved_tf, "peak": peak_tf, "unit": "TFLOP/s",
        "frac": (achieved_tf / peak_tf) if achieved_tf else None,
        "traffic": traffic_db.get("k_far_wing") if prec == abi.PREC_FP64 else None,
        "peak_source": f"nominal {'FP64' if lanes == 64 else 'FP32'} vector rate: "
                       f"{N_SM} SMs x {lanes} lanes x 2 x 1965 MHz (MEASURED_PEAKS.json "
                       "holds HBM and bf16 only)",
        "work": f"{evals:.4g} line-point evaluations x {F4_FLOPS} flops per launch",
        "launch_ms": fw_ms,
    }
    # HBM roofline of the merge: each launch merges a run of layers on one
    # grid, reading every layer's FP64 optical depth once and the radiance
    # and transmittance below the run (16 B per point) and writing them
    # (16 B per point)
    mg = stats.get("merge", (0.0, 0, 0.0))
    merge_bytes = merge_bytes_per_step(run, layers)
    merge_ms = mg[0] / nstep
    roof_merge = {"bound": "hbm", "kernel": "k_merge_run (EMIN/RADNN over same-grid layers)",
                  "achieved": merge_bytes / (merge_ms / 1e3) / 1e9 if merge_ms > 0 else None,
                  "peak": hbm_peak, "unit": "GB/s",
                  "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback 6650"}
    if roof_merge["achieved"]:
        roof_merge["frac"] = roof_merge["achieved"] / hbm_peak
    launches = sum(v[1] for v in stats.values()) // max(nstep, 1)
    stage_ms = {k: round(v[0] / nstep, 4) for k, v in stats.items()}
    stage_work = {k: v[2] / nstep for k, v in stats.items() if v[2]}
    print("forward step ms", round(step_ms, 3), "stage ms", json.dumps(stage_ms),
          "autotune", json.dumps(tuning), file=sys.stderr, flush=True)

    jleg = None
    if not a.no_jacobian:
        jleg = jacobian_leg(ctx, prec, torch)
    bleg = None
    if not a.no_batch:
        bleg = batch_leg(ctx, torch, dist, world, rank, nprof=a.batch_profiles)
    pleg = c2leg = None
    if not a.no_precision:
        pleg = precision_leg(ctx)
        c2leg = config2_leg(ctx, torch)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        workers = a.cpu_workers or default_workers()
        r = cpu_run(a.nlines, workers, reps=1)[0]
        cpu = {"value": r[0] / r[1], "unit": UNIT, "cores": workers, "kind": "port",
               "cpu": cpu_model(),
               "sample": f"{workers} concurrent config-1 forwards (restated reference, "
                         f"C++ FP64 oracle), wall {r[1]:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == abi.PREC_FP64 else "f32/f64",
            "data": "synthetic (seeded lines and atmosphere)",
            "config": {"workload": WORKLOAD.format(nlines=a.nlines),
                       "nlines": a.nlines, "layers": len(layers),
                       "layer_points_per_step": pts, "precision": a.precision,
                       "l2": "256 MB buffer written between timed steps",
                       "parallelism": f"replica x{world}"},
            "roofline": roofline, "roofline_far_wing": roof_fw, "roofline_merge": roof_merge,
            "stage_ms": stage_ms, "stage_work": stage_work,
            "autotune": tuning or None,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "jacobian": jleg,
            "batch": bleg,
            "precision": pleg,
            "config2": c2leg,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
    else:
        gpu_arm(a)


if __name__ == "__main__":
    main()
