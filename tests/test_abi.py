"""C ABI checks that need no GPU: the library loads, exports every entry
point declared in include/lblgpu.h, and its host-side functions agree with
the oracle; argument validation returns status codes (no exits)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle_lib as O
from lblrtm_b200 import abi, configs, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "lblgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lbl_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_function():
    lib = gpu.load()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(gpu.SIGNATURES), set(names) - set(gpu.SIGNATURES)


def test_ctx_create_status_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    h = C.c_void_p()
    assert gpu.load().lbl_ctx_create(0, C.byref(h)) == 11  # LBL_E_NODEVICE


@pytest.mark.parametrize("cfgf", [configs.config0, configs.config1])
def test_dv_rule_and_npts_match_oracle(cfgf):
    cfg = cfgf()
    run = abi.make_run(**cfg["run"])
    a = abi.make_layers(cfg["profile"])
    b = abi.make_layers(cfg["profile"])
    dv_g, it_g = gpu.dv_rule(run, a)
    dv_o, it_o = O.dv_rule(run, b)
    assert np.array_equal(dv_g, dv_o) and np.array_equal(it_g, it_o)
    for d in dv_g[::7]:
        assert gpu.layer_npts(run, d) == O.npts(run, d)


def test_dv_rule_rejects_steep_profile():
    run = abi.make_run(v1=500.0, v2=1500.0, iemit=1)
    lays = abi.make_layers(configs.atmosphere(6))  # 5 decades in 6 layers
    rc = gpu.load().lbl_dv_rule(C.byref(run), lays, len(lays))
    assert rc == 7  # LBL_E_RANGE ('PATH; ISTOP EQ 1')
    assert gpu.load().lbl_dv_rule(C.byref(run), lays, 0) == 1


def test_brightness_temperature_matches_oracle():
    v1, dv = 600.0, 0.01
    rad = 1e-6 * (1.0 + 0.1 * np.sin(np.arange(1000) / 37.0))
    bt = gpu.brightness_temperature(rad, v1, dv)
    L = O.lib()
    for i in (0, 511, 999):
        assert abs(bt[i] - L.orc_brightness_temperature(v1 + i * dv, rad[i])) < 1e-10


def test_layer_npts_invalid():
    run = abi.make_run(v1=600.0, v2=500.0)
    assert gpu.layer_npts(run, 0.01) == -1


def test_noalloc_rejects_bad_iemit_before_device_work():
    """IEMIT other than 0 or 1 is refused before any CUDA call (so the GPU
    never sees the emission branch with a NULL transmittance output)."""
    lib = gpu.load()
    lay = abi.Layer()
    lay.tave = 250.0
    lay.dv = 0.01
    buf = [np.zeros(8) for _ in range(2)]
    P = [C.c_void_p(b.ctypes.data) for b in buf]
    for iemit in (2, -1):
        run = abi.make_run(v1=600.0, v2=700.0, iemit=iemit)
        assert lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lay), 1, 0.0, None, None,
                                           0, P[0], P[1], None, 8, None) == 1
    run = abi.make_run(v1=-5.0, v2=700.0, iemit=0)
    assert lib.lbl_merge_layer_noalloc(0, C.byref(run), C.byref(lay), 1, 0.0, None, None, 0,
                                       P[0], P[1], None, 8, None) == 1


def test_tangent_path_needs_lower_level_temperature():
    """IPATHL=2 radiates each layer's far crossing at TZL: the DV rule (run
    by every forward before any device work) rejects a layer without it."""
    run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ipathl=2)
    lays = abi.make_layers(configs.atmosphere(6, ptop=300.0))
    gpu.dv_rule(run, lays)
    lays[3].tzl = 0.0
    with pytest.raises(gpu.LblError) as e:
        gpu.dv_rule(run, lays)
    assert e.value.code == 1  # LBL_E_ARG


def test_reflected_atmosphere_needs_lower_level_temperature():
    """IPATHL=1 with BNDRFL > 0 is the reflected atmosphere, whose layers
    radiate downward at TZL: the DV rule (run by every forward before any
    device work) rejects a layer without it, and accepts it without BNDRFL."""
    run = abi.make_run(v1=600.0, v2=650.0, iemit=1, ipathl=1)
    lays = abi.make_layers(configs.atmosphere(6, ptop=300.0))
    lays[2].tzl = 0.0
    gpu.dv_rule(run, lays)
    run.bndrfl = 0.2
    with pytest.raises(gpu.LblError) as e:
        gpu.dv_rule(run, lays)
    assert e.value.code == 1  # LBL_E_ARG
