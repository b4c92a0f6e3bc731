"""ctypes binding of the CPU FP64 oracle (oracle/_build/liblbl_oracle.so).

Test infrastructure only: the tests, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use it as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from lblrtm_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def lib(variant=""):
    global _LIB
    path = os.path.join(ROOT, "oracle", "_build", f"liblbl_oracle{variant}.so")
    if _LIB is None or variant:
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_last_error.restype = C.c_char_p
        L.orc_layer_npts.restype = C.c_int64
        L.orc_layer_npts.argtypes = [C.POINTER(abi.Run), C.c_double]
        L.orc_planck.restype = C.c_double
        L.orc_planck.argtypes = [C.c_double, C.c_double]
        L.orc_radfn.restype = C.c_double
        L.orc_radfn.argtypes = [C.c_double, C.c_double]
        L.orc_brightness_temperature.restype = C.c_double
        L.orc_brightness_temperature.argtypes = [C.c_double, C.c_double]
        if variant:
            return L
        _LIB = L
    return _LIB


def check(rc, L=None):
    if rc != 0:
        msg = (L or lib()).orc_last_error().decode()
        raise RuntimeError(f"oracle: {abi.STATUS.get(rc, rc)}: {msg}")


def dv_rule(run, layers):
    check(lib().orc_dv_rule(C.byref(run), layers, len(layers)))
    return np.array([l.dv for l in layers]), np.array([l.itype for l in layers])


def npts(run, dv):
    return int(lib().orc_layer_npts(C.byref(run), C.c_double(dv)))


def layer_od(run, layer, lines_h, mtckd_h=None, jrad=None):
    n = npts(run, layer.dv)
    od = np.zeros(n)
    j = C.c_int32(run.jrad if jrad is None else jrad)
    ck = C.byref(mtckd_h.struct) if mtckd_h is not None else None
    check(lib().orc_layer_od(C.byref(run), C.byref(layer), C.byref(lines_h.struct), ck,
                             C.byref(j), od.ctypes.data_as(C.POINTER(C.c_double)),
                             C.c_int64(n)))
    return od, j.value


def forward(run, layers, lines_h, mtckd_h=None, variant=""):
    L = lib(variant) if variant else lib()
    check(L.orc_dv_rule(C.byref(run), layers, len(layers)), L)
    L.orc_layer_npts.restype = C.c_int64
    n = int(L.orc_layer_npts(C.byref(run), C.c_double(layers[len(layers) - 1].dv)))
    rad = np.zeros(n)
    tr = np.zeros(n)
    ck = C.byref(mtckd_h.struct) if mtckd_h is not None else None
    check(L.orc_forward(C.byref(run), layers, len(layers), C.byref(lines_h.struct), ck,
                        rad.ctypes.data_as(C.POINTER(C.c_double)),
                        tr.ctypes.data_as(C.POINTER(C.c_double)), C.c_int64(n)), L)
    return rad, tr


def merge_layer(run, layer, first, dv_old, rad_in, tr_in, od):
    n_new = len(od)
    rad = np.zeros(n_new)
    tr = np.zeros(n_new)
    P = C.POINTER(C.c_double)
    ri = rad_in.ctypes.data_as(P) if rad_in is not None else None
    ti = tr_in.ctypes.data_as(P) if tr_in is not None else None
    check(lib().orc_merge_layer(C.byref(run), C.byref(layer), int(first), C.c_double(dv_old),
                                ri, ti, C.c_int64(0 if rad_in is None else len(rad_in)),
                                od.ctypes.data_as(P), rad.ctypes.data_as(P),
                                tr.ctypes.data_as(P), C.c_int64(n_new)))
    return rad, tr


def shape_table(which):
    out = np.zeros(2601)
    lib().orc_shape_table(which, out.ctypes.data_as(C.POINTER(C.c_double)), 2601)
    return out


def tips_scor(mol, iso, t):
    s = C.c_double()
    check(lib().orc_tips_scor(mol, iso, C.c_double(t), C.byref(s)))
    return s.value


def jacobian(run, layers, lines_h, mols, mode, mtckd_h=None):
    """TOA radiance and Jacobian rows (1 + len(mols), nlay, npts) of the
    oracle's analytic-Jacobian restatement (mode 1: the reference's
    definitions; mode 0: central differences)."""
    L = lib()
    check(L.orc_dv_rule(C.byref(run), layers, len(layers)))
    n = npts(run, layers[len(layers) - 1].dv)
    nl = len(layers)
    rad = np.zeros(n)
    jac = np.zeros((1 + len(mols), nl, n))
    m = (C.c_int * max(len(mols), 1))(*mols)
    ck = C.byref(mtckd_h.struct) if mtckd_h is not None else None
    P = C.POINTER(C.c_double)
    check(L.orc_jacobian(C.byref(run), layers, nl, C.byref(lines_h.struct), ck, m, len(mols),
                         int(mode), rad.ctypes.data_as(P), jac.ctypes.data_as(P), C.c_int64(n)))
    return rad, jac


def pnlint(run, dv, dvout, od):
    """PNLINT re-grid of a layer optical depth (oracle restatement)."""
    L = lib()
    od = np.ascontiguousarray(od, dtype=np.float64)
    n = C.c_int64(0)
    args = [C.byref(run), C.c_double(dv), C.c_double(dvout), od.ctypes.data_as(C.POINTER(C.c_double)),
            C.c_int64(len(od))]
    check(L.orc_pnlint(*args, None, C.c_int64(0), C.byref(n)))
    out = np.zeros(n.value)
    check(L.orc_pnlint(*args, out.ctypes.data_as(C.POINTER(C.c_double)), C.c_int64(len(out)),
                       C.byref(n)))
    return out


def scan(sc, spec, v1_in, dv_in):
    """SCANFN convolution (oracle restatement)."""
    L = lib()
    spec = np.ascontiguousarray(spec, dtype=np.float64)
    n = C.c_int64(0)
    dvo = C.c_double(0.0)
    P = C.POINTER(C.c_double)
    args = [C.byref(sc), spec.ctypes.data_as(P), C.c_int64(len(spec)), C.c_double(v1_in),
            C.c_double(dv_in)]
    check(L.orc_scan(*args, None, C.c_int64(0), C.byref(n), C.byref(dvo)))
    out = np.zeros(n.value)
    check(L.orc_scan(*args, out.ctypes.data_as(P), C.c_int64(len(out)), C.byref(n), C.byref(dvo)))
    return out, dvo.value


def scnint(spec, v1_in, dv_in, dvo):
    """SCNINT/INTERP (oracle restatement): spec onto the spacing dvo."""
    L = lib()
    spec = np.ascontiguousarray(spec, dtype=np.float64)
    P = C.POINTER(C.c_double)
    num = int((len(spec) - 1) * dv_in / dvo + 0.5) + 1
    out = np.zeros(num + 2400)
    n = C.c_int64(0)
    check(L.orc_scnint(spec.ctypes.data_as(P), C.c_int64(len(spec)), C.c_double(v1_in),
                       C.c_double(dv_in), C.c_double(dvo), out.ctypes.data_as(P),
                       C.c_int64(len(out)), C.byref(n)))
    return out[:n.value]
