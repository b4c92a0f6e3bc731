"""Python binding of the CUDA library's C ABI (include/lblgpu.h).

The product path: every call goes through lblrtm_b200/_lib/liblblgpu.so.
There is no CPU fallback -- if the library or a CUDA device is missing the
calls raise.
"""
import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "liblblgpu.so")
_LIB = None

P_D = C.POINTER(C.c_double)
P_I32 = C.POINTER(C.c_int32)
P_I64 = C.POINTER(C.c_int64)

# every entry point of include/lblgpu.h with its ctypes signature
SIGNATURES = {
    "lbl_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "lbl_ctx_destroy": (C.c_int, [C.c_void_p]),
    "lbl_last_error": (C.c_char_p, [C.c_void_p]),
    "lbl_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "lbl_lines_upload": (C.c_int, [C.c_void_p, C.POINTER(abi.Lines)]),
    "lbl_lines_load_tape3": (C.c_int, [C.c_void_p, C.c_char_p, P_I64]),
    "lbl_mtckd_upload": (C.c_int, [C.c_void_p, C.POINTER(abi.Mtckd)]),
    "lbl_dv_rule": (C.c_int, [C.POINTER(abi.Run), C.POINTER(abi.Layer), C.c_int32]),
    "lbl_layer_npts": (C.c_int64, [C.POINTER(abi.Run), C.c_double]),
    "lbl_pnlint_npts": (C.c_int64, [C.POINTER(abi.Run), C.c_double, C.c_double]),
    "lbl_scan_npts": (C.c_int64, [C.POINTER(abi.Scan), C.c_double, P_D]),
    "lbl_scan_spectrum": (C.c_int, [C.c_void_p, C.POINTER(abi.Scan), C.c_void_p, C.c_int64,
                                    C.c_double, C.c_double, C.c_void_p, C.c_int64]),
    "lbl_pnlint": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.c_double, C.c_double, C.c_void_p,
                             C.c_int64, C.c_void_p, C.c_int64]),
    "lbl_layer_od": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer), P_I32,
                               C.c_void_p, C.c_int64, C.c_int32]),
    "lbl_merge_layer": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer),
                                  C.c_int32, C.c_double, C.c_void_p, C.c_void_p, C.c_int64,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64]),
    "lbl_forward": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer), C.c_int32,
                              C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]),
    "lbl_forward_batch": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer), P_I32,
                                    C.c_int32, C.c_void_p, C.c_void_p, P_I64, C.c_int64,
                                    C.c_int32]),
    "lbl_jacobian": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer), C.c_int32,
                               P_I32, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32]),
    "lbl_adjoint_batch": (C.c_int, [C.c_void_p, C.POINTER(abi.Run), C.POINTER(abi.Layer), P_I32,
                                    C.c_int32, P_I32, C.c_int32, C.c_int32, C.c_double,
                                    C.c_void_p, P_I64, C.c_int64, C.c_void_p, P_I64, C.c_int64,
                                    C.c_int32]),
    "lbl_brightness_temperature": (C.c_int, [P_D, C.c_int64, C.c_double, C.c_double, P_D]),
    "lbl_merge_layer_noalloc": (C.c_int, [C.c_int, C.POINTER(abi.Run), C.POINTER(abi.Layer),
                                          C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                          C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_int64, C.c_void_p]),
    "lbl_set_memory_limit": (C.c_int, [C.c_void_p, C.c_int64]),
    "lbl_memory_used": (C.c_int64, [C.c_void_p]),
    "lbl_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "lbl_profile_read": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, P_I32]),
}


class StageStat(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("ms", C.c_double), ("launches", C.c_int64),
                ("work", C.c_double)]


class LblError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.STATUS.get(code, code)}: {msg}")
        self.code = code


def load():
    """Load the library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built; run python -m lblrtm_b200.build")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _LIB = lib
    return _LIB


def _ptr(a):
    """Data pointer of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)


def dv_rule(run, layers):
    rc = load().lbl_dv_rule(C.byref(run), layers, len(layers))
    if rc:
        raise LblError(rc, "DV rule")
    return np.array([l.dv for l in layers]), np.array([l.itype for l in layers])


def layer_npts(run, dv):
    return int(load().lbl_layer_npts(C.byref(run), C.c_double(dv)))


def pnlint_npts(run, dv, dvout):
    """Points of the DVOUT grid PNLINT writes for a layer of spacing dv."""
    n = int(load().lbl_pnlint_npts(C.byref(run), C.c_double(dv), C.c_double(dvout)))
    if n < 0:
        raise LblError(-n, f"pnlint_npts: {abi.STATUS.get(-n, -n)}")
    return n


def scan_npts(sc, dv_in):
    """Output points and spacing of a SCANFN convolution for input spacing dv_in."""
    dvo = C.c_double(0.0)
    n = int(load().lbl_scan_npts(C.byref(sc), C.c_double(dv_in), C.byref(dvo)))
    if n < 0:
        raise LblError(-n, f"scan_npts: {abi.STATUS.get(-n, -n)}")
    return n, dvo.value


def brightness_temperature(rad, v1, dv):
    rad = np.ascontiguousarray(rad, dtype=np.float64)
    bt = np.empty_like(rad)
    load().lbl_brightness_temperature(rad.ctypes.data_as(P_D), len(rad), v1, dv,
                                      bt.ctypes.data_as(P_D))
    return bt


class Context:
    """One device context: resident lines and tables, reusable buffers."""

    def __init__(self, device=0):
        self.lib = load()
        h = C.c_void_p()
        rc = self.lib.lbl_ctx_create(device, C.byref(h))
        if rc:
            raise LblError(rc, "lbl_ctx_create")
        self.h = h
        self._keep = []

    def close(self):
        if self.h:
            self.lib.lbl_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            raise LblError(rc, f"{what}: {self.lib.lbl_last_error(self.h).decode()}")

    def profile(self, enable=True):
        self._check(self.lib.lbl_profile(self.h, int(enable)), "profile")

    def profile_read(self):
        """Per-stage {name: (ms, launches, work)} since the last read."""
        buf = (StageStat * 32)()
        n = C.c_int32()
        self._check(self.lib.lbl_profile_read(self.h, buf, 32, C.byref(n)), "profile_read")
        return {buf[i].name.decode(): (buf[i].ms, buf[i].launches, buf[i].work)
                for i in range(n.value)}

    def set_memory_limit(self, nbytes):
        """Cap the device memory this context may hold (0: no cap)."""
        self._check(self.lib.lbl_set_memory_limit(self.h, int(nbytes)), "set_memory_limit")

    def memory_used(self):
        return int(self.lib.lbl_memory_used(self.h))

    def set_stream(self, stream_ptr):
        self._check(self.lib.lbl_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    def upload_lines(self, lines):
        lh = lines if isinstance(lines, abi.LinesHandle) else abi.LinesHandle(lines)
        self._check(self.lib.lbl_lines_upload(self.h, C.byref(lh.struct)), "lines_upload")

    def load_tape3(self, path):
        n = C.c_int64()
        self._check(self.lib.lbl_lines_load_tape3(self.h, path.encode(), C.byref(n)), "tape3")
        return n.value

    def upload_mtckd(self, table):
        th = table if isinstance(table, abi.MtckdHandle) else abi.MtckdHandle(table)
        self._check(self.lib.lbl_mtckd_upload(self.h, C.byref(th.struct)), "mtckd_upload")

    def layer_od(self, run, layer, jrad=None, precision=abi.PREC_FP64, out=None):
        n = layer_npts(run, layer.dv)
        od = np.zeros(n) if out is None else out
        j = C.c_int32(run.jrad if jrad is None else jrad)
        self._check(self.lib.lbl_layer_od(self.h, C.byref(run), C.byref(layer), C.byref(j),
                                          _ptr(od), n, precision), "layer_od")
        return od, j.value

    def pnlint(self, run, dv, dvout, od, out=None):
        """PNLINT: a layer optical depth (numpy or CUDA tensor) on its own
        grid re-gridded to DVOUT."""
        n = pnlint_npts(run, dv, dvout)
        res = np.zeros(n) if out is None else out
        self._check(self.lib.lbl_pnlint(self.h, C.byref(run), C.c_double(dv), C.c_double(dvout),
                                        _ptr(od), len(od), _ptr(res), n), "pnlint")
        return res

    def scan_spectrum(self, sc, spec, v1_in, dv_in, out=None):
        """SCANFN convolution of a spectrum (numpy or CUDA tensor) on
        v1_in + i*dv_in; returns the output on sc.v1 + j*DVOUT."""
        n, _ = scan_npts(sc, dv_in)
        res = np.zeros(n) if out is None else out
        self._check(self.lib.lbl_scan_spectrum(self.h, C.byref(sc), _ptr(spec), len(spec),
                                               C.c_double(v1_in), C.c_double(dv_in), _ptr(res),
                                               n), "scan_spectrum")
        return res

    def merge_layer(self, run, layer, first, dv_old, rad_in, tr_in, od):
        n = len(od)
        rad = np.zeros(n)
        tr = np.zeros(n)
        self._check(self.lib.lbl_merge_layer(
            self.h, C.byref(run), C.byref(layer), int(first), C.c_double(dv_old),
            _ptr(rad_in), _ptr(tr_in), 0 if rad_in is None else len(rad_in), _ptr(od),
            _ptr(rad), _ptr(tr), n), "merge_layer")
        return rad, tr

    def forward(self, run, layers, precision=abi.PREC_FP64, rad=None, tr=None):
        dv, _ = dv_rule(run, layers)
        n = layer_npts(run, dv[-1])
        rad = np.zeros(n) if rad is None else rad
        trb = np.zeros(n) if tr is None else tr
        self._check(self.lib.lbl_forward(self.h, C.byref(run), layers, len(layers), _ptr(rad),
                                         _ptr(trb), n, precision), "forward")
        return rad, trb

    def forward_batch(self, run, profiles, precision=abi.PREC_FP64, rad=None, tr=None):
        """Many profiles in one call: profiles is a list of lbl_layer arrays.
        Returns a list of (rad, tr) per profile on each profile's top grid.
        rad/tr may be given as flat buffers (numpy arrays or CUDA tensors)
        holding all profiles' points."""
        counts = [len(p) for p in profiles]
        allL = (abi.Layer * sum(counts))()
        k = 0
        for p in profiles:
            C.memmove(C.byref(allL, k * C.sizeof(abi.Layer)), p, C.sizeof(abi.Layer) * len(p))
            k += len(p)
        total = 0
        for p in profiles:
            q = abi.make_layers_like(p)
            dv, _ = dv_rule(run, q)
            total += layer_npts(run, dv[-1])
        rad = np.zeros(total) if rad is None else rad
        tr = np.zeros(total) if tr is None else tr
        off = np.zeros(len(profiles) + 1, dtype=np.int64)
        nl = (C.c_int32 * len(profiles))(*counts)
        self._check(self.lib.lbl_forward_batch(self.h, C.byref(run), allL, nl, len(profiles),
                                               _ptr(rad), _ptr(tr),
                                               off.ctypes.data_as(C.POINTER(C.c_int64)), total,
                                               precision), "forward_batch")
        return [(rad[off[i]:off[i + 1]], tr[off[i]:off[i + 1]]) for i in range(len(profiles))]

    def adjoint_batch(self, run, profiles, mols, mode=abi.JAC_REFERENCE, dv_chan=0.0,
                      precision=abi.PREC_FP64, rad=None, jac=None):
        """Forward and Jacobians of many profiles in one call.  Returns a list
        of (rad, jac) per profile, jac of shape (1 + len(mols), nlay, n);
        n is the profile's top-grid length (dv_chan = 0) or the number of
        channels of width dv_chan.  rad/jac may be given as flat buffers
        (numpy arrays or CUDA tensors) large enough for all profiles."""
        counts = [len(p) for p in profiles]
        allL = (abi.Layer * sum(counts))()
        k = 0
        for p in profiles:
            C.memmove(C.byref(allL, k * C.sizeof(abi.Layer)), p, C.sizeof(abi.Layer) * len(p))
            k += len(p)
        np_ = 1 + len(mols)
        if dv_chan > 0:
            nch = int(np.floor((run.v2 - run.v1) / dv_chan + 1e-9))
            nout = [nch] * len(profiles)
        else:
            nout = []
            for p in profiles:
                q = abi.make_layers_like(p)
                dv, _ = dv_rule(run, q)
                nout.append(layer_npts(run, dv[-1]))
        nrad = sum(nout)
        njac = sum(np_ * c * n for c, n in zip(counts, nout))
        rad = np.zeros(nrad) if rad is None else rad
        jac = np.zeros(njac) if jac is None else jac
        off = np.zeros(len(profiles) + 1, dtype=np.int64)
        joff = np.zeros(len(profiles) + 1, dtype=np.int64)
        nl = (C.c_int32 * len(profiles))(*counts)
        m = (C.c_int32 * max(len(mols), 1))(*mols)
        self._check(self.lib.lbl_adjoint_batch(
            self.h, C.byref(run), allL, nl, len(profiles), m, len(mols), int(mode),
            C.c_double(dv_chan), _ptr(rad), off.ctypes.data_as(P_I64), int(nrad), _ptr(jac),
            joff.ctypes.data_as(P_I64), int(njac), precision), "adjoint_batch")
        out = []
        for i, (c, n) in enumerate(zip(counts, nout)):
            r = rad[off[i]:off[i + 1]]
            j = jac[joff[i]:joff[i + 1]]
            out.append((r, j.reshape(np_, c, n) if hasattr(j, "reshape") else j))
        return out

    def jacobian(self, run, layers, mols, precision=abi.PREC_FP64, rad=None, jac=None):
        """TOA radiance and its Jacobians, shape (1 + len(mols), nlay, npts):
        row 0 d rad/d T_l, row k d rad/d ln W_{mols[k-1]},l.  rad/jac may be
        given (numpy arrays or CUDA tensors of that size)."""
        dv, _ = dv_rule(run, layers)
        n = layer_npts(run, dv[-1])
        nl = len(layers)
        m = (C.c_int32 * max(len(mols), 1))(*mols)
        rad = np.zeros(n) if rad is None else rad
        jac = np.zeros((1 + len(mols), nl, n)) if jac is None else jac
        self._check(self.lib.lbl_jacobian(self.h, C.byref(run), layers, nl, m, len(mols),
                                          _ptr(rad), _ptr(jac), n, precision), "jacobian")
        return rad, jac
