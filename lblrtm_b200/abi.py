"""ctypes mirrors of the structs in include/lblgpu.h.

These are the only Python definitions of the C ABI; both the CUDA library
wrapper and the test harness build their arguments with them.
"""
import ctypes as C

import numpy as np

LBL_WKDIM = 60

STATUS = {
    0: "LBL_OK", 1: "LBL_E_ARG", 2: "LBL_E_UNSORTED", 3: "LBL_E_NREC",
    4: "LBL_E_ITYPE", 5: "LBL_E_CUDA", 6: "LBL_E_NOMEM", 7: "LBL_E_RANGE",
    8: "LBL_E_NOTREADY", 9: "LBL_E_CONVERGE", 10: "LBL_E_FORMAT",
    11: "LBL_E_NODEVICE",
}

PREC_FP64 = 0
PREC_SPLIT = 1

JAC_CENTRAL = 0     # lbl_jac_mode: central differences, exact merge derivative
JAC_REFERENCE = 1   # the reference's analytic-Jacobian definitions


class Run(C.Structure):
    """lbl_run: TAPE5 records 1.2/1.2a/1.3/1.4 subset."""

    _fields_ = [
        ("ihirac", C.c_int32), ("ilblf4", C.c_int32), ("icntnm", C.c_int32),
        ("iemit", C.c_int32), ("ipathl", C.c_int32), ("jrad", C.c_int32),
        ("v1", C.c_double), ("v2", C.c_double), ("sample", C.c_double),
        ("dvset", C.c_double), ("alfal0", C.c_double), ("avmass", C.c_double),
        ("dptmin", C.c_double), ("dptfac", C.c_double), ("xself", C.c_double),
        ("xfrgn", C.c_double), ("tmpbnd", C.c_double), ("bndemi", C.c_double),
        ("xrayl", C.c_double), ("xco2c", C.c_double), ("xo2cn", C.c_double),
        ("xn2cn", C.c_double), ("bndrfl", C.c_double),
    ]


class Scan(C.Structure):
    """lbl_scan: SCANFN controls (HWHM, V1, V2, SAMPL, JFN, JEMIT=-1)."""

    _fields_ = [
        ("hwhm", C.c_double), ("v1", C.c_double), ("v2", C.c_double), ("sampl", C.c_double),
        ("jfn", C.c_int32), ("jabs", C.c_int32),
    ]


def make_scan(hwhm, v1, v2, jfn=2, sampl=0.0, jabs=0):
    sc = Scan()
    sc.hwhm, sc.v1, sc.v2, sc.sampl, sc.jfn, sc.jabs = hwhm, v1, v2, sampl, jfn, jabs
    return sc


class Layer(C.Structure):
    """lbl_layer: the /FILHDR/ quantities of one layer."""

    _fields_ = [
        ("pave", C.c_double), ("tave", C.c_double), ("pzl", C.c_double),
        ("pzu", C.c_double), ("tzl", C.c_double), ("tzu", C.c_double),
        ("wk", C.c_double * LBL_WKDIM), ("wbroad", C.c_double),
        ("nmol", C.c_int32), ("itype", C.c_int32), ("dv", C.c_double),
    ]


class Lines(C.Structure):
    """lbl_lines: TAPE3 records as structure of arrays."""

    _fields_ = [
        ("n", C.c_int64),
        ("vnu", C.POINTER(C.c_double)), ("sp", C.POINTER(C.c_float)),
        ("alfa", C.POINTER(C.c_float)), ("epp", C.POINTER(C.c_float)),
        ("mol", C.POINTER(C.c_int32)), ("hwhms", C.POINTER(C.c_float)),
        ("tmpalf", C.POINTER(C.c_float)), ("pshift", C.POINTER(C.c_float)),
        ("iflg", C.POINTER(C.c_int32)), ("nblock", C.c_int64),
        ("block_start", C.POINTER(C.c_int64)),
    ]


class Mtckd(C.Structure):
    """lbl_mtckd: continuum coefficient table."""

    _fields_ = [
        ("n", C.c_int64), ("v0", C.c_double), ("dv", C.c_double),
        ("self_absco_ref", C.POINTER(C.c_double)),
        ("for_absco_ref", C.POINTER(C.c_double)),
        ("self_texp", C.POINTER(C.c_double)),
        ("ref_press", C.c_double), ("ref_temp", C.c_double),
    ]


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def make_run(**kw):
    """lbl_run with the reference defaults (src/lblrtm.f90:911-913, 950-951)."""
    d = dict(ihirac=1, ilblf4=1, icntnm=0, iemit=0, ipathl=1, jrad=1,
             v1=0.0, v2=0.0, sample=4.0, dvset=0.0, alfal0=0.04, avmass=36.0,
             dptmin=2e-4, dptfac=1e-3, xself=1.0, xfrgn=1.0, tmpbnd=0.0,
             bndemi=1.0, xrayl=1.0, xco2c=1.0, xo2cn=1.0, xn2cn=1.0, bndrfl=0.0)
    d.update(kw)
    r = Run()
    for k, v in d.items():
        setattr(r, k, v)
    return r


def make_layers_like(layers):
    """A new lbl_layer array holding a copy of layers."""
    n = len(layers)
    arr = (Layer * n)()
    C.memmove(arr, layers, C.sizeof(Layer) * n)
    return arr


def make_layers(profile):
    """Array of lbl_layer from a profile dict of numpy arrays."""
    n = len(profile["pave"])
    arr = (Layer * n)()
    for l in range(n):
        L = arr[l]
        L.pave = float(profile["pave"][l])
        L.tave = float(profile["tave"][l])
        L.pzl = float(profile["pzl"][l])
        L.pzu = float(profile["pzu"][l])
        L.tzl = float(profile["tzl"][l])
        L.tzu = float(profile["tzu"][l])
        wk = profile["wk"][l]
        for m in range(len(wk)):
            L.wk[m] = float(wk[m])
        L.wbroad = float(profile["wbroad"][l])
        L.nmol = int(profile["nmol"])
        L.itype = 0
        L.dv = 0.0
    return arr


class LinesHandle:
    """Keeps the numpy arrays alive while a Lines struct points at them."""

    def __init__(self, lines):
        self.a = {k: np.ascontiguousarray(v) for k, v in lines.items()}
        a = self.a
        s = Lines()
        s.n = len(a["vnu"])
        s.vnu = _ptr(a["vnu"].astype(np.float64, copy=False), C.c_double)
        for k in ("sp", "alfa", "epp", "hwhms", "tmpalf", "pshift"):
            setattr(s, k, _ptr(a[k], C.c_float))
        s.mol = _ptr(a["mol"], C.c_int32)
        s.iflg = _ptr(a["iflg"], C.c_int32)
        if "block_start" in a:
            s.nblock = len(a["block_start"]) - 1
            s.block_start = _ptr(a["block_start"], C.c_int64)
        else:
            s.nblock = 0
            s.block_start = None
        self.struct = s


class MtckdHandle:
    def __init__(self, table):
        self.a = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in table.items()
                  if k in ("self_absco_ref", "for_absco_ref", "self_texp")}
        s = Mtckd()
        s.n = len(self.a["self_absco_ref"])
        s.v0 = float(table["v0"])
        s.dv = float(table["dv"])
        s.self_absco_ref = _ptr(self.a["self_absco_ref"], C.c_double)
        s.for_absco_ref = _ptr(self.a["for_absco_ref"], C.c_double)
        s.self_texp = _ptr(self.a["self_texp"], C.c_double)
        s.ref_press = float(table.get("ref_press", 1013.0))
        s.ref_temp = float(table.get("ref_temp", 296.0))
        self.struct = s
