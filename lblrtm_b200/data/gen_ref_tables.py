"""Generate ``ref_tables.h`` from the numeric DATA statements of LBLRTM.

Build-time step, run once in a checkout that has the LBLRTM sources.  The
generated header is committed, so nothing at run time reads the Fortran.

The tables must be bit-for-bit the reference's numbers for the line-shape
and partition-sum arithmetic to agree, so they are extracted mechanically
rather than retyped:

* ``BLOCK DATA VOICON``  (src/oprop.f90:1993-2144): AVRAT, CGAUSS, CF1, CF2,
  CF3, CER -- the zeta-indexed Voigt-width and sub-function weights.
* ``BLOCK DATA BD_TDAT`` (src/oprop.f90:6295-6315): the 119 TIPS temperatures.
* ``QT_H2O .. QT_O2``    (src/oprop.f90:6588-8233): TIPS Q(T) tables for
  HITRAN molecules 1-7, every isotopologue listed there.
* ``BLOCK DATA Isotop``  (src/oprop.f90:2697-2896): ISO_MAX and SMASS.

Usage:  python gen_ref_tables.py <lblrtm-src-dir> <out.h>
"""
import re
import sys


def _strip_comments(lines):
    out = []
    for ln in lines:
        s = ln.rstrip("\n")
        if s.lstrip().startswith("!"):
            continue
        # drop trailing comment (no strings containing '!' in numeric DATA)
        if "!" in s:
            s = s[: s.index("!")]
        out.append(s)
    return out


def _collect_data(text_lines, start_idx):
    """Return the numbers of the DATA statement starting at ``start_idx``."""
    buf = []
    i = start_idx
    while "/" not in text_lines[i]:
        i += 1
    first = text_lines[i]
    j = first.index("/")
    rest = first[j + 1 :]
    while True:
        seg = rest.replace("&", " ")
        if "/" in seg:
            buf.append(seg[: seg.index("/")])
            break
        buf.append(seg)
        i += 1
        rest = text_lines[i]
    body = " ".join(buf)
    vals = []
    for tok in body.split(","):
        tok = tok.strip()
        if not tok:
            continue
        rep = 1
        if "*" in tok:
            r, tok = tok.split("*", 1)
            rep = int(r)
        vals.extend([float(tok.replace("D", "E").replace("d", "e"))] * rep)
    return vals


def _find(lines, pattern, start=0):
    rx = re.compile(pattern, re.IGNORECASE)
    for k in range(start, len(lines)):
        if rx.search(lines[k]):
            return k
    raise KeyError(pattern)


def extract(src):
    with open(f"{src}/oprop.f90", encoding="latin-1") as f:
        raw = f.readlines()
    L = _strip_comments(raw)
    t = {}
    # VOICON
    names = ["AV01", "AV51", "CG01", "CG51", "CFA01", "CFA51", "CFB01",
             "CFB51", "CFC01", "CFC51", "CER01", "CER51"]
    k0 = _find(L, r"BLOCK DATA VOICON")
    got = {}
    for nm in names:
        k = _find(L, r"^\s*DATA\s+%s\s*/" % nm, k0)
        got[nm] = _collect_data(L, k)
    for out, (a, b) in {"AVRAT": ("AV01", "AV51"), "CGAUSS": ("CG01", "CG51"),
                        "CF1": ("CFA01", "CFA51"), "CF2": ("CFB01", "CFB51"),
                        "CF3": ("CFC01", "CFC51"), "CER": ("CER01", "CER51")}.items():
        v = got[a] + got[b]
        assert len(v) == 102, (out, len(v))
        t[out] = v
    # TIPS temperatures
    k = _find(L, r"data\s+Tdat\s*/")
    t["TDAT"] = _collect_data(L, k)
    assert len(t["TDAT"]) == 119
    # Q(T) tables, molecules 1..7
    qnames = ["QT_H2O", "QT_CO2", "QT_O3", "QT_N2O", "QT_CO", "QT_CH4", "QT_O2"]
    qt = []
    for m, nm in enumerate(qnames, start=1):
        ks = _find(L, r"^\s*Subroutine\s+%s\b" % nm)
        ke = _find(L, r"^\s*end\s+subroutine\s+%s\b" % nm, ks)
        isos = []
        k = ks
        while True:
            try:
                k = _find(L, r"data\s*\(QofT\(\s*(\d+),J\),J=1,119\)\s*/", k)
            except KeyError:
                break
            if k > ke:
                break
            iso = int(re.search(r"QofT\(\s*(\d+)", L[k]).group(1))
            v = _collect_data(L, k)
            assert len(v) == 119, (nm, iso, len(v))
            isos.append((iso, v))
            k += 1
        isos.sort()
        assert [i for i, _ in isos] == list(range(1, len(isos) + 1)), nm
        qt.append([v for _, v in isos])
    t["QOFT"] = qt
    # ISO_MAX and SMASS
    k0 = _find(L, r"BLOCK DATA Isotop")
    k = _find(L, r"DATA\s*\(ISO_MAX\(I\),I=1,NMOL\)\s*/", k0)
    t["ISO_MAX"] = [int(x) for x in _collect_data(L, k)]
    assert len(t["ISO_MAX"]) == 47
    smass = [[0.0] * 10 for _ in range(47)]
    for m in range(1, 48):
        k = _find(L, r"data\s*\(smass\(%d,i\),i=1,(\d+)\)" % m, k0)
        v = _collect_data(L, k)
        for i, x in enumerate(v):
            smass[m - 1][i] = x
    t["SMASS"] = smass
    return t


def _fmt(v):
    return repr(float(v))


def write_header(t, out):
    lines = []
    w = lines.append
    w("/* Generated by gen_ref_tables.py from the LBLRTM sources; do not edit.")
    w(" * Numeric DATA tables that the line-shape and partition-sum arithmetic")
    w(" * needs verbatim (src/oprop.f90 BLOCK DATA VOICON, BD_TDAT, Isotop and")
    w(" * the QT_* TIPS tables for HITRAN molecules 1-7). */")
    w("#ifndef LBL_REF_TABLES_H")
    w("#define LBL_REF_TABLES_H")
    for nm in ["AVRAT", "CGAUSS", "CF1", "CF2", "CF3", "CER"]:
        w("static const double LBL_%s[102] = {%s};" % (nm, ", ".join(map(_fmt, t[nm]))))
    w("static const double LBL_TDAT[119] = {%s};" % ", ".join(map(_fmt, t["TDAT"])))
    w("#define LBL_NQMOL %d" % len(t["QOFT"]))
    niso = [len(q) for q in t["QOFT"]]
    w("static const int LBL_QNISO[%d] = {%s};" % (len(niso), ", ".join(map(str, niso))))
    w("#define LBL_QMAXISO %d" % max(niso))
    w("static const double LBL_QOFT[%d][%d][119] = {" % (len(niso), max(niso)))
    for q in t["QOFT"]:
        rows = q + [[0.0] * 119] * (max(niso) - len(q))
        w("  {" + ",\n   ".join("{" + ", ".join(map(_fmt, r)) + "}" for r in rows) + "},")
    w("};")
    w("static const int LBL_ISO_MAX[47] = {%s};" % ", ".join(map(str, t["ISO_MAX"])))
    w("static const double LBL_SMASS[47][10] = {")
    for r in t["SMASS"]:
        w("  {" + ", ".join(map(_fmt, r)) + "},")
    w("};")
    w("#endif")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    write_header(extract(sys.argv[1]), sys.argv[2])
