"""Generate ``cont_tables.h`` from the CO2 continuum DATA of LBLRTM.

Build-time step, run once in a checkout that has the LBLRTM sources (like
``gen_ref_tables.py``).  The generated header is committed; nothing at run
time reads the Fortran.  The coefficients must be the reference's numbers
for the continuum optical depth to agree, so they are extracted
mechanically:

* ``BLOCK DATA BFCO2`` (src/contnm.f90:1355-2491): the CO2 continuum
  coefficients, -4 to 10000 cm-1 every 2 cm-1 (5003 values, F0000..F5001).
* ``XFACCO2`` (src/contnm.f90:95-179): the mt_ckd_2.5 scaling of the CO2
  continuum from 2000 to 2998 cm-1 (500 values).
* ``tdep_bandhead``, ``t_eff`` (src/contnm.f90:1300-1313): the temperature
  dependence of coefficients 1196-1220 (2386-2434 cm-1).
* ``BLOCK DATA bo2f`` (src/contnm.f90:7320-7382): the O2 collision-induced
  fundamental, 1340-1850 cm-1 every 5 cm-1 (coefficients and temperature
  exponents, 103 each).
* ``BLOCK DATA BN2T296``, ``BN2T220`` (src/contnm.f90:2569-2664): the N2
  collision-induced rotational band at 296 K and 220 K, -10-350 cm-1 every
  5 cm-1 (coefficients and O2 scale factors, 73 each).
* ``BLOCK DATA bn2f`` (src/contnm.f90:2756-2912): the N2 collision-induced
  fundamental at 272 K and 228 K and the H2O broadening efficiency, 228
  points from 1997.78 cm-1.
* ``BLOCK DATA bn2f1`` (src/contnm.f90:2970-3020): the N2 collision-induced
  first overtone, 4340-4910 cm-1 every 3 cm-1 (191 values).
* ``BLOCK DATA bo2inf1`` (src/contnm.f90:7441-7562): the O2 1.27 um
  collision-induced band (Mate et al.), 7536-8500 cm-1 every 2 cm-1 (483).

Usage:  python gen_cont_tables.py <lblrtm-src-dir> <out.h>
"""
import re
import sys

from gen_ref_tables import _collect_data, _find, _fmt, _strip_comments


def extract(src):
    with open(f"{src}/contnm.f90", encoding="latin-1") as f:
        L = _strip_comments(f.readlines())
    t = {}
    k = _find(L, r"^\s*DATA\s+XFACCO2\s*/")
    t["XFACCO2"] = _collect_data(L, k)
    assert len(t["XFACCO2"]) == 500, len(t["XFACCO2"])
    ks = _find(L, r"^\s*SUBROUTINE\s+FRNCO2\b")
    k = _find(L, r"data\s*\(tdep_bandhead\(i\),i=1196,1220\)\s*/", ks)
    t["TDEP"] = _collect_data(L, k)
    assert len(t["TDEP"]) == 25
    k = _find(L, r"data\s+t_eff\s*/", ks)
    t["TEFF"] = _collect_data(L, k)[0]
    kb = _find(L, r"^\s*BLOCK DATA BFCO2\b")
    k = _find(L, r"DATA\s+V1\s*,\s*V2\s*,\s*DV\s*,\s*NPT\s*/", kb)
    v1, v2, dv, npt = _collect_data(L, k)
    t["HDR"] = (v1, v2, dv, int(npt))
    vals = []
    names = ["F0000"] + ["F%04d" % n for n in range(1, 5002, 50)]
    for nm in names:
        k = _find(L, r"^\s*DATA\s+%s\s*/" % nm, kb)
        vals.extend(_collect_data(L, k))
    assert len(vals) == int(npt), (len(vals), npt)
    t["FCO2"] = vals

    def block(name, arrays, hdr):
        kb = _find(L, r"^\s*BLOCK DATA %s\b" % name)
        k = _find(L, r"^\s*DATA\s+%s" % hdr, kb)
        h = _collect_data(L, k)
        out = {}
        for nm, parts in arrays.items():
            v = []
            for part in parts:
                k = _find(L, r"^\s*DATA\s+%s\s*/" % part, kb)
                v.extend(_collect_data(L, k))
            assert len(v) == int(h[3]), (name, nm, len(v))
            out[nm] = v
        return (h[0], h[1], h[2], int(h[3])), out

    t["O2F"] = block("bo2f", {"XO2": ["o0001", "o0051", "o0101"],
                              "XO2T": ["ot0001", "ot0051", "ot0101"]}, r"V1S\s*,")
    t["N2R296"] = block("BN2T296", {"C": ["CT296"], "SF": ["sf_296"]}, r"V1N2CR\s*,")
    t["N2R220"] = block("BN2T220", {"C": ["CT220"], "SF": ["sf_220"]}, r"V1N2CR\s*,")
    t["N2F"] = block("bn2f", {"X272": ["xn2_272"], "X228": ["xn2_228"], "AH2O": ["a_h2o"]},
                     r"V1n2f\s*,")
    t["N2O1"] = block("bn2f1", {"X": ["xn2"]}, r"V1n2f\s*,")
    t["O2I1"] = block("bo2inf1", {"X": ["o%04d" % k for k in range(1, 482, 50)]}, r"V1\s*,")
    return t


def write_header(t, out):
    v1, v2, dv, npt = t["HDR"]
    lines = [
        "/* Generated by gen_cont_tables.py from the LBLRTM sources; do not edit.",
        " * The CO2 continuum of CONTNM (src/contnm.f90 BLOCK DATA BFCO2, XFACCO2,",
        " * FRNCO2's tdep_bandhead and t_eff) and the O2 and N2 collision-induced",
        " * bands (BLOCK DATA bo2f, BN2T296, BN2T220, bn2f), as initializer lists",
        " * so that host and device arrays can be defined from them. */",
        "#ifndef LBL_CONT_TABLES_H",
        "#define LBL_CONT_TABLES_H",
        "#define LBL_FCO2_V1 %s" % _fmt(v1),
        "#define LBL_FCO2_V2 %s" % _fmt(v2),
        "#define LBL_FCO2_DV %s" % _fmt(dv),
        "#define LBL_FCO2_N %d" % npt,
        "#define LBL_CO2_TEFF %s" % _fmt(t["TEFF"]),
        "#define LBL_FCO2_VALUES \\",
    ]
    vals = t["FCO2"]
    for i in range(0, len(vals), 8):
        tail = ", \\" if i + 8 < len(vals) else ""
        lines.append("  " + ", ".join(map(_fmt, vals[i:i + 8])) + tail)
    lines.append("#define LBL_XFACCO2_VALUES \\")
    vals = t["XFACCO2"]
    for i in range(0, len(vals), 8):
        tail = ", \\" if i + 8 < len(vals) else ""
        lines.append("  " + ", ".join(map(_fmt, vals[i:i + 8])) + tail)
    lines.append("#define LBL_CO2_TDEP_VALUES \\")
    lines.append("  " + ", ".join(map(_fmt, t["TDEP"])))
    for key, tag in (("O2F", "O2F"), ("N2R296", "N2R296"), ("N2R220", "N2R220"),
                     ("N2F", "N2F"), ("N2O1", "N2O1"), ("O2I1", "O2I1")):
        (a, b, d, n), arrays = t[key]
        lines.append("#define LBL_%s_V1 %s" % (tag, _fmt(a)))
        lines.append("#define LBL_%s_V2 %s" % (tag, _fmt(b)))
        lines.append("#define LBL_%s_DV %s" % (tag, _fmt(d)))
        lines.append("#define LBL_%s_N %d" % (tag, n))
        for nm, vals in arrays.items():
            lines.append("#define LBL_%s_%s_VALUES \\" % (tag, nm))
            for i in range(0, len(vals), 8):
                tail = ", \\" if i + 8 < len(vals) else ""
                lines.append("  " + ", ".join(map(_fmt, vals[i:i + 8])) + tail)
    lines.append("#endif")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    write_header(extract(sys.argv[1]), sys.argv[2])
