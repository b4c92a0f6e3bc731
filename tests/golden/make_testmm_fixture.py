"""Generate tests/golden/testmm_lines.npz from the reference's built-in test
line list (BLOCK DATA BTEST of src/testmm.f90, 1,068 records, 0-80 cm-1),
as TESTMM writes it with line coupling switched off (LINCPL=0, :136-141:
coupling records dropped, flags zeroed).  Run in a checkout that has the
LBLRTM sources:  python make_testmm_fixture.py <lblrtm-src-dir>
"""
import os
import re
import sys

import numpy as np


def numbers(text):
    out = []
    for tok in text.replace("&", " ").split(","):
        tok = tok.strip()
        if tok:
            out.append(float(tok.replace("D", "E")))
    return out


def main(src):
    t = open(os.path.join(src, "testmm.f90"), encoding="latin-1").read()
    t = t[t.index("BLOCK DATA BTEST"):]
    lines = [ln for ln in t.splitlines() if not ln.lstrip().startswith("!")]
    t = "\n".join(lines)
    c, d = [], []
    for m in re.finditer(r"DATA\s+([CD])(\d{4})\s*/(.*?)/", t, re.S):
        (c if m.group(1) == "C" else d).extend(numbers(m.group(3)))
    xc = np.array(c).reshape(-1, 5)
    xd = np.array(d).reshape(-1, 6)
    assert len(xc) == len(xd) == 1068
    keep = xd[:, 5] >= 0
    xc, xd = xc[keep], xd[keep]
    iso = (xc[:, 0] / 100.0).astype(int)
    mol = np.mod(xc[:, 0], 100.0).astype(int) + 100 * iso
    out = {
        "vnu": xc[:, 1].astype(np.float64), "sp": xc[:, 2].astype(np.float32),
        "alfa": xc[:, 3].astype(np.float32), "epp": xc[:, 4].astype(np.float32),
        "mol": mol.astype(np.int32), "hwhms": xd[:, 2].astype(np.float32),
        "tmpalf": xd[:, 3].astype(np.float32), "pshift": xd[:, 4].astype(np.float32),
        "iflg": np.zeros(len(xc), np.int32),
    }
    np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "testmm_lines.npz"), **out)
    print(len(xc), "records")


if __name__ == "__main__":
    main(sys.argv[1])
