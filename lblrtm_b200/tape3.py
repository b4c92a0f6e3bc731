"""TAPE3 line files: Fortran unformatted sequential records, 4-byte markers.

Layout (src/struct_types.f90:106-125, RDLIN src/oprop.f90:741-779):
  record 1        file header (HLINID(10) as 80 characters, then counts);
  per panel:      INPUT_HEADER  VMIN, VMAX (f8), NREC, NWDS (i4)
                  INPUT_BLOCK   250 slots of VNU (f8), SP, ALFA, EPP (f4),
                                MOL (i4), HWHM, TMPALF, PSHIFT (f4), IFLG (i4),
                                BRD_MOL_FLG_IN(7) (i4), BRD_MOL_DAT(21) (f4),
                                SPEED_DEP (f4)
"""
import struct

import numpy as np

NL = 250
FIELDS = [("vnu", "<f8"), ("sp", "<f4"), ("alfa", "<f4"), ("epp", "<f4"), ("mol", "<i4"),
          ("hwhms", "<f4"), ("tmpalf", "<f4"), ("pshift", "<f4"), ("iflg", "<i4")]
BLOCK_BYTES = NL * 156


def _record(f, payload):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write(path, lines, per_panel=NL):
    n = len(lines["vnu"])
    with open(path, "wb") as f:
        hid = b"LBLRTM-B200 synthetic TAPE3".ljust(80)
        _record(f, hid + bytes(1664 - 80))
        for s in range(0, n, per_panel):
            e = min(n, s + per_panel)
            k = e - s
            blk = bytearray(BLOCK_BYTES)
            off = 0
            for name, dt in FIELDS:
                a = np.zeros(NL, dtype=dt)
                a[:k] = lines[name][s:e]
                blk[off:off + a.nbytes] = a.tobytes()
                off += a.nbytes
            _record(f, struct.pack("<ddii", float(lines["vnu"][s]), float(lines["vnu"][e - 1]),
                                   k, BLOCK_BYTES // 4))
            _record(f, bytes(blk))


def read(path):
    out = {name: [] for name, _ in FIELDS}
    starts = [0]
    with open(path, "rb") as f:
        data = f.read()
    pos = 0

    def rec():
        nonlocal pos
        (n1,) = struct.unpack_from("<i", data, pos)
        body = data[pos + 4: pos + 4 + n1]
        (n2,) = struct.unpack_from("<i", data, pos + 4 + n1)
        if n1 != n2:
            raise ValueError("TAPE3: record markers differ")
        pos += 8 + n1
        return body

    hdr = rec()
    if hdr[6 * 8 + 7:6 * 8 + 8] == b"^":
        rec()
    while pos < len(data):
        h = rec()
        vmin, vmax, nrec, nwds = struct.unpack("<ddii", h)
        b = rec()
        off = 0
        for name, dt in FIELDS:
            a = np.frombuffer(b, dtype=dt, count=NL, offset=off)
            out[name].append(a[:nrec].copy())
            off += a.nbytes
        if nrec > 0:
            starts.append(starts[-1] + nrec)
    res = {k: np.concatenate(v) for k, v in out.items()}
    res["block_start"] = np.array(starts, dtype=np.int64)
    return res
