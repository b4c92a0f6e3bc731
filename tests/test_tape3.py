"""TAPE3 line files through the C reader (lbl_lines_load_tape3 with no
context: read and check only, no device) and the Python writer/reader:
a round trip, and every malformed-file path returning its status code
(the reference STOPs on these, RDLIN src/oprop.f90:741-779)."""
import ctypes as C
import struct

import numpy as np
import pytest

from lblrtm_b200 import abi, configs, gpu, tape3

LBL_OK, LBL_E_ARG, LBL_E_UNSORTED, LBL_E_NREC, LBL_E_FORMAT = 0, 1, 2, 3, 10


def load_check(path):
    n = C.c_int64(-1)
    rc = gpu.load().lbl_lines_load_tape3(None, str(path).encode(), C.byref(n))
    return rc, n.value


@pytest.fixture()
def lines():
    return configs.gen_lines(1234, 600.0, 700.0, seed=31, mols=configs.MOLS)


def test_round_trip(tmp_path, lines):
    p = tmp_path / "TAPE3"
    tape3.write(p, lines)
    rc, n = load_check(p)
    assert rc == LBL_OK and n == 1234
    back = tape3.read(p)
    for k in ("vnu", "sp", "alfa", "epp", "mol", "hwhms", "tmpalf", "pshift", "iflg"):
        assert np.array_equal(back[k], lines[k]), k
    assert list(back["block_start"]) == list(range(0, 1234, 250)) + [1234]


def test_short_panels_keep_their_boundaries(tmp_path, lines):
    p = tmp_path / "TAPE3"
    tape3.write(p, lines, per_panel=97)
    rc, n = load_check(p)
    assert rc == LBL_OK and n == 1234
    assert list(tape3.read(p)["block_start"]) == list(range(0, 1234, 97)) + [1234]


def test_missing_file():
    assert load_check("/nonexistent/TAPE3")[0] == LBL_E_ARG


def test_bad_header(tmp_path):
    p = tmp_path / "TAPE3"
    body = b"short header"
    p.write_bytes(struct.pack("<i", len(body)) + body + struct.pack("<i", len(body)))
    assert load_check(p)[0] == LBL_E_FORMAT


def test_record_markers_differ(tmp_path, lines):
    p = tmp_path / "TAPE3"
    tape3.write(p, lines)
    b = bytearray(p.read_bytes())
    # the trailing marker of the header record
    n1 = struct.unpack_from("<i", b, 0)[0]
    struct.pack_into("<i", b, 4 + n1, n1 + 4)
    p.write_bytes(bytes(b))
    assert load_check(p)[0] == LBL_E_FORMAT


@pytest.mark.parametrize("cut", [3, 10, 200, 30000])
def test_truncated_file(tmp_path, lines, cut):
    """Cut inside a panel header marker, a panel header, or a data block."""
    p = tmp_path / "TAPE3"
    tape3.write(p, lines)
    b = p.read_bytes()
    hdr = 8 + struct.unpack_from("<i", b, 0)[0]
    p.write_bytes(b[:hdr + cut])
    assert load_check(p)[0] == LBL_E_FORMAT


def test_nrec_above_250(tmp_path, lines):
    p = tmp_path / "TAPE3"
    tape3.write(p, lines)
    b = bytearray(p.read_bytes())
    hdr = 8 + struct.unpack_from("<i", b, 0)[0]
    # NREC of the first panel header (VMIN, VMAX f8, then NREC i4)
    struct.pack_into("<i", b, hdr + 4 + 16, 300)
    p.write_bytes(bytes(b))
    assert load_check(p)[0] == LBL_E_NREC


def test_unsorted_centres(tmp_path, lines):
    bad = {k: v.copy() for k, v in lines.items()}
    bad["vnu"][500], bad["vnu"][501] = bad["vnu"][501], bad["vnu"][500]
    p = tmp_path / "TAPE3"
    tape3.write(p, bad)
    assert load_check(p)[0] == LBL_E_UNSORTED


def test_coupling_record_without_line(tmp_path, lines):
    bad = {k: v.copy() for k, v in lines.items()}
    bad["iflg"][10] = -1
    p = tmp_path / "TAPE3"
    tape3.write(p, bad)
    assert load_check(p)[0] == LBL_E_FORMAT


def test_lines_upload_needs_context(lines):
    lh = abi.LinesHandle(lines)
    assert gpu.load().lbl_lines_upload(None, C.byref(lh.struct)) == LBL_E_ARG
