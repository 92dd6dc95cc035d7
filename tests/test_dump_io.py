"""Fortran 'binary' dumps and the MRI history file, host side (no GPU).

The committed fixtures under tests/golden/ were written by this package and read back by
the reference's own reader, dumpy (make_dump_golden.py records what it checked).  Here the
same seeded inputs must reproduce those files byte for byte, and the readers must return
them; the gfortran subrecord framing of records over 2 GiB is checked on small records
(with a small subrecord limit on the writer side, and on a hand-framed file on the reader
side).
"""
import hashlib
import json
import pathlib
import shutil
import struct
import subprocess
import sys

import numpy as np
import pytest

import dumses_hybrid_b200 as dg

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))
from make_dump_golden import HIST_SEED, HIST_TIMES, PARAMS, SEED, seeded_sums, seeded_uin  # noqa: E402

META = json.loads((GOLDEN / "dump_golden.json").read_text())


def test_dump_matches_golden_bytes(tmp_path):
    p = dg.Params(**PARAMS)
    path = dg.dump_filename(1, 0, tmp_path)
    assert path.relative_to(tmp_path).as_posix() == "output_000001/data.000000.bin"
    dg.write_dump(path, p, seeded_uin(p, SEED), META["time"], META["dt"])
    data = path.read_bytes()
    assert len(data) == META["dump_bytes"]
    assert hashlib.sha256(data).hexdigest() == META["dump_sha256"]
    assert data == (GOLDEN / META["dump"]).read_bytes()


def test_dump_layout():
    """Records of output.f90:228-232 with 4-byte markers, as dumpy's reader seeks them."""
    data = (GOLDEN / META["dump"]).read_bytes()
    p = dg.Params(**PARAMS)
    assert struct.unpack_from("<i6ii", data, 0) == (24, 4, 3, 3, 1, 1, 1, 24)
    t, dt, dx, dy, dz = struct.unpack_from("<5d", data, 32 + 4)
    assert (t, dt) == (META["time"], META["dt"])
    assert (dx, dy, dz) == ((p.xmax - p.xmin) / p.nx, (p.ymax - p.ymin) / p.ny, (p.zmax - p.zmin) / p.nz)
    off = 6 * 4 + 13 * 8 + 2 * 4 * 4  # dumpy's offset of the uin record (rd_dumses.py:642)
    n = int(np.prod(p.shape)) * 8
    assert struct.unpack_from("<i", data, off)[0] == n
    assert struct.unpack_from("<i", data, off + 4 + n)[0] == n
    assert len(data) == off + n + 8


def test_read_golden_dump():
    p = dg.Params(**PARAMS)
    u, t, dt = dg.read_dump(GOLDEN / META["dump"], p)
    assert (t, dt) == (META["time"], META["dt"])
    assert np.array_equal(u, seeded_uin(p, SEED))
    h = dg.dump_header(GOLDEN / META["dump"])
    assert (h["nx"], h["ny"], h["nz"], h["nxslice"]) == (4, 3, 3, 1)
    assert (h["gamma"], h["ciso"], h["uin_bytes"]) == (p.gamma, p.ciso, int(np.prod(p.shape)) * 8)


def test_read_dump_wrong_grid(tmp_path):
    p = dg.Params(**{**PARAMS, "nx": 5})
    with pytest.raises(dg.DumsesError, match="DG_ERR_ARG"):
        dg.read_dump(GOLDEN / META["dump"], p)
    q = dg.Params(**{**PARAMS, "gamma": 1.4})
    with pytest.raises(dg.DumsesError, match="DG_ERR_ARG"):
        dg.read_dump(GOLDEN / META["dump"], q)


def test_damaged_dumps_are_errors_not_crashes(tmp_path):
    """A dump cut short anywhere, or with a record marker changed, is refused with an error
    code; the reader never reads past a record it was not promised."""
    p = dg.Params(**PARAMS)
    good = (GOLDEN / META["dump"]).read_bytes()
    path = tmp_path / "bad.bin"
    off = 6 * 4 + 13 * 8 + 2 * 4 * 4
    cuts = sorted({0, 3, 4, 20, 31, 32, 60, 100, off - 1, off, off + 4, off + 1000, len(good) - 5, len(good) - 1})
    for cut in cuts:
        path.write_bytes(good[:cut])
        with pytest.raises(dg.DumsesError):
            dg.read_dump(path, p)
    # record markers: the header's leading and trailing ones, and the uin record's
    for pos, value in ((0, 28), (28, 20), (0, -24), (off, 16), (off, 2 ** 31 - 1), (len(good) - 4, 8)):
        bad = bytearray(good)
        struct.pack_into("<i", bad, pos, value)
        path.write_bytes(bytes(bad))
        with pytest.raises(dg.DumsesError):
            dg.read_dump(path, p)
    # trailing bytes after the last record are not part of a dump either
    path.write_bytes(good + b"\0" * 8)
    u, t, _ = dg.read_dump(path, p)  # the reference reads its records and stops, as this does
    assert t == META["time"] and np.array_equal(u, seeded_uin(p, SEED))


def test_read_dump_of_a_decomposed_run(tmp_path):
    data = bytearray((GOLDEN / META["dump"]).read_bytes())
    struct.pack_into("<i", data, 4 + 5 * 4, 2)  # nzslice = 2
    path = tmp_path / "d.bin"
    path.write_bytes(bytes(data))
    with pytest.raises(dg.DumsesError, match="DG_ERR_UNSUPPORTED"):
        dg.read_dump(path, dg.Params(**PARAMS))


def frame_subrecords(payload: bytes, sizes: list[int]) -> bytes:
    """gfortran framing: leading marker negative when a subrecord follows, trailing
    marker negative when one precedes."""
    out, pos = bytearray(), 0
    for s, n in enumerate(sizes):
        chunk = payload[pos: pos + n]
        pos += n
        out += struct.pack("<i", -n if s < len(sizes) - 1 else n) + chunk + struct.pack("<i", -n if s > 0 else n)
    assert pos == len(payload)
    return bytes(out)


def test_read_subrecords(tmp_path):
    p = dg.Params(ndim=2, nx=3, ny=3, nz=1)
    u = seeded_uin(p, 5)
    gold = tmp_path / "one.bin"
    dg.write_dump(gold, p, u, 0.5, 0.25)
    data = gold.read_bytes()
    off = 6 * 4 + 13 * 8 + 2 * 4 * 4
    payload = data[off + 4: -4]
    n = len(payload)
    split = tmp_path / "split.bin"
    split.write_bytes(data[:off] + frame_subrecords(payload, [1000, 1000, 3000, n - 5000]))
    v, t, dt = dg.read_dump(split, p)
    assert (t, dt) == (0.5, 0.25) and np.array_equal(u, v)
    assert dg.dump_header(split)["uin_bytes"] == n
    # a record one subrecord short is refused
    short = tmp_path / "short.bin"
    short.write_bytes(data[:off] + frame_subrecords(payload[:-8], [1000, n - 1008]))
    with pytest.raises(dg.DumsesError):
        dg.read_dump(short, p)


WRITER_CHECK = r"""
#include "dump_io.h"
#include <vector>
int main(int argc, char **argv) {
    FILE *f = std::fopen(argv[1], "wb");
    std::vector<unsigned char> a(2500);
    for (size_t q = 0; q < a.size(); q++) a[q] = (unsigned char)(q * 7);
    dg::dump::RecordWriter w(f, 2500, 1000);
    bool ok = w.write(a.data(), 700) && w.write(a.data() + 700, 1800) && w.close();
    dg::dump::RecordWriter e(f, 2000, 1000);  // an exact multiple of the limit
    ok = ok && e.write(a.data(), 2000) && e.close();
    std::fclose(f);
    return ok ? 0 : 1;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_writer_subrecords(tmp_path):
    src = tmp_path / "w.cpp"
    src.write_text(WRITER_CHECK)
    exe = tmp_path / "w"
    csrc = pathlib.Path(dg.__file__).resolve().parent / "csrc"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(csrc), str(src), "-o", str(exe)], check=True)
    out = tmp_path / "rec.bin"
    subprocess.run([str(exe), str(out)], check=True)
    a = bytes((q * 7) % 256 for q in range(2500))
    assert out.read_bytes() == frame_subrecords(a, [1000, 1000, 500]) + frame_subrecords(a[:2000], [1000, 1000])


def test_history_file_matches_golden(tmp_path):
    path = tmp_path / "history.txt"
    for (t, dt), s in zip(HIST_TIMES, seeded_sums(HIST_SEED, len(HIST_TIMES))):
        dg.write_history(path, t, dt, s)
    assert path.read_bytes() == (GOLDEN / META["history"]).read_bytes()
    assert hashlib.sha256(path.read_bytes()).hexdigest() == META["history_sha256"]


def test_history_format():
    """('# ', A11, 1X, A12, 1X, 9(A14,1X)) and (1X, 1PE12.5, 1X, 1PE12.5, 1X, 9(E14.5,1X)),
    the scale factor carrying over to the E14.5 fields (history.f90:152-168)."""
    head = dg.history_header()
    assert head.startswith("#        time           dt           mass        maxwell")
    assert len(head) == 2 + 11 + 1 + 12 + 1 + 9 * 15
    line = dg.history_line(1.5, 2.0e-3, np.array([1.0, -2.5e-4, 0.0, 1e-300, 12345.678, 0, 0, 0, -1e-17]))
    assert line == ("  1.50000E+00  2.00000E-03    1.00000E+00   -2.50000E-04    0.00000E+00    1.00000-300"
                    "    1.23457E+04    0.00000E+00    0.00000E+00    0.00000E+00   -1.00000E-17 ")
