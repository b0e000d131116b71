"""Field files (OVF 1.0 / 2.0, dump) and the Go number format (CPU only).

Pins: the element values test/loadfile.mx3 expects from the reference's
fixture files (read from the reference tree when it is present), byte-exact
rewrites of files the reference itself wrote, and lossless round trips."""
import os

import numpy as np
import pytest

from oracle import build_ref
from umagnus_b200 import fileio

REF = build_ref.reference_root()
DATA = os.path.join(REF, "test", "testdata") if REF else ""
needs_ref = pytest.mark.skipif(not (REF and os.path.isdir(DATA)), reason="reference test data not present")


@needs_ref
@pytest.mark.parametrize("fname,ncomp,size,elem,want", [
    # test/loadfile.mx3:17-60: s.get(c, ix, iy, iz)
    ("binary4.dump", 3, (100, 25, 1), (2, 99, 24, 0), -2.052794059181906e-07),
    ("binary4.ovf", 3, (100, 25, 1), (2, 99, 24, 0), -2.052794059181906e-07),
    ("binary8.ovf", 3, (100, 25, 1), (2, 99, 24, 0), -17100.58203125),
    ("oommf_ovf1_binary8.omf", 3, (100, 25, 1), (2, 99, 24, 0), -17100.58203125),
    ("m2.dump", 3, (128, 64, 1), (2, 99, 24, 0), -0.002278769388794899),
    ("movf2.ovf", 3, (64, 68, 1), (1, 2, 3, 0), 0.1468590646982193),
    ("scalarovf2.ovf", 1, (64, 64, 1), (0, 2, 3, 0), 0.0),
])
def test_loadfile_pins(fname, ncomp, size, elem, want):
    arr, meta = fileio.read(os.path.join(DATA, fname))
    assert arr.shape == (ncomp, size[2], size[1], size[0])
    c, ix, iy, iz = elem
    assert arr[c, iz, iy, ix] == np.float32(want)


@needs_ref
def test_ovf1_text_equals_binary4():
    """oommf_ovf1_text.omf and oommf_ovf1_binary4.omf hold the same field."""
    a, ma = fileio.read(os.path.join(DATA, "oommf_ovf1_text.omf"))
    b, mb = fileio.read(os.path.join(DATA, "oommf_ovf1_binary4.omf"))
    assert a.shape == b.shape == (3, 1, 10, 25)
    np.testing.assert_array_equal(a, b)
    assert ma["cellsize"] == (2e-08, 2e-08, 2e-08)


@needs_ref
@pytest.mark.parametrize("fname", ["randommag4x4x1.ovf", "regions.ovf"])
def test_rewrite_is_byte_identical(fname, tmp_path):
    """Files the reference wrote (WriteOVF2, binary 4) come out byte for byte
    the same from this writer given their data and header values."""
    src = os.path.join(DATA, fname)
    arr, meta = fileio.read(src)
    unit = "" if meta["unit"] == "1" else meta["unit"]
    out = tmp_path / "out.ovf"
    fileio.write_ovf(out, arr, meta["cellsize"], name=meta["name"], unit=unit, time=meta["time"])
    assert out.read_bytes() == open(src, "rb").read()


@pytest.mark.parametrize("kind", ["ovf2-bin", "ovf2-text", "ovf1-bin", "ovf1-text", "dump"])
def test_round_trip(kind, tmp_path):
    rng = np.random.default_rng(3)
    arr = rng.standard_normal((3, 2, 5, 7)).astype(np.float32) * np.float32(1e-3)
    arr[0, 0, 0, 0] = 0.0
    arr[1, 1, 2, 3] = np.float32(1234567.0)
    cell = (1e-9, 2.5e-9, 3e-9)
    p = tmp_path / "f"
    if kind == "dump":
        fileio.write_dump(p, arr, cell, name="m", unit="T", time=1.5e-10)
    else:
        v = 2 if kind.startswith("ovf2") else 1
        fileio.write_ovf(p, arr, cell, name="m", unit="T", time=1.5e-10,
                         format="text" if kind.endswith("text") else "binary 4", version=v)
    back, meta = fileio.read(p)
    np.testing.assert_array_equal(back, arr)
    assert meta["cellsize"] == cell
    assert meta["time"] == pytest.approx(1.5e-10, rel=1e-15)


def test_scalar_ovf2_round_trip(tmp_path):
    arr = np.arange(24, dtype=np.float32).reshape(1, 2, 3, 4)
    fileio.write_ovf(tmp_path / "s.ovf", arr, (1, 1, 1), name="Kc1", unit="J/m3")
    back, meta = fileio.read(tmp_path / "s.ovf")
    np.testing.assert_array_equal(back, arr)
    assert meta["name"] == "Kc1" and meta["unit"] == "J/m3"


@pytest.mark.parametrize("v,bits,want", [
    (0.0, 64, "0"), (1.0, 64, "1"), (100.0, 64, "100"), (0.5, 64, "0.5"), (1e-9, 64, "1e-09"),
    (6.4e-07, 64, "6.4e-07"), (1234567.0, 64, "1.234567e+06"), (123456.0, 64, "123456"),
    (0.0001, 64, "0.0001"), (0.00001, 64, "1e-05"), (-2.5e-9, 64, "-2.5e-09"),
    (2.000377037076917e-10, 64, "2.000377037076917e-10"),
    (np.float32(0.1), 32, "0.1"), (np.float32(-17100.58203125), 32, "-17100.582"), (np.float32(1e10), 32, "1e+10"),
])
def test_go_float_format(v, bits, want):
    assert fileio.go_float(v, bits) == want


class _StubSim:
    def __init__(self):
        self.t = 0.0

    def state(self):
        return {"time": self.t}

    def average_m(self):
        return [0.1, -0.25, 0.9669625163078308]


def test_table_format(tmp_path):
    """engine/table.go: '# t (s)\\tmx ()\\tmy ()\\tmz ()', rows of Go-formatted numbers."""
    t = fileio.Table(tmp_path / "table.txt")
    s = _StubSim()
    t.save(s)
    s.t = 1.5e-10
    t.save(s)
    t.close()
    lines = (tmp_path / "table.txt").read_text().splitlines()
    assert lines[0] == "# t (s)\tmx ()\tmy ()\tmz ()"
    assert lines[1] == "0\t0.1\t-0.25\t0.9669625"
    assert lines[2] == "1.5e-10\t0.1\t-0.25\t0.9669625"
