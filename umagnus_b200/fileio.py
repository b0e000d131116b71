"""Field files and the data table, on top of the library's native readers and
writers (libumagnus_b200.so umag_field_* / umag_ovf_write / umag_dump_write).

Mirrors the reference's `oommf` package (OVF 1.0 / 2.0: oommf/oommf.go Read,
oommf/ovf1.go WriteOVF1, oommf/ovf2.go WriteOVF2), the legacy `dump` format
(dump/read.go, dump/write.go), the engine's SaveAs / LoadFile and the data
table (engine/table.go).  Arrays are float32 shaped (ncomp, Nz, Ny, Nx).
These calls need no GPU.
"""
import ctypes
import os

import numpy as np

from . import _lib
from ._lib import check


class FieldInfo(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int * 3), ("ncomp", ctypes.c_int), ("cell", ctypes.c_double * 3),
                ("time", ctypes.c_double), ("title", ctypes.c_char * 64), ("unit", ctypes.c_char * 32)]


def _info(ncomp, N, cell, title, unit, time):
    i = FieldInfo()
    i.N[:] = [int(n) for n in N]
    i.ncomp = int(ncomp)
    i.cell[:] = [float(c) for c in cell]
    i.time = float(time)
    i.title = title.encode()[:63]
    i.unit = unit.encode()[:31]
    return i


def read(path):
    """oommf.ReadFile / dump.ReadFile: (array (ncomp, Nz, Ny, Nx) float32, meta)
    with meta = dict(name, unit, time, cellsize)."""
    L = _lib.load()
    info = FieldInfo()
    p = os.fsencode(path)
    check(L.umag_field_read_info(p, ctypes.byref(info)))
    N = tuple(info.N)
    arr = np.empty((info.ncomp, N[2], N[1], N[0]), np.float32)
    check(L.umag_field_read(p, arr.ctypes.data, arr.size, ctypes.byref(info)))
    meta = dict(name=info.title.decode(), unit=info.unit.decode(), time=info.time, cellsize=tuple(info.cell))
    return arr, meta


def _field(arr):
    a = np.ascontiguousarray(arr, np.float32)
    if a.ndim == 3:
        a = a[None]
    if a.ndim != 4:
        raise ValueError("field must be shaped (ncomp, Nz, Ny, Nx) or (Nz, Ny, Nx)")
    return a


def write_ovf(path, arr, cellsize, name="m", unit="", time=0.0, format="binary 4", version=2):
    """oommf.WriteOVF2 (version 2) / WriteOVF1 (version 1); format "text" or "binary 4"."""
    a = _field(arr)
    info = _info(a.shape[0], (a.shape[3], a.shape[2], a.shape[1]), cellsize, name, unit, time)
    check(_lib.load().umag_ovf_write(os.fsencode(path), a.ctypes.data, ctypes.byref(info), format.encode(),
                                     int(version)))


def write_dump(path, arr, cellsize, name="m", unit="", time=0.0):
    """dump.WriteFile."""
    a = _field(arr)
    info = _info(a.shape[0], (a.shape[3], a.shape[2], a.shape[1]), cellsize, name, unit, time)
    check(_lib.load().umag_dump_write(os.fsencode(path), a.ctypes.data, ctypes.byref(info)))


def go_float(v, bits=64):
    """A number as Go's fmt %v prints it (float64 or float32)."""
    buf = ctypes.create_string_buffer(64)
    check(_lib.load().umag_format_float(float(v), int(bits), buf, 64))
    return buf.value.decode()


def save_m(sim, path, format="binary 4", version=2):
    """engine SaveAs(m, path): the simulation's m as OVF."""
    m = sim.get_m().cpu().numpy()
    write_ovf(path, m, sim.params.cell[:], name="m", unit="", time=sim.state()["time"], format=format,
              version=version)


def load_m(sim, path):
    """engine m.LoadFile(path) (engine/magnetization.go:55-57)."""
    arr, _ = read(path)
    if arr.shape != (3,) + sim.shape:
        raise ValueError(f"{path}: field {arr.shape} does not match the mesh {(3,) + sim.shape}")
    sim.set_m(arr)


class Table:
    """engine/table.go data table: header '# t (s)' then one tab-separated
    column per component of each quantity ('mx ()' ...); every row is the
    time (float64) then the quantities' values as float32, formatted as Go's
    %v (engine/table.go:112-133, 145-165)."""

    def __init__(self, path, quantities=(("m", "", 3, None),)):
        # quantities: (name, unit, ncomp, fn(sim) -> sequence of ncomp floats); fn None = average m
        self.path = path
        self.q = list(quantities)
        self.f = None

    def _init(self):
        if self.f is not None:
            return
        self.f = open(self.path, "w")
        head = "# t (s)"
        for name, unit, ncomp, _ in self.q:
            if ncomp == 1:
                head += "\t" + name + " (" + unit + ")"
            else:
                for c in range(ncomp):
                    head += "\t" + name + "xyz"[c] + " (" + unit + ")"
        self.f.write(head + "\n")
        self.f.flush()

    def save(self, sim):
        self._init()
        row = go_float(sim.state()["time"], 64)
        for name, unit, ncomp, fn in self.q:
            vals = sim.average_m() if fn is None else fn(sim)
            for v in list(vals)[:ncomp]:
                row += "\t" + go_float(np.float32(v), 32)
        self.f.write(row + "\n")

    def close(self):
        if self.f is not None:
            self.f.close()
            self.f = None
