"""Gauge configurations from and to files: the GaugeConf_* initialisers of
IroIro (lib/Main/gaugeConf.hpp:23-107, gaugeConf.cpp:23-228) and
CCIO::SaveOnDisk (lib/IO/fields_io.hpp:48-139), over the library's host-only
readers (iro_gauge_read / iro_gauge_write).

Every configuration is a Format_G array of 18*4*V doubles (the layout
iro_gauge_upload takes): link (site, mu) at 18*(site + V*mu), site =
x + Lx*(y + Ly*(z + Lz*t)).  Like GaugeConf_*::init_conf, init_conf(u) fills
the caller's array in place; it also returns it.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import IroError, BAD_ARG, _ptr, lib

(GAUGE_BINARY, GAUGE_JLQCD_LEGACY, GAUGE_NERSC, GAUGE_ILDG, GAUGE_ILDG_FORTRAN, GAUGE_CSDT,
 GAUGE_TEXT, GAUGE_UNIT) = range(8)
IO_ERROR, FORMAT_ERROR, UNSUPPORTED = 8, 9, 10

_WRITERS = {"Binary": GAUGE_BINARY, "NERSC": GAUGE_NERSC, "ILDG": GAUGE_ILDG}


class GaugeInfo(ctypes.Structure):
    """What a read learned: the plaquette and link trace of the field
    (Staples::plaquette, link_trace) and, for NERSC, the header's stored values
    and the data checksum as the reader forms it."""
    _fields_ = [("plaquette", ctypes.c_double), ("link_trace", ctypes.c_double),
                ("stored_plaquette", ctypes.c_double), ("stored_link_trace", ctypes.c_double),
                ("checksum", ctypes.c_uint32), ("stored_checksum", ctypes.c_uint32),
                ("is3x2", ctypes.c_int), ("bits", ctypes.c_int)]


def _io_error(rc: int, what: str) -> IroError:
    msg = lib().iro_io_last_error()
    return IroError(rc, f"{what}: {msg.decode() if msg else ''}")


def _lattice(L):
    L = [int(v) for v in L]
    if len(L) != 4 or min(L) < 1:
        raise IroError(BAD_ARG, f"bad lattice {L}")
    return L, (ctypes.c_int * 4)(*L), int(np.prod(L))


def _field(u, V):
    if u is None:
        return np.empty(18 * 4 * V)
    if not (isinstance(u, np.ndarray) and u.dtype == np.float64 and u.flags.c_contiguous
            and u.size == 18 * 4 * V):
        raise IroError(BAD_ARG, f"u must be a contiguous float64 array of {18 * 4 * V} doubles")
    return u


def read_gauge(path, fmt: int, L, u=None, offset: int = 0) -> tuple[np.ndarray, GaugeInfo]:
    """CCIO::ReadFromDisk<Format_G> (fields_io.hpp:250-360) for one format."""
    L, cL, V = _lattice(L)
    u = _field(u, V)
    info = GaugeInfo()
    p = None if path is None else str(path).encode()
    rc = lib().iro_gauge_read(p, fmt, cL, offset, _ptr(u), ctypes.byref(info))
    if rc:
        raise _io_error(rc, f"reading {path}")
    return u, info


def plaquette(u, L) -> float:
    """Staples::plaquette (lib/Measurements/GaugeM/staples.cpp:35-38)."""
    return _measure(u, L)[0]


def link_trace(u, L) -> float:
    """Staples::link_trace (staples.cpp:24-33)."""
    return _measure(u, L)[1]


def _measure(u, L):
    L, cL, V = _lattice(L)
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.size != 18 * 4 * V:
        raise IroError(BAD_ARG, "u does not match the lattice")
    p, t = ctypes.c_double(), ctypes.c_double()
    rc = lib().iro_gauge_plaquette(cL, _ptr(u), ctypes.byref(p), ctypes.byref(t))
    if rc:
        raise _io_error(rc, "plaquette")
    return p.value, t.value


def save_on_disk(u, L, filename, append_mode: bool = False, writer: str = "Binary") -> int:
    """CCIO::SaveOnDisk<Format_G>(u, filename, append_mode, writerID)
    (fields_io.hpp:48-139): "Binary" writes [site][mu][18] doubles in host
    byte order (BinaryWriter), "NERSC" a 3x3 IEEE64BIG file with the header of
    NERSCWriter.  Returns 0 like the reference."""
    L, cL, V = _lattice(L)
    if writer not in _WRITERS:
        raise IroError(BAD_ARG, f"unknown writer {writer!r}")
    u = np.ascontiguousarray(u, dtype=np.float64)
    if u.size != 18 * 4 * V:
        raise IroError(BAD_ARG, "u does not match the lattice")
    rc = lib().iro_gauge_write(str(filename).encode(), _WRITERS[writer], cL, _ptr(u), int(append_mode))
    if rc:
        raise _io_error(rc, f"writing {filename}")
    return 0


class GaugeConf:
    """GaugeConf (gaugeConf.hpp:23-44): initialises a Format_G field of the
    lattice L.  `info` holds what the last init_conf read."""
    FORMAT = None

    def __init__(self, L, fname=None):
        self.L = [int(v) for v in L]
        self.file = fname
        self.info = None

    def init_conf(self, u=None, do_check: bool = True) -> np.ndarray:
        """Fills u (or a new array) from the configuration.  do_check is
        accepted for the reference's signature; its check is commented out
        there (fields_io.hpp:346-352), so nothing is checked here either:
        compare self.info's plaquette and checksum fields to verify."""
        u, self.info = read_gauge(self.file, self.FORMAT, self.L, u)
        return u


class GaugeConf_bin(GaugeConf):
    """Binary file, [site][mu][18] big-endian doubles (BinaryReader,
    lib/IO/binary_reader.cpp:21-35; GaugeConf_bin::init_conf gaugeConf.cpp:23-26)."""
    FORMAT = GAUGE_BINARY


class GaugeConf_JLQCDLegacy(GaugeConf):
    """JLQCD legacy file: a 4-byte Fortran record word, then [mu][site][18]
    doubles in host byte order (GaugeConf_JLQCDLegacy, gaugeConf.cpp:28-33)."""
    FORMAT = GAUGE_JLQCD_LEGACY


class GaugeConf_NERSC(GaugeConf):
    """NERSC file (NERSCReader, lib/IO/NERSC_reader.cpp): 3x2 or 3x3, IEEE32
    or IEEE64BIG; the header's dimensions must match L."""
    FORMAT = GAUGE_NERSC


class GaugeConf_ILDG(GaugeConf):
    """ILDG file: needs the lime library, which is absent; init_conf raises."""
    FORMAT = GAUGE_ILDG


class GaugeConf_ILDG_FORTRAN(GaugeConf):
    FORMAT = GAUGE_ILDG_FORTRAN


class GaugeConf_csdt(GaugeConf):
    """(c, s, d, t) binary file: a 4-byte record word, then
    [t][mu][z][y][x][a][b] big-endian complex doubles (gaugeConf.cpp:66-140)."""
    FORMAT = GAUGE_CSDT


class GaugeConf_txt(GaugeConf):
    """Text file, [t][z][y][x][mu][a][b] "re im" (gaugeConf.cpp:142-209)."""
    FORMAT = GAUGE_TEXT


class GaugeConf_unit(GaugeConf):
    """Unit links (gaugeConf.cpp:211-228)."""
    FORMAT = GAUGE_UNIT

    def __init__(self, L):
        super().__init__(L, None)
