"""Writers of the gauge-file layouts that the reference reads but never writes,
for the golden fixtures (make_golden.py) and the IO tests: each turns a
Format_G array u (link (site, mu) at 18*(site + V*mu), site = x + Lx*(y +
Ly*(z + Lz*t))) into the byte layout the reference's reader expects.

  csdt         GaugeConf_csdt::init_conf (lib/Main/gaugeConf.cpp:66-140)
  text         GaugeConf_txt::init_conf (gaugeConf.cpp:142-209)
  JLQCDLegacy  GaugeConf_JLQCDLegacy (gaugeConf.cpp:28-33), as its reader intends
  Binary (BE)  BinaryReader::read (lib/IO/binary_reader.cpp:21-29)
  NERSC        NERSCReader (lib/IO/NERSC_reader.cpp): 3x2 / 3x3, IEEE32BIG / IEEE64BIG
"""
import numpy as np


def links(u, L):
    """u as an array [mu][t][z][y][x][18]."""
    Lx, Ly, Lz, Lt = L
    return np.asarray(u, dtype=np.float64).reshape(4, Lt, Lz, Ly, Lx, 18)


def site_major(u, L):
    """[t][z][y][x][mu][18] (the site-major order of Binary and NERSC)."""
    return np.ascontiguousarray(links(u, L).transpose(1, 2, 3, 4, 0, 5))


RECORD = b"\0\0\0\0"  # the 4-byte Fortran record word skipped by the reader


def write_csdt(u, L, path):
    a = np.ascontiguousarray(links(u, L).transpose(1, 0, 2, 3, 4, 5))  # [t][mu][z][y][x][18]
    with open(path, "wb") as f:
        f.write(RECORD)
        f.write(a.astype(">f8").tobytes())


def write_text(u, L, path):
    a = site_major(u, L).reshape(-1, 2)
    with open(path, "w") as f:
        for re, im in a:
            f.write("%.17g %.17g\n" % (re, im))


def write_jlqcd_legacy(u, L, path):
    with open(path, "wb") as f:
        f.write(RECORD)
        f.write(np.asarray(u, dtype=np.float64).astype("=f8").tobytes())


def write_binary_be(u, L, path):
    with open(path, "wb") as f:
        f.write(site_major(u, L).astype(">f8").tobytes())


def nersc_checksum(data: bytes) -> int:
    """The reader's checksum: the data's 32-bit words in host (little-endian)
    order, summed modulo 2^32 (NERSC_reader.cpp:126-153)."""
    return int(np.frombuffer(data, dtype="<u4").sum(dtype=np.uint64) & 0xFFFFFFFF)


def write_nersc(u, L, path, is3x2=False, bits=64, plaquette=0.0, link_trace=0.0):
    a = site_major(u, L)
    if is3x2:
        a = a[..., :12]
    data = a.astype(">f4" if bits == 32 else ">f8").tobytes()
    hdr = ["BEGIN_HEADER", "HDR_VERSION = 1.0",
           "DATATYPE = " + ("4D_SU3_GAUGE" if is3x2 else "4D_SU3_GAUGE_3x3"),
           "STORAGE_FORMAT = 1.0"]
    hdr += [f"DIMENSION_{d + 1} = {L[d]}" for d in range(4)]
    hdr += [f"LINK_TRACE = {link_trace:1.15g}", f"PLAQUETTE = {plaquette:1.15g}",
            f"CHECKSUM = {nersc_checksum(data):x}", "ENSEMBLE_ID = test", "SEQUENCE_NUMBER = 0",
            "FLOATING_POINT = " + ("IEEE32BIG" if bits == 32 else "IEEE64BIG"), "END_HEADER"]
    with open(path, "wb") as f:
        f.write(("\n".join(hdr) + "\n").encode())
        f.write(data)
