"""Gauge-configuration readers and writers (host-only, no GPU) against the
reference's own: files its writers made (NERSC, Binary) and what its readers
(GaugeConf_bin / NERSC / csdt / txt / unit, lib/Main/gaugeConf.cpp) made of
those and of the layouts.py files, plus Staples::plaquette / link_trace.  Byte
layouts, header and checksums are exact; plaquette and link trace agree to
round-off (different summation order)."""
import sys

import numpy as np
import pytest

import iroiro_b200 as ib
from conftest import GOLDEN, load_golden

sys.path.insert(0, str(GOLDEN))
import layouts  # noqa: E402

LATTICES = ["4x4x4x4", "6x2x4x4"]


@pytest.fixture(scope="module", params=LATTICES)
def g(request):
    d = load_golden(request.param)
    d["name"] = request.param
    d["Ls"] = [int(v) for v in d["L"]]
    return d


def header(path):
    raw = open(path, "rb").read()
    head, data = raw.split(b"END_HEADER\n", 1)
    kv = dict(line.split(" = ", 1) for line in head.decode().splitlines()[1:])
    return kv, data


def test_plaquette_and_link_trace(g):
    p, t = ib.plaquette(g["u"], g["Ls"]), ib.link_trace(g["u"], g["Ls"])
    assert abs(p - float(g["plaquette"])) < 1e-14
    assert abs(t - float(g["link_trace"])) < 1e-14
    unit = ib.GaugeConf_unit(g["Ls"]).init_conf()
    assert ib.plaquette(unit, g["Ls"]) == 1.0 and ib.link_trace(unit, g["Ls"]) == 1.0


def test_read_reference_nersc(g):
    """GaugeConf_NERSC on the file NERSCWriter wrote: the field bit for bit,
    the header's checksum equal to the reader's."""
    gc = ib.GaugeConf_NERSC(g["Ls"], GOLDEN / f"gauge_{g['name']}.nersc")
    u = gc.init_conf()
    assert np.array_equal(u, g["u"])
    i = gc.info
    assert i.bits == 64 and i.is3x2 == 0
    assert i.checksum == i.stored_checksum
    assert abs(i.stored_plaquette - float(g["plaquette"])) < 1e-14
    assert abs(i.plaquette - i.stored_plaquette) < 1e-14


def test_write_nersc_as_reference(g, tmp_path):
    """save_on_disk(..., "NERSC"): the same data bytes and header keys as
    NERSCWriter's file; numeric header values to round-off."""
    p = tmp_path / "c.nersc"
    assert ib.save_on_disk(g["u"], g["Ls"], p, writer="NERSC") == 0
    ours, ours_data = header(p)
    ref, ref_data = header(GOLDEN / f"gauge_{g['name']}.nersc")
    assert ours_data == ref_data
    assert ours.keys() == ref.keys()
    for k in ours:
        if k in ("PLAQUETTE", "LINK_TRACE"):
            assert abs(float(ours[k]) - float(ref[k])) < 1e-14, k
        else:
            assert ours[k] == ref[k], k


def test_binary_as_reference(g, tmp_path):
    """BinaryWriter stores host byte order and BinaryReader expects
    big-endian: writing matches the reference's file byte for byte, and reading
    its own file gives the reference's (byte-swapped) values bit for bit."""
    p = tmp_path / "c.bin"
    ib.save_on_disk(g["u"], g["Ls"], p, writer="Binary")
    assert p.read_bytes() == (GOLDEN / f"gauge_{g['name']}.bin").read_bytes()
    u = ib.GaugeConf_bin(g["Ls"], p).init_conf()
    assert np.array_equal(u.view(np.uint64), g["bin_ref_read"])


@pytest.mark.parametrize("kind,cls,write", [
    ("bin_be", ib.GaugeConf_bin, layouts.write_binary_be),
    ("csdt", ib.GaugeConf_csdt, layouts.write_csdt),
    ("txt", ib.GaugeConf_txt, layouts.write_text),
])
def test_read_layouts_as_reference(g, tmp_path, kind, cls, write):
    p = tmp_path / kind
    write(g["u"], g["Ls"], p)
    u = cls(g["Ls"], p).init_conf()
    assert np.array_equal(u, g[f"{kind}_ref_read"])
    assert np.array_equal(u, g["u"])


def test_read_nersc_3x2_ieee32(g, tmp_path):
    """Two stored rows in 32 bits: row 2 rebuilt as conj(row0 x row1), as the
    reference's reader does, to FP64 round-off of the same float inputs."""
    p = tmp_path / "n32"
    layouts.write_nersc(g["u"], g["Ls"], p, is3x2=True, bits=32)
    gc = ib.GaugeConf_NERSC(g["Ls"], p)
    u = gc.init_conf()
    assert gc.info.is3x2 == 1 and gc.info.bits == 32 and gc.info.checksum == gc.info.stored_checksum
    assert float(np.abs(u - g["nersc32_ref_read"]).max()) < 1e-15
    assert float(np.abs(u - g["u"]).max()) < 1e-6


def test_jlqcd_legacy_layout(g, tmp_path):
    """No reference output to compare with (its reader overruns its row buffer
    for mu > 0); the layout its reader intends: record word, [mu][site][18]."""
    p = tmp_path / "jl"
    layouts.write_jlqcd_legacy(g["u"], g["Ls"], p)
    assert np.array_equal(ib.GaugeConf_JLQCDLegacy(g["Ls"], p).init_conf(), g["u"])


def test_unit_as_reference(g):
    assert np.array_equal(ib.GaugeConf_unit(g["Ls"]).init_conf(), g["unit_ref"])


def test_fills_callers_array_and_append(g, tmp_path):
    """init_conf fills the caller's array in place (GaugeConf::init_conf(Field&));
    SaveOnDisk's append mode stacks configurations, read back by offset."""
    p = tmp_path / "two.bin"
    ib.save_on_disk(g["u"], g["Ls"], p, writer="Binary")
    ib.save_on_disk(2.0 * g["u"], g["Ls"], p, append_mode=True, writer="Binary")
    one = g["u"].nbytes
    assert p.stat().st_size == 2 * one
    # Binary is read big-endian: swap the host-order file first
    raw = np.fromfile(p, dtype="<f8").astype(">f8")
    q = tmp_path / "two_be.bin"
    raw.tofile(q)
    u = np.empty_like(g["u"])
    out, _ = ib.read_gauge(q, ib.gaugeconf.GAUGE_BINARY, g["Ls"], u, offset=one)
    assert out is u and np.array_equal(u, 2.0 * g["u"])


def test_errors(g, tmp_path):
    L = g["Ls"]
    with pytest.raises(ib.IroError) as e:
        ib.GaugeConf_ILDG(L, tmp_path / "x").init_conf()
    assert e.value.code == ib.UNSUPPORTED
    with pytest.raises(ib.IroError) as e:
        ib.GaugeConf_bin(L, tmp_path / "missing").init_conf()
    assert e.value.code == ib.IO_ERROR
    short = tmp_path / "short"
    short.write_bytes(b"\0" * 100)
    with pytest.raises(ib.IroError) as e:
        ib.GaugeConf_bin(L, short).init_conf()
    assert e.value.code == ib.IO_ERROR
    # a NERSC file of another lattice: the header's dimension check
    other = [L[0] * 2] + L[1:]
    p = tmp_path / "other.nersc"
    ib.save_on_disk(ib.GaugeConf_unit(other).init_conf(), other, p, writer="NERSC")
    with pytest.raises(ib.IroError) as e:
        ib.GaugeConf_NERSC(L, p).init_conf()
    assert e.value.code == ib.FORMAT_ERROR
    bad = tmp_path / "bad.nersc"
    bad.write_bytes(b"not a header\n")
    with pytest.raises(ib.IroError) as e:
        ib.GaugeConf_NERSC(L, bad).init_conf()
    assert e.value.code == ib.FORMAT_ERROR
    with pytest.raises(ib.IroError):
        ib.save_on_disk(g["u"], L, tmp_path / "t.txt", writer="text")


@pytest.mark.gpu
@pytest.mark.parametrize("name", LATTICES)
def test_configuration_file_drives_the_operator(name):
    """The reference's NERSC file, read and uploaded, gives the reference's
    Dirac_Wilson / Dirac_Wilson_EvenOdd outputs on the GPU."""
    from conftest import TOL_FP64, rel
    d = load_golden(name)
    L = [int(v) for v in d["L"]]
    u = ib.GaugeConf_NERSC(L, GOLDEN / f"gauge_{name}.nersc").init_conf()
    c = ib.context(L)
    c.upload_gauge(u, force=True)
    m = float(d["mass"])
    assert rel(c.apply(ib.OP_WILSON_FULL, m, 0, 0, d["f_full"]), d["wilson_full_0"]) < TOL_FP64
    assert rel(c.apply(ib.OP_WILSON_SCHUR_EE, m, 0, 1, d["f_half"]), d["wilson_eo_1"]) < TOL_FP64
