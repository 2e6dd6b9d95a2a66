"""CPU oracle for the fermion-solve hot path -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may load this package, and only to check results against: the
product (``iroiro_b200``) never imports it.

Two implementations live here:

* ``port()`` -- liboracle_port.so, a plain-C restatement (port/iro_oracle.c)
  of the reference's Wilson/clover operators, CG and multishift CG, citing
  the reference lines it follows.
* ``ref()`` -- oracle/_ref/libiroiro_ref.so, the reference's own classes
  compiled from its sources by oracle/Makefile (built only where the
  reference tree is present; the built library travels with the repository
  working copy).  It keeps the lattice in process-wide singletons, so one
  process can serve one lattice size.

The port is pinned against the reference through tests/golden/, which
tests/golden/make_golden.py generates by running the reference library.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle_port.so"
REF_LIB = HERE / "_ref" / "libiroiro_ref.so"

WILSON_FULL, WILSON_EO, CLOVER_FULL = 0, 1, 2

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int
_port = None
_ref = None


def build(ref: bool = False) -> None:
    """make -C oracle port [ref]."""
    targets = ["port"] + (["ref"] if ref else [])
    subprocess.run(["make", "-s", "-C", str(HERE), *targets], check=True)


def _p(a):
    return a.ctypes.data_as(_D)


def port() -> "Port":
    global _port
    if _port is None:
        if not PORT_LIB.exists():
            build()
        _port = Port(ctypes.CDLL(str(PORT_LIB)))
    return _port


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> "Ref":
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise FileNotFoundError(f"{REF_LIB} not built (make -C oracle ref)")
        _ref = Ref(ctypes.CDLL(str(REF_LIB)))
    return _ref


class Port:
    """The C restatement; any lattice size per call."""

    def __init__(self, lib):
        self.lib = lib
        D, L4 = ctypes.c_double, ctypes.POINTER(ctypes.c_int)
        lib.orc_gamma5.argtypes = [ctypes.c_long, _D, _D]
        lib.orc_wilson_full.argtypes = [L4, _D, D, _I, _D, _D]
        lib.orc_wilson_hop.argtypes = [L4, _D, D, _I, _I, _D, _D]
        lib.orc_wilson_eo.argtypes = [L4, _D, D, _I, _D, _D]
        lib.orc_field_strength.argtypes = [L4, _D, _I, _I, _D]
        lib.orc_clover_full.argtypes = [L4, _D, D, D, _I, _D, _D]
        lib.orc_cg.argtypes = [L4, _D, _I, D, D, _D, _D, D, _I, _D, ctypes.POINTER(_I)]
        lib.orc_multishift.argtypes = [L4, _D, _I, D, D, _D, _I, _D, _D, D, _I, _D,
                                       ctypes.POINTER(_I)]
        lib.orc_eo_invert.argtypes = [L4, _D, D, _D, _D, D, _I, _D, ctypes.POINTER(_I)]
        lib.orc_md_force.argtypes = [L4, _D, D, _I, _D, _D, _D]
        lib.orc_rational.argtypes = [L4, _D, _I, D, D, _D, _I, _D, _D, D, _D, D, _I, _D,
                                     ctypes.POINTER(_I)]
        lib.orc_synth_gauge.argtypes = [L4, D, ctypes.c_ulonglong, _I, _D]
        lib.orc_synth_gaussian.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong, _D]

    @staticmethod
    def _L(L):
        return (ctypes.c_int * 4)(*[int(v) for v in L])

    def gamma5(self, f):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f)
        self.lib.orc_gamma5(f.size // 24, _p(f), _p(out))
        return out

    def wilson_full(self, L, u, mass, dag, f):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f)
        self.lib.orc_wilson_full(self._L(L), _p(u), mass, int(dag), _p(f), _p(out))
        return out

    def wilson_hop(self, L, u, mass, eo, dag, f):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f)
        self.lib.orc_wilson_hop(self._L(L), _p(u), mass, int(eo), int(dag), _p(f), _p(out))
        return out

    def wilson_eo(self, L, u, mass, dag, f):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f)
        self.lib.orc_wilson_eo(self._L(L), _p(u), mass, int(dag), _p(f), _p(out))
        return out

    def field_strength(self, L, u, mu, nu):
        out = np.empty(18 * int(np.prod(L)))
        self.lib.orc_field_strength(self._L(L), _p(u), mu, nu, _p(out))
        return out

    def clover_full(self, L, u, mass, csw, dag, f):
        f = np.ascontiguousarray(f, np.float64)
        out = np.empty_like(f)
        self.lib.orc_clover_full(self._L(L), _p(u), mass, csw, int(dag), _p(f), _p(out))
        return out

    def cg(self, L, u, op, mass, csw, b, prec, maxiter):
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty_like(b)
        diff = ctypes.c_double()
        it = ctypes.c_int()
        self.lib.orc_cg(self._L(L), _p(u), op, mass, csw, _p(b), _p(x), prec, maxiter,
                        ctypes.byref(diff), ctypes.byref(it))
        return x, it.value, diff.value

    def multishift(self, L, u, op, mass, csw, b, shifts, prec, maxiter):
        b = np.ascontiguousarray(b, np.float64)
        sh = np.ascontiguousarray(shifts, np.float64)
        x = np.empty(b.size * sh.size)
        diff = ctypes.c_double()
        nc = ctypes.c_int()
        self.lib.orc_multishift(self._L(L), _p(u), op, mass, csw, _p(b), sh.size, _p(sh), _p(x),
                                prec, maxiter, ctypes.byref(diff), ctypes.byref(nc))
        return x.reshape(sh.size, b.size), nc.value, diff.value


def _port_eo_invert(self, L, u, mass, src, prec, maxiter):
    """Inverter_WilsonLike::invert (Wilson e/o) of one full-lattice source."""
    src = np.ascontiguousarray(src, np.float64)
    sol = np.empty_like(src)
    diff = ctypes.c_double()
    it = ctypes.c_int()
    self.lib.orc_eo_invert(self._L(L), _p(u), mass, _p(src), _p(sol), prec, maxiter,
                           ctypes.byref(diff), ctypes.byref(it))
    return sol, it.value, diff.value


def _port_rational(self, L, u, op, mass, csw, b, poles, residues, c0, prec, maxiter):
    """RationalSolver_CG::solve: c0 b + sum_i r_i (A + p_i)^-1 b."""
    b = np.ascontiguousarray(b, np.float64)
    p = np.ascontiguousarray(poles, np.float64)
    r = np.ascontiguousarray(residues, np.float64)
    sol = np.empty_like(b)
    diff = ctypes.c_double()
    nc = ctypes.c_int()
    self.lib.orc_rational(self._L(L), _p(u), op, mass, csw, _p(b), p.size, _p(p), _p(r), c0, _p(sol),
                          prec, maxiter, ctypes.byref(diff), ctypes.byref(nc))
    return sol, nc.value, diff.value


def _port_md_force(self, L, u, mass, eo, eta, zeta):
    """md_force of the full (eo=False) or e/o (eo=True) Wilson operator."""
    F = np.empty(72 * int(np.prod(L)))
    self.lib.orc_md_force(self._L(L), _p(u), mass, 1 if eo else -1, _p(np.ascontiguousarray(eta)),
                          _p(np.ascontiguousarray(zeta)), _p(F))
    return F


def _port_synth_gauge(self, L, eps, seed, gauge_transform=False):
    """The seeded exp(i eps H) field of the product's synth_gauge, bit for bit
    (Format_G, 18*4*V doubles), without loading the product library."""
    u = np.empty(72 * int(np.prod(L)))
    if self.lib.orc_synth_gauge(self._L(L), float(eps), int(seed), int(gauge_transform), _p(u)):
        raise ValueError(f"bad lattice {L}")
    return u


def _port_synth_gaussian(self, nsites, seed):
    """N(0,1) in every real component of nsites Format_F sites, as the
    product's synth_gaussian."""
    f = np.empty(24 * int(nsites))
    self.lib.orc_synth_gaussian(int(nsites), int(seed), _p(f))
    return f


def synth_point_sources(nsites, site):
    """The 12 Source_local point sources at `site` (1.0 at index_r(c,s,site),
    source_types.hpp:40-60), shape (12, 24*nsites)."""
    f = np.zeros((12, 24 * int(nsites)))
    for k in range(12):
        f[k, 24 * int(site) + 2 * k] = 1.0
    return f


Port.synth_gauge = _port_synth_gauge
Port.synth_gaussian = _port_synth_gaussian
Port.eo_invert = _port_eo_invert
Port.md_force = _port_md_force
Port.rational = _port_rational


class Ref:
    """The reference's own classes; one lattice per process (ref_init)."""

    def __init__(self, lib):
        self.lib = lib
        D = ctypes.c_double
        lib.ref_init.argtypes = [_I, _I, _I, _I]
        lib.ref_wilson_mult.argtypes = [_D, D, _I, _D, _D]
        lib.ref_wilson_hop.argtypes = [_D, D, _I, _I, _D, _D]
        lib.ref_wilson_eo_mult.argtypes = [_D, D, _I, _D, _D]
        lib.ref_clover_mult.argtypes = [_D, D, D, _I, _D, _D]
        lib.ref_field_strength.argtypes = [_D, _I, _I, _D]
        lib.ref_cg_solve.argtypes = [_D, _I, D, D, _D, _D, D, _I, _D, ctypes.POINTER(_I), _D]
        lib.ref_multishift_solve.argtypes = [_D, _I, D, D, _D, _I, _D, _D, D, _I, _D,
                                             ctypes.POINTER(_I)]
        lib.ref_eo_mult_throughput.argtypes = [_D, D, _D, _D, _I, _I, _D]
        lib.ref_eo_invert.argtypes = [_D, D, _D, _D, _I, D, _I]
        lib.ref_md_force.argtypes = [_D, _I, D, _D, _D, _D]
        lib.ref_gauge_save.argtypes = [_D, ctypes.c_char_p, _I]
        lib.ref_gauge_load.argtypes = [ctypes.c_char_p, _I, _D]
        lib.ref_plaquette.argtypes = [_D, _D, _D]
        lib.ref_rational_solve.argtypes = [_D, _I, D, D, _D, _I, _D, _D, D, _D, D, _I, _D,
                                           ctypes.POINTER(_I)]
        self.L = None

    def init(self, L):
        rc = self.lib.ref_init(*[int(v) for v in L])
        if rc:
            raise RuntimeError(f"reference already initialised with another lattice than {L}")
        self.L = list(L)

    def _chk(self, rc, what):
        if rc:
            raise RuntimeError(f"{what} returned {rc}")

    def wilson_full(self, u, mass, dag, f):
        out = np.empty_like(f)
        self._chk(self.lib.ref_wilson_mult(_p(u), mass, int(dag), _p(f), _p(out)), "ref_wilson_mult")
        return out

    def wilson_hop(self, u, mass, eo, dag, f):
        out = np.empty_like(f)
        self._chk(self.lib.ref_wilson_hop(_p(u), mass, int(eo), int(dag), _p(f), _p(out)), "ref_wilson_hop")
        return out

    def wilson_eo(self, u, mass, dag, f):
        out = np.empty_like(f)
        self._chk(self.lib.ref_wilson_eo_mult(_p(u), mass, int(dag), _p(f), _p(out)), "ref_wilson_eo_mult")
        return out

    def clover_full(self, u, mass, csw, dag, f):
        out = np.empty_like(f)
        self._chk(self.lib.ref_clover_mult(_p(u), mass, csw, int(dag), _p(f), _p(out)), "ref_clover_mult")
        return out

    def field_strength(self, u, mu, nu):
        out = np.empty(18 * int(np.prod(self.L)))
        self._chk(self.lib.ref_field_strength(_p(u), mu, nu, _p(out)), "ref_field_strength")
        return out

    def cg(self, u, op, mass, csw, b, prec, maxiter):
        x = np.empty_like(b)
        diff = ctypes.c_double()
        it = ctypes.c_int()
        ms = ctypes.c_double()
        self._chk(self.lib.ref_cg_solve(_p(u), op, mass, csw, _p(b), _p(x), prec, maxiter,
                                        ctypes.byref(diff), ctypes.byref(it), ctypes.byref(ms)),
                  "ref_cg_solve")
        return x, it.value, diff.value, ms.value

    def multishift(self, u, op, mass, csw, b, shifts, prec, maxiter):
        sh = np.ascontiguousarray(shifts, np.float64)
        x = np.empty(b.size * sh.size)
        diff = ctypes.c_double()
        nc = ctypes.c_int()
        self._chk(self.lib.ref_multishift_solve(_p(u), op, mass, csw, _p(b), sh.size, _p(sh), _p(x),
                                                prec, maxiter, ctypes.byref(diff), ctypes.byref(nc)),
                  "ref_multishift_solve")
        return x.reshape(sh.size, b.size), nc.value, diff.value

    def eo_invert(self, u, mass, srcs, prec, maxiter):
        """Inverter_WilsonLike::invert of each full-lattice source (rows of srcs)."""
        srcs = np.ascontiguousarray(np.atleast_2d(srcs), np.float64)
        sol = np.empty_like(srcs)
        self._chk(self.lib.ref_eo_invert(_p(u), mass, _p(srcs), _p(sol), srcs.shape[0], prec, maxiter),
                  "ref_eo_invert")
        return sol

    def rational(self, u, op, mass, csw, b, poles, residues, c0, prec, maxiter):
        p = np.ascontiguousarray(poles, np.float64)
        r = np.ascontiguousarray(residues, np.float64)
        sol = np.empty_like(b)
        diff = ctypes.c_double()
        nc = ctypes.c_int()
        self._chk(self.lib.ref_rational_solve(_p(u), op, mass, csw, _p(b), p.size, _p(p), _p(r), c0,
                                              _p(sol), prec, maxiter, ctypes.byref(diff),
                                              ctypes.byref(nc)), "ref_rational_solve")
        return sol, nc.value, diff.value

    def md_force(self, u, op, mass, eta, zeta):
        """Dirac_Wilson[_EvenOdd]::md_force(eta, zeta) as a Format_G array."""
        F = np.empty(72 * int(np.prod(self.L)))
        self._chk(self.lib.ref_md_force(_p(u), op, mass, _p(eta), _p(zeta), _p(F)), "ref_md_force")
        return F

    def gauge_save(self, u, path, writer):
        """CCIO::SaveOnDisk<Format_G>(u, path, false, "Binary" (0) | "NERSC" (2))."""
        self._chk(self.lib.ref_gauge_save(_p(u), str(path).encode(), writer), "ref_gauge_save")

    def gauge_load(self, path, kind):
        """GaugeConf_{bin (0), NERSC (2), csdt (5), txt (6), unit (7)}::init_conf."""
        u = np.zeros(72 * int(np.prod(self.L)))
        self._chk(self.lib.ref_gauge_load(str(path).encode(), kind, _p(u)), "ref_gauge_load")
        return u

    def plaquette(self, u):
        """(Staples::plaquette, Staples::link_trace)."""
        p, t = ctypes.c_double(), ctypes.c_double()
        self._chk(self.lib.ref_plaquette(_p(u), ctypes.byref(p), ctypes.byref(t)), "ref_plaquette")
        return p.value, t.value

    def eo_mult_throughput(self, u, mass, f, nthreads, reps):
        out = np.empty_like(f)
        secs = ctypes.c_double()
        self._chk(self.lib.ref_eo_mult_throughput(_p(u), mass, _p(f), _p(out), nthreads, reps,
                                                  ctypes.byref(secs)), "ref_eo_mult_throughput")
        return out, secs.value
