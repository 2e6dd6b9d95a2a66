"""B200-native fermion-solve hot path of IroIro, behind the reference's interfaces.

The classes here mirror the reference's operator and solver API for this path
(names, argument meaning and error behaviour), on numpy arrays in the
reference's own host layouts (Format_F spinors, Format_G links):

=============================  ==============================================
this package                   reference
=============================  ==============================================
``Dirac_Wilson``               lib/Dirac_ops/dirac_wilson.hpp:89-175
``Dirac_Wilson_EvenOdd``       lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:14-119
``Dirac_Clover``               lib/Dirac_ops/dirac_clover.hpp:14-100
``Fopr_DdagD``                 lib/Fopr/fopr.h:146-153
``Solver_CG``                  lib/Solver/solver_CG.hpp:20-50
``MultiShiftSolver_CG``        lib/Solver/multiShiftSolver_CG.hpp:30-90
``SolverOutput``               lib/Solver/solver.hpp:16-22
=============================  ==============================================

Every computation runs in libiroiro_b200.so (CUDA, sm_100a) through its C
ABI (include/iroiro_b200.h); there is no CPU fallback: importing works
without a GPU, but the first operator call raises if the library or a CUDA
device is missing.
"""
from __future__ import annotations

import ctypes
import weakref
import os
import threading
from dataclasses import dataclass
from pathlib import Path

import numpy as np

__all__ = [
    "IroError", "ConvergenceError", "lib", "Context", "context", "init",
    "Dirac_Wilson", "Dirac_Wilson_EvenOdd", "Dirac_Clover", "Dirac_Clover_EvenOdd",
    "Fopr_DdagD", "Solver_CG", "MultiShiftSolver_CG", "SolverOutput",
    "synth_gauge", "synth_gaussian", "synth_point_sources",
    "OP_WILSON_FULL", "OP_WILSON_HOP_EO", "OP_WILSON_HOP_OE", "OP_WILSON_SCHUR_EE",
    "OP_CLOVER_FULL", "OP_CLOVER_SCHUR_EE", "OP_CLOVER_HOP_OE_INV", "PREC_DOUBLE", "PREC_SINGLE", "PREC_HALF",
    "GaugeConf", "GaugeConf_bin", "GaugeConf_JLQCDLegacy", "GaugeConf_NERSC", "GaugeConf_ILDG",
    "GaugeConf_ILDG_FORTRAN", "GaugeConf_csdt", "GaugeConf_txt", "GaugeConf_unit", "GaugeInfo",
    "read_gauge", "save_on_disk", "plaquette", "link_trace",
    "Source_local", "Inverter_WilsonLike", "Qprop_EvenOdd", "Qprop", "Qprop_MultiShift",
    "RationalApprox", "RationalSolver_CG", "DeviceField",
]

_HERE = Path(__file__).resolve().parent
_LIBPATH = _HERE / "libiroiro_b200.so"

(OK, NOT_CONVERGED, BAD_ARG, CUDA_ERROR, TIMEOUT, NO_GAUGE, NO_CLOVER, OUT_OF_MEMORY, IO_ERROR,
 FORMAT_ERROR, UNSUPPORTED) = range(11)
(OP_WILSON_FULL, OP_WILSON_HOP_EO, OP_WILSON_HOP_OE, OP_WILSON_SCHUR_EE,
 OP_CLOVER_FULL, OP_CLOVER_SCHUR_EE, OP_CLOVER_HOP_OE_INV) = range(7)
PREC_DOUBLE, PREC_SINGLE, PREC_HALF = range(3)
_PREC = {"double": PREC_DOUBLE, "single": PREC_SINGLE, "half": PREC_HALF,
         PREC_DOUBLE: PREC_DOUBLE, PREC_SINGLE: PREC_SINGLE, PREC_HALF: PREC_HALF}


class IroError(RuntimeError):
    """A status other than IRO_OK from the library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class ConvergenceError(IroError):
    """Solver did not converge: Solver_CG aborts through Errors::ConvergenceErr
    (lib/Solver/solver_CG.cpp:63-67) and MultiShiftSolver_CG throws
    "Not converged." (lib/Solver/multiShiftSolver_CG.cpp:163)."""


class SolverOut(ctypes.Structure):
    _fields_ = [("diff", ctypes.c_double), ("iterations", ctypes.c_int),
                ("timing_ms", ctypes.c_double), ("reliable_updates", ctypes.c_int),
                ("operator_applies", ctypes.c_int)]


class CGParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_double), ("max_iter", ctypes.c_int),
                ("inner_prec", ctypes.c_int), ("delta", ctypes.c_double),
                ("use_graph", ctypes.c_int)]


_lib = None
_lib_lock = threading.Lock()
_D = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p


def _declare(L):
    I, D = ctypes.c_int, ctypes.c_double
    L4 = ctypes.POINTER(ctypes.c_int)
    sig = {
        "iro_ctx_create": (I, [L4, I, ctypes.POINTER(_VP)]),
        "iro_ctx_destroy": (I, [_VP]),
        "iro_last_error": (ctypes.c_char_p, [_VP]),
        "iro_ctx_get_stream": (_VP, [_VP]),
        "iro_ctx_set_stream": (I, [_VP, _VP]),
        "iro_autotune_report": (I, [_VP, ctypes.c_char_p, I]),
        "iro_gauge_upload": (I, [_VP, _D]),
        "iro_clover_setup": (I, [_VP, D, D]),
        "iro_field_strength": (I, [_VP, I, I, _D]),
        "iro_dirac_apply": (I, [_VP, I, D, D, I, I, _D, _D, I]),
        "iro_gamma5": (I, [_VP, _D, _D, ctypes.c_int64]),
        "iro_field_create": (I, [_VP, I, I, I, ctypes.POINTER(_VP)]),
        "iro_field_destroy": (I, [_VP]),
        "iro_field_upload": (I, [_VP, _VP, _D]),
        "iro_field_download": (I, [_VP, _VP, _D]),
        "iro_dirac_apply_field": (I, [_VP, I, D, D, I, _VP, _VP]),
        "iro_field_norm": (I, [_VP, _VP, _D]),
        "iro_field_dot": (I, [_VP, _VP, _VP, _D]),
        "iro_norm_noalloc": (I, [_VP, ctypes.c_int64, _VP, _VP]),
        "iro_selftest_bounded_wait": (I, [_VP, D, _D]),
        "iro_cg_solve": (I, [_VP, I, D, D, ctypes.POINTER(CGParams), _D, _D, I,
                             ctypes.POINTER(SolverOut)]),
        "iro_cg_solve_field": (I, [_VP, I, D, D, ctypes.POINTER(CGParams), _VP, _VP,
                                   ctypes.POINTER(SolverOut)]),
        "iro_multishift_cg_solve": (I, [_VP, I, D, D, _D, I, _D, _D, D, I,
                                        ctypes.POINTER(SolverOut), ctypes.POINTER(I)]),
        "iro_multishift_cg_solve_mixed": (I, [_VP, I, D, D, _D, I, _D, _D, D, I, I,
                                              ctypes.POINTER(SolverOut), ctypes.POINTER(I)]),
        "iro_multishift_cg_solve_field": (I, [_VP, I, D, D, _VP, I, _D, _VP, D, I, I,
                                              ctypes.POINTER(SolverOut), ctypes.POINTER(I)]),
        "iro_rational_cg_solve": (I, [_VP, I, D, D, _D, I, _D, _D, D, _D, D, I,
                                      ctypes.POINTER(SolverOut), ctypes.POINTER(I)]),
        "iro_eo_invert": (I, [_VP, I, D, D, ctypes.POINTER(CGParams), _D, _D, I,
                              ctypes.POINTER(SolverOut)]),
        "iro_qprop_point": (I, [_VP, I, D, D, ctypes.POINTER(CGParams), ctypes.c_int64, I, I, _D,
                                ctypes.POINTER(SolverOut)]),
        "iro_md_force": (I, [_VP, I, D, D, _D, _D, _D]),
        "iro_synth_gauge": (I, [L4, D, ctypes.c_uint64, I, _D]),
        "iro_synth_gaussian": (I, [ctypes.c_int64, ctypes.c_uint64, _D]),
        "iro_synth_point_sources": (I, [ctypes.c_int64, ctypes.c_int64, _D]),
        "iro_gauge_read": (I, [ctypes.c_char_p, I, L4, ctypes.c_int64, _D, _VP]),
        "iro_gauge_write": (I, [ctypes.c_char_p, I, L4, _D, I]),
        "iro_gauge_plaquette": (I, [L4, _D, _D, _D]),
        "iro_io_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def lib() -> ctypes.CDLL:
    """The loaded libiroiro_b200.so; raises if it has not been built."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not _LIBPATH.exists():
                raise IroError(CUDA_ERROR, f"{_LIBPATH} is missing: run python -m iroiro_b200.build")
            L = ctypes.CDLL(str(_LIBPATH))
            _declare(L)
            _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _f64(a, n=None, name="field") -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise IroError(BAD_ARG, f"{name} has {a.size} doubles, expected {n}")
    return a


# ---- synthetic inputs ----------------------------------------------------------------

def synth_gauge(L, eps: float, seed: int, gauge_transform: bool = False) -> np.ndarray:
    """Seeded SU(3) field exp(i eps H) in Format_G (18*4*V doubles)."""
    L = [int(v) for v in L]
    V = int(np.prod(L))
    u = np.empty(18 * 4 * V)
    rc = lib().iro_synth_gauge((ctypes.c_int * 4)(*L), eps, seed, int(gauge_transform), _ptr(u))
    if rc:
        raise IroError(rc, "iro_synth_gauge")
    return u


def synth_gaussian(nsites: int, seed: int) -> np.ndarray:
    """N(0,1) in every real component of nsites Format_F sites."""
    f = np.empty(24 * nsites)
    rc = lib().iro_synth_gaussian(nsites, seed, _ptr(f))
    if rc:
        raise IroError(rc, "iro_synth_gaussian")
    return f


def synth_point_sources(nsites: int, site: int) -> np.ndarray:
    """The 12 point sources at `site` (Source_local semantics), shape (12, 24*nsites)."""
    f = np.empty(12 * 24 * nsites)
    rc = lib().iro_synth_point_sources(nsites, site, _ptr(f))
    if rc:
        raise IroError(rc, "iro_synth_point_sources")
    return f.reshape(12, 24 * nsites)


# ---- context -------------------------------------------------------------------------

class Context:
    """One lattice on one GPU: the geometry singletons of the reference
    (CommonPrms, SiteIndex_EvenOdd) plus the resident gauge/clover data."""

    def __init__(self, L, device: int = 0):
        self.L = [int(v) for v in L]
        self.V = int(np.prod(self.L))
        self.Vh = self.V // 2
        self._lib = lib()
        h = _VP()
        rc = self._lib.iro_ctx_create((ctypes.c_int * 4)(*self.L), device, ctypes.byref(h))
        if rc:
            raise IroError(rc, f"iro_ctx_create({self.L}, device={device})")
        self.h = h
        self._gauge_key = None
        # fields and networks of this context, closed before it
        self._owned = weakref.WeakSet()

    def check(self, rc: int, what: str):
        if rc == OK:
            return
        msg = self._lib.iro_last_error(self.h).decode()
        if rc == NOT_CONVERGED:
            raise ConvergenceError(rc, f"{what}: {msg}")
        raise IroError(rc, f"{what}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            for obj in list(getattr(self, "_owned", ())):
                obj.close()
            self._lib.iro_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return int(self._lib.iro_ctx_get_stream(self.h) or 0)

    def autotune_report(self) -> list:
        """The stencil autotuner's choices (one dict per tuned launch shape)."""
        import json
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(self._lib.iro_autotune_report(self.h, buf, len(buf)), "iro_autotune_report")
        return json.loads(buf.value.decode())

    def set_stream(self, stream_handle: int):
        self.check(self._lib.iro_ctx_set_stream(self.h, _VP(stream_handle)), "set_stream")

    def upload_gauge(self, u: np.ndarray, force: bool = False):
        u = _f64(u, 72 * self.V, "gauge field")
        key = (id(u), u.ctypes.data)
        if force or key != self._gauge_key:
            self.check(self._lib.iro_gauge_upload(self.h, _ptr(u)), "iro_gauge_upload")
            self._gauge_key = key
            self._gauge_ref = u

    def apply(self, op: int, mass: float, csw: float, dag: bool, f: np.ndarray, prec=PREC_DOUBLE,
              nrhs: int = 1, out: np.ndarray = None) -> np.ndarray:
        """`out`, when given, is a contiguous float64 array of the result's size
        (e.g. page-locked memory: the Schur operator between page-locked arrays
        overlaps its copies with the stencils)."""
        full = op in (OP_WILSON_FULL, OP_CLOVER_FULL)
        n = (24 * self.V if full else 12 * self.V) * nrhs
        f = _f64(f, n, "spinor")
        if out is None:
            out = np.empty(n)
        elif (not isinstance(out, np.ndarray) or out.dtype != np.float64 or out.size != n
              or not out.flags.c_contiguous or not out.flags.writeable):
            raise IroError(BAD_ARG, f"apply: out must be a writable contiguous float64 array of {n}")
        self.check(self._lib.iro_dirac_apply(self.h, op, mass, csw, int(bool(dag)), _PREC[prec],
                                             _ptr(f), _ptr(out), nrhs), "iro_dirac_apply")
        return out

    def gamma5(self, f: np.ndarray) -> np.ndarray:
        f = _f64(f)
        if f.size % 24:
            raise IroError(BAD_ARG, "gamma5: spinor size not a multiple of 24")
        out = np.empty_like(f)
        self.check(self._lib.iro_gamma5(self.h, _ptr(f), _ptr(out), f.size // 24), "iro_gamma5")
        return out

    def field_strength(self, mu: int, nu: int) -> np.ndarray:
        out = np.empty(18 * self.V)
        self.check(self._lib.iro_field_strength(self.h, mu, nu, _ptr(out)), "iro_field_strength")
        return out


class DeviceField:
    """A spinor field resident on the GPU (iro_field): subset 0 even half,
    1 odd half, 2 full lattice; nrhs right-hand sides in the device layout
    of `prec`.  upload/download convert from/to Format_F host arrays."""

    def __init__(self, ctx: Context, subset: int, prec="double", nrhs: int = 1):
        self.ctx, self.subset, self.prec, self.nrhs = ctx, subset, _PREC[prec], nrhs
        h = _VP()
        ctx.check(ctx._lib.iro_field_create(ctx.h, subset, self.prec, nrhs, ctypes.byref(h)),
                  "iro_field_create")
        self.h = h
        ctx._owned.add(self)

    @property
    def size(self) -> int:
        return (24 if self.subset == 2 else 12) * self.ctx.V * self.nrhs

    def upload(self, f):
        f = _f64(f, self.size, "spinor")
        self.ctx.check(self.ctx._lib.iro_field_upload(self.ctx.h, self.h, _ptr(f)), "iro_field_upload")
        return self

    def download(self) -> np.ndarray:
        out = np.empty(self.size)
        self.ctx.check(self.ctx._lib.iro_field_download(self.ctx.h, self.h, _ptr(out)),
                       "iro_field_download")
        return out

    def norm(self) -> np.ndarray:
        """Field::norm() per right-hand side (include/field.h:74-78)."""
        out = np.empty(self.nrhs)
        self.ctx.check(self.ctx._lib.iro_field_norm(self.ctx.h, self.h, _ptr(out)), "iro_field_norm")
        return out

    def dot(self, other: "DeviceField") -> np.ndarray:
        """Field::operator* per right-hand side (lib/Fields/field.inl:58-62)."""
        out = np.empty(self.nrhs)
        self.ctx.check(self.ctx._lib.iro_field_dot(self.ctx.h, self.h, other.h, _ptr(out)),
                       "iro_field_dot")
        return out

    def close(self):
        if getattr(self, "h", None):
            self.ctx._lib.iro_field_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_contexts: dict = {}


def context(L, device: int = 0) -> Context:
    """The shared context of lattice L on `device` (created on first use)."""
    key = (tuple(int(v) for v in L), device)
    if key not in _contexts:
        _contexts[key] = Context(L, device)
    return _contexts[key]


_default_L = None


def init(L, device: int = 0) -> Context:
    """Sets the lattice used by operators built without an explicit context,
    as CommonPrms::instance(Lattice) does for the reference."""
    global _default_L
    _default_L = (tuple(int(v) for v in L), device)
    return context(L, device)


def _ctx_for(u: np.ndarray, ctx):
    if ctx is not None:
        return ctx
    if _default_L is None:
        raise IroError(BAD_ARG, "no lattice: call iroiro_b200.init(L) or pass ctx=")
    return context(*_default_L)


# ---- operators ---------------------------------------------------------------------

class _Dirac:
    op: int
    csw = 0.0

    def __init__(self, mass: float, u: np.ndarray, ctx=None, prec="double"):
        self.ctx = _ctx_for(u, ctx)
        self.mass = float(mass)
        self.u = u
        self.prec = _PREC[prec]
        self.ctx.upload_gauge(u)

    def update_internal_state(self):
        """Re-reads the gauge field (Dirac::update_internal_state, dirac.hpp:28)."""
        self.ctx.upload_gauge(self.u, force=True)

    def _apply(self, op, dag, f, nrhs=1):
        self.ctx.upload_gauge(self.u)
        return self.ctx.apply(op, self.mass, self.csw, dag, f, self.prec, nrhs)

    def mult(self, f):
        return self._apply(self.op, False, f)

    def mult_dag(self, f):
        return self._apply(self.op, True, f)

    def gamma5(self, f):
        return self.ctx.gamma5(f)

    def getKappa(self) -> float:
        return 0.5 / (4.0 + self.mass)

    def getMass(self) -> float:
        return self.mass

    def gsize(self) -> int:
        return 72 * self.ctx.V

    def getGaugeField_ptr(self):
        return self.u

    def md_force(self, eta: np.ndarray, zeta: np.ndarray) -> np.ndarray:
        """The MD force zeta^dag dD/dU eta as a Format_G field (gsize doubles),
        Re Tr(X F_mu(x)) = d/de Re(zeta^dag D(U_mu(x) -> (1 + e X) U_mu(x)) eta):
        Dirac_Wilson::md_force (lib/Dirac_ops/dirac_wilson.cpp:41-58) for the
        full operator, Dirac_Wilson_EvenOdd::md_force
        (dirac_wilson_EvenOdd.hpp:95-117) for the e/o one, Dirac_Clover::md_force
        (dirac_clover.cpp:356-532) for the full clover operator."""
        if self.op not in (OP_WILSON_FULL, OP_WILSON_SCHUR_EE, OP_CLOVER_FULL):
            raise IroError(BAD_ARG, "md_force: Wilson full or even/odd, or full clover operator")
        self.ctx.upload_gauge(self.u)
        n = self.fsize()
        eta, zeta = _f64(eta, n, "eta"), _f64(zeta, n, "zeta")
        F = np.empty(self.gsize())
        self.ctx.check(self.ctx._lib.iro_md_force(self.ctx.h, self.op, self.mass, self.csw,
                                                  _ptr(eta), _ptr(zeta), _ptr(F)), "iro_md_force")
        return F


class Dirac_Wilson(_Dirac):
    """Dirac_Wilson(mass, u[, tag]).  tag None: full lattice, mult = f - kappa H f;
    "EO": -kappa D_eo (odd -> even); "OE": -kappa D_oe (even -> odd)
    (lib/Dirac_ops/dirac_wilson.hpp:89-128)."""

    def __init__(self, mass, u, tag=None, ctx=None, prec="double"):
        super().__init__(mass, u, ctx, prec)
        self.tag = tag
        self.op = {None: OP_WILSON_FULL, "EO": OP_WILSON_HOP_EO, "OE": OP_WILSON_HOP_OE}[tag]

    def fsize(self) -> int:
        return 24 * self.ctx.V if self.tag is None else 12 * self.ctx.V


class Dirac_Wilson_EvenOdd(_Dirac):
    """Dirac_Wilson_EvenOdd<Dirac_Wilson>: the Schur operator f - Deo(Doe f) on
    even half fields (lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:24-92)."""

    op = OP_WILSON_SCHUR_EE

    def fsize(self) -> int:
        return 12 * self.ctx.V

    def mult_eo(self, f):
        return self._apply(OP_WILSON_HOP_EO, False, f)

    def mult_oe(self, f):
        return self._apply(OP_WILSON_HOP_OE, False, f)

    def mult_eo_dag(self, f):  # Doe_.mult_dag (dirac_wilson_EvenOdd.hpp:70-73)
        return self._apply(OP_WILSON_HOP_OE, True, f)

    def mult_oe_dag(self, f):  # Deo_.mult_dag (dirac_wilson_EvenOdd.hpp:75-78)
        return self._apply(OP_WILSON_HOP_EO, True, f)

    def mult_ee(self, f):
        return np.array(f, dtype=np.float64, copy=True)

    mult_oo = mult_ee_inv = mult_oo_inv = mult_ee

    def getDeo(self):
        return Dirac_Wilson(self.mass, self.u, "EO", self.ctx, self.prec)

    def getDoe(self):
        return Dirac_Wilson(self.mass, self.u, "OE", self.ctx, self.prec)


class Dirac_Clover(_Dirac):
    """Dirac_Clover(Dw, csw, u): Wilson plus clover, full lattice
    (lib/Dirac_ops/dirac_clover.hpp:57-69).  Unlike the reference it does not
    take ownership of (or delete) Dw; it only reads its mass."""

    op = OP_CLOVER_FULL

    def __init__(self, Dw, csw, u, ctx=None, prec="double"):
        super().__init__(Dw.getMass(), u, ctx or getattr(Dw, "ctx", None), prec)
        self.csw = float(csw)
        self.ctx.check(self.ctx._lib.iro_clover_setup(self.ctx.h, self.mass, self.csw),
                       "iro_clover_setup")

    def fsize(self) -> int:
        return 24 * self.ctx.V

    def update_internal_state(self):
        super().update_internal_state()
        self.ctx.check(self.ctx._lib.iro_clover_setup(self.ctx.h, self.mass, self.csw),
                       "iro_clover_setup")


class Dirac_Clover_EvenOdd(Dirac_Clover):
    """The even-odd Schur complement of Dirac_Clover, A_ee - kappa^2 H_eo A_oo^-1 H_oe,
    on even half fields.  The reference has no e/o clover operator."""

    op = OP_CLOVER_SCHUR_EE

    def __init__(self, mass, csw, u, ctx=None, prec="double"):
        _Dirac.__init__(self, mass, u, ctx, prec)
        self.csw = float(csw)
        self.ctx.check(self.ctx._lib.iro_clover_setup(self.ctx.h, self.mass, self.csw),
                       "iro_clover_setup")

    def fsize(self) -> int:
        return 12 * self.ctx.V


class Fopr_DdagD:
    """D^dagger D (lib/Fopr/fopr.h:146-153)."""

    def __init__(self, D):
        self.D = D

    def mult(self, f):
        return self.D.mult_dag(self.D.mult(f))

    def mult_dag(self, f):
        return self.mult(f)

    def func(self, x):
        return x

    def fsize(self):
        return self.D.fsize()


# ---- solvers -----------------------------------------------------------------------

@dataclass
class SolverOutput:
    """lib/Solver/solver.hpp:16-22."""

    diff: float
    Iterations: int
    timing: float
    Msg: str
    reliable_updates: int = 0
    operator_applies: int = 0

    def print(self, Msg2: str = ""):
        print(f" {self.Msg} {Msg2}\n  Iterations = {self.Iterations}\n  Residual   = "
              f"{self.diff:.6e}\n  Timing     = {self.timing:.3f} ms")


_SOLVER_OPS = (OP_WILSON_FULL, OP_WILSON_SCHUR_EE, OP_CLOVER_FULL, OP_CLOVER_SCHUR_EE)


class Solver_CG:
    """Solver_CG(prec, MaxIter, Fopr_DdagD(D)) (lib/Solver/solver_CG.hpp:28-31).

    ``prec`` is the squared relative residual target (GoalPrecision).
    ``inner`` selects the reference's FP64 CG ("double") or the reliable-update
    mixed-precision CG with FP32 ("single") or FP16 ("half") inner storage."""

    def __init__(self, prec: float, MaxIter: int, fopr: Fopr_DdagD, inner="double",
                 delta: float = 0.1, use_graph: bool = True):
        if not isinstance(fopr, Fopr_DdagD) or fopr.D.op not in _SOLVER_OPS:
            raise IroError(BAD_ARG, "Solver_CG needs Fopr_DdagD of a full or Schur operator")
        self.fopr = fopr
        self.params = CGParams(float(prec), int(MaxIter), _PREC[inner], float(delta),
                               int(bool(use_graph)))

    def check_DdagD(self) -> bool:
        return True

    def solve_many(self, b: np.ndarray, nrhs: int):
        """Solves nrhs right-hand sides together (one link load serves all).
        Returns (x, [SolverOutput]) without raising on non-convergence."""
        D = self.fopr.D
        D.ctx.upload_gauge(D.u)
        b = _f64(b, D.fsize() * nrhs, "source")
        x = np.empty_like(b)
        outs = (SolverOut * nrhs)()
        rc = D.ctx._lib.iro_cg_solve(D.ctx.h, D.op, D.mass, D.csw, ctypes.byref(self.params),
                                     _ptr(b), _ptr(x), nrhs, outs)
        if rc not in (OK, NOT_CONVERGED):
            D.ctx.check(rc, "iro_cg_solve")
        res = [SolverOutput(o.diff, o.iterations, o.timing_ms, "CG solver", o.reliable_updates,
                            o.operator_applies) for o in outs]
        return x, res, rc

    def solve_field(self, b: "DeviceField", x: "DeviceField"):
        """Solves on device-resident FP64 fields (all right-hand sides of b
        together), without host traffic.  Returns ([SolverOutput], status)."""
        D = self.fopr.D
        D.ctx.upload_gauge(D.u)
        outs = (SolverOut * b.nrhs)()
        rc = D.ctx._lib.iro_cg_solve_field(D.ctx.h, D.op, D.mass, D.csw, ctypes.byref(self.params),
                                           b.h, x.h, outs)
        if rc not in (OK, NOT_CONVERGED):
            D.ctx.check(rc, "iro_cg_solve_field")
        return [SolverOutput(o.diff, o.iterations, o.timing_ms, "CG solver", o.reliable_updates,
                             o.operator_applies) for o in outs], rc

    def solve(self, xq: np.ndarray, b: np.ndarray) -> SolverOutput:
        """Solver_CG::solve(Field& xq, const Field& b) (solver_CG.cpp:29-80)."""
        x, res, rc = self.solve_many(b, 1)
        if rc == NOT_CONVERGED:
            raise ConvergenceError(rc, "CG solver not converged")
        xq[...] = x.reshape(xq.shape)
        return res[0]


class MultiShiftSolver_CG:
    """MultiShiftSolver_CG(Fopr_DdagD(D), stop_cond, Niter)
    (lib/Solver/multiShiftSolver_CG.hpp:61-65).  inner="double" is the
    reference's FP64 solver; "single" or "half" the mixed-precision one
    (FP32 multishift with FP64 recurrences, then a reliable-update CG
    refinement of all shifts as one block in that storage), with the same
    FP64 true-residual contract."""

    def __init__(self, fopr: Fopr_DdagD, stop_cond: float, Niter: int, inner: str = "double"):
        if not isinstance(fopr, Fopr_DdagD) or fopr.D.op not in _SOLVER_OPS:
            raise IroError(BAD_ARG, "MultiShiftSolver_CG needs Fopr_DdagD of a full or Schur operator")
        self.fopr = fopr
        self.prec = float(stop_cond)
        self.niter = int(Niter)
        self.inner = _PREC[inner]

    def solve(self, xq: list, b: np.ndarray, shifts) -> SolverOutput:
        """solve(vector_Field& x, const Field& b, const vector_double& shifts,
        double& diff, int& Nconv) (multiShiftSolver_CG.cpp:95-185).  The
        returned SolverOutput carries .diff and .Nconv; xq[i] are filled."""
        D = self.fopr.D
        D.ctx.upload_gauge(D.u)
        n = D.fsize()
        b = _f64(b, n, "source")
        sh = _f64(shifts)
        x = np.empty(n * sh.size)
        o = SolverOut()
        nconv = ctypes.c_int(-1)
        rc = D.ctx._lib.iro_multishift_cg_solve_mixed(D.ctx.h, D.op, D.mass, D.csw, _ptr(b),
                                                      sh.size, _ptr(sh), _ptr(x), self.prec,
                                                      self.niter, self.inner, ctypes.byref(o),
                                                      ctypes.byref(nconv))
        D.ctx.check(rc, "iro_multishift_cg_solve")
        x = x.reshape(sh.size, n)
        for i in range(sh.size):
            if i < len(xq):
                xq[i][...] = x[i]
            else:
                xq.append(x[i].copy())
        out = SolverOutput(o.diff, o.iterations, o.timing_ms, "Multishift CG solver",
                           o.reliable_updates, o.operator_applies)
        out.Nconv = nconv.value
        return out

    def solve_field(self, b: "DeviceField", x: "DeviceField", shifts) -> SolverOutput:
        """The solve on device-resident FP64 fields, without host traffic: b
        one right-hand side, x one right-hand side per shift."""
        D = self.fopr.D
        D.ctx.upload_gauge(D.u)
        sh = _f64(shifts)
        o = SolverOut()
        nconv = ctypes.c_int(-1)
        rc = D.ctx._lib.iro_multishift_cg_solve_field(D.ctx.h, D.op, D.mass, D.csw, b.h, sh.size,
                                                      _ptr(sh), x.h, self.prec, self.niter,
                                                      self.inner, ctypes.byref(o),
                                                      ctypes.byref(nconv))
        D.ctx.check(rc, "iro_multishift_cg_solve_field")
        out = SolverOutput(o.diff, o.iterations, o.timing_ms, "Multishift CG solver",
                           o.reliable_updates, o.operator_applies)
        out.Nconv = nconv.value
        return out


# ---- rational functions of D^dag D ---------------------------------------------------

class RationalApprox:
    """The numbers RationalSolver_CG takes from RationalApprox
    (lib/Tools/RationalApprox/rationalapprox.hpp:85-91):
    f(x) = Const + sum_i Residuals[i] / (x + Poles[i]) and its inverse.  The
    reference computes them with a GMP Remez algorithm; here they are given."""

    def __init__(self, const, residues, poles, inv_const=0.0, inv_residues=(), inv_poles=()):
        self._c, self._r, self._p = float(const), [float(v) for v in residues], [float(v) for v in poles]
        self._ic, self._ir = float(inv_const), [float(v) for v in inv_residues]
        self._ip = [float(v) for v in inv_poles]
        if len(self._r) != len(self._p) or len(self._ir) != len(self._ip):
            raise IroError(BAD_ARG, "residues and poles differ in number")

    def Residuals(self): return list(self._r)
    def Poles(self): return list(self._p)
    def Const(self): return self._c
    def InvResiduals(self): return list(self._ir)
    def InvPoles(self): return list(self._ip)
    def InvConst(self): return self._ic


class RationalSolver_CG:
    """RationalSolver_CG(MultiShiftSolver_CG, RationalApprox)
    (lib/Solver/rationalSolver_CG.hpp:35-44).  solve(sol, b):
    sol = Const b + sum_i Residuals[i] (D^dag D + Poles[i])^-1 b, reconstructed
    on the device; solve_inv uses the inverse approximation;
    solve_noReconstruct(_inv) return the shifted solutions."""

    def __init__(self, ms: "MultiShiftSolver_CG", ra: RationalApprox = None):
        self.ms = ms
        self.ra = ra

    def set_Approx(self, ra: RationalApprox):
        self.ra = ra

    def _solve(self, sol, b, c0, res, poles, what):
        if self.ra is None or not res:
            raise IroError(BAD_ARG, f"[RationalSolver] {what} rational approximation not initialized yet")
        D = self.ms.fopr.D
        D.ctx.upload_gauge(D.u)
        n = D.fsize()
        b = _f64(b, n, "source")
        p, r = _f64(poles), _f64(res)
        out = np.empty(n)
        o = SolverOut()
        nconv = ctypes.c_int(-1)
        rc = D.ctx._lib.iro_rational_cg_solve(D.ctx.h, D.op, D.mass, D.csw, _ptr(b), p.size, _ptr(p),
                                              _ptr(r), c0, _ptr(out), self.ms.prec, self.ms.niter,
                                              ctypes.byref(o), ctypes.byref(nconv))
        D.ctx.check(rc, "iro_rational_cg_solve")
        sol[...] = out
        res_out = SolverOutput(o.diff, o.iterations, o.timing_ms, "Multishift CG solver", 0,
                               o.operator_applies)
        res_out.Nconv = nconv.value
        return res_out

    def solve(self, sol: np.ndarray, b: np.ndarray) -> SolverOutput:
        ra = self.ra
        return self._solve(sol, b, ra.Const() if ra else 0.0, ra.Residuals() if ra else [],
                           ra.Poles() if ra else [], "")

    def solve_inv(self, sol: np.ndarray, b: np.ndarray) -> SolverOutput:
        ra = self.ra
        return self._solve(sol, b, ra.InvConst() if ra else 0.0, ra.InvResiduals() if ra else [],
                           ra.InvPoles() if ra else [], "Inverse")

    def solve_noReconstruct(self, shifted_sol: list, b: np.ndarray) -> SolverOutput:
        if self.ra is None or not self.ra.InvPoles():
            raise IroError(BAD_ARG, "[RationalSolver] Inverse rational approximation not initialized yet")
        return self.ms.solve(shifted_sol, b, self.ra.InvPoles())

    def solve_noReconstruct_inv(self, shifted_sol: list, b: np.ndarray) -> SolverOutput:
        if self.ra is None or not self.ra.Poles():
            raise IroError(BAD_ARG, "[RationalSolver] Rational approximation not initialized yet")
        return self.ms.solve(shifted_sol, b, self.ra.Poles())


# ---- propagators: e/o inversion and the 12 spin-colour sources --------------------------

class Source_local:
    """Source_local (lib/Measurements/FermionicM/source_types.hpp:22-66): a
    point source at lattice coordinates sp = [x, y, z, t]; mksrc(s, c) is the
    full-lattice Format_F field with 1 at index_r(c, s, site)."""

    def __init__(self, sp, L):
        self.sp, self.L = [int(v) for v in sp], [int(v) for v in L]
        x, y, z, t = (self.sp[i] % self.L[i] for i in range(4))
        self.site = x + self.L[0] * (y + self.L[1] * (z + self.L[2] * t))
        self.V = int(np.prod(self.L))

    def mksrc(self, s: int, c: int) -> np.ndarray:
        f = np.zeros(24 * self.V)
        f[2 * (c + 3 * s) + 24 * self.site] = 1.0
        return f


class Inverter_WilsonLike:
    """EvenOddUtils::Inverter_WilsonLike(D, solver) (lib/Dirac_ops/eoUtils.hpp:23-48)
    for D a Dirac_Wilson_EvenOdd or Dirac_Clover_EvenOdd and solver a
    Solver_CG on Fopr_DdagD(D): invert(sol, src) solves the full-lattice
    system through the Schur complement (eoUtils.cpp:43-81)."""

    def __init__(self, D, solver: "Solver_CG"):
        if D.op not in (OP_WILSON_SCHUR_EE, OP_CLOVER_SCHUR_EE):
            raise IroError(BAD_ARG, "Inverter_WilsonLike needs an even/odd operator")
        self.D, self.slv = D, solver

    def invert_many(self, src: np.ndarray, nrhs: int):
        """nrhs full-lattice sources at once; returns (sol, [SolverOutput], status)."""
        D = self.D
        D.ctx.upload_gauge(D.u)
        n = 24 * D.ctx.V
        src = _f64(src, n * nrhs, "source")
        sol = np.empty_like(src)
        outs = (SolverOut * nrhs)()
        rc = D.ctx._lib.iro_eo_invert(D.ctx.h, D.op, D.mass, D.csw, ctypes.byref(self.slv.params),
                                      _ptr(src), _ptr(sol), nrhs, outs)
        if rc not in (OK, NOT_CONVERGED):
            D.ctx.check(rc, "iro_eo_invert")
        res = [SolverOutput(o.diff, o.iterations, o.timing_ms, "CG solver", o.reliable_updates,
                            o.operator_applies) for o in outs]
        return sol, res, rc

    def invert(self, sol: np.ndarray, src: np.ndarray) -> SolverOutput:
        x, res, rc = self.invert_many(src, 1)
        if rc != OK:
            raise ConvergenceError(rc, "Inverter_WilsonLike: CG not converged")
        sol[...] = x
        return res[0]


class Qprop_EvenOdd:
    """Qprop_EvenOdd(D, solver) (lib/Measurements/FermionicM/qprop_EvenOdd.hpp:17-36):
    calc(src) returns the 12 solutions D^-1 src.mksrc(s, c), s-major, computed
    as ONE block of 12 right-hand sides (the reference runs 12 inversions,
    qprop_EvenOdd.cpp:10-21)."""

    def __init__(self, D, solver: "Solver_CG"):
        self.inv = Inverter_WilsonLike(D, solver)
        self.last_outputs = []

    def calc(self, src, s=None, c=None, out=None) -> list:
        """The 12 solutions (s-major), or with s and c the one solution of
        source (s, c) as the reference's calc(xq, src, s, c)
        (qprop_EvenOdd.cpp:24-28).  The point sources of a Source_local are
        built on the device (iro_qprop_point) instead of as host fields.
        `out`, an array of (number of sources) * 24 * V doubles that the
        caller keeps across calls (the reference's prop_t xq), receives the
        solutions; the returned arrays are views of it."""
        one = s is not None
        nsrc = 1 if one else (len(src) if isinstance(src, (list, tuple)) else 12)
        D, slv = self.inv.D, self.inv.slv
        n = 24 * D.ctx.V
        if out is not None:
            o = _f64(out, n * nsrc, "out")
            if not np.shares_memory(o, out):
                raise IroError(BAD_ARG, "out must be a contiguous float64 array")
        if isinstance(src, Source_local):
            D.ctx.upload_gauge(D.u)
            x = np.empty(n * nsrc) if out is None else o
            outs = (SolverOut * nsrc)()
            first = 3 * s + c if one else 0
            rc = D.ctx._lib.iro_qprop_point(D.ctx.h, D.op, D.mass, D.csw, ctypes.byref(slv.params),
                                            src.site, first, nsrc, _ptr(x), outs)
            if rc not in (OK, NOT_CONVERGED):
                D.ctx.check(rc, "iro_qprop_point")
            res = [SolverOutput(o.diff, o.iterations, o.timing_ms, "CG solver", o.reliable_updates,
                                o.operator_applies) for o in outs]
        else:
            if isinstance(src, (list, tuple)):
                srcs = np.stack([_f64(f) for f in src])
            elif one:
                srcs = src.mksrc(s, c)[None, :]
            else:
                srcs = np.stack([src.mksrc(sp, cp) for sp in range(4) for cp in range(3)])
            x, res, rc = self.inv.invert_many(srcs.ravel(), nsrc)
            if out is not None:
                o.reshape(-1)[...] = x
                x = o
        self.last_outputs = res
        if rc != OK:
            raise ConvergenceError(rc, "Qprop_EvenOdd: CG not converged")
        return list(x.reshape(nsrc, -1))


class Qprop:
    """Qprop(D, solver) (lib/Measurements/FermionicM/qprop.cpp:8-25) on the
    full-lattice operator: sol = (D^dag D)^-1 D^dag src for the 12 point
    sources, solved as one block."""

    def __init__(self, D, solver: "Solver_CG"):
        if D.op not in (OP_WILSON_FULL, OP_CLOVER_FULL):
            raise IroError(BAD_ARG, "Qprop needs a full-lattice operator")
        self.D, self.slv = D, solver
        self.last_outputs = []

    def calc(self, src) -> list:
        if isinstance(src, (list, tuple)):
            srcs = [_f64(f) for f in src]
        else:
            srcs = [src.mksrc(s, c) for s in range(4) for c in range(3)]
        b = np.concatenate([self.D.mult_dag(f) for f in srcs])
        x, res, rc = self.slv.solve_many(b, len(srcs))
        self.last_outputs = res
        if rc != OK:
            raise ConvergenceError(rc, "Qprop: CG not converged")
        return list(x.reshape(len(srcs), -1))


class Qprop_MultiShift:
    """Qprop_MultiShift(D, solver) (lib/Measurements/FermionicM/qprop_MultiShift.hpp:20-42):
    calc(src, mass_shifts) solves, source by source (s-major, as
    qprop_MultiShift.cpp:11-31), (D^dag D + sigma_m) x_m = src.mksrc(s, c) for
    every shift with the multishift solver and returns D x_m, one propagator
    per source and shift (shift fastest).  The reference sizes its solution
    vector to Nc * Nd = 12 whatever the number of shifts, so it returns 12
    fields per source (the trailing ones zero when fewer shifts are given);
    this returns one per shift."""

    def __init__(self, D, solver: "MultiShiftSolver_CG"):
        self.D, self.slv = D, solver
        self.last_outputs = []

    def calc(self, src, mass_shifts) -> list:
        srcs = list(src) if isinstance(src, (list, tuple)) else \
            [src.mksrc(s, c) for s in range(4) for c in range(3)]
        out, self.last_outputs = [], []
        for b in srcs:
            xs = []
            self.last_outputs.append(self.slv.solve(xs, b, mass_shifts))
            out.extend(self.D.mult(x) for x in xs)
        return out


# gauge-configuration files (GaugeConf_*, CCIO::SaveOnDisk, Staples::plaquette)
from .gaugeconf import (GaugeConf, GaugeConf_bin, GaugeConf_csdt, GaugeConf_ILDG,  # noqa: E402
                        GaugeConf_ILDG_FORTRAN, GaugeConf_JLQCDLegacy, GaugeConf_NERSC,
                        GaugeConf_txt, GaugeConf_unit, GaugeInfo, link_trace, plaquette,
                        read_gauge, save_on_disk)
