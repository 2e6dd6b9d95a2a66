"""Runs the reference's own classes (oracle/_ref/libiroiro_ref.so) in a child
process -- test infrastructure.

The compiled reference keeps its lattice in process-wide singletons
(CommonPrms, SiteIndex, SiteIndex_EvenOdd), so one process serves one lattice
size.  The parity tests at the benchmark configurations need several
lattices, so each batch of reference computations runs in a fresh child:
``run(L, arrays, jobs)`` writes the input arrays to a temporary directory,
starts ``python tests/refproc.py <dir>``, which calls the reference for every
job, and returns the outputs.

A job is a dict with "op" one of
  wilson_full  Dirac_Wilson::mult / mult_dag            (dirac_wilson.cpp:28-36)
  wilson_eo    Dirac_Wilson_EvenOdd::mult / mult_dag    (dirac_wilson_EvenOdd.hpp:80-92)
  clover_full  Dirac_Clover::mult / mult_dag            (dirac_clover.cpp:334-353)
  cg           Solver_CG::solve on Fopr_DdagD(D)        (solver_CG.cpp:29-80)
and the names of its input arrays ("u", "f" or "b") plus its scalars.  The
OpenMP thread count of the reference's CG is pinned to 4 (its BLAS loops drop
tail elements when the thread count does not divide the field size).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


ADAPTER_LIB = ROOT / "oracle" / "_ref" / "libadapter_check.so"


def available() -> bool:
    return (ROOT / "oracle" / "_ref" / "libiroiro_ref.so").exists()


def adapter_available() -> bool:
    return ADAPTER_LIB.exists()


def run(L, arrays: dict, jobs: list, timeout: float = 1800.0, lib: str = "ref") -> list:
    with tempfile.TemporaryDirectory() as d:
        for k, v in arrays.items():
            np.save(os.path.join(d, k + ".npy"), np.ascontiguousarray(v, np.float64))
        with open(os.path.join(d, "jobs.json"), "w") as fh:
            json.dump({"L": [int(v) for v in L], "jobs": jobs, "lib": lib}, fh)
        env = dict(os.environ, OMP_NUM_THREADS="4", PYTHONPATH=str(ROOT))
        r = subprocess.run([sys.executable, str(Path(__file__).resolve()), d], env=env,
                           capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference child failed ({r.returncode}):\n{r.stderr[-3000:]}")
        out = []
        for i, job in enumerate(jobs):
            res = {k[len(f"out{i}_"):-4]: np.load(os.path.join(d, k))
                   for k in os.listdir(d) if k.startswith(f"out{i}_") and k.endswith(".npy")}
            res["x"] = np.load(os.path.join(d, f"out{i}.npy"))
            meta = os.path.join(d, f"out{i}.json")
            if os.path.exists(meta):
                with open(meta) as fh:
                    res.update(json.load(fh))
            out.append(res)
        return out


def _child(d: str) -> int:
    import resource

    # the reference's improved kernels keep boundary slices in stack arrays
    try:
        resource.setrlimit(resource.RLIMIT_STACK, (resource.RLIM_INFINITY, resource.RLIM_INFINITY))
    except (ValueError, OSError):
        pass
    import oracle

    with open(os.path.join(d, "jobs.json")) as fh:
        spec = json.load(fh)
    if spec.get("lib") == "adapter":
        return _adapter_child(d, spec)
    ref = oracle.ref()
    ref.init(spec["L"])
    cache = {}

    def arr(name):
        if name not in cache:
            cache[name] = np.load(os.path.join(d, name + ".npy"))
        return cache[name]

    for i, job in enumerate(spec["jobs"]):
        op = job["op"]
        u = arr(job.get("u", "u"))
        meta = None
        if op == "wilson_full":
            x = ref.wilson_full(u, job["mass"], job.get("dag", 0), arr(job["f"]))
        elif op == "wilson_eo":
            x = ref.wilson_eo(u, job["mass"], job.get("dag", 0), arr(job["f"]))
        elif op == "clover_full":
            x = ref.clover_full(u, job["mass"], job["csw"], job.get("dag", 0), arr(job["f"]))
        elif op == "cg":
            x, it, diff, ms = ref.cg(u, job["kind"], job["mass"], job.get("csw", 0.0), arr(job["b"]),
                                     job["prec"], job["maxiter"])
            meta = {"iterations": it, "diff": diff, "ms": ms}
        else:
            raise ValueError(op)
        np.save(os.path.join(d, f"out{i}.npy"), x)
        if meta is not None:
            with open(os.path.join(d, f"out{i}.json"), "w") as fh:
                json.dump(meta, fh)
    return 0


def _adapter_child(d: str, spec: dict) -> int:
    """The adapter check library (oracle/ref/adapter_check.cpp): each job runs
    the reference's classes and the adapters over libiroiro_b200; "x" is the
    adapters' result, "ref" the reference's."""
    import ctypes

    D = ctypes.POINTER(ctypes.c_double)
    lib = ctypes.CDLL(str(ADAPTER_LIB))
    lib.ref_init.argtypes = [ctypes.c_int] * 4
    if lib.ref_init(*spec["L"]):
        raise RuntimeError("ref_init failed")
    p = lambda a: a.ctypes.data_as(D)  # noqa: E731
    V = int(np.prod(spec["L"]))
    for i, job in enumerate(spec["jobs"]):
        u = np.load(os.path.join(d, job.get("u", "u") + ".npy"))
        meta = None
        if job["op"] == "adapter_eo_mult":
            f = np.load(os.path.join(d, job["f"] + ".npy"))
            xb, xr = np.empty_like(f), np.empty_like(f)
            rc = lib.adapter_eo_mult(p(u), ctypes.c_double(job["mass"]), job.get("dag", 0), p(f),
                                     p(xb), p(xr))
        elif job["op"] == "adapter_cg":
            b = np.load(os.path.join(d, job["b"] + ".npy"))
            xb, xr = np.empty_like(b), np.empty_like(b)
            diff = (ctypes.c_double * 2)()
            its = (ctypes.c_int * 2)()
            rc = lib.adapter_cg(p(u), int(job["eo"]), ctypes.c_double(job["mass"]), p(b),
                                ctypes.c_double(job["prec"]), int(job["maxiter"]), p(xb), p(xr),
                                diff, its)
            meta = {"diff": [diff[0], diff[1]], "iterations": [its[0], its[1]]}
        elif job["op"] == "adapter_qprop_multishift":
            sh = np.ascontiguousarray(job["shifts"], np.float64)
            n = 12 * 12 * 24 * V
            xb, xr = np.empty(n), np.empty(n)
            site = (ctypes.c_int * 4)(*job["site"])
            rc = lib.adapter_qprop_multishift(p(u), ctypes.c_double(job["mass"]), site, sh.size, p(sh),
                                              ctypes.c_double(job["prec"]), int(job["maxiter"]),
                                              p(xb), p(xr))
        else:
            raise ValueError(job["op"])
        if rc:
            raise RuntimeError(f"{job['op']} returned {rc}")
        np.save(os.path.join(d, f"out{i}.npy"), xb)
        np.save(os.path.join(d, f"out{i}_ref.npy"), xr)
        if meta is not None:
            with open(os.path.join(d, f"out{i}.json"), "w") as fh:
                json.dump(meta, fh)
    return 0


if __name__ == "__main__":
    sys.exit(_child(sys.argv[1]))
