"""Build recipe of libiroiro_b200.so for sm_100a (B200).

Compiles every CUDA/C++ source under csrc/ with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into ``_build/`` and links the
shared library in-tree, next to this file, so that it travels with the
repository.  Sources compile in parallel; a source is rebuilt when it or any
header under csrc/ or include/ is newer than its object.

Usage: ``python -m iroiro_b200.build [-j N] [--force]``
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
BUILD = HERE / "_build"
LIB = HERE / "libiroiro_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = Path(cuda) / "bin" / "nvcc"
    return str(path) if path.exists() else (shutil.which("nvcc") or "nvcc")


def _host_cxx() -> str:
    # the system compiler links libstdc++ dynamically, which is what a library
    # loaded into a Python process next to torch needs
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else (shutil.which("g++") or "g++")


def _flags() -> list[str]:
    return ARCH + [
        "-O3", "-lineinfo", "-std=c++17", "-ccbin", _host_cxx(),
        "-Xcompiler", "-fPIC,-fopenmp", "-Xptxas", "-warn-spills",
        "-I", str(INCLUDE), "-I", str(CSRC),
    ]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src: Path, obj: Path, verbose: bool) -> tuple[Path, str]:
    cmd = [_nvcc(), *(_flags()), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [_nvcc(), "-x", "cu", *(_flags()), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(jobs: int = 0, force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    todo = [(s, o) for s, o in zip(srcs, objs) if force or _stale(s, o, newest)]
    if todo:
        n = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            for obj, err in ex.map(lambda so: _compile(so[0], so[1], verbose), todo):
                warn = [ln for ln in err.splitlines() if "spill" in ln.lower() and " 0 bytes" not in ln]
                if warn and verbose:
                    print(f"{obj.name}: " + "\n".join(warn))
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-ccbin", _host_cxx(), "-o", str(LIB),
               *[str(o) for o in objs], "-l:libgomp.so.1"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-j", "--jobs", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    lib = build(a.jobs, a.force, a.verbose)
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
