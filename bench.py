"""Benchmark of the even-odd Wilson Dslash hot path on B200.

Workload (one "step"): one application of the even-odd Schur operator
Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult, M f_e = f_e - kappa^2 H_eo H_oe f_e
(lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:80-84), on a 24^3x48 lattice, kappa =
0.12, seeded synthetic SU(3) links exp(i*0.2*H) followed by a random gauge
transformation, FP64 storage and arithmetic (the reference's own arithmetic),
reconstruct-12 links.  One step = two launches of the hopping kernel.

value     algorithmic GB/s of the step, fields resident in HBM, L2 flushed
          (256 MiB written) before every step, CUDA events on the launching
          stream around each step; summed over ranks (replicas) / max time.
e2e       the same metric through the C ABI with host buffers:
          iro_dirac_apply() on pinned Format_F arrays, H2D + D2H inside the
          timed region.
roofline  achieved = algorithmic bytes per hopping launch / its mean
          duration; bytes per even output site 2496 (8 neighbour spinors,
          8 two-row links, 1 output spinor) for the first hop and 2688
          (+ the f_e read of the fused x + a*y epilogue) for the second.
solve     time to a 1e-10 FP64 true relative residual on the e/o Wilson-
          clover Schur operator (csw=1.0) of the same field, for the
          reference's FP64 CG and the mixed-precision reliable-update CG.

--impl reference runs the reference's own C++ (compiled from its sources
into oracle/_ref) on the host cores for the same metric, config and step.
"""
from __future__ import annotations

import argparse
import re
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L = [24, 24, 24, 48]
KAPPA = 0.12
MASS = 0.5 / KAPPA - 4.0
CSW = 1.0
EPS = 0.2
SEED = 20240601
BYTES_HOP = 2496          # FP64, reconstruct-12, per even/odd output site
BYTES_XPAY = 192          # extra f_e read of the fused epilogue
FLOPS_SCHUR = 2 * 1320 + 48
METRIC = "EO-Wilson Dslash GB/s (FP64 Schur operator, algorithmic bytes)"
WORKLOAD = "Dirac_Wilson_EvenOdd::mult 24^3x48, kappa=0.12, FP64, recon-12"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self, wait_s: float = 15.0):
        """Starts sampling every 100 ms and waits for the first sample, so that
        the sampler's start-up does not fall inside the timed region."""
        import threading
        self.lines = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        first = threading.Event()

        def reader():
            for line in self.proc.stdout:
                self.lines.append((time.perf_counter(), line))
                first.set()

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()
        first.wait(wait_s)

    def mark(self):
        self.t_begin = time.perf_counter()

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        t_end = time.perf_counter()
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        t0 = getattr(self, "t_begin", 0.0)
        inside = [ln for t, ln in self.lines if t0 <= t <= t_end + 0.15]
        out = "".join(inside or [ln for _, ln in self.lines[-3:]])
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend: str = None):
    """One process per GPU (torchrun env); NCCL on GPUs, gloo when asked (the
    CPU tests of the replica path)."""
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = backend or "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def reduce_max(v: float, world: int) -> float:
    """Max over ranks (device times are reported as the slowest replica)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(step_bytes: float, steps: int, t_ms: float, world: int) -> float:
    """Whole-job GB/s of N independent replicas: every rank moves step_bytes
    per step, the job takes as long as its slowest rank."""
    t_max = reduce_max(t_ms, world)
    return world * step_bytes * steps / (t_max * 1e-3) / 1e9


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def traffic_per_launch(vh: int):
    """DRAM bytes (read + write) of one Schur application (both hop launches)
    from the committed ncu summary, scaled from the captured lattice to this
    one by the sites processed."""
    p = ROOT / "profiles" / "hop_fp64_24x24x24x48.txt"
    if not p.exists():
        return None
    m = re.search(r"^dram_bytes_per_site_schur:\s*([0-9.]+)", p.read_text(), re.M)
    return float(m.group(1)) * vh if m else None


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- reference arm ----------------------------------------------------------------------

def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libiroiro_ref.so was not built (needs the reference tree)"}))
        return 0
    import iroiro_b200 as ib
    V = int(np.prod(L))
    u = ib.synth_gauge(L, EPS, SEED, gauge_transform=True)
    f = ib.synth_gaussian(V // 2, SEED + 1)
    ref = oracle.ref()
    ref.init(L)
    threads = cpu_cores()
    for _ in range(min(args.warmup, 2)):
        ref.eo_mult_throughput(u, MASS, f, threads, 1)
    t = 0.0
    nsteps = max(1, min(args.steps, 20))  # bounded sample: a step takes ~1 s on the host
    for _ in range(nsteps):
        _, s = ref.eo_mult_throughput(u, MASS, f, threads, 1)
        t += s
    steps_bytes = (2 * BYTES_HOP + BYTES_XPAY) * (V // 2) * threads * nsteps
    val = steps_bytes / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": nsteps, "warmup": min(args.warmup, 2),
        "ms_per_step": round(1e3 * t / nsteps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": L, "kappa": KAPPA,
                   "sample": f"{threads} concurrent Dirac_Wilson_EvenOdd::mult per step"},
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"{threads} threads x 1 mult per step, {nsteps} steps (at most 20: one step takes about a second)"},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def schur_fp64_32(torch, device, steps, peak):
    """FP64 e/o Wilson Schur operator at 32^3x64, L2 flushed before every
    application, CUDA events on the launching stream; DRAM bytes per site
    from the ncu summary of this lattice."""
    import iroiro_b200 as ib
    Lb = [32, 32, 32, 64]
    Vh = int(np.prod(Lb)) // 2
    ctx = ib.Context(Lb, device)
    st = torch.cuda.current_stream()
    ctx.set_stream(st.cuda_stream)
    ctx.upload_gauge(ib.synth_gauge(Lb, EPS, SEED + 5, gauge_transform=True), force=True)
    a = ib.DeviceField(ctx, 0, "double").upload(ib.synth_gaussian(Vh, SEED + 6))
    b = ib.DeviceField(ctx, 0, "double")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=torch.device("cuda", device))
    lib = ctx._lib
    for _ in range(3):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, ib.OP_WILSON_SCHUR_EE, MASS, 0.0, 0, a.h, b.h), "apply")
    torch.cuda.synchronize()
    n = max(10, min(steps, 500))
    tot = 0.0
    for _ in range(n):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(st)
        ctx.check(lib.iro_dirac_apply_field(ctx.h, ib.OP_WILSON_SCHUR_EE, MASS, 0.0, 0, a.h, b.h), "apply")
        e.record(st)
        e.synchronize()
        tot += s.elapsed_time(e)
    ms = tot / n
    alg = (2 * BYTES_HOP + BYTES_XPAY) * Vh / (ms * 1e-3) / 1e9
    traffic = None
    p = ROOT / "profiles" / "hop_fp64_32x32x32x64_dram.txt"
    if p.exists():
        m = re.search(r"^dram_bytes_per_site_schur_32x32x32x64:\s*([0-9.]+)", p.read_text(), re.M)
        traffic = float(m.group(1)) * Vh if m else None
    out = {"ms_per_op": round(ms, 4), "GBps": round(alg, 1), "frac_of_measured_hbm": round(alg / peak, 3)}
    if traffic:
        dram = traffic / (ms * 1e-3) / 1e9
        out.update({"dram_GBps": round(dram, 1), "dram_frac_of_measured_hbm": round(dram / peak, 3)})
    ctx.close()
    return out


def timed_solves(ctx, D, b, nrhs, torch, inners=("double", "single", "half"), prec=1e-20,
                 delta=0.1):
    """Wall time of iro_cg_solve_field to a 1e-10 FP64 true residual for the
    reference's FP64 CG and the mixed-precision CG (device-resident fields)."""
    import iroiro_b200 as ib
    sub = 0 if D.op in (ib.OP_WILSON_SCHUR_EE, ib.OP_CLOVER_SCHUR_EE) else 2
    B = ib.DeviceField(ctx, sub, "double", nrhs).upload(b)
    X = ib.DeviceField(ctx, sub, "double", nrhs)
    res = {}
    for inner in inners:
        slv = ib.Solver_CG(prec, 20000, ib.Fopr_DdagD(D), inner=inner, delta=delta)
        slv.solve_field(B, X)  # warm-up: workspaces, autotuning, graph capture
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs, rc = slv.solve_field(B, X)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[inner] = {"ms": round(dt * 1e3, 2), "iterations": max(o.Iterations for o in outs),
                      "true_residual_max": max(o.diff for o in outs),
                      "reliable_updates": max(o.reliable_updates for o in outs),
                      "converged": rc == ib.OK}
    if "double" in res:
        for k in res:
            if k != "double":
                res[k]["speedup_vs_fp64_cg"] = round(res["double"]["ms"] / res[k]["ms"], 2)
    B.close()
    X.close()
    return res


def batched_solves(torch, device):
    """Batched configuration: 32^3x64 even-odd Wilson, kappa=0.12; the 12
    spin-colour point sources at one seeded site solved together (one
    launch sequence, every link load shared by the 12 right-hand sides) in
    mixed precision, against 12 sequential plain FP64 CG solves; and
    multishift CG with 12 shifts 1e-4..10 on one Gaussian source."""
    import iroiro_b200 as ib
    Lb = [32, 32, 32, 64]
    Vb = int(np.prod(Lb))
    ctx = ib.Context(Lb, device)
    s = torch.cuda.current_stream()
    ctx.set_stream(s.cuda_stream)
    u = ib.synth_gauge(Lb, EPS, SEED + 7, gauge_transform=False)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
    site = int(np.random.default_rng(SEED).integers(Vb // 2))
    src = ib.synth_point_sources(Vb // 2, site)
    out = {"op": "e/o Wilson Schur 32^3x64, kappa=0.12, 12 point sources at half-site %d" % site}
    # plain FP64 CG, one source after the other (what Qprop does, qprop.cpp:14-24)
    seq = timed_solves(ctx, D, src[0], 1, torch, inners=("double",))
    out["fp64_cg_one_source_ms"] = seq["double"]["ms"]
    out["fp64_cg_12_sequential_ms"] = round(12 * seq["double"]["ms"], 2)
    out["fp64_cg_iterations"] = seq["double"]["iterations"]
    # reliable updates when |r| fell by 0.02 (6 FP64 residual recomputations to
    # 1e-10, against 8 at 0.05, for 2-3 more iterations).  The FP16 block solve
    # is timed first, right after the FP64 baseline above, so that the two
    # numbers compared both follow one warm-up solve; timed after the FP64 and
    # FP32 block solves (seconds at the 1000 W cap) it ran at reduced clocks.
    blk = timed_solves(ctx, D, src.ravel(), 12, torch, inners=("half", "single", "double"),
                       delta=0.02)
    out["reliable_update_delta"] = 0.02
    for k, v in blk.items():
        v.pop("speedup_vs_fp64_cg", None)
        v["speedup_vs_12_fp64_cg"] = round(out["fp64_cg_12_sequential_ms"] / v["ms"], 2)
    out["block12"] = blk
    # multishift, 12 shifts geometrically spaced 1e-4..10, one Gaussian source
    shifts = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
    g = ib.synth_gaussian(Vb // 2, SEED + 9)
    ms = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 20000)
    xs = []
    ms.solve(xs, g, shifts)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    o = ms.solve(xs, g, shifts)
    torch.cuda.synchronize()
    out["multishift12"] = {"ms": round((time.perf_counter() - t0) * 1e3, 2), "iterations": o.Nconv,
                           "max_true_residual": o.diff}
    out["autotune"] = ctx.autotune_report()
    ctx.close()
    return out


def learned_solves(torch, device, nfields=24, epochs=15, widths=(4, 8, 8, 4), nkrylov=16):
    """Learned preconditioner: a PTC network trained by the library's own
    forward/backward kernels on pairs (b = D^dag D v, v) from `nfields` seeded
    16^3x32 gauge fields (eps=0.2, kappa=0.12), then applied inside flexible
    GCR at 32^3x64 (unseen field, one Gaussian source) against GCR without it
    and against CG on the same full-lattice D^dag D: FP64 and mixed precision.
    Every solve stops on the FP64 true residual 1e-10."""
    import iroiro_b200 as ib
    from iroiro_b200 import learned
    t0 = time.perf_counter()
    pairs = learned.make_pairs([16, 16, 16, 32], nfields, seed0=SEED + 300, device=device)
    net0 = learned.PTCNet(pairs[0].ctx, widths)
    hist = learned.train(net0, pairs, epochs=epochs, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    W = net0.W
    for pr in pairs:
        pr.ctx.close()
    Lb = [32, 32, 32, 64]
    Vb = int(np.prod(Lb))
    ctx = ib.Context(Lb, device)
    s = torch.cuda.current_stream()
    ctx.set_stream(s.cuda_stream)
    u = ib.synth_gauge(Lb, EPS, SEED + 301)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson(MASS, u, ctx=ctx)
    b = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(Vb, SEED + 302))
    net = learned.PTCNet(ctx, widths, W)
    out = {"op": "full-lattice Wilson D^dag D 32^3x64, kappa=0.12, one Gaussian source",
           "network": {"widths": list(widths), "train_fields": nfields, "train_lattice": "16^3x32",
                       "epochs": epochs, "train_s": round(train_s, 1),
                       "loss_first": round(hist[0], 4), "loss_last": round(hist[-1], 4)}}

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3, r

    for name, n in (("gcr_network", net), ("gcr_plain", None)):
        x = ib.DeviceField(ctx, 2, "double")
        slv = learned.Solver_GCR(D, n, nkrylov=nkrylov)
        ms, (o, rc) = timed(lambda: slv.solve_field(b, x))
        out[name] = {"ms": round(ms, 1), "iterations": o.iterations, "true_residual": o.diff,
                     "cg_fallback": bool(o.fallback), "converged": rc == ib.OK}
        x.close()
    for inner in ("double", "single", "half"):
        x = ib.DeviceField(ctx, 2, "double")
        slv = ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D), inner=inner)
        ms, (outs, rc) = timed(lambda: slv.solve_field(b, x))
        out["cg_" + inner] = {"ms": round(ms, 1), "iterations": outs[0].Iterations,
                              "true_residual": outs[0].diff, "converged": rc == ib.OK}
        x.close()
    a = ib.DeviceField(ctx, 2, "single").upload(ib.synth_gaussian(Vb, SEED + 303))
    c2 = ib.DeviceField(ctx, 2, "single")
    apply_ms, _ = timed(lambda: ctx.check(net.L.iro_ptc_apply_field(ctx.h, net.h, a.h, c2.h), "apply"))
    out["network_apply_ms"] = round(apply_ms, 3)
    best_cg = min(out["cg_single"]["ms"], out["cg_half"]["ms"])
    out["gcr_network_vs_best_mixed_cg"] = round(best_cg / out["gcr_network"]["ms"], 2)
    out["iteration_ratio_vs_gcr_plain"] = round(out["gcr_plain"]["iterations"] /
                                                max(1, out["gcr_network"]["iterations"]), 2)
    ctx.close()
    return out


def callers(torch, device):
    """The callers of the solvers (through the public API, host arrays in the
    reference's layouts, so host<->device copies are inside the times):
    Qprop_EvenOdd on the 12 point sources at 32^3x64 as one mixed-precision
    block against the reference's 12 sequential FP64 inversions; the
    RationalSolver_CG with 12 poles and the Wilson e/o MD force at 24^3x48."""
    import iroiro_b200 as ib
    out = {}
    Lb = [32, 32, 32, 64]
    Vb = int(np.prod(Lb))
    ctx = ib.Context(Lb, device)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    u = ib.synth_gauge(Lb, EPS, SEED + 7, gauge_transform=False)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
    rng = np.random.default_rng(SEED)
    sp = [int(v) for v in rng.integers(0, 32, 3)] + [int(rng.integers(0, 64))]
    src = ib.Source_local(sp, Lb)
    res = {}
    # the caller keeps the 12 propagators' storage across calls (the
    # reference's prop_t xq); the warm-up call of each arm touches it
    buf = np.empty((12, 24 * Vb))
    for name, inner, delta in (("block12_half", "half", 0.02), ("block12_double", "double", 0.1)):
        qp = ib.Qprop_EvenOdd(D, ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D), inner=inner, delta=delta))
        qp.calc(src, out=buf)
        torch.cuda.synchronize()
        t = time.perf_counter()
        qp.calc(src, out=buf)
        torch.cuda.synchronize()
        res[name] = {"ms": round((time.perf_counter() - t) * 1e3, 1),
                     "true_residual_max": max(o.diff for o in qp.last_outputs),
                     "iterations": max(o.Iterations for o in qp.last_outputs)}
        if name == "block12_half":
            x_half = buf.copy()
    # the reference's way: one FP64 e/o inversion per source, calc(xq, src, s, c)
    # (qprop_EvenOdd.cpp:24-28); the comparison with the block runs after the
    # timed region
    qp = ib.Qprop_EvenOdd(D, ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D)))
    for k in range(12):
        qp.calc(src, k // 3, k % 3, out=buf[k])
    torch.cuda.synchronize()
    t = time.perf_counter()
    for k in range(12):
        qp.calc(src, k // 3, k % 3, out=buf[k])
    torch.cuda.synchronize()
    res["sequential12_fp64_ms"] = round((time.perf_counter() - t) * 1e3, 1)
    res["block12_half_error_vs_fp64"] = max(
        float(np.linalg.norm(x_half[k] - buf[k]) / np.linalg.norm(buf[k])) for k in range(12))
    res["speedup_block12_half_vs_sequential_fp64"] = round(res["sequential12_fp64_ms"] /
                                                           res["block12_half"]["ms"], 2)
    res["note"] = ("point sources built on the device (iro_qprop_point); 12 x 24 V doubles "
                   "of propagators copied to the caller's host storage in both arms")
    out["qprop_evenodd_32x32x32x64"] = res
    ctx.close()
    # RationalSolver_CG and md_force at 24^3x48
    ctx = ib.Context(L, device)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    u = ib.synth_gauge(L, EPS, SEED, gauge_transform=True)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
    Vh = int(np.prod(L)) // 2
    b = ib.synth_gaussian(Vh, SEED + 11)
    poles = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
    ra = ib.RationalApprox(0.5, [0.1 / (k + 1) for k in range(12)], poles)
    rs = ib.RationalSolver_CG(ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 20000), ra)
    sol = np.empty_like(b)
    rs.solve(sol, b)
    torch.cuda.synchronize()
    t = time.perf_counter()
    o = rs.solve(sol, b)
    torch.cuda.synchronize()
    out["rational_12poles_24x24x24x48"] = {"ms": round((time.perf_counter() - t) * 1e3, 1),
                                           "nconv": o.Nconv, "true_residual_max": o.diff}
    e, z = ib.synth_gaussian(Vh, SEED + 12), ib.synth_gaussian(Vh, SEED + 13)
    D.md_force(e, z)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(5):
        D.md_force(e, z)
    torch.cuda.synchronize()
    out["md_force_evenodd_24x24x24x48_ms"] = round((time.perf_counter() - t) * 1e3 / 5, 2)
    # Dirac_Clover::md_force: the Wilson force plus the clover term's leaf derivatives
    Dc = ib.Dirac_Clover(ib.Dirac_Wilson(MASS, u, ctx=ctx), CSW, u, ctx=ctx)
    ef, zf = ib.synth_gaussian(2 * Vh, SEED + 14), ib.synth_gaussian(2 * Vh, SEED + 15)
    Dc.md_force(ef, zf)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(5):
        Dc.md_force(ef, zf)
    torch.cuda.synchronize()
    out["md_force_clover_24x24x24x48_ms"] = round((time.perf_counter() - t) * 1e3 / 5, 2)
    out["md_force_note"] = "host arrays: 2 spinors in, the 72*V-double Format_G force out (382 MB)"
    ctx.close()
    return out


def mixed48(torch, device):
    """Mixed-precision configuration: 48^3x96 even-odd Wilson-clover
    (csw=1.0, kappa=0.124, eps=0.25 field), 12 Gaussian right-hand sides
    solved together with FP16 storage (per-site norms, reconstruct-12 links),
    FP32 arithmetic and FP64 reliable updates, against the FP64 block CG on
    the same sources; every result's error against the FP64 solution."""
    import iroiro_b200 as ib
    Lb = [48, 48, 48, 96]
    Vb = int(np.prod(Lb))
    kappa = 0.124
    mass = 0.5 / kappa - 4.0
    ctx = ib.Context(Lb, device)
    s = torch.cuda.current_stream()
    ctx.set_stream(s.cuda_stream)
    u = ib.synth_gauge(Lb, 0.25, SEED + 400)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Clover_EvenOdd(mass, CSW, u, ctx=ctx)
    src = np.concatenate([ib.synth_gaussian(Vb // 2, SEED + 401 + r) for r in range(12)])
    B = ib.DeviceField(ctx, 0, "double", 12).upload(src)
    del src
    out = {"op": "e/o Wilson-clover Schur 48^3x96, kappa=0.124, csw=1.0, eps=0.25, 12 Gaussian sources"}
    X64 = ib.DeviceField(ctx, 0, "double", 12)
    # outside the timed solves: the clover set-up and the autotuning of the
    # 12-RHS operator shapes of both precisions (D and D^dag)
    lib = ctx._lib
    for dag in (0, 1):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, D.op, mass, CSW, dag, B.h, X64.h), "apply")
    # (FP16 scratch fields: the tuning only times the launch shapes)
    H = [ib.DeviceField(ctx, 0, "half", 12) for _ in range(2)]
    for dag in (0, 1):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, D.op, mass, CSW, dag, H[0].h, H[1].h), "apply")
    for h in H:
        h.close()
    torch.cuda.synchronize()
    res = {}
    # (FP32 storage is left out here: its 12-RHS workspaces would not fit
    # beside the FP64 and FP16 ones and the clover terms in 180 GB)
    for inner, X in (("double", X64), ("half", None)):
        X = X or ib.DeviceField(ctx, 0, "double", 12)
        slv = ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D), inner=inner, delta=0.1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        outs, rc = slv.solve_field(B, X)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t) * 1e3
        res[inner] = {"ms": round(ms, 1), "iterations": max(o.Iterations for o in outs),
                      "true_residual_max": max(o.diff for o in outs),
                      "reliable_updates": max(o.reliable_updates for o in outs),
                      "converged": rc == ib.OK}
        if inner != "double":
            x = X.download().reshape(12, -1)
            x64 = X64.download().reshape(12, -1)
            res[inner]["error_vs_fp64_per_rhs"] = [
                float(np.linalg.norm(x[r] - x64[r]) / np.linalg.norm(x64[r])) for r in range(12)]
            res[inner]["speedup_vs_fp64_block_cg"] = round(res["double"]["ms"] / ms, 2)
            X.close()
    out.update(res)
    out["note"] = ("single timed solve each, after the clover set-up and the operator autotuning; "
                   "the solver workspaces are allocated inside the first call of each precision")
    ctx.close()
    return out


def cpu_baseline_leg():
    """The reference's own e/o mult on the host cores, a bounded sample."""
    import oracle
    import iroiro_b200 as ib
    if not oracle.ref_available():
        return None
    V = int(np.prod(L))
    u = ib.synth_gauge(L, EPS, SEED, gauge_transform=True)
    f = ib.synth_gaussian(V // 2, SEED + 1)
    ref = oracle.ref()
    ref.init(L)
    threads = cpu_cores()
    ref.eo_mult_throughput(u, MASS, f, threads, 1)
    reps = 3
    _, s = ref.eo_mult_throughput(u, MASS, f, threads, reps)
    val = (2 * BYTES_HOP + BYTES_XPAY) * (V // 2) * threads * reps / s / 1e9
    return {"value": round(val, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"{threads} threads x {reps} Dirac_Wilson_EvenOdd::mult at 24^3x48 "
                      f"({s:.1f} s)"}


# ---- our arm --------------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch
    import iroiro_b200 as ib

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V = int(np.prod(L))
    Vh = V // 2
    u = ib.synth_gauge(L, EPS, SEED + rank, gauge_transform=True)
    h = ib.synth_gaussian(Vh, SEED + 100 + rank)
    ctx = ib.Context(L, local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    ctx.upload_gauge(u, force=True)
    lib = ctx._lib
    import ctypes
    fin = ctypes.c_void_p()
    fout = ctypes.c_void_p()
    ctx.check(lib.iro_field_create(ctx.h, 0, ib.PREC_DOUBLE, 1, ctypes.byref(fin)), "field")
    ctx.check(lib.iro_field_create(ctx.h, 0, ib.PREC_DOUBLE, 1, ctypes.byref(fout)), "field")
    ctx.check(lib.iro_field_upload(ctx.h, fin, h.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
              "upload")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        ctx.check(lib.iro_dirac_apply_field(ctx.h, ib.OP_WILSON_SCHUR_EE, MASS, 0.0, 0, fin, fout),
                  "apply")

    for _ in range(max(args.warmup, 3)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clocks = Clocks(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    clocks.mark()
    torch.cuda.profiler.start()  # ncu --profile-from-start off captures exactly this region
    for s, e in ev:
        flush.zero_()
        s.record(stream)
        step()
        e.record(stream)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    barrier(world)
    ck = clocks.stop()
    t_ms = sum(s.elapsed_time(e) for s, e in ev)
    step_bytes = (2 * BYTES_HOP + BYTES_XPAY) * Vh
    t_max = reduce_max(t_ms, world)
    value = replica_value(step_bytes, args.steps, t_ms, world)
    achieved = step_bytes / ((t_ms / args.steps) * 1e-3) / 1e9
    peak, peak_kind = measured_peak()

    # e2e: through the C ABI with pinned host buffers (H2D + D2H inside)
    hin = torch.from_numpy(h).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    pin_in = ctypes.cast(hin.data_ptr(), ctypes.POINTER(ctypes.c_double))
    pin_out = ctypes.cast(hout.data_ptr(), ctypes.POINTER(ctypes.c_double))

    def e2e_step():
        ctx.check(lib.iro_dirac_apply(ctx.h, ib.OP_WILSON_SCHUR_EE, MASS, 0.0, 0, ib.PREC_DOUBLE,
                                      pin_in, pin_out, 1), "iro_dirac_apply")

    for _ in range(3):
        e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    es, ee = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    es.record(stream)
    for _ in range(args.steps):
        e2e_step()
    ee.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(es.elapsed_time(ee), world)
    e2e_val = world * step_bytes * args.steps / (e2e_ms * 1e-3) / 1e9

    # FP32 / FP16 Schur and clover variants, same protocol (reported, not the headline)
    variants = {}
    for name, op, csw, prec, bps in (
            ("wilson_fp32", ib.OP_WILSON_SCHUR_EE, 0.0, ib.PREC_SINGLE, 2 * 1248 + 96),
            ("wilson_fp16", ib.OP_WILSON_SCHUR_EE, 0.0, ib.PREC_HALF, 2 * 660 + 52),
            ("clover_fp64", ib.OP_CLOVER_SCHUR_EE, CSW, ib.PREC_DOUBLE, 2 * (2496 + 576) + 192),
            ("clover_fp32", ib.OP_CLOVER_SCHUR_EE, CSW, ib.PREC_SINGLE, 2 * (1248 + 288) + 96)):
        a, b = ctypes.c_void_p(), ctypes.c_void_p()
        ctx.check(lib.iro_field_create(ctx.h, 0, prec, 1, ctypes.byref(a)), "field")
        ctx.check(lib.iro_field_create(ctx.h, 0, prec, 1, ctypes.byref(b)), "field")
        ctx.check(lib.iro_field_upload(ctx.h, a, h.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "up")
        for _ in range(3):
            ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, csw, 0, a, b), "apply")
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(args.steps):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, csw, 0, a, b), "apply")
            e.record(stream)
            e.synchronize()
            tot += s.elapsed_time(e)
        ms = tot / args.steps
        variants[name] = {"ms_per_op": round(ms, 4), "GBps": round(bps * Vh / (ms * 1e-3) / 1e9, 1),
                          "frac_of_measured_hbm": round(bps * Vh / (ms * 1e-3) / 1e9 / peak, 3)}
        lib.iro_field_destroy(a)
        lib.iro_field_destroy(b)

    # the FP64 Schur operator on the 32^3x64 lattice (same protocol)
    variants["wilson_fp64_32x32x32x64"] = schur_fp64_32(torch, local, args.steps, peak)

    # time to a 1e-10 FP64 true residual, e/o Wilson-clover, FP64 CG vs mixed
    # precision; fields resident on the device (iro_cg_solve_field)
    solve = {}
    if not args.no_solve:
        D = ib.Dirac_Clover_EvenOdd(MASS, CSW, u, ctx=ctx)
        solve = timed_solves(ctx, D, h, 1, torch)
        solve["op"] = "e/o Wilson-clover Schur 24^3x48, kappa=0.12, csw=1.0, one Gaussian source"
    batched = {}
    if not args.no_solve and not args.no_batched:
        batched = batched_solves(torch, local)
    learned_res = {}
    if not args.no_solve and not args.no_learned:
        learned_res = learned_solves(torch, local)
    mixed = {}
    if args.mixed48:
        mixed = mixed48(torch, local)
    caller_res = {}
    if not args.no_solve and not args.no_callers:
        caller_res = callers(torch, local)

    lib.iro_field_destroy(fin)
    lib.iro_field_destroy(fout)
    if rank != 0:
        return 0
    cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline_leg()
    traffic = traffic_per_launch(Vh)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": L, "kappa": KAPPA, "eps": EPS,
                   "gauge_transform": True, "l2": "flushed (256 MiB write) before every step",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 3), "traffic": traffic,
                     "peak_kind": peak_kind,
                     "dram_GBps": None if traffic is None else
                     round(traffic / ((t_ms / args.steps) * 1e-3) / 1e9, 1),
                     "dram_frac": None if traffic is None else
                     round(traffic / ((t_ms / args.steps) * 1e-3) / 1e9 / peak, 3),
                     "bytes_model": "per even site: hop 2496 + hop 2496 + f_e 192 (FP64, recon-12)",
                     "gflops": round(FLOPS_SCHUR * Vh / ((t_ms / args.steps) * 1e-3) / 1e9, 1)},
        "e2e": {"value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": 24 * 8 * Vh,
                "d2h_bytes_per_step": 24 * 8 * Vh, "ms_per_step": round(e2e_ms / args.steps, 3)},
        "gpu_launches": 2 * args.steps,
        "autotune": ctx.autotune_report(),
        "clocks": ck,
        "variants": variants,
        "solve": solve,
        "batched": batched,
        "learned": learned_res,
        "mixed48": mixed,
        "callers": caller_res,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    return 0


def kernel_only(args):
    """Profiling driver: `steps` applications of one operator on device
    fields inside a cudaProfilerStart/Stop range (after autotuning), for
    `ncu --profile-from-start off`.  --kernel OP,PREC,NRHS with OP one of
    wilson_eo, clover_eo, wilson_full; --lattice Lx,Ly,Lz,Lt."""
    import ctypes
    import torch
    import iroiro_b200 as ib
    Lk = [int(v) for v in args.lattice.split(",")]
    if args.kernel.startswith(("ptc,", "batched,")) or args.kernel in ("md_force_eo", "md_force_clover"):
        return kernel_only_other(args, Lk)
    opn, prec, nrhs = args.kernel.split(",")
    nrhs = int(nrhs)
    op = {"wilson_eo": ib.OP_WILSON_SCHUR_EE, "clover_eo": ib.OP_CLOVER_SCHUR_EE,
          "wilson_full": ib.OP_WILSON_FULL}[opn]
    sub = 2 if op == ib.OP_WILSON_FULL else 0
    V = int(np.prod(Lk))
    ctx = ib.Context(Lk, 0)
    ctx.upload_gauge(ib.synth_gauge(Lk, EPS, SEED, gauge_transform=True), force=True)
    a = ib.DeviceField(ctx, sub, prec, nrhs).upload(
        ib.synth_gaussian((V if sub == 2 else V // 2) * nrhs, SEED + 3))
    b = ib.DeviceField(ctx, sub, prec, nrhs)
    lib = ctx._lib
    for _ in range(3):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, CSW, 0, a.h, b.h), "apply")
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(args.steps):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, CSW, 0, a.h, b.h), "apply")
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"kernel": args.kernel, "lattice": Lk, "autotune": ctx.autotune_report()}))
    return 0


def kernel_only_other(args, Lk):
    """Profiling driver for the other kernels: --kernel ptc,4-16-16-16-4 applies
    that network `steps` times to an FP32 field; --kernel md_force_eo computes
    one even/odd Wilson MD force, --kernel md_force_clover one full-lattice
    Wilson-clover MD force; --kernel batched,INNER,DELTA runs the batched
    configuration's solve (the 12 point sources on the seeded field of
    batched_solves, on the lattice given) once untimed and once profiled; all
    inside cudaProfilerStart/Stop."""
    import torch
    import iroiro_b200 as ib
    from iroiro_b200 import learned
    V = int(np.prod(Lk))
    ctx = ib.Context(Lk, 0)
    if args.kernel.startswith("batched,"):
        _, inner, delta = args.kernel.split(",")
        st = torch.cuda.Stream()
        torch.cuda.set_stream(st)
        ctx.set_stream(st.cuda_stream)  # a capturable stream: the solver's CUDA graphs
        u = ib.synth_gauge(Lk, EPS, SEED + 7, gauge_transform=False)
        ctx.upload_gauge(u, force=True)
        D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
        site = int(np.random.default_rng(SEED).integers(V // 2))
        B = ib.DeviceField(ctx, 0, "double", 12).upload(ib.synth_point_sources(V // 2, site).ravel())
        X = ib.DeviceField(ctx, 0, "double", 12)
        slv = ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D), inner=inner, delta=float(delta))
        slv.solve_field(B, X)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        t0 = time.perf_counter()
        outs, rc = slv.solve_field(B, X)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": args.kernel, "lattice": Lk, "ms": round(ms, 2),
                          "iterations": max(o.Iterations for o in outs),
                          "reliable_updates": max(o.reliable_updates for o in outs), "rc": rc}))
        return 0
    u = ib.synth_gauge(Lk, EPS, SEED, gauge_transform=True)
    ctx.upload_gauge(u, force=True)
    if args.kernel.startswith("ptc,"):
        widths = tuple(int(v) for v in args.kernel.split(",")[1].split("-"))
        net = learned.PTCNet(ctx, widths, learned.init_weights(widths, 1, 0.3))
        a = ib.DeviceField(ctx, 2, "single").upload(ib.synth_gaussian(V, SEED + 1))
        b = ib.DeviceField(ctx, 2, "single")
        run = lambda: ctx.check(net.L.iro_ptc_apply_field(ctx.h, net.h, a.h, b.h), "apply")
        reps = args.steps
    elif args.kernel == "md_force_clover":
        D = ib.Dirac_Clover(ib.Dirac_Wilson(MASS, u, ctx=ctx), CSW, u, ctx=ctx)
        e, z = ib.synth_gaussian(V, SEED + 1), ib.synth_gaussian(V, SEED + 2)
        run = lambda: D.md_force(e, z)
        reps = 1
    else:
        D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
        e, z = ib.synth_gaussian(V // 2, SEED + 1), ib.synth_gaussian(V // 2, SEED + 2)
        run = lambda: D.md_force(e, z)
        reps = 1
    run()
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(reps):
        run()
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"kernel": args.kernel, "lattice": Lk}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-callers", action="store_true")
    ap.add_argument("--mixed48", action="store_true",
                    help="also run the 48^3x96 mixed-precision 12-RHS configuration (~1 min)")
    ap.add_argument("--kernel", default=None, help="profiling driver: OP,PREC,NRHS")
    ap.add_argument("--lattice", default="24,24,24,48")
    args = ap.parse_args()
    if args.kernel:
        return kernel_only(args)
    world, rank, local = (1, 0, 0) if args.impl == "reference" and _env_int("WORLD_SIZE", 1) == 1 \
        else ((_env_int("WORLD_SIZE", 1), _env_int("RANK", 0), _env_int("LOCAL_RANK", 0))
              if args.impl == "reference" else dist_setup())
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1 and args.impl != "reference":
            import torch.distributed as dist
            if dist.is_initialized():
                dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
