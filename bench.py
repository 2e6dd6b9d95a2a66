"""Benchmark of the even-odd Wilson Dslash hot path on B200.

Workload (one "step"): one application of the even-odd Schur operator
Dirac_Wilson_EvenOdd<Dirac_Wilson>::mult, M f_e = f_e - kappa^2 H_eo H_oe f_e
(lib/Dirac_ops/dirac_wilson_EvenOdd.hpp:79-83), on a 32^3x64 lattice, kappa =
0.12, seeded synthetic SU(3) links exp(i*0.2*H) followed by a random gauge
transformation, FP64 storage and arithmetic (the reference's own arithmetic),
reconstruct-12 links.  One step = two launches of the hopping kernel.

value     GB/s of the step on compulsory bytes, fields resident in HBM, L2
          flushed (256 MiB written) before every step, CUDA events on the
          launching stream around each step; summed over ranks (replicas) /
          max time.  Compulsory bytes per even site: 2496 = hop 1152 (4 own
          links 384 + 4 neighbours' links 384 + input spinor 192 + output
          192, each byte once) + hop 1152 + the f_e read (192) of the fused
          f - x epilogue.  The model that counts every neighbour spinor and
          link once per reading site (5184 B per even site) is reported as
          roofline.algorithmic_GBps.
e2e       the same metric through the C ABI with host buffers:
          iro_dirac_apply() on pinned Format_F arrays, H2D + D2H inside the
          timed region (the library moves the field in chunks of t-slices,
          both copy directions overlapped with each other and the stencils;
          equals_plain_path: the result equals the unchunked path's bitwise).
roofline  achieved = compulsory bytes per step / mean step time; traffic =
          DRAM bytes (read + write) of one step from the committed ncu
          capture of this lattice, scaled by the sites processed.
reference_beside  the reference's full-lattice Wilson CG, e/o multishift CG (12
          shifts) and full-lattice clover mult on one host core at 8^3x16,
          beside ours through the host-array API (same inputs; iteration
          counts reported for both).
summary   (last key) the headline numbers of every configuration.

--impl reference runs the reference's own C++ (compiled from its sources
into oracle/_ref) on the host cores for the same metric, config and step, on
inputs made by the oracle's copy of the generator (the product library is
not loaded).
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

L = [32, 32, 32, 64]          # headline lattice
L_C2 = [24, 24, 24, 48]       # the Wilson-clover configuration's lattice
KAPPA = 0.12
MASS = 0.5 / KAPPA - 4.0
CSW = 1.0
EPS = 0.2
SEED = 20240601
BYTES_HOP = 1152          # FP64 recon-12, per output site, each byte once
BYTES_XPAY = 192          # f_e read of the fused epilogue
BYTES_STEP = 2 * BYTES_HOP + BYTES_XPAY           # 2496 per even site
BYTES_STEP_ALG = 2 * 2496 + 192                   # every neighbour counted per reader
FLOPS_SCHUR = 2 * 1320 + 48
METRIC = "EO-Wilson Dslash GB/s (% of HBM peak)"
WORKLOAD = "Dirac_Wilson_EvenOdd::mult 32^3x64, kappa=0.12, FP64, recon-12"
PROFILE_32 = "profiles/hop_fp64_32x32x32x64_dram.txt"


def config_for(world: int) -> dict:
    """The config object of the JSON line, identical in both arms."""
    return {"workload": WORKLOAD, "lattice": L, "kappa": KAPPA, "eps": EPS,
            "gauge_transform": True, "seed": SEED,
            "bytes_model": "compulsory, 2496 B per even site",
            "l2": "GPU arm: 256 MiB written before every step (fields 1.0 GB > 126 MB L2)",
            "parallelism": f"replicas x{world}"}


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


def traffic_per_step(vh: int):
    """DRAM bytes (read + write) of one Schur application (both hop launches)
    from the committed ncu capture of the 32^3x64 lattice, scaled to `vh`
    even sites by the sites processed; (bytes, source) or (None, None)."""
    p = ROOT / PROFILE_32
    if not p.exists():
        return None, None
    m = re.search(r"^dram_bytes_per_site_schur_32x32x32x64:\s*([0-9.]+)", p.read_text(), re.M)
    if not m:
        return None, None
    return float(m.group(1)) * vh, f"{PROFILE_32} (ncu, DRAM read+write per even site x sites)"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- reference arm ----------------------------------------------------------------------

REF_MAX_STEPS = 40   # a step takes about 3 s on the host at 32^3x64


def ref_inputs():
    """The headline's gauge field and source, made by the oracle's copy of the
    generator (bit-identical to the product's), without the product library."""
    import oracle
    P = oracle.port()
    V = int(np.prod(L))
    return P.synth_gauge(L, EPS, SEED, True), P.synth_gaussian(V // 2, SEED + 100)


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libiroiro_ref.so was not built (needs the reference tree)"}))
        return 0
    V = int(np.prod(L))
    u, f = ref_inputs()
    ref = oracle.ref()
    ref.init(L)
    threads = cpu_cores()
    warm = max(args.warmup, 3)
    nsteps = max(1, min(args.steps, REF_MAX_STEPS))
    for _ in range(warm):
        ref.eo_mult_throughput(u, MASS, f, threads, 1)
    t = 0.0
    for _ in range(nsteps):
        _, s = ref.eo_mult_throughput(u, MASS, f, threads, 1)
        t += s
    step_bytes = BYTES_STEP * (V // 2) * threads
    val = step_bytes * nsteps / t / 1e9
    sample = (f"{threads} host threads, each one Dirac_Wilson_EvenOdd::mult per step on its own "
              f"copy of the source ({nsteps} steps, at most {REF_MAX_STEPS})")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": nsteps, "warmup": warm,
        "ms_per_step": round(1e3 * t / nsteps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_for(args.gpus),
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def schur_timing(torch, ctx, st, prec, op, csw, vh, steps, flush, nrhs=1, source=None):
    """Mean event-timed ms of one Schur application (op, precision) on device
    fields, L2 flushed before every application."""
    import iroiro_b200 as ib
    lib = ctx._lib
    a = ib.DeviceField(ctx, 0, prec, nrhs).upload(
        source if source is not None else ib.synth_gaussian(vh * nrhs, SEED + 6))
    b = ib.DeviceField(ctx, 0, prec, nrhs)
    for _ in range(3):
        ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, csw, 0, a.h, b.h), "apply")
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(st)
        ctx.check(lib.iro_dirac_apply_field(ctx.h, op, MASS, csw, 0, a.h, b.h), "apply")
        e.record(st)
        e.synchronize()
        tot += s.elapsed_time(e)
    a.close()
    b.close()
    return tot / steps


def variant_line(ms, bytes_per_site, vh, peak):
    gbs = bytes_per_site * vh / (ms * 1e-3) / 1e9
    return {"ms": round(ms, 4), "GBps": round(gbs, 1), "frac": round(gbs / peak, 3)}


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
    # FP64 (the reference's solver) against the mixed-precision one, on
    # device-resident fields (source in, the 12 solutions out)
    msr = {}
    G = ib.DeviceField(ctx, 0, "double").upload(g)
    XS = ib.DeviceField(ctx, 0, "double", 12)
    x64 = None
    for inner in ("double", "single", "half"):
        ms = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 20000, inner=inner)
        ms.solve_field(G, XS, shifts)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = ms.solve_field(G, XS, shifts)
        torch.cuda.synchronize()
        msr[inner] = {"ms": round((time.perf_counter() - t0) * 1e3, 2), "iterations": o.Nconv,
                      "max_true_residual": o.diff, "reliable_updates": o.reliable_updates}
        xs = XS.download().reshape(12, -1)
        if inner == "double":
            x64 = xs
        else:
            msr[inner]["max_error_vs_fp64"] = max(
                float(np.linalg.norm(xs[k] - x64[k]) / np.linalg.norm(x64[k])) for k in range(12))
            msr[inner]["speedup_vs_fp64"] = round(msr["double"]["ms"] / msr[inner]["ms"], 2)
    G.close()
    XS.close()
    out["multishift12"] = msr
    ctx.close()
    return out


def learned_solves(torch, device, nfields=100, epochs=15, widths=(4, 4, 4, 4), nkrylov=16, delta=0.03,
                   krylov="half"):
    """Learned preconditioner: a PTC network trained by the library's own
    forward/backward kernels on pairs (b = D^dag D v, v) from `nfields` seeded
    16^3x32 gauge fields (eps=0.2, kappa=0.12), then applied inside flexible
    GCR at 32^3x64 and 48^3x96 (unseen fields, one Gaussian source each)
    against GCR without it and against CG on the same full-lattice D^dag D:
    FP64 and mixed precision.  GCR restarts after `nkrylov` directions or once
    its iterated residual has fallen by `delta`; its directions z_j, w_j are
    stored in `krylov` precision (FP16: D^dag D applied in mixed FP16).  Every solve stops on the FP64
    true residual 1e-10; each is timed after an untimed call, as the median
    (and the minimum) of 9 runs at 32^3x64 and one run at 48^3x96."""
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
    out = {"op": "full-lattice Wilson D^dag D, kappa=0.12, one Gaussian source, unseen field",
           "network": {"widths": list(widths), "train_fields": nfields, "train_lattice": "16^3x32",
                       "epochs": epochs, "train_s": round(train_s, 1),
                       "loss_first": round(hist[0], 4), "loss_last": round(hist[-1], 4)},
           "gcr": {"nkrylov": nkrylov, "delta": delta, "krylov": krylov}}

    samples = {}

    def timed(fn, reps=1):
        # one untimed call (tuning, workspaces), then the median of `reps`
        # timed calls: the solves sync with the host every iteration, and
        # single runs of GCR here have varied by up to 3.7x (box-side jitter)
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t) * 1e3)
        samples["last"] = [round(v, 1) for v in ts]
        samples["min"] = round(min(ts), 1)
        return statistics.median(ts), r

    for Lb, tag, seed, reps in (([32, 32, 32, 64], "", SEED + 301, 9),
                                ([48, 48, 48, 96], "_48x48x48x96", SEED + 311, 1)):
        Vb = int(np.prod(Lb))
        ctx = ib.Context(Lb, device)
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        u = ib.synth_gauge(Lb, EPS, seed)
        ctx.upload_gauge(u, force=True)
        D = ib.Dirac_Wilson(MASS, u, ctx=ctx)
        b = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(Vb, seed + 1))
        net = learned.PTCNet(ctx, widths, W)
        res = {}
        for name, n in (("gcr_network", net), ("gcr_plain", None)):
            x = ib.DeviceField(ctx, 2, "double")
            slv = learned.Solver_GCR(D, n, nkrylov=nkrylov, delta=delta, krylov=krylov)
            ms, (o, rc) = timed(lambda: slv.solve_field(b, x), reps)
            res[name] = {"ms": round(ms, 1), "ms_min": samples["min"], "ms_samples": samples["last"],
                         "iterations": o.iterations,
                         "true_residual": o.diff, "cg_fallback": bool(o.fallback), "converged": rc == ib.OK}
            x.close()
        for inner in ("double", "single", "half"):
            x = ib.DeviceField(ctx, 2, "double")
            slv = ib.Solver_CG(1e-20, 20000, ib.Fopr_DdagD(D), inner=inner)
            ms, (outs, rc) = timed(lambda: slv.solve_field(b, x), reps)
            res["cg_" + inner] = {"ms": round(ms, 1), "ms_min": samples["min"], "ms_samples": samples["last"],
                                  "iterations": outs[0].Iterations, "true_residual": outs[0].diff,
                                  "converged": rc == ib.OK}
            x.close()
        a = ib.DeviceField(ctx, 2, "single").upload(ib.synth_gaussian(Vb, seed + 2))
        c2 = ib.DeviceField(ctx, 2, "single")
        apply_ms, _ = timed(lambda: ctx.check(net.L.iro_ptc_apply_field(ctx.h, net.h, a.h, c2.h), "apply"))
        res["network_apply_ms"] = round(apply_ms, 3)
        best_cg = min(res["cg_single"]["ms"], res["cg_half"]["ms"])
        res["gcr_network_vs_best_mixed_cg"] = round(best_cg / res["gcr_network"]["ms"], 2)
        res["iteration_ratio_vs_gcr_plain"] = round(res["gcr_plain"]["iterations"] /
                                                    max(1, res["gcr_network"]["iterations"]), 2)
        if tag:
            out["at" + tag] = res
        else:
            out.update(res)
        for f in (a, c2, b):
            f.close()
        net.close()
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
    ctx = ib.Context(L_C2, device)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    u = ib.synth_gauge(L_C2, EPS, SEED, gauge_transform=True)
    ctx.upload_gauge(u, force=True)
    D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
    Vh = int(np.prod(L_C2)) // 2
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
    res = {}
    # (FP32 storage is left out here: its 12-RHS workspaces would not fit
    # beside the FP64 and FP16 ones and the clover terms in 180 GB)
    # Outside the timed solves: the clover set-up, the autotuning of every
    # operator shape on the real sources, the solver workspaces and graphs --
    # one 16-iteration solve per precision.
    for inner in ("double", "half"):
        Xw = ib.DeviceField(ctx, 0, "double", 12)
        ib.Solver_CG(1e-20, 16, ib.Fopr_DdagD(D), inner=inner, delta=0.1).solve_field(B, Xw)
        Xw.close()
    torch.cuda.synchronize()
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
            res[inner]["error_vs_fp64_max"] = max(
                float(np.linalg.norm(x[r] - x64[r]) / np.linalg.norm(x64[r])) for r in range(12))
            res[inner]["speedup_vs_fp64_block_cg"] = round(res["double"]["ms"] / ms, 2)
            X.close()
    out.update(res)
    out["note"] = ("one timed solve each, after an untimed 16-iteration solve per precision "
                   "(clover set-up, autotuning, workspaces, graphs)")
    ctx.close()
    return out


def cpu_baseline_leg():
    """The reference's own e/o mult on the host cores, a bounded sample of
    the headline workload (inputs from the oracle's generator)."""
    import oracle
    if not oracle.ref_available():
        return None
    V = int(np.prod(L))
    u, f = ref_inputs()
    ref = oracle.ref()
    ref.init(L)
    threads = cpu_cores()
    ref.eo_mult_throughput(u, MASS, f, threads, 1)
    reps = 3
    _, s = ref.eo_mult_throughput(u, MASS, f, threads, reps)
    val = BYTES_STEP * (V // 2) * threads * reps / s / 1e9
    return {"value": round(val, 3), "unit": "GB/s", "cores": threads, "kind": "reference",
            "sample": f"{threads} threads x {reps} Dirac_Wilson_EvenOdd::mult at 32^3x64 "
                      f"({s:.1f} s)"}


# The reference's solvers and clover operator on the host cores, beside ours on the GPU, at a
# size where the reference finishes in seconds (8^3x16): full-lattice Wilson CG (D^dag D to
# |r|^2/|b|^2 < 1e-20), e/o multishift CG (12 shifts 1e-4..10) and the full-lattice clover mult
# (the reference's took ~24 s per call at 24^3x48 on one core of the build machine).  The reference keeps one
# lattice per process, so it runs in a child process that loads only oracle/ libraries; its
# results go to a file (the reference's clover prints on every call).
REF_SOLVER_SPECS = {
    "8x8x8x16": {"L": [8, 8, 8, 16], "seed": SEED + 500},
}
SHIFTS12 = [1e-4 * (1e5) ** (k / 11) for k in range(12)]


def ref_solver_child(name, path):
    import oracle
    spec = REF_SOLVER_SPECS[name]
    Lr = spec["L"]
    V = int(np.prod(Lr))
    P = oracle.port()
    R = oracle.ref()
    R.init(Lr)
    u = P.synth_gauge(Lr, EPS, spec["seed"], True)
    out = {}
    b = P.synth_gaussian(V, spec["seed"] + 1)
    t = time.perf_counter()
    _, it, diff, _ = R.cg(u, oracle.WILSON_FULL, MASS, 0.0, b, 1e-20, 5000)
    out["cg_wilson_full"] = {"ms": (time.perf_counter() - t) * 1e3, "iterations": it, "diff": diff}
    bh = P.synth_gaussian(V // 2, spec["seed"] + 2)
    t = time.perf_counter()
    _, nc, diff = R.multishift(u, oracle.WILSON_EO, MASS, 0.0, bh, SHIFTS12, 1e-20, 5000)
    out["multishift12_wilson_eo"] = {"ms": (time.perf_counter() - t) * 1e3, "nconv": nc, "diff": diff}
    f = P.synth_gaussian(V, spec["seed"] + 3)
    R.clover_full(u, MASS, 1.0, 0, f)
    t = time.perf_counter()
    R.clover_full(u, MASS, 1.0, 0, f)
    out["clover_full_mult"] = {"ms": (time.perf_counter() - t) * 1e3}
    with open(path, "w") as fh:
        json.dump(out, fh)


def reference_solvers_beside(torch, device):
    """Each item: the reference (host cores, one thread: its Dslash has no
    threading) and ours (GPU, through the host-array API, copies included)."""
    import tempfile
    import oracle
    import iroiro_b200 as ib
    if not oracle.ref_available():
        return None
    res = {}
    for name, spec in REF_SOLVER_SPECS.items():
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "ref.json")
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--ref-solver-child", name, path],
                               stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=600)
            if r.returncode != 0 or not os.path.exists(path):
                res[name] = {"error": r.stderr.decode(errors="replace")[-300:]}
                continue
            with open(path) as fh:
                ref = json.load(fh)
        Lr = spec["L"]
        V = int(np.prod(Lr))
        ctx = ib.Context(Lr, device)
        u = ib.synth_gauge(Lr, EPS, spec["seed"], gauge_transform=True)
        ctx.upload_gauge(u, force=True)

        def timed(fn):
            fn()
            torch.cuda.synchronize()
            t = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            return (time.perf_counter() - t) * 1e3, r

        D = ib.Dirac_Wilson(MASS, u, ctx=ctx)
        b = ib.synth_gaussian(V, spec["seed"] + 1)
        x = np.empty_like(b)
        ms, o = timed(lambda: ib.Solver_CG(1e-20, 5000, ib.Fopr_DdagD(D)).solve(x, b))
        rc = ref["cg_wilson_full"]
        res["cg_wilson_full_" + name] = {
            "reference_ms": round(rc["ms"], 2), "reference_iterations": rc["iterations"],
            "ours_ms": round(ms, 2), "ours_iterations": o.Iterations, "speedup": round(rc["ms"] / ms, 1)}
        De = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
        bh = ib.synth_gaussian(V // 2, spec["seed"] + 2)
        xs = []
        ms, o = timed(lambda: ib.MultiShiftSolver_CG(ib.Fopr_DdagD(De), 1e-20, 5000).solve(xs, bh, SHIFTS12))
        rm = ref["multishift12_wilson_eo"]
        res["multishift12_wilson_eo_" + name] = {
            "reference_ms": round(rm["ms"], 2), "reference_nconv": rm["nconv"],
            "ours_ms": round(ms, 2), "ours_nconv": o.Nconv, "speedup": round(rm["ms"] / ms, 1)}
        f = ib.synth_gaussian(V, spec["seed"] + 3)
        ms, _ = timed(lambda: ctx.apply(ib.OP_CLOVER_FULL, MASS, 1.0, 0, f))
        rk = ref["clover_full_mult"]
        res["clover_full_mult_" + name] = {
            "reference_ms": round(rk["ms"], 2), "ours_ms": round(ms, 3), "speedup": round(rk["ms"] / ms, 1)}
        ctx.close()
    res["note"] = ("reference: oracle/_ref on one host core in a child process; ours: the host-array "
                   "API on the GPU, copies included; same seeded inputs")
    return res


# ---- our arm --------------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch
    import iroiro_b200 as ib

    if world > 1:
        # replicas: every rank runs the headline (and its e2e and variants);
        # the solver sections are single-GPU configurations and would only
        # hold the other GPUs while they run
        args.no_solve = True
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
    step_bytes = BYTES_STEP * Vh
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
    # page-locked arrays take the overlapped path, pageable ones the plain one
    e2e_exact = bool(np.array_equal(hout.numpy(), ctx.apply(ib.OP_WILSON_SCHUR_EE, MASS, 0.0, 0, h)))

    # other precisions and operators, same protocol (reported, not the headline)
    nvar = max(10, min(args.steps, 200))
    variants = {}
    for name, op, csw, prec, bps in (
            ("wilson_fp32", ib.OP_WILSON_SCHUR_EE, 0.0, "single", 2 * 576 + 96),
            ("wilson_fp16", ib.OP_WILSON_SCHUR_EE, 0.0, "half", 2 * 296 + 52)):
        ms = schur_timing(torch, ctx, stream, prec, op, csw, Vh, nvar, flush, source=h)
        variants[name + "_32x32x32x64"] = variant_line(ms, bps, Vh, peak)
    lib.iro_field_destroy(fin)
    lib.iro_field_destroy(fout)
    ctx.close()
    # the Wilson-clover configuration's lattice: 24^3x48, gauge-transformed field
    ctx2 = ib.Context(L_C2, local)
    ctx2.set_stream(stream.cuda_stream)
    u2 = ib.synth_gauge(L_C2, EPS, SEED + 1, gauge_transform=True)
    ctx2.upload_gauge(u2, force=True)
    Vh2 = int(np.prod(L_C2)) // 2
    h2 = ib.synth_gaussian(Vh2, SEED + 101)
    for name, op, csw, prec, bps in (
            ("wilson_fp64", ib.OP_WILSON_SCHUR_EE, 0.0, "double", BYTES_STEP),
            ("wilson_fp32", ib.OP_WILSON_SCHUR_EE, 0.0, "single", 2 * 576 + 96),
            ("wilson_fp16", ib.OP_WILSON_SCHUR_EE, 0.0, "half", 2 * 296 + 52),
            # + the clover blocks A_oo^-1 and A_ee, 72 reals per site each
            ("clover_fp64", ib.OP_CLOVER_SCHUR_EE, CSW, "double", BYTES_STEP + 2 * 576),
            ("clover_fp32", ib.OP_CLOVER_SCHUR_EE, CSW, "single", 2 * 576 + 96 + 2 * 288)):
        ms = schur_timing(torch, ctx2, stream, prec, op, csw, Vh2, nvar, flush, source=h2)
        variants[name + "_24x24x24x48"] = variant_line(ms, bps, Vh2, peak)

    # time to a 1e-10 FP64 true residual, e/o Wilson-clover, FP64 CG vs mixed
    # precision; fields resident on the device (iro_cg_solve_field)
    solve = {}
    if not args.no_solve:
        D = ib.Dirac_Clover_EvenOdd(MASS, CSW, u2, ctx=ctx2)
        solve = timed_solves(ctx2, D, h2, 1, torch)
        solve["op"] = "e/o Wilson-clover Schur 24^3x48, kappa=0.12, csw=1.0, one Gaussian source"
    ctx2.close()
    batched = {}
    if not args.no_solve and not args.no_batched:
        batched = batched_solves(torch, local)
    learned_res = {}
    if not args.no_solve and not args.no_learned:
        learned_res = learned_solves(torch, local)
    caller_res = {}
    if not args.no_solve and not args.no_callers:
        caller_res = callers(torch, local)
    mixed = {}
    if not args.no_solve and not args.no_mixed48:
        mixed = mixed48(torch, local)

    if rank != 0:
        return 0
    cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline_leg()
    beside = None if args.no_cpu_baseline or world > 1 else reference_solvers_beside(torch, local)
    traffic, traffic_src = traffic_per_step(Vh)
    t_step = (t_ms / args.steps) * 1e-3
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_for(world),
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 3), "traffic": traffic,
                     "traffic_source": traffic_src, "peak_kind": peak_kind,
                     "dram_GBps": None if traffic is None else round(traffic / t_step / 1e9, 1),
                     "dram_frac": None if traffic is None else
                     round(traffic / t_step / 1e9 / peak, 3),
                     "bytes_model": "compulsory per even site: hop 1152 + hop 1152 + f_e 192 "
                                    "(FP64, recon-12)",
                     "algorithmic_GBps": round(BYTES_STEP_ALG * Vh / t_step / 1e9, 1),
                     "algorithmic_bytes_model": "5184 B per even site: 2 hops x (8 neighbour "
                                                "spinors + 8 links + output) + f_e",
                     "gflops": round(FLOPS_SCHUR * Vh / t_step / 1e9, 1)},
        "e2e": {"value": round(e2e_val, 2), "unit": "GB/s", "h2d_bytes_per_step": 24 * 8 * Vh,
                "d2h_bytes_per_step": 24 * 8 * Vh, "ms_per_step": round(e2e_ms / args.steps, 3),
                "equals_plain_path": e2e_exact},
        "gpu_launches": 2 * args.steps,
        "clocks": ck,
        "cpu_baseline": cpu,
        "reference_beside": beside,
        "variants": variants,
        "solve": solve,
        "learned": learned_res,
        "callers": caller_res,
        "mixed48": mixed,
        "batched": batched,
    }
    line["summary"] = summarise(line, peak)
    print(json.dumps(line))
    return 0


def summarise(line, peak):
    """The headline numbers of every configuration, short enough to survive
    any truncation of the printed line (the last key)."""
    g = lambda d, *k: _dig(d, k)  # noqa: E731
    out = {"headline_32x32x32x64_fp64": {"ms": line["ms_per_step"], "GBps": line["value"],
                                         "frac_of_hbm_peak": line["roofline"]["frac"],
                                         "peak_kind": line["roofline"]["peak_kind"],
                                         "dram_frac": line["roofline"]["dram_frac"]}}
    v = line["variants"]
    out["schur_fp64_24x24x24x48_frac"] = g(v, "wilson_fp64_24x24x24x48", "frac")
    out["clover_fp64_24x24x24x48_ms"] = g(v, "clover_fp64_24x24x24x48", "ms")
    out["clover_solve_24x24x24x48_ms"] = {k: g(line["solve"], k, "ms") for k in ("double", "single", "half")}
    b = line["batched"]
    if b:
        out["batched_32x32x32x64"] = {
            "fp64_cg_12_sequential_ms": b.get("fp64_cg_12_sequential_ms"),
            "block12_ms": {k: g(b, "block12", k, "ms") for k in ("half", "single", "double")},
            "block12_half_speedup_vs_12_fp64_cg": g(b, "block12", "half", "speedup_vs_12_fp64_cg"),
            "block12_half_residual": g(b, "block12", "half", "true_residual_max"),
            "multishift12_ms": {k: g(b, "multishift12", k, "ms") for k in ("double", "single", "half")},
            "multishift12_max_error_vs_fp64": {k: g(b, "multishift12", k, "max_error_vs_fp64")
                                               for k in ("single", "half")}}
    lr = line["learned"]
    if lr:
        out["learned_32x32x32x64_ms"] = {k: g(lr, k, "ms") for k in
                                         ("gcr_network", "gcr_plain", "cg_double", "cg_single", "cg_half")}
        out["learned_32x32x32x64_ms_min"] = {k: g(lr, k, "ms_min") for k in ("gcr_network", "cg_half")}
        out["learned_iterations"] = {k: g(lr, k, "iterations") for k in ("gcr_network", "cg_half")}
        out["learned_network_apply_ms"] = lr.get("network_apply_ms")
        out["gcr_network_vs_best_mixed_cg"] = lr.get("gcr_network_vs_best_mixed_cg")
        l48 = lr.get("at_48x48x48x96")
        if l48:
            out["learned_48x48x48x96_ms"] = {k: g(l48, k, "ms") for k in
                                             ("gcr_network", "gcr_plain", "cg_half")}
            out["learned_48x48x48x96_iterations"] = {k: g(l48, k, "iterations") for k in
                                                     ("gcr_network", "gcr_plain", "cg_half")}
    m = line["mixed48"]
    if m:
        out["mixed48_clover_12rhs"] = {"fp64_ms": g(m, "double", "ms"), "fp16_ms": g(m, "half", "ms"),
                                       "speedup": g(m, "half", "speedup_vs_fp64_block_cg"),
                                       "max_error_vs_fp64": g(m, "half", "error_vs_fp64_max")}
    rb = line.get("reference_beside")
    if rb:
        out["reference_beside_8x8x8x16_speedup"] = {k.replace("_8x8x8x16", ""): g(rb, k, "speedup")
                                                     for k in rb if k != "note"}
    c = line["callers"]
    if c:
        out["qprop_block12_half_speedup"] = g(c, "qprop_evenodd_32x32x32x64",
                                              "speedup_block12_half_vs_sequential_fp64")
    return out


def _dig(d, keys):
    for k in keys:
        if not isinstance(d, dict) or k not in d:
            return None
        d = d[k]
    return d


def kernel_only(args):
    """Profiling driver: `steps` applications of one operator on device
    fields inside a cudaProfilerStart/Stop range (after autotuning), for
    `ncu --profile-from-start off`.  --kernel OP,PREC,NRHS with OP one of
    wilson_eo, clover_eo, wilson_full; --lattice Lx,Ly,Lz,Lt."""
    import ctypes
    import torch
    import iroiro_b200 as ib
    Lk = [int(v) for v in args.lattice.split(",")]
    if args.kernel.startswith(("ptc,", "batched,", "multishift,", "gcr,")) or \
            args.kernel in ("md_force_eo", "md_force_clover"):
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
    batched_solves, on the lattice given) once untimed and once profiled;
    --kernel gcr,W-W-...,KRYLOV trains that network as learned_solves does and
    runs its GCR solve (learned_solves' field and source, on the lattice given)
    once untimed and once profiled; all inside cudaProfilerStart/Stop."""
    import torch
    import iroiro_b200 as ib
    from iroiro_b200 import learned
    V = int(np.prod(Lk))
    ctx = ib.Context(Lk, 0)
    if args.kernel.startswith("multishift,"):
        inner = args.kernel.split(",")[1]
        st = torch.cuda.Stream()
        torch.cuda.set_stream(st)
        ctx.set_stream(st.cuda_stream)
        u = ib.synth_gauge(Lk, EPS, SEED + 7, gauge_transform=False)
        ctx.upload_gauge(u, force=True)
        D = ib.Dirac_Wilson_EvenOdd(MASS, u, ctx=ctx)
        g = ib.synth_gaussian(V // 2, SEED + 9)
        shifts = [1e-4 * (1e5) ** (k / 11) for k in range(12)]
        ms = ib.MultiShiftSolver_CG(ib.Fopr_DdagD(D), 1e-20, 20000, inner=inner)
        G = ib.DeviceField(ctx, 0, "double").upload(g)
        XS = ib.DeviceField(ctx, 0, "double", 12)
        ms.solve_field(G, XS, shifts)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        t0 = time.perf_counter()
        o = ms.solve_field(G, XS, shifts)
        torch.cuda.synchronize()
        ms_t = (time.perf_counter() - t0) * 1e3
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": args.kernel, "lattice": Lk, "ms": round(ms_t, 2),
                          "iterations": o.Nconv, "residual": o.diff,
                          "reliable_updates": o.reliable_updates}))
        return 0
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
    if args.kernel.startswith("gcr,"):
        _, wtxt, krylov = args.kernel.split(",")
        widths = tuple(int(v) for v in wtxt.split("-"))
        pairs = learned.make_pairs([16, 16, 16, 32], 100, seed0=SEED + 300, device=0)
        net0 = learned.PTCNet(pairs[0].ctx, widths)
        learned.train(net0, pairs, epochs=15, lr=3e-3)
        for pr in pairs:
            pr.ctx.close()
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        u = ib.synth_gauge(Lk, EPS, SEED + 301)
        ctx.upload_gauge(u, force=True)
        D = ib.Dirac_Wilson(MASS, u, ctx=ctx)
        b = ib.DeviceField(ctx, 2, "double").upload(ib.synth_gaussian(V, SEED + 302))
        x = ib.DeviceField(ctx, 2, "double")
        net = learned.PTCNet(ctx, widths, net0.W)
        slv = learned.Solver_GCR(D, net, nkrylov=16, delta=0.03, krylov=krylov)
        slv.solve_field(b, x)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        t0 = time.perf_counter()
        o, rc = slv.solve_field(b, x)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        torch.cuda.profiler.stop()
        print(json.dumps({"kernel": args.kernel, "lattice": Lk, "ms": round(ms, 2),
                          "iterations": o.iterations, "restarts": o.restarts, "residual": o.diff,
                          "rc": rc}))
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
    ap.add_argument("--no-mixed48", action="store_true",
                    help="skip the 48^3x96 mixed-precision 12-RHS configuration (~1 min)")
    ap.add_argument("--kernel", default=None, help="profiling driver: OP,PREC,NRHS")
    ap.add_argument("--lattice", default="24,24,24,48")
    ap.add_argument("--ref-solver-child", nargs=2, default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ref_solver_child:
        ref_solver_child(*args.ref_solver_child)
        return 0
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
