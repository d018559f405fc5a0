#!/usr/bin/env python3
"""Benchmark of the RHMC hot path on B200.

Headline workload: the even/odd staggered Dslash on a 32^4 lattice (Haar-random SU(3) links,
unit-variance Gaussian spinors, fixed seeds; synthetic data).  One step = one full Dslash,
D_oe then D_eo (two half-Dslash launches), with FP64 links (18 reals) and FP64 spinors.
`value` is the algorithmic HBM traffic of those launches per second (GB/s, whole job over all
ranks); the other link formats are reported under `variants`.  The 32^4 FP64 links (604 MB)
are larger than the 126 MB L2, so no L2 flush is needed between steps.

Multi-GPU: independent replicas (the path has no data exchange), one process per GPU,
"scaling": "weak", value = sum over ranks of the per-rank work / max over ranks of the time.

`--impl reference` times the reference's own CPU Dslash (Doe/Deo of
lib/Action/fermionmatrix.cc, compiled unmodified into oracle/_ref/libref_b32.so) on the
host cores, one process per core.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rhmc-on-gpu_b200"))

DIMS = (32, 32, 32, 32)
METRIC = "multi-shift CG s/solve @1e-10 & Dslash GB/s at 32^4: mixed+batched vs plain FP64"

# algorithmic bytes per output site of one half-Dslash: 8 links + 1 input + 1 output spinor
LINK_BYTES = {0: 144, 1: 96, 2: 72, 3: 48}
SPINOR_BYTES = {0: 48, 1: 48, 2: 24, 3: 24}
FLOPS_PER_SITE = 570


def half_dslash_bytes(fmt, Vh, nrhs=1):
    return Vh * (8 * LINK_BYTES[fmt] + 2 * SPINOR_BYTES[fmt] * nrhs)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", "clocks_bench_%d.csv" % index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_dslash(seconds=12.0, procs=1, tag="b32"):
    """Reference Doe/Deo on the host: GB/s of algorithmic bytes, per process count."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(seconds, tag, i) for i in range(procs)])
    gbs = sum(r[0] for r in res)
    return gbs, res


def _cpu_worker(args):
    """One host process applying the reference Dslash (Doe then Deo) at 32^4 for `seconds`.
    The reference's own ordered start (Conf(0), lib/Main/Conf/conf.cc:23-39) supplies the
    links; the timing of the stencil does not depend on their values."""
    seconds, tag, idx = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    from rhmc_b200 import fields as F
    dims = DIMS
    Vh = int(np.prod(dims)) // 2
    x = F.random_spinor(dims, seed=2002 + idx)
    try:
        ref = oracle.RefLib(tag)
        kind = "reference"
    except Exception:
        ref = None
        kind = "port"
    if ref is not None:
        ref.lib.ref_dslash_loop(1, x.ctypes.data_as(oracle._D))  # warm-up
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < seconds:
            ref.lib.ref_dslash_loop(1, x.ctypes.data_as(oracle._D))
            n += 1
        dt = time.perf_counter() - t0
    else:
        orc = oracle.Oracle(dims)
        u = F.random_links(dims, seed=1001 + idx, kind="near1")
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < seconds:
            h = orc.doe(u, x)
            orc.deo(u, h)
            n += 1
        dt = time.perf_counter() - t0
    by = 2 * half_dslash_bytes(0, Vh) * n
    return by / dt / 1e9, n, dt, kind


def host_processes():
    """Processes for the host reference arm: one per core, bounded by memory (the reference
    allocates about 3.5 GB of fields per 32^4 process)."""
    n = os.cpu_count() or 1
    try:
        import psutil
        n = min(n, max(1, int(psutil.virtual_memory().available / 4.5e9)))
    except Exception:
        n = min(n, 4)
    return max(1, min(n, 32))


def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    procs = host_processes()
    steps = max(1, a.steps)
    # each step: a bounded sample of every process applying the full Dslash at 32^4
    seconds = 10.0
    t0 = time.perf_counter()
    gbs, res = cpu_reference_dslash(seconds=seconds, procs=procs)
    wall = time.perf_counter() - t0
    kind = res[0][3]
    napps = sum(r[1] for r in res)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s",
        "n_gpus": a.gpus, "steps": steps, "warmup": a.warmup,
        "ms_per_step": round(1000.0 * sum(r[2] for r in res) / max(1, napps), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "Dslash Doe+Deo 32^4 FP64 (reference CPU, lib/Action/fermionmatrix.cc)",
                   "lattice": list(DIMS), "precision": "f64", "processes": procs},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": procs, "kind": kind,
                         "sample": "%d full Dslash applications at 32^4 over %d processes, %.0f s each" % (napps, procs, seconds)},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 1),
    }
    print(json.dumps(line))
    return 0


MS_DIMS = (24, 24, 24, 32)


def msolve_bench(rb, F, np, torch, rank, dev, stream, nrhs=4, nshift=16, res=1e-10):
    from rhmc_b200 import replicas as RP
    """Multi-shift CG at 24^3x32, am=0.01: 16 poles log-spaced in [1e-4, 50], 4 Gaussian RHS,
    true residual 1e-10.  Plain FP64 single-RHS (the reference algorithm, RHS after RHS, then
    FP64 CG refinement of every system whose FP64 true residual is still above 1e-10) against
    the mixed batched solver; both checked by FP64 true residuals.  The reference algorithm
    without the refinement is reported too (it stops on its iterated residual)."""
    ctx = rb.Context(MS_DIMS, mass=0.01, beta=5.7, device=dev.index or 0)
    ctx.set_stream(stream.cuda_stream)
    u = F.random_links(MS_DIMS, seed=RP.replica_seed(1001, rank))
    ctx.set_gauge(u)
    Vh = ctx.Vh
    shifts = 1e-4 * (5e5) ** (np.arange(nshift) / (nshift - 1.0))
    b_host = F.random_spinor(MS_DIMS, seed=RP.replica_seed(2002, rank), n=nrhs)
    b = torch.zeros(nrhs * 6 * Vh, dtype=torch.float64, device=dev)
    ctx.spinor_to_internal(rb.LINKS_F64_18, b, b_host, nrhs)
    x = torch.zeros(nrhs * nshift * 6 * Vh, dtype=torch.float64, device=dev)
    out = {}
    for name, mode, fmt, batched, cert in (("fp64_single_rhs", rb.MSOLVE_FP64, rb.LINKS_F64_18, False, 1),
                                           ("fp64_single_rhs_uncertified", rb.MSOLVE_FP64, rb.LINKS_F64_18, False, 0),
                                           ("mixed_batched", rb.MSOLVE_MIXED, rb.LINKS_F64_12, True, 0),
                                           ("mixed_batched_f32_bulk", rb.MSOLVE_MIXED, rb.LINKS_F32_12, True, 0)):
        # warm-up on a loose residual (graphs, derived link formats)
        ctx.msolve(x, b, shifts, 1e-4, nrhs=nrhs if batched else 1, mode=mode, fmt=fmt)
        stream.synchronize()
        t0 = time.perf_counter()
        infos = []
        if batched:
            infos.append(ctx.msolve(x, b, shifts, res, nrhs=nrhs, mode=mode, fmt=fmt))
        else:
            for r in range(nrhs):
                infos.append(ctx.msolve(x[r * nshift * 6 * Vh:], b[r * 6 * Vh:], shifts, res, nrhs=1, mode=mode, fmt=fmt,
                                        certify=cert))
        stream.synchronize()
        dt = time.perf_counter() - t0
        tr = ctx.true_residuals(x, b, shifts, nrhs=nrhs)
        out[name] = {"s_per_solve": round(dt, 4), "max_true_residual": float(tr.max()),
                     "iters": [i["iters"][0] for i in infos] if not batched else infos[0]["iters"][:nrhs],
                     "refine_iters": sum(i["refine_iters"] for i in infos),
                     "links": rb.FMT_NAMES[fmt]}
    out["speedup_mixed_vs_fp64"] = round(out["fp64_single_rhs"]["s_per_solve"] / out["mixed_batched"]["s_per_solve"], 3)
    out["config"] = {"lattice": list(MS_DIMS), "mass": 0.01, "nshift": nshift, "shifts": [float(shifts[0]), float(shifts[-1])],
                     "nrhs": nrhs, "residual": res, "links": "Haar (beta=5.7 labels the run)"}
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--no-msolve", action="store_true")
    a = ap.parse_args()
    a.warmup = max(3, a.warmup)
    if a.impl == "reference":
        return run_reference_arm(a)

    import numpy as np
    import torch
    import rhmc_b200 as rb
    from rhmc_b200 import fields as F
    from rhmc_b200 import replicas as RP

    global DIMS
    DIMS = tuple(int(v) for v in a.dims.split(","))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    V = int(np.prod(DIMS))
    Vh = V // 2
    ctx = rb.Context(DIMS, mass=0.01, beta=5.8, device=local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    u = F.random_links(DIMS, seed=RP.replica_seed(1001, rank))
    ctx.set_gauge(u)
    x = F.random_spinor(DIMS, seed=RP.replica_seed(2002, rank))

    peak, peak_kind = load_peaks()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return RP.max_over_ranks(v, dist, dev)

    results = {}
    for fmt in (rb.LINKS_F64_18, rb.LINKS_F64_12, rb.LINKS_F32_18, rb.LINKS_F32_12):
        f64 = fmt in (rb.LINKS_F64_18, rb.LINKS_F64_12)
        dt = torch.float64 if f64 else torch.float32
        xe = torch.zeros(6 * Vh, dtype=dt, device=dev)
        xo = torch.zeros(6 * Vh, dtype=dt, device=dev)
        ctx.spinor_to_internal(fmt, xe, x)
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                ctx.dslash(fmt, 1, xo, xe)
                ctx.dslash(fmt, 0, xe, xo)
        stream.synchronize()
        clocks = ClockSampler(local) if fmt == rb.LINKS_F64_18 else None
        if clocks:
            clocks.start()
        barrier()
        torch.cuda.synchronize()
        n0 = ctx.launch_count()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            ctx.dslash_repeat(fmt, xe, xo, 1, a.steps)  # steps x (D_oe, D_eo) issued from C
            ev1.record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        barrier()
        launches = ctx.launch_count() - n0
        cl = clocks.stop() if clocks else None
        total_ms = ev0.elapsed_time(ev1)
        per_launch = [total_ms / (2 * a.steps)]
        total_ms = max_over_ranks(total_ms)
        by_launch = half_dslash_bytes(fmt, Vh)
        avg_launch_ms = sum(per_launch) / len(per_launch)
        results[fmt] = dict(total_ms=total_ms, avg_launch_ms=avg_launch_ms, launches=launches, clocks=cl,
                            gbs=world * 2 * by_launch * a.steps / (total_ms * 1e-3) / 1e9,
                            achieved=by_launch / (avg_launch_ms * 1e-3) / 1e9,
                            gflops=world * 2 * FLOPS_PER_SITE * Vh * a.steps / (total_ms * 1e-3) / 1e9)
        del xe, xo

    # end to end: reference-facing host call (host spinors in/out, copies inside the timing)
    xin = np.ascontiguousarray(x)
    pin_in = torch.from_numpy(xin.view(np.float64).reshape(-1).copy()).pin_memory()
    pin_out = torch.zeros(6 * Vh, dtype=torch.float64).pin_memory()
    e2e_steps = max(3, min(a.steps, 50))
    for _ in range(3):
        ctx.dslash_host(1, pin_out.numpy(), pin_in.numpy())
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.dslash_host(1, pin_out.numpy(), pin_in.numpy())
        ctx.dslash_host(0, pin_in.numpy(), pin_out.numpy())
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_gbs = world * 2 * half_dslash_bytes(0, Vh) * e2e_steps / e2e_s / 1e9

    ms = None
    if not a.no_msolve:
        try:
            ms = msolve_bench(rb, F, np, torch, rank, dev, stream)
        except Exception as e:  # reported in the JSON line, the Dslash numbers stand
            ms = {"error": str(e)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            gbs, res = cpu_reference_dslash(seconds=12.0, procs=1)
            cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": 1, "kind": res[0][3],
                   "sample": "%d full Dslash (Doe+Deo) applications at 32^4 FP64 in %.1f s" % (res[0][1], res[0][2])}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "GB/s", "cores": 1, "kind": "reference", "sample": "failed: %s" % e}

    r = results[rb.LINKS_F64_18]
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(r["gbs"], 2), "unit": "GB/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(r["total_ms"] / a.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (Haar links seed 1001+rank, Gaussian spinor seed 2002+rank)",
            "config": {"workload": "Dslash D_oe+D_eo 32^4 FP64 links(18 real) + FP64 spinors, 1 RHS",
                       "lattice": list(DIMS), "parallelism": "replicas%d" % world,
                       "l2": "inputs larger than L2 (links 604 MB)"},
            "roofline": {"bound": "hbm", "achieved": round(r["achieved"], 1), "peak": peak, "unit": "GB/s",
                         "frac": round(r["achieved"] / peak, 4), "traffic": None,
                         "peak_kind": peak_kind, "kernel": "dslash_kernel<L64_18,1>",
                         "bytes_per_launch": half_dslash_bytes(0, Vh)},
            "gflops": round(r["gflops"], 1),
            "variants": {rb.FMT_NAMES[f]: {"gbs": round(v["gbs"], 1), "achieved": round(v["achieved"], 1),
                                            "frac": round(v["achieved"] / peak, 4),
                                            "us_per_half_dslash": round(1000 * v["avg_launch_ms"], 2),
                                            "sites_per_s": round(2 * Vh * a.steps / (v["total_ms"] * 1e-3) * world, 1)}
                         for f, v in results.items()},
            "e2e": {"value": round(e2e_gbs, 2), "unit": "GB/s", "h2d_bytes_per_step": 2 * 48 * Vh,
                    "d2h_bytes_per_step": 2 * 48 * Vh, "api": "rhmc_dslash_host (host spinors, pinned)"},
            "msolve": ms,
            "cpu_baseline": cpu,
            "gpu_launches": r["launches"],
            "clocks": r["clocks"],
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
