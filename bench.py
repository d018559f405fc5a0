#!/usr/bin/env python3
"""Benchmark of the RHMC hot path on B200.

Headline workload: the even/odd staggered Dslash on a 32^4 lattice (Haar-random SU(3) links,
unit-variance Gaussian spinors, fixed seeds; synthetic data).  One step = the 1000 half-Dslash
applications of the Dslash benchmark configuration: 500 full Dslash, D_oe then D_eo, with FP64
links (18 reals) and FP64 spinors, each output the next input (after a few hundred applications
the values overflow; the kernel's time does not depend on them, and its output is checked
against the reference's Deo/Doe at this lattice by tests/test_dslash32_gpu.py).  `value` is
the algorithmic HBM traffic of those launches per second (GB/s, whole job over all ranks); the
other link formats are reported under `variants`.  The 32^4 FP64 links (604 MB) are larger
than the 126 MB L2, so no L2 flush is needed between steps.

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
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rhmc-on-gpu_b200"))

DIMS = (32, 32, 32, 32)
PAIRS = 500  # full Dslash (D_oe, D_eo) per step: 1000 half-Dslash applications
METRIC ="multi-shift CG s/solve @1e-10 & Dslash GB/s at 32^4: mixed+batched vs plain FP64"

# algorithmic bytes per output site of one half-Dslash: 8 links + 1 input + 1 output spinor
LINK_BYTES = {0: 144, 1: 96, 2: 72, 3: 48, 4: 24}
SPINOR_BYTES = {0: 48, 1: 48, 2: 24, 3: 24, 4: 16}  # 4: half with a per-site scale (16-byte vector)
FLOPS_PER_SITE = 570


def approx_report(groups):
    """Each approximation's degree, method and maximum relative error on its interval (what the
    reference prints for every approximation it builds, lib/Tools/RationalApprox/
    rationalapprox_calc.cc:42): groups = one [first, md, last] list per species."""
    roles = ("first (heatbath)", "md (force)", "last (action)")
    return [{"species": si, "role": roles[j], "power": c["power"], "poles": len(c["b"]),
             "method": c.get("method", "lsq"), "max_rel_err": c["max_rel_err"]}
            for si, g in enumerate(groups) for j, c in enumerate(g)]


def solver_summary(ctx):
    """What the driver's solves of the last trajectory cost (rhmc_driver_solver_stats), force
    solves and heatbath/action solves separately; resets the sums."""
    keys = ("iters_total", "iters_max", "iters_fp64", "ms_reliable_updates", "refine_iters", "systems_refined",
            "seconds", "seconds_phase_a")
    md = ctx.driver_solver_stats(0)
    metro = ctx.driver_solver_stats(1, reset=True)
    return {"md": {k: (round(md[k], 3) if isinstance(md[k], float) else md[k]) for k in keys},
            "metro": {k: (round(metro[k], 3) if isinstance(metro[k], float) else metro[k]) for k in keys}}


def half_dslash_bytes(fmt, Vh, nrhs=1):
    return Vh * (8 * LINK_BYTES[fmt] + 2 * SPINOR_BYTES[fmt] * nrhs)


def tuned_shapes(rb, Vh):
    """The launch shape (threads per block, minimum blocks per SM) the autotuner chose for each
    Dslash instantiation timed at this volume, with the candidates' times in microseconds."""
    out = {}
    for e in rb.tune_report().get("entries", []):
        dev, vh, what = (e["key"].split("|") + ["", ""])[:3]
        if vh == "vh=%d" % Vh and what.startswith("dslash"):
            out[what] = {"block": e["shapes"][e["choice"]][0], "min_blocks": e["shapes"][e["choice"]][1],
                         "candidates_us": dict(("%dx%d" % tuple(s), t) for s, t in zip(e["shapes"], e["us"]))}
    return out


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
        # the raw samples go to RHMC_CLOCKS_CSV when set (kept for inspection), else a temporary file
        self.path = os.environ.get("RHMC_CLOCKS_CSV") or os.path.join(
            tempfile.gettempdir(), "rhmc_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
            d = os.path.dirname(self.path)
            if d:
                os.makedirs(d, exist_ok=True)
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


def msolve_bench(rb, F, np, torch, rank, dev, stream, dims=None, relative=False, nrhs=4, nshift=16, res=1e-10, only=(),
                 mass=0.01, warmup=True, cpu=False):
    """Multi-shift CG, am=0.01: 16 poles log-spaced in [1e-4, 50], 4 Gaussian RHS, true residual
    1e-10 for every (RHS, pole) system: absolute |b - (M^dag M + s) x| <= 1e-10 (the reference's
    stopping criterion, inverter.cc:287) or, with relative, <= 1e-10 |b| (at 32^4 the absolute
    1e-10 is below the FP64 rounding floor of the smallest poles).  Plain FP64 single-RHS (the
    reference algorithm, RHS after RHS, then FP64 CG refinement of every system whose FP64 true
    residual is still above target) against the mixed batched solver; both checked by FP64 true
    residuals.  The reference algorithm without the refinement is reported too (it stops on its
    iterated residual).  Every variant runs once untimed, then timed."""
    from rhmc_b200 import replicas as RP
    dims = dims or MS_DIMS
    ctx = rb.Context(dims, mass=mass, beta=5.7, device=dev.index or 0)
    ctx.set_stream(stream.cuda_stream)
    u = F.random_links(dims, seed=RP.replica_seed(1001, rank))
    ctx.set_gauge(u)
    Vh = ctx.Vh
    shifts = 1e-4 * (5e5) ** (np.arange(nshift) / (nshift - 1.0))
    b_host = F.random_spinor(dims, seed=RP.replica_seed(2002, rank), n=nrhs)
    res_target = res
    if relative:
        res = res * float(np.sqrt(min((np.abs(bb) ** 2).sum() for bb in b_host)))
    b = torch.zeros(nrhs * 6 * Vh, dtype=torch.float64, device=dev)
    ctx.spinor_to_internal(rb.LINKS_F64_18, b, b_host, nrhs)
    x = torch.zeros(nrhs * nshift * 6 * Vh, dtype=torch.float64, device=dev)
    out = {}
    for name, mode, fmt, batched, cert in (("fp64_single_rhs", rb.MSOLVE_FP64, rb.LINKS_F64_18, False, 1),
                                           ("fp64_single_rhs_uncertified", rb.MSOLVE_FP64, rb.LINKS_F64_18, False, 0),
                                           ("mixed_batched", rb.MSOLVE_MIXED, rb.LINKS_F64_12, True, 0),
                                           ("mixed_batched_f32_bulk", rb.MSOLVE_MIXED, rb.LINKS_F32_12, True, 0),
                                           ("mixed_batched_f32_bulk_f16_refine", rb.MSOLVE_MIXED, rb.LINKS_F16_12, True, 0)):
        if only and name not in only:
            continue
        def solve():
            infos = []
            if batched:
                infos.append(ctx.msolve(x, b, shifts, res, nrhs=nrhs, mode=mode, fmt=fmt))
            else:
                for r in range(nrhs):
                    infos.append(ctx.msolve(x[r * nshift * 6 * Vh:], b[r * 6 * Vh:], shifts, res, nrhs=1, mode=mode,
                                            fmt=fmt, certify=cert))
            return infos

        # warm-up: the identical solve, untimed (module loading, graphs, workspaces, derived links)
        if warmup:
            solve()
        stream.synchronize()
        t0 = time.perf_counter()
        infos = solve()
        stream.synchronize()
        dt = time.perf_counter() - t0
        tr = ctx.true_residuals(x, b, shifts, nrhs=nrhs)
        out[name] = {"s_per_solve": round(dt, 4), "max_true_residual": float(tr.max()),
                     "iters": [i["iters"][0] for i in infos] if not batched else infos[0]["iters"][:nrhs],
                     "refine_iters": sum(i["refine_iters"] for i in infos),
                     "s_phase_a": round(sum(i["seconds_phase_a"] for i in infos), 4),
                     "systems_refined": sum(i["systems_refined"] for i in infos),
                     "iters_fp64": sum(i["iters_fp64"] for i in infos) if batched else None,
                     "ms_reliable_updates": sum(i["ms_reliable_updates"] for i in infos),
                     "links": rb.FMT_NAMES[fmt]}
    mixed = [k for k in ("mixed_batched", "mixed_batched_f32_bulk", "mixed_batched_f32_bulk_f16_refine") if k in out]
    if "fp64_single_rhs" in out and mixed:
        best = min(mixed, key=lambda k: out[k]["s_per_solve"])
        out["speedup_mixed_vs_fp64"] = round(out["fp64_single_rhs"]["s_per_solve"] / out[best]["s_per_solve"], 3)
        out["speedup_variant"] = best
    out["config"] = {"lattice": list(dims), "mass": mass, "nshift": nshift, "shifts": [float(shifts[0]), float(shifts[-1])],
                     "nrhs": nrhs, "residual": res_target,
                     "residual_kind": "relative to |b| (absolute %.3g)" % res if relative else "absolute",
                     "links": "Haar (beta=5.7 labels the run)"}
    free, total = torch.cuda.mem_get_info(dev)
    out["device_memory_in_use_gb"] = round((total - free) / 1e9, 2)  # workspaces of all variants, at the end
    ctx.close()
    # the bounded reference builds: lattice -> (tag, poles, mass) they were compiled for
    tag, ref_nshift, ref_mass = {(24, 24, 24, 32): ("m24", 16, 0.01), (32, 32, 32, 32): ("m32", 16, 0.01),
                                 (48, 48, 48, 48): ("m48", 20, 0.005)}.get(tuple(dims), (None, 0, 0.0))
    if cpu and tag and nshift == ref_nshift and abs(mass - ref_mass) < 1e-12:
        out["cpu_reference"] = reference_msolve_timing(tag, u, b_host[0], shifts, np,
                                                       out.get("fp64_single_rhs", {}).get("iters", [None])[0], nrhs)
    return out


def reference_msolve_timing(tag, u, b, shifts, np, iters, nrhs):
    """The reference's own CPU multi-shift solver (multips_shifted_invert,
    lib/Action/Inverter/inverter.cc:142-339, unmodified, behind the harness in
    oracle/_ref/libref_<tag>.so, built with max_cg = 100 (24^3x32), 60 (32^4) or 10 (48^4)) on the same links,
    right-hand side and poles, on one host core: seconds per iteration over its first max_cg
    iterations (all 16 poles still active, so an upper figure for the average iteration), and
    that figure times the B200 solve's iteration count as the estimated CPU time of the solve."""
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        ref = oracle.RefLib(tag)
    except Exception as e:
        return {"unavailable": str(e)[:200]}
    ref.set_links(u)
    ref.set_chi(np.asarray(b)[None])
    n_it = int(ref.lib.ref_param(5))  # max_cg of the build
    t0 = time.perf_counter()
    ref.msolve(1e-10, shifts)
    dt = time.perf_counter() - t0
    out = {"kind": "reference", "cores": 1, "iterations_timed": n_it, "s_per_iteration": round(dt / n_it, 5),
           "sample": "first %d iterations of one right-hand side, %d poles, FP64" % (n_it, len(shifts))}
    if iters:
        out["est_s_per_solve"] = round(dt / n_it * iters * nrhs, 1)
        out["est_basis"] = "%d iterations x %d right-hand sides" % (iters, nrhs)
    return out


NF_ML, NF_MS, NF_BETA, NF_DEG = 0.01, 0.05, 5.8, 15

# DRAM bytes per output site of dslash_kernel<L64_18,1>, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum of its first timed launch at 24^4:
# 200,237,056 + 6,219,008 bytes over Vh = 165,888 sites); the kernel streams per site, so the
# traffic of a launch is this times Vh
DSLASH_F64_18_DRAM_PER_SITE = (200237056 + 6219008) / 165888


def _timed(torch, stream, fn, reps):
    """Average device time (ms) of fn() issued reps times on stream, CUDA events on that stream."""
    fn()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / reps


def nf2p1_bench(a, rb, F, np, torch, rank, dev, stream):
    """N_f = 2+1 RHMC at 32^4 (light am=0.01 with N_f=2, strange am=0.05 with N_f=1, one
    pseudofermion each, degree-15 rational approximations, beta=5.8, Haar hot start seed 1001,
    momenta seed 3003, phi seeds 2002/2003, Metropolis uniform seed 4004; synthetic data).

    1. MD kernels at this volume: device time and algorithmic bytes of the gauge force, the
       fermion force (both species' 30 shifted solutions), the momentum and the link update.
    2. The fermion force against central finite differences of S_f (md approximation, both
       species) with eps = 1e-5 along fd_dirs random su(3) directions (seed 5005) on fd_links
       random links (seed 6006).  At this volume S_f ~ 1e6, so S(+eps) - S(-eps) taken as the
       difference of two separately summed actions loses ~11 digits; the central difference is
       therefore also evaluated exactly as sum_i a_i Re<x_i(+), (A(-) - A(+)) x_i(-)> with
       A = M^dag M + b_i and x_i(+-) the solutions at the two perturbed configurations (the
       second resolvent identity, no approximation): A(-) - A(+) is non-zero only next to the
       perturbed link, so nothing cancels.  Both are reported.
    3. One leapfrog trajectory (tau = 1, 20 steps) with all-FP64 solves and with the mixed
       solver for the force (FP64 heatbath/action solves): seconds per trajectory, Delta H,
       acceptance and plaquette of both."""
    from scipy.linalg import expm
    from rhmc_b200 import rational as R
    from rhmc_b200 import replicas as RP
    # torch work (link edits, inner products) must be ordered with the library's launches
    torch.cuda.set_stream(stream)
    dims = DIMS
    V = int(np.prod(dims))
    Vh = V // 2
    ctx = rb.Context(dims, mass=NF_ML, beta=NF_BETA, device=dev.index or 0)
    ctx.set_stream(stream.cuda_stream)
    u = F.random_links(dims, seed=RP.replica_seed(1001, rank))
    u_traj = u if a.nf_start == "haar" else F.random_links(dims, seed=RP.replica_seed(1001, rank), kind="near1", eps=0.3)
    ctx.set_gauge(u)
    P0 = F.random_momenta(dims, seed=RP.replica_seed(3003, rank))
    phis = [F.random_spinor(dims, seed=RP.replica_seed(2002, rank), n=1),
            F.random_spinor(dims, seed=RP.replica_seed(2003, rank), n=1)]
    uniform = float(np.random.Generator(np.random.Philox(RP.replica_seed(4004, rank))).random())
    # spectral bounds: lambda_max by power iteration, lambda_min = m^2 (M^dag M = m^2 - D_eo D_oe >= m^2)
    lmax = ctx.find_max(F.random_spinor(dims, seed=7007))
    species = [(NF_ML, 2), (NF_MS, 1)]
    bounds, approx = [], []
    for m, nf in species:
        lo, hi = m * m, lmax + m * m - NF_ML * NF_ML
        eps = 0.95 * lo / (1.05 * hi)
        bounds.append((lo, hi))
        approx.append([R.rational_power(nf / 8.0, NF_DEG, eps), R.rational_power(-nf / 4.0, NF_DEG, eps),
                       R.rational_power(-nf / 4.0, NF_DEG, eps)])
    out = {"config": {"lattice": list(dims), "beta": NF_BETA, "species": [{"mass": m, "no_flavours": nf, "no_ps": 1}
                                                                         for m, nf in species],
                      "degree": NF_DEG, "eig_bounds": bounds, "start": "Haar (hot) for kernels and finite differences; "
                      + ("Haar" if a.nf_start == "haar" else "exp(i 0.3 H) of a Gaussian algebra element H per link")
                      + " for the trajectories",
                      "approx_max_rel_err": max(c["max_rel_err"] for ap_ in approx for c in ap_),
                      "approximations": approx_report(approx)}}

    def configure(md_mode, md_fmt, residue_md, no_md=20):
        ctx.driver_setup(no_flavours=2, no_ps=1, no_md=no_md, integrator=rb.INT_LEAPFROG, residue_metro=1e-10,
                         residue_md=residue_md, md_mode=md_mode, md_fmt=md_fmt)
        if not getattr(ctx, "_nf_species", False):
            ctx._nf_species = ctx.add_species(NF_MS, 1, 1)
        for s in range(2):
            ctx.select_species(s)
            for w in range(3):
                ctx.set_approx(w, approx[s][w])
            ctx.set_eig_bounds(*bounds[s])
            ctx.set_phi(phis[s])
        ctx.select_species(0)

    # ---- 1. MD kernels
    configure(rb.MSOLVE_FP64, rb.LINKS_F64_18, 1e-10)
    ctx.first_inv_approx_calc(1e-10)
    ctx.set_momenta(P0)
    nv = 2 * NF_DEG
    xk = torch.randn(nv * 6 * Vh, dtype=torch.float64, device=dev)
    coef = np.linspace(0.1, 1.0, nv)
    reps = 5
    kern = {}
    kern["gauge_force"] = (_timed(torch, stream, lambda: ctx.gauge_force(0), reps), 4 * V * (144 + 64))
    kern["fermion_force_30_vectors"] = (_timed(torch, stream, lambda: ctx.fermion_force(xk, coef, nrhs=1, add=1), reps),
                                        4 * V * (144 + 128) + -(-nv // 8) * 4 * V * 144 + nv * (Vh * 96 + V * 48))
    kern["mom_update"] = (_timed(torch, stream, lambda: ctx.mom_update(0.0), reps), 4 * V * 3 * 64)
    kern["link_update"] = (_timed(torch, stream, lambda: ctx.link_update(0.0), reps), 4 * V * (64 + 2 * 144))
    # rational sum chi = a0 b + sum_i a_i x_i over one pole set (15 shifted vectors)
    chi_out = torch.zeros(6 * Vh, dtype=torch.float64, device=dev)
    kern["rational_sum_15_poles"] = (_timed(torch, stream, lambda: ctx.rational_sum(chi_out, xk, xk[:6 * Vh], 0.5,
                                                                                    coef[:NF_DEG]), reps),
                                     (NF_DEG + 2) * Vh * 48)
    # actions and plaquette: one pass over the links (or momenta) and an FP64 reduction; these
    # return host values, so the time includes the synchronisation and the read-back
    kern["gauge_action"] = (_timed(torch, stream, lambda: ctx.gauge_action(), reps), 4 * V * 144)
    kern["plaquette"] = (_timed(torch, stream, lambda: ctx.plaquette(), reps), 4 * V * 144)
    kern["momentum_action"] = (_timed(torch, stream, lambda: ctx.momentum_action(), reps), 4 * V * 64)
    del chi_out
    peak, _ = load_peaks()
    fp64_peak = ctx.fma_peak(True)
    out["kernels"] = {k: {"ms": round(t, 4), "alg_bytes": b, "gbs": round(b / (t * 1e-3) / 1e9, 1),
                          "frac": round(b / (t * 1e-3) / 1e9 / peak, 4)} for k, (t, b) in kern.items()}
    # the FP64 CUDA-core roofline of the compute-leaning kernels (algorithmic flops per link)
    for k, fl in (("gauge_force", 2700), ("link_update", 1300)):
        tf = fl * 4 * V / (kern[k][0] * 1e-3) / 1e12
        out["kernels"][k].update({"flops_per_link": fl, "tflops": round(tf, 2), "frac_fp64": round(tf / fp64_peak, 4)})
    out["kernels"]["fp64_fma_peak_tflops"] = round(fp64_peak, 2)
    out["kernels"]["fp32_fma_peak_tflops"] = round(ctx.fma_peak(False), 2)
    out["kernels"]["note"] = ("fermion_force = D_oe of the 30 vectors batched 8 per link read, then the outer-product/TA "
                              "kernel; bytes: links + ipdot read-modify-write, links once per 8 vectors, per vector "
                              "the spinor in/out of D_oe and the x and h reads of the force kernel")
    del xk
    ctx.set_gauge(u)

    # ---- 2. finite differences of S_f
    if a.fd_links > 0:
        configure(rb.MSOLVE_FP64, rb.LINKS_F64_18, 1e-10)
        ctx.first_inv_approx_calc(1e-10)
        chis = []
        for s in range(2):
            ctx.select_species(s)
            c_int = torch.zeros(6 * Vh, dtype=torch.float64, device=dev)
            ctx.spinor_to_internal(rb.LINKS_F64_18, c_int, ctx.get_chi()[0])
            chis.append(c_int)
        ctx.select_species(0)
        ctx.calc_ipdot_fermion()
        ip = ctx.get_ipdot()
        md = []
        for s, (m, nf) in enumerate(species):
            r = R.rescale(approx[s][1], 1.05 * bounds[s][1], -nf / 4.0)
            md.append((np.array(r["b"]) + (m * m - NF_ML * NF_ML), np.array(r["a"]), r["a0"]))
        rng = np.random.Generator(np.random.Philox(6006))
        links = rng.choice(4 * V, size=a.fd_links, replace=False)
        Qs = F.random_algebra(a.fd_dirs, np.random.Generator(np.random.Philox(5005)))
        u_dev = torch.from_numpy(u).to(dev)
        xs = {k: torch.zeros(NF_DEG * 6 * Vh, dtype=torch.float64, device=dev) for k in ("m0", "m1", "p0", "p1")}
        w1 = [torch.zeros(NF_DEG * 6 * Vh, dtype=torch.float64, device=dev) for _ in range(2)]
        w2 = torch.zeros(NF_DEG * 6 * Vh, dtype=torch.float64, device=dev)
        h = 1e-5
        errs, errs_plain, t_fd = [], [], time.perf_counter()
        for l in links:
            ul = u[l].copy()
            for Q in Qs:
                exact = float((1j * np.trace(Q @ ip[l])).real)
                scale = float(np.linalg.norm(Q) * np.linalg.norm(ip[l]))
                S = {}
                for sign in (-1, 1):
                    u_dev[l] = torch.from_numpy(expm(1j * sign * h * Q) @ ul).to(dev)
                    ctx.set_gauge(u_dev)
                    tag = "m" if sign < 0 else "p"
                    for s in range(2):
                        x = xs[tag + str(s)]
                        ctx.msolve(x, chis[s], md[s][0], 1e-10, certify=1)
                        xv = x.view(NF_DEG, 6 * Vh)
                        S[(sign, s)] = md[s][2] * float(torch.dot(chis[s], chis[s])) + float(
                            (torch.as_tensor(md[s][1], device=dev) * (xv @ chis[s])).sum())
                        if sign < 0:
                            ctx.mdagm(rb.LINKS_F64_18, w1[s], xs["m" + str(s)], 0.0, NF_DEG)
                        else:
                            ctx.mdagm(rb.LINKS_F64_18, w2, xs["m" + str(s)], 0.0, NF_DEG)
                            d = (xs["p" + str(s)].view(NF_DEG, 6 * Vh) * (w1[s] - w2).view(NF_DEG, 6 * Vh)).sum(1)
                            S[("id", s)] = float((torch.as_tensor(md[s][1], device=dev) * d).sum())
                u_dev[l] = torch.from_numpy(ul).to(dev)
                fd_id = (S[("id", 0)] + S[("id", 1)]) / (2 * h)
                fd_plain = sum(S[(1, s)] - S[(-1, s)] for s in range(2)) / (2 * h)
                errs.append(abs(fd_id - exact) / scale)
                errs_plain.append(abs(fd_plain - exact) / scale)
            print("fd: link %d done, %d pairs, max rel err %.3g, %.1f s" % (l, len(errs), max(errs), time.perf_counter() - t_fd),
                  file=sys.stderr, flush=True)
        ctx.set_gauge(u)
        out["fd_check"] = {"pairs": len(errs), "links": int(a.fd_links), "directions": int(a.fd_dirs), "eps": h,
                           "solve_true_residual": 1e-10,
                           "max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs)),
                           "max_rel_err_plain_difference": float(max(errs_plain)),
                           "rel_err_definition": "|FD - Re i Tr(Q ipdot_l)| / (|Q| |ipdot_l|)",
                           "target": 1e-8, "seconds": round(time.perf_counter() - t_fd, 1)}
        del u_dev, xs, w1, w2

    # ---- 3. trajectories: the MD evolution alone (plaquette of the proposal), then the full update
    traj = {}
    bounds_traj = bounds
    if a.nf_start != "haar":
        ctx.set_gauge(u_traj)
        lmax_t = ctx.find_max(F.random_spinor(dims, seed=7007))
        bounds_traj = [(m * m, lmax_t + m * m - NF_ML * NF_ML) for m, _ in species]
        if lmax_t > lmax:
            raise RuntimeError("trajectory start has a larger spectral radius than the approximations cover")
    for name, mode, fmt in (("fp64", rb.MSOLVE_FP64, rb.LINKS_F64_18), ("mixed", rb.MSOLVE_MIXED, rb.LINKS_F64_12),
                            ("mixed_f32_schedule", rb.MSOLVE_MIXED, rb.LINKS_F32_12)):
        configure(mode, fmt, 1e-8, no_md=a.nf_steps)
        for s in range(2):
            ctx.select_species(s)
            ctx.set_eig_bounds(*bounds_traj[s])
        ctx.select_species(0)
        ctx.set_gauge(u_traj)
        ctx.set_momenta(P0)
        ctx.first_inv_approx_calc(1e-10)
        stream.synchronize()
        t0 = time.perf_counter()
        ctx.update_nometro()
        stream.synchronize()
        t_md = time.perf_counter() - t0
        plaq_md = ctx.plaquette()
        ctx.set_gauge(u_traj)
        ctx.set_momenta(P0)
        stream.synchronize()
        ctx.driver_solver_stats(0, reset=True)
        n0 = ctx.launch_count()
        t0 = time.perf_counter()
        dS, acc = ctx.update(uniform)
        stream.synchronize()
        dt = time.perf_counter() - t0
        traj[name] = {"s_per_trajectory": round(dt, 3), "s_md_only": round(t_md, 3), "delta_H": dS, "accepted": acc,
                      "plaquette_proposal": plaq_md, "plaquette_after": ctx.plaquette(),
                      "gpu_launches": ctx.launch_count() - n0, "solves": solver_summary(ctx)}
    traj["speedup_mixed_vs_fp64"] = round(traj["fp64"]["s_per_trajectory"] / traj["mixed"]["s_per_trajectory"], 3)
    traj["speedup_mixed_f32_schedule_vs_fp64"] = round(traj["fp64"]["s_per_trajectory"]
                                                       / traj["mixed_f32_schedule"]["s_per_trajectory"], 3)
    traj["delta_H_abs_diff"] = max(abs(traj["fp64"]["delta_H"] - traj[k]["delta_H"]) for k in ("mixed", "mixed_f32_schedule"))
    traj["integrator"] = "leapfrog tau=1, %d steps; md residual 1e-8, metro residual 1e-10 (FP64)" % a.nf_steps
    traj["plaquette_proposal_abs_diff"] = max(abs(p - q) for k in ("mixed", "mixed_f32_schedule")
                                              for p, q in zip(traj["fp64"]["plaquette_proposal"], traj[k]["plaquette_proposal"]))
    out["trajectory"] = traj
    ctx.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return out


B5_ML, B5_MS, B5_BETA, B5_DEG = 0.005, 0.04, 5.8, 20
B5_POLE_GROUP = 5  # poles per group in the pole-group arm (20 poles: 4 groups)


def batched_rhmc_bench(a, rb, F, np, torch, rank, dev, stream):
    """Large batched RHMC: N_f = 2+1 staggered (light am=0.005 with N_f=2, strange am=0.04 with
    N_f=1) on b5_dims (48^4 by default), beta=5.8, degree-20 rational approximations per pole set,
    b5_ps pseudofermions per species (4 + 4 = 8 right-hand sides: the two species have the same
    pole count, so every multi-shift solve runs all 8 together), start exp(i 0.3 H) per link
    (seed 1001), momenta seed 3003, phi seeds 2002/2003, Metropolis uniform seed 4004; synthetic
    data.  One leapfrog trajectory (tau = 1, b5_steps steps; force solves to 1e-8, heatbath and
    action solves to 1e-10) five times: every solve in plain FP64 (18-real links) one
    pseudofermion at a time (the reference's loop), the same with all right-hand sides batched,
    every solve in the mixed batched solver (FP64 12-real multi-shift + FP32 refinement, same
    targets), the same with the FP32 precision schedule, and the mixed batched solver with the
    poles taken B5_POLE_GROUP at a time (only one group's shifted solutions on the device):
    seconds per trajectory, Delta H, acceptance, plaquette, the library's workspace and the
    device memory in use."""
    from rhmc_b200 import rational as R
    from rhmc_b200 import replicas as RP
    torch.cuda.set_stream(stream)
    dims = tuple(int(d) for d in a.b5_dims.split(","))
    nps = a.b5_ps
    ctx = rb.Context(dims, mass=B5_ML, beta=B5_BETA, device=dev.index or 0)
    ctx.set_stream(stream.cuda_stream)
    u0 = F.random_links(dims, seed=RP.replica_seed(1001, rank), kind="near1", eps=0.3)
    ctx.set_gauge(u0)
    P0 = F.random_momenta(dims, seed=RP.replica_seed(3003, rank))
    phis = [F.random_spinor(dims, seed=RP.replica_seed(2002 + s, rank), n=nps) for s in range(2)]
    uniform = float(np.random.Generator(np.random.Philox(RP.replica_seed(4004, rank))).random())
    lmax = ctx.find_max(F.random_spinor(dims, seed=7007))
    species = [(B5_ML, 2), (B5_MS, 1)]
    bounds, approx = [], []
    for m, nf in species:
        lo, hi = m * m, lmax + m * m - B5_ML * B5_ML
        eps = 0.95 * lo / (1.05 * hi)
        bounds.append((lo, hi))
        approx.append([R.rational_power(nf / (8.0 * nps), B5_DEG, eps), R.rational_power(-nf / (4.0 * nps), B5_DEG, eps),
                       R.rational_power(-nf / (4.0 * nps), B5_DEG, eps)])
    out = {"config": {"lattice": list(dims), "beta": B5_BETA,
                      "species": [{"mass": m, "no_flavours": nf, "no_ps": nps} for m, nf in species],
                      "rhs_batched": 2 * nps, "degree": B5_DEG, "eig_bounds": bounds,
                      "start": "exp(i 0.3 H) of a Gaussian algebra element H per link",
                      "integrator": "leapfrog tau=1, %d steps; force solves 1e-8, heatbath/action solves 1e-10"
                                    % a.b5_steps,
                      "approx_max_rel_err": max(c["max_rel_err"] for ap_ in approx for c in ap_),
                      "approximations": approx_report(approx)}}
    have_ms = False
    traj = {}
    # (name, solver mode, link format, single_rhs, pole_group): pole_group G > 0 solves and uses the
    # poles G at a time, holding one group's shifted solutions instead of all of them
    arms = (("fp64_single_rhs", rb.MSOLVE_FP64, rb.LINKS_F64_18, 1, 0),
            ("fp64_batched", rb.MSOLVE_FP64, rb.LINKS_F64_18, 0, 0),
            ("mixed_batched", rb.MSOLVE_MIXED, rb.LINKS_F64_12, 0, 0),
            ("mixed_batched_f32_schedule", rb.MSOLVE_MIXED, rb.LINKS_F32_12, 0, 0),
            ("mixed_batched_pole_groups_%d" % B5_POLE_GROUP, rb.MSOLVE_MIXED, rb.LINKS_F64_12, 0, B5_POLE_GROUP))
    only = [v for v in a.b5_arms.split(",") if v]
    arms = tuple(x for x in arms if not only or x[0] in only)
    for name, mode, fmt, single, pgroup in arms:
        ctx.workspace_release()  # each arm's workspace high-water mark is its own
        ctx.driver_setup(no_flavours=2, no_ps=nps, no_md=a.b5_steps, integrator=rb.INT_LEAPFROG, residue_metro=1e-10,
                         residue_md=1e-8, metro_mode=mode, metro_fmt=fmt, md_mode=mode, md_fmt=fmt, single_rhs=single,
                         pole_group=pgroup)
        if not have_ms:
            ctx.add_species(B5_MS, 1, nps)
            have_ms = True
        for s in range(2):
            ctx.select_species(s)
            for w in range(3):
                ctx.set_approx(w, approx[s][w])
            ctx.set_eig_bounds(*bounds[s])
            ctx.set_phi(phis[s])
        ctx.select_species(0)
        ctx.set_gauge(u0)
        ctx.set_momenta(P0)
        stream.synchronize()
        ctx.driver_solver_stats(0, reset=True)
        n0 = ctx.launch_count()
        t0 = time.perf_counter()
        dS, acc = ctx.update(uniform)
        stream.synchronize()
        dt = time.perf_counter() - t0
        solves = solver_summary(ctx)
        free, total = torch.cuda.mem_get_info(dev)
        traj[name] = {"s_per_trajectory": round(dt, 2), "delta_H": dS, "accepted": acc,
                      "plaquette_after": ctx.plaquette(), "gpu_launches": ctx.launch_count() - n0,
                      "workspace_gb": round(ctx.workspace_bytes() / 1e9, 2),
                      "device_memory_in_use_gb": round((total - free) / 1e9, 2), "solves": solves}
        print("rhmc48: %s trajectory %.1f s, dH %.6g" % (name, dt, dS), file=sys.stderr, flush=True)
    if "fp64_single_rhs" in traj:
        for k in [n for n, *_ in arms if n != "fp64_single_rhs"]:
            traj["speedup_%s_vs_fp64_single_rhs" % k] = round(traj["fp64_single_rhs"]["s_per_trajectory"]
                                                              / traj[k]["s_per_trajectory"], 3)
        traj["delta_H_abs_diff_max"] = max(abs(traj[k]["delta_H"] - traj["fp64_single_rhs"]["delta_H"])
                                           for k, *_ in arms)
    traj["memory_note"] = ("workspace_gb: the library's workspaces after the arm (released before it: solver "
                           "vectors, shifted solutions, driver fields; links, momenta and ipdot come on top); "
                           "device_memory_in_use_gb: the whole device after the arm")
    out["trajectory"] = traj
    ctx.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return out


def rhmc4_bench(a, rb, F, np, torch, rank, dev, stream):
    """Plain RHMC as the reference CPU build runs it: N_f=2 staggered on 4^4, beta=5.5, am=0.1,
    degree-8 approximations of x^(1/4) (heatbath) and x^(-1/2) (force, action) on [1e-3, 64],
    Haar hot start (seed 1001), leapfrog tau=1 with 10 steps, FP64, CG residual 1e-10, 5
    trajectories; momenta (seed 3003+i), pseudofermions (seed 2002+i) and Metropolis uniforms
    (seed 4004) injected identically into the B200 driver and into the reference's own CPU code
    (oracle/_ref/libref_t4.so, the unmodified sources behind the harness; its leapfrog kicks with
    the sign of the wired integrators).  Reports Delta H, acceptance and plaquette per trajectory
    for both, their largest differences, and seconds per trajectory of each."""
    from rhmc_b200 import rational as R
    dims = (4, 4, 4, 4)
    lo, hi = 1e-3, 64.0 / 1.05  # the rescale widens the top by 1.05: range [1e-3, 64]
    eps = 0.95 * lo / 64.0      # ... and the bottom by 0.95 (rationalapprox.cc:147-170)
    ap_ = [R.rational_power(0.25, 8, eps), R.rational_power(-0.5, 8, eps), R.rational_power(-0.5, 8, eps)]
    ntraj = 5
    uni = np.random.Generator(np.random.Philox(4004)).random(ntraj)
    u0 = F.random_links(dims, seed=1001)
    ctx = rb.Context(dims, mass=0.1, beta=5.5, device=dev.index or 0)
    ctx.set_stream(stream.cuda_stream)
    ctx.set_gauge(u0)
    ctx.driver_setup(no_flavours=2, no_ps=1, no_md=10, integrator=rb.INT_LEAPFROG, residue_metro=1e-10, residue_md=1e-10)
    for w in range(3):
        ctx.set_approx(w, ap_[w])
    ctx.set_eig_bounds(lo, hi)
    gpu, t_gpu = [], []
    for i in range(ntraj):
        ctx.set_momenta(F.random_momenta(dims, seed=3003 + i))
        ctx.set_phi(F.random_spinor(dims, seed=2002 + i, n=1))
        stream.synchronize()
        t0 = time.perf_counter()
        de, acc = ctx.update(float(uni[i]))
        stream.synchronize()
        t_gpu.append(time.perf_counter() - t0)
        gpu.append({"delta_H": de, "accepted": acc, "plaquette": list(ctx.plaquette())})
    u_gpu = ctx.get_gauge()
    ctx.close()
    out = {"config": {"lattice": list(dims), "no_flavours": 2, "mass": 0.1, "beta": 5.5, "degree": 8, "range": [lo, 64.0],
                      "integrator": "leapfrog tau=1, 10 steps", "residual": 1e-10, "trajectories": ntraj,
                      "approx_max_rel_err": max(c["max_rel_err"] for c in ap_),
                      "approximations": approx_report([ap_])},
           "b200": gpu, "b200_s_per_trajectory": round(float(np.median(t_gpu)), 5)}
    try:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        ref = oracle.RefLib("t4")
    except Exception as e:  # the reference harness is built where the reference sources are
        out["reference"] = {"unavailable": str(e)[:200]}
        return out
    ref.set_links(u0)
    for w in range(3):
        ref.set_approx(w, ap_[w])
    ref.set_minmax(lo, hi)
    cpu, t_cpu = [], []
    for i in range(ntraj):
        ref.set_momenta(F.random_momenta(dims, seed=3003 + i))
        ref.set_phi(F.random_spinor(dims, seed=2002 + i, n=1))
        t0 = time.perf_counter()
        de, acc = ref.trajectory(3, float(uni[i]))
        t_cpu.append(time.perf_counter() - t0)
        cpu.append({"delta_H": de, "accepted": acc, "plaquette": list(ref.plaquette())})
    out["reference"] = cpu
    out["reference_s_per_trajectory"] = round(float(np.median(t_cpu)), 5)
    out["reference_cores"] = 1
    out["max_abs_diff"] = {
        "delta_H": max(abs(g["delta_H"] - c["delta_H"]) for g, c in zip(gpu, cpu)),
        "plaquette": max(abs(x - y) for g, c in zip(gpu, cpu) for x, y in zip(g["plaquette"], c["plaquette"])),
        "acceptance_mismatches": sum(g["accepted"] != c["accepted"] for g, c in zip(gpu, cpu)),
        "links_after": float(np.abs(u_gpu - ref.get_links()).max())}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--no-msolve", action="store_true")
    ap.add_argument("--workload", default="dslash", choices=["dslash", "nf2p1", "msolve", "rhmc4", "rhmc48"],
                    help="dslash: the headline line (Dslash + multi-shift CG); nf2p1: N_f=2+1 forces, "
                         "finite-difference check and trajectories; msolve: the multi-shift CG comparison alone")
    ap.add_argument("--ms-relative", action="store_true", help="msolve workload: residual relative to |b|")
    ap.add_argument("--ms-variants", default="", help="msolve workload: comma-separated subset of the variants")
    ap.add_argument("--ms-nrhs", type=int, default=4)
    ap.add_argument("--ms-nshift", type=int, default=16)
    ap.add_argument("--ms-mass", type=float, default=0.01)
    ap.add_argument("--ms-no-warmup", action="store_true", help="msolve workload: time the first solve")
    ap.add_argument("--fd-links", type=int, default=16)
    ap.add_argument("--fd-dirs", type=int, default=8)
    ap.add_argument("--nf-steps", type=int, default=20)
    ap.add_argument("--nf-start", default="near1", choices=["haar", "near1"])
    ap.add_argument("--ms-dims", default="24,24,24,32", help="lattice of the multi-shift CG comparison")
    ap.add_argument("--b5-dims", default="48,48,48,48", help="rhmc48 workload: lattice")
    ap.add_argument("--b5-steps", type=int, default=10, help="rhmc48 workload: leapfrog steps per trajectory")
    ap.add_argument("--b5-ps", type=int, default=4, help="rhmc48 workload: pseudofermions per species")
    ap.add_argument("--b5-arms", default="", help="rhmc48 workload: comma-separated subset of the arms")
    a = ap.parse_args()
    a.warmup = max(3, a.warmup)
    if a.impl == "reference":
        return run_reference_arm(a)

    import numpy as np
    import torch
    import rhmc_b200 as rb
    from rhmc_b200 import fields as F
    from rhmc_b200 import replicas as RP

    global DIMS, MS_DIMS
    DIMS = tuple(int(v) for v in a.dims.split(","))
    MS_DIMS = tuple(int(v) for v in a.ms_dims.split(","))
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

    if a.workload == "rhmc4":
        stream = torch.cuda.Stream(device=dev)
        res = rhmc4_bench(a, rb, F, np, torch, rank, dev, stream)
        if rank == 0:
            print(json.dumps({"workload": "rhmc4", "n_gpus": world, "data": "synthetic", **res}))
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    if a.workload == "msolve":
        stream = torch.cuda.Stream(device=dev)
        only = [v for v in a.ms_variants.split(",") if v]
        res = msolve_bench(rb, F, np, torch, rank, dev, stream, relative=a.ms_relative, only=only, nrhs=a.ms_nrhs,
                           nshift=a.ms_nshift, mass=a.ms_mass, warmup=not a.ms_no_warmup,
                           cpu=rank == 0 and world == 1 and not a.no_cpu_baseline)

        if rank == 0:
            print(json.dumps({"workload": "msolve", "n_gpus": world, "data": "synthetic", **res}))
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    if a.workload == "rhmc48":
        stream = torch.cuda.Stream(device=dev)
        res = batched_rhmc_bench(a, rb, F, np, torch, rank, dev, stream)
        if rank == 0:
            print(json.dumps({"workload": "rhmc48", "n_gpus": world, "data": "synthetic", **res}))
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    if a.workload == "nf2p1":
        stream = torch.cuda.Stream(device=dev)
        res = nf2p1_bench(a, rb, F, np, torch, rank, dev, stream)
        if rank == 0:
            print(json.dumps({"workload": "nf2p1", "n_gpus": world, "data": "synthetic", **res}))
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

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
    for fmt in (rb.LINKS_F64_18, rb.LINKS_F64_12, rb.LINKS_F32_18, rb.LINKS_F32_12, rb.LINKS_F16_12):
        f64 = fmt in (rb.LINKS_F64_18, rb.LINKS_F64_12)
        dt = torch.float64 if f64 else torch.float32
        xe = torch.zeros(rb.spinor_floats(fmt, Vh), dtype=dt, device=dev)
        xo = torch.zeros(rb.spinor_floats(fmt, Vh), dtype=dt, device=dev)
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
            ctx.dslash_repeat(fmt, xe, xo, 1, a.steps * PAIRS)  # steps x PAIRS x (D_oe, D_eo) issued from C
            ev1.record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        barrier()
        launches = ctx.launch_count() - n0
        cl = clocks.stop() if clocks else None
        total_ms = ev0.elapsed_time(ev1)
        per_launch = [total_ms / (2 * PAIRS * a.steps)]
        total_ms = max_over_ranks(total_ms)
        by_launch = half_dslash_bytes(fmt, Vh)
        avg_launch_ms = sum(per_launch) / len(per_launch)
        results[fmt] = dict(total_ms=total_ms, avg_launch_ms=avg_launch_ms, launches=launches, clocks=cl,
                            gbs=world * 2 * PAIRS * by_launch * a.steps / (total_ms * 1e-3) / 1e9,
                            achieved=by_launch / (avg_launch_ms * 1e-3) / 1e9,
                            gflops=world * 2 * PAIRS * FLOPS_PER_SITE * Vh * a.steps / (total_ms * 1e-3) / 1e9)
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

    ms = ms32 = None
    if not a.no_msolve:
        cpu_ms = rank == 0 and world == 1 and not a.no_cpu_baseline
        try:
            ms = msolve_bench(rb, F, np, torch, rank, dev, stream, cpu=cpu_ms)
        except Exception as e:  # reported in the JSON line, the Dslash numbers stand
            ms = {"error": str(e)[:300]}
        try:
            ms32 = msolve_bench(rb, F, np, torch, rank, dev, stream, dims=(32, 32, 32, 32), relative=True, cpu=cpu_ms)
        except Exception as e:
            ms32 = {"error": str(e)[:300]}

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
                       "half_dslash_per_step": 2 * PAIRS,
                       "l2": "inputs larger than L2 (links 604 MB)",
                       "launch_shapes": tuned_shapes(rb, Vh)},
            "roofline": {"bound": "hbm", "achieved": round(r["achieved"], 1), "peak": peak, "unit": "GB/s",
                         "frac": round(r["achieved"] / peak, 4), "traffic": round(DSLASH_F64_18_DRAM_PER_SITE * Vh),
                         "traffic_note": "ncu dram read+write of this kernel at 24^4 (1244.8 B per output site), "
                                         "scaled to this launch by Vh",
                         "peak_kind": peak_kind, "kernel": "dslash_kernel<L64_18,1>",
                         "bytes_per_launch": half_dslash_bytes(0, Vh)},
            "gflops": round(r["gflops"], 1),
            "variants": {rb.FMT_NAMES[f]: {"gbs": round(v["gbs"], 1), "achieved": round(v["achieved"], 1),
                                            "frac": round(v["achieved"] / peak, 4),
                                            "us_per_half_dslash": round(1000 * v["avg_launch_ms"], 2),
                                            "sites_per_s": round(2 * PAIRS * Vh * a.steps / (v["total_ms"] * 1e-3) * world, 1)}
                         for f, v in results.items()},
            "e2e": {"value": round(e2e_gbs, 2), "unit": "GB/s", "h2d_bytes_per_step": 2 * 48 * Vh,
                    "d2h_bytes_per_step": 2 * 48 * Vh, "api": "rhmc_dslash_host (host spinors, pinned)"},
            "msolve": ms,
            "msolve_32": ms32,
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
