"""Benchmark of the pressure-projection step (computeSource -> solveFPS ->
makeVelocityDivFree -> computeContinuityError) on the 512x384x256 channel.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one projection of the whole channel.  ``value`` is measured with all
inputs resident in HBM (device entry point, out-of-place velocity so every step
projects the same u*); ``e2e`` goes through the host entry point with pinned
host buffers, host<->device copies inside the timed region.  Inputs (~0.4 GB
per field) are larger than L2, so no flush is needed between steps.

With N > 1 (torchrun, one rank per GPU) every rank projects its own,
independently seeded channel: the ensemble shards as independent channels per
GPU with no data-path collective (weak scaling); the time is the max over ranks.

``--impl reference`` times the CPU restatement of the reference path (the
oracle; the Fortran reference cannot be built here) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "projection solves/s and Gcell/s, mixed vs FP64 on 1 B200 at rel. residual 1e-10"
UNIT = "Gcell/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--mg", action="store_true", help="also time the MG_MODE projection (default for c5)")
    ap.add_argument("--no-mg", action="store_true", help="skip the MG_MODE leg")
    ap.add_argument("--no-vof", action="store_true", help="skip the material-properties leg")
    ap.add_argument("--no-momentum", action="store_true", help="skip the momentum-predictor leg")
    ap.add_argument("--no-st", action="store_true", help="skip the surface-tension leg")
    ap.add_argument("--slabs", action="store_true",
                    help="one channel split over the ranks (z/kx slabs, two all-to-alls) instead of replicas")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the legs on the other workloads (mixed 1024x512x512, MG 256x256x128, ensemble)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML (read-only queries)
    every few milliseconds while the timed region runs."""

    def __init__(self, index: int, period_s: float = 0.005):
        self.index = index
        self.period = period_s
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.ok = False
        self._stop = threading.Event()

    def start(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
            self.names = {nv.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                          nv.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                          nv.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                          nv.nvmlClocksEventReasonSwPowerCap: "sw_power_cap",
                          nv.nvmlClocksEventReasonHwPowerBrakeSlowdown: "hw_power_brake_slowdown"}
            self.ok = True
        except Exception:
            self.ok = False
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for b, n in self.names.items():
                    if bits & b:
                        self.reasons.add(n)
            except Exception:
                pass
            time.sleep(self.period)

    def stop(self):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"], "samples": 0}
        self._stop.set()
        self.t.join(timeout=2)
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def alg_bytes(nx, ny, nz):
    """Compulsory HBM bytes of the stage sequence (FP64, no surface tension)."""
    N = nx * ny * nz
    K = (nx // 2 + 1) * ny * nz
    return {
        "recip": 16.0 * N,
        "rhs_fftx": 48.0 * N + 16.0 * K,
        "fftz_fwd": 32.0 * K,
        "tridiag": 32.0 * K,
        "fftz_inv": 32.0 * K,
        "fftx_inv": 16.0 * K + 8.0 * N,
        "correct": 80.0 * N,
        "div": 24.0 * N,
        "b_alg": 128.0 * N + 64.0 * K,
    }


def config_dict(spec, cells, world):
    """The workload's config, identical in both arms of the benchmark."""
    return {"workload": spec.name, "cells": cells, "precision": "fp64",
            "parallelism": f"independent channel per GPU x{world}",
            "l2": "inputs larger than L2 (0.4 GB per field)"}


def host_inputs(spec, seed, device):
    """The benchmark inputs as host numpy arrays (synthesised on `device`)."""
    from tbfsolver_b200 import synth

    inp = synth.make_inputs(spec, seed=seed, device=device)
    np_ = lambda f: f.a.detach().cpu().numpy().copy()  # noqa: E731
    return inp, [np_(f) for f in (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho, inp.psi_n, inp.psi_nm1)]


def cpu_projection_timer(grid, arrays, dt, alpha, rho0, min_seconds=10.0, min_reps=1, nthreads=0):
    """Time the C/OpenMP oracle projection on this host.  u* is restored from a
    pristine copy before every repetition, outside the timed interval.
    Returns (seconds per projection, repetitions, threads, psi, [ux, uy, uz],
    max|div u|) with the oracle's pressure, projected velocity and continuity
    error."""
    import numpy as np

    from oracle import cref

    ux, uy, uz, rho, pn, pnm1 = arrays
    work = [ux.copy(), uy.copy(), uz.copy()]
    psi = np.zeros_like(pn)
    thr = nthreads or cref.max_threads()
    cref.projection(grid, *work, rho, pn, pnm1, dt, alpha, rho0, psi, thr)  # warm-up
    reps, total = 0, 0.0
    while reps < min_reps or total < min_seconds:
        for w, a in zip(work, (ux, uy, uz)):
            w[...] = a
        t0 = time.perf_counter()
        md = cref.projection(grid, *work, rho, pn, pnm1, dt, alpha, rho0, psi, thr)
        total += time.perf_counter() - t0
        reps += 1
    return total / reps, reps, thr, psi, work, md


def run_reference(args, world, rank):
    """The CPU restatement of the reference path on all host cores (rank 0 only)."""
    if rank != 0:
        return
    import torch

    from tbfsolver_b200 import synth

    spec = synth.CONFIGS[args.config]
    dev = "cuda" if torch.cuda.is_available() else "cpu"  # input synthesis only
    inp, arrays = host_inputs(spec, args.seed, dev)
    g = inp.grid
    from oracle import cref

    import numpy as np

    thr = cref.max_threads()
    ux, uy, uz, rho, pn, pnm1 = arrays
    # calls 1 and 2 of the chain (untimed), as the GPU arm does, then time call 3
    for _ in range(2):
        w = [a.copy() for a in (ux, uy, uz)]
        psi = np.zeros_like(pn)
        cref.projection(g, *w, rho, pn, pnm1, inp.dt, inp.alpha, inp.rho0, psi, thr)
        pnm1, pn = pn, psi
    work = [a.copy() for a in (ux, uy, uz)]
    psi = np.zeros_like(pn)
    secs = []
    for it in range(args.warmup + args.steps):
        for wk, a in zip(work, (ux, uy, uz)):
            wk[...] = a
        t0 = time.perf_counter()
        cref.projection(g, *work, rho, pn, pnm1, inp.dt, inp.alpha, inp.rho0, psi, thr)
        if it >= args.warmup:
            secs.append(time.perf_counter() - t0)
    sec = sum(secs) / len(secs)
    gcell = g.ncells / sec / 1e9
    sample = f"C/OpenMP oracle, full {spec.name} projection per step, {thr} threads"
    line = {"metric": METRIC, "value": gcell, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(spec, g.ncells, args.gpus),
            "impl": "reference",
            "cpu_baseline": {"value": gcell, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample},
            "e2e": {"value": gcell, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def ensemble_measure(args, world, rank, local, precisions=("fp64",)):
    """Config 4: 64 channels of the minimal box with seeded sizes, one
    tbfp_ensemble call per step -- in the form the autotuner picks, and in each
    form forced: the multi-stream CUDA graph and the one persistent launch
    (mixed members run in the graph with their refinement loops on the device)
    -- against the same 64 projections made one after another through the
    single-channel FP64 entry point.  Returns a dict on rank 0, else None."""
    import torch
    import torch.distributed as dist

    from tbfsolver_b200 import synth
    from tbfsolver_b200.fields import Field, VField
    from tbfsolver_b200.solver import Ensemble, PoissonEqn

    torch.cuda.set_device(local)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    specs = synth.ensemble_specs(64, seed=args.seed + rank)
    inps = [synth.make_inputs(sp, seed=args.seed + 1000 * rank + c, device="cuda") for c, sp in enumerate(specs)]
    ncells = sum(sp.ncells for sp in specs)
    dt, alpha, rho0 = inps[0].dt, inps[0].alpha, min(specs[0].rhol, specs[0].rhog)
    seq = [PoissonEqn(i.grid, sp.rhol, sp.rhog) for i, sp in zip(inps, specs)]
    members = []
    for inp, eqn in zip(inps, seq):  # calls 1 and 2 of the chain build psi^n, psi^{n-1}
        pn, pnm1 = inp.psi_n, inp.psi_nm1
        uo = VField(*[Field.like(f, f.a.clone()) for f in inp.u.components()])
        for _ in range(2):
            psi = Field.like(pn, torch.zeros_like(pn.a))
            eqn.projection(psi, pn, pnm1, inp.rho, inp.u, dt, alpha, u_out=uo, want_stats=False)
            pnm1, pn = pn, psi
        members.append((Field.like(pn, torch.zeros_like(pn.a)), pn, pnm1, inp.rho, inp.u, uo))
    torch.cuda.synchronize()

    def timed(fn, steps):
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        if world > 1:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    res = {}
    clocks = None
    # FP64: the form the autotuner picks (measured on the first call), then each form forced;
    # mixed members run in the graph form (device-side refinement loops)
    runs = [("fp64", "fp64", "auto"), ("fp64_graph", "fp64", "graph"), ("fp64_persistent", "fp64", "persistent")]
    runs = [r for r in runs if r[1] in precisions] + [("mixed", "mixed", "auto")] * ("mixed" in precisions)
    for key, prec, mode in runs:
        # one stream per member: 2.96 ms against 3.27 ms with a pool of 8 (graph form, B200)
        ens = Ensemble([i.grid for i in inps], nstreams=len(inps), precision=prec, tol=1e-10, max_iter=8,
                       mode=mode)
        clk = ClockSampler(local)
        clk.start()
        ms = timed(lambda: ens.projection(members, dt, alpha, rho0, want_stats=False), args.steps)
        c = clk.stop()
        clocks = clocks or c
        st = ens.projection(members, dt, alpha, rho0)
        form, param, tuned = ens.mode()
        ens.close()
        res[key] = {"value": world * ncells / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
                    "solves_per_s": world * 64e3 / ms, "max_div": max(x.max_div for x in st),
                    "max_sweeps": max(x.iterations for x in st), "form": form, "form_param": param}
        if mode == "auto" and prec == "fp64":
            res[key]["tuned_ms"] = {"graph": tuned[0], "persistent_1_block_per_sm": tuned[1],
                                    "persistent_2_blocks_per_sm": tuned[2]}

    def sequential():
        for (psi, pn, pnm1, rho, u, uo), eqn in zip(members, seq):
            eqn.projection(psi, pn, pnm1, rho, u, dt, alpha, u_out=uo, want_stats=False)

    ms_seq = timed(sequential, max(1, args.steps // 4))
    for eqn in seq:
        eqn.close()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return None
    seqd = {"value": world * ncells / (ms_seq * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms_seq,
            "solves_per_s": world * 64e3 / ms_seq,
            "note": "the same 64 projections one after another, single-channel FP64 entry point"}
    for prec in res:
        res[prec]["vs_sequential"] = ms_seq / res[prec]["ms_per_step"]
    return {"workload": f"c4-ensemble-64ch-{ncells}cells", "channels": 64, "cells": ncells, "clocks": clocks,
            "sequential": seqd, **res}


def run_ensemble(args, world, rank, local):
    """--config c4: the ensemble as the headline line (FP64 members)."""
    r = ensemble_measure(args, world, rank, local, precisions=("fp64", "mixed"))
    if r is None:
        return
    f = r["fp64"]
    line = {
        "metric": METRIC, "value": f["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": f["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": r["workload"], "channels": 64, "cells": r["cells"],
                   "precision": "fp64", "parallelism": f"64 independent channels per GPU x{world}",
                   "l2": "inputs larger than L2 (6 GB per step)", "timing": "events around synchronous calls"},
        "max_div": f["max_div"], "form": f["form"], "form_param": f["form_param"],
        "tuned_ms": f.get("tuned_ms"), "fp64_graph": r.get("fp64_graph"),
        "fp64_persistent": r.get("fp64_persistent"), "mixed": r["mixed"], "sequential": r["sequential"],
        "e2e": None, "gpu_launches": None, "clocks": r["clocks"], "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def _rel(a, b):
    """max|a - b| / max|b| over torch tensors or numpy arrays."""
    import torch

    a = torch.as_tensor(a, device="cpu") if not isinstance(a, torch.Tensor) else a.detach().cpu()
    b = torch.as_tensor(b, device="cpu") if not isinstance(b, torch.Tensor) else b.detach().cpu()
    den = float(b.abs().max())
    return float((a - b).abs().max()) / (den if den > 0 else 1.0)


def parity_report(opsi, ou, omd, psi64, u64, u_fields, md):
    """The GPU FP64 projection against the C restatement of the reference path
    (epsilon pivot for the singular (0,0) system) on the benchmarked inputs:
    psi over the whole array (ghosts included), u over the interior faces."""
    from tbfsolver_b200.fields import Field

    u_err = max(_rel(Field.like(f, g).interior(), Field.like(f, o).interior())
                for f, g, o in zip(u_fields.components(), u64, ou))
    return {"oracle": "C restatement of the reference projection (oracle/tbfp_oracle.c), epsilon pivot",
            "psi_rel_linf": _rel(psi64, opsi), "u_rel_linf": u_err, "max_div_abs_diff": abs(md - omd),
            "tolerance": 1e-12}


def mixed_bytes(N, K, n):
    """Compulsory bytes of a mixed projection with n FP32 solves and n FP64
    residual passes: 1/rho 16N, RHS 56N, first solve 16N + 64K (FP32 spectrum),
    each residual pass 16N + 8K, each further sweep 16N + 56K (psi += c2r),
    correction 80N."""
    return (168 + 16 * n + 16 * (n - 1)) * N + (64 + 8 * n + 56 * (n - 1)) * K


def mixed_report(g, mms, mst, psi, u_fields, psi64, u64):
    """The mixed leg: throughput, the loop's outcome and the error against the
    FP64 GPU path on the same input (psi L2 and L-infinity over the interior,
    u L-infinity), with the fraction of its own byte model."""
    import torch

    pk, _ = peaks()
    N, K = g.ncells, (g.nx // 2 + 1) * g.ny * g.nz
    pi = lambda t: t[1:-1, 1:-1, 1:-1]  # noqa: E731  (psi has halo 1)
    d = pi(psi.a) - pi(psi64)
    l2 = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(pi(psi64)))
    from tbfsolver_b200.fields import Field

    u_err = max(_rel(Field.like(f, f.a).interior(), Field.like(f, w).interior())
                for f, w in zip(u_fields.components(), u64))
    mb = mixed_bytes(N, K, max(1, mst.iterations))
    return {"value": N / (mms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": mms, "solves_per_s": 1e3 / mms,
            "sweeps": mst.iterations, "rel_residual": mst.rel_residual, "max_div": mst.max_div,
            "psi_rel_l2_vs_fp64": l2, "psi_rel_linf_vs_fp64": _rel(pi(psi.a), pi(psi64)),
            "u_rel_linf_vs_fp64": u_err, "alg_bytes_model": mb,
            "frac_of_model": mb / (mms * 1e-3) / 1e9 / pk, "vs_fp64": None}


def _stream_timer(stream, fn, steps, warmup):
    """Mean device time of fn() per call, CUDA events on the library's stream."""
    import torch

    for _ in range(max(3, warmup)):
        fn()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    stream.synchronize()
    return e0.elapsed_time(e1) / steps


def _chain(eqn, inp, u_out, new_psi, calls=2):
    """Calls 1 and 2 of a projection chain: returns (psi^n, psi^{n-1}) for call 3."""
    pn, pnm1 = inp.psi_n, inp.psi_nm1
    for _ in range(calls):
        psi = new_psi()
        eqn.projection(psi, pn, pnm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out, want_stats=False)
        pnm1, pn = pn, psi
    return pn, pnm1


def leg_mixed_large(args, name="c3"):
    """The mixed-precision projection on the 1024x512x512 workload (the size
    its metric is written for) against the FP64 path on the same input."""
    import torch

    from tbfsolver_b200 import synth
    from tbfsolver_b200.fields import Field, VField
    from tbfsolver_b200.solver import PoissonEqn

    spec = synth.CONFIGS[name]
    inp = synth.make_inputs(spec, seed=args.seed, device="cuda")
    g = inp.grid
    stream = torch.cuda.Stream()
    new = lambda: Field("cl", 1, g.nx, g.ny, g.nz, torch.zeros_like(inp.psi_n.a))  # noqa: E731
    u_out = VField(*[Field.like(f, torch.empty_like(f.a)) for f in inp.u.components()])
    out = {"workload": spec.name}
    f64 = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream, asynchronous=True)
    try:
        with torch.cuda.stream(stream):
            pn, pnm1 = _chain(f64, inp, u_out, new)
        psi = new()
        step = lambda e: e.projection(psi, pn, pnm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out,  # noqa: E731
                                      want_stats=False)
        ms64 = _stream_timer(stream, lambda: step(f64), args.steps, args.warmup)
        st64 = f64.projection(psi, pn, pnm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out)
        psi64, u64 = psi.a.clone(), [f.a.clone() for f in u_out.components()]
    finally:
        f64.close()
    mx = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream, asynchronous=True, precision="mixed",
                    tol=1e-10, max_iter=8)
    try:
        mms = _stream_timer(stream, lambda: step(mx), args.steps, args.warmup)
        mst = mx.projection(psi, pn, pnm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out)
        out.update(mixed_report(g, mms, mst, psi, u_out, psi64, u64))
    finally:
        mx.close()
    out["fp64_ms_per_step"] = ms64
    out["fp64_value"] = g.ncells / (ms64 * 1e-3) / 1e9
    out["fp64_max_div"] = st64.max_div
    out["vs_fp64"] = ms64 / mms
    return out


def leg_mg(args, name="c5"):
    """MG_MODE (FP64 PCG + FP32 V-cycles, 6 levels, 2+2 sweeps, tolPCG 1e-10,
    tolMG 0.4) on the 256x256x128 workload, compared with the split FFT
    projection (call 3 of its chain) on the same input: the pressures after
    removing their means, and max|div u| of both."""
    import torch

    from tbfsolver_b200 import synth
    from tbfsolver_b200.fields import Field, VField
    from tbfsolver_b200.solver import PCG, PoissonEqn

    spec = synth.CONFIGS[name]
    inp = synth.make_inputs(spec, seed=args.seed, device="cuda")
    g = inp.grid
    stream = torch.cuda.Stream()
    new = lambda: Field("cl", 1, g.nx, g.ny, g.nz, torch.zeros_like(inp.psi_n.a))  # noqa: E731
    u_out = VField(*[Field.like(f, torch.empty_like(f.a)) for f in inp.u.components()])
    fast = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream)
    try:
        with torch.cuda.stream(stream):
            pn, pnm1 = _chain(fast, inp, u_out, new)
        pf = new()
        fst = fast.projection(pf, pn, pnm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out)
    finally:
        fast.close()
    pcg = PCG(g, n_levels=6, n_pre=2, n_post=2, tol_mg=0.4, tol_pcg=1e-10, stream=stream.cuda_stream)
    try:
        pm = new()

        def step():
            pm.a.zero_()
            return pcg.projection(pm, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out)

        nmg = max(1, min(args.steps, 5))
        with torch.cuda.stream(stream):
            gms = _stream_timer(stream, step, nmg, 1)
            mst = step()
    finally:
        pcg.close()
    inner = lambda t: t[1:-1, 1:-1, 1:-1]  # noqa: E731
    a, b = inner(pm.a), inner(pf.a)
    return {"workload": spec.name, "value": g.ncells / (gms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": gms,
            "steps": nmg, "pcg_iterations": mst.iterations, "v_cycles": int(mst.ms_stage[0]),
            "rel_residual": mst.rel_residual, "max_div": mst.max_div, "fast_max_div": fst.max_div,
            "psi_rel_linf_vs_fast": _rel(a - a.mean(), b - b.mean()),
            "note": "variable-coefficient PCG from a zero guess vs the split FFT projection (call 3 of its chain) "
                    "on the same input; the two methods solve different pressure equations"}


def leg_ensemble(args):
    """The 64-channel ensemble (FP64 and mixed members) against 64 sequential
    single-channel FP64 projections."""
    return ensemble_measure(args, 1, 0, torch_local(), precisions=("fp64", "mixed"))


def torch_local():
    import torch

    return torch.cuda.current_device()


def extra_legs(args):
    legs = {}
    for key, fn in (("mixed_c3", leg_mixed_large), ("mg", leg_mg), ("ensemble", leg_ensemble)):
        try:
            legs[key] = fn(args)
        except Exception as e:  # a failed leg is reported, not hidden
            legs[key] = {"error": f"{type(e).__name__}: {e}"}
        import gc

        import torch

        gc.collect()
        torch.cuda.empty_cache()
    return legs


def run_slabs(args, world, rank, local):
    """One channel split over the ranks (the reference's pencil decomposition
    with py = 1): z slabs in physical space, kx slabs in spectral space, two
    all-to-alls per solve (library packing, zero-copy send / receive buffers)
    and the z ghost planes of psi.  A step: split RHS, solveFPS, correction,
    every rank on its slab.  Strong scaling: the channel is the same at every
    N.  The inputs' ghost planes come from the whole-channel synthesis on each
    rank, so only the exchanges of a step run inside the timed region."""
    import torch
    import torch.distributed as dist

    from tbfsolver_b200 import synth
    from tbfsolver_b200.dist import SlabChannel
    from tbfsolver_b200.fields import Field, VField
    from tbfsolver_b200.solver import PoissonEqn, make_velocity_div_free

    torch.cuda.set_device(local)
    group = None
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    spec = synth.CONFIGS[args.config]
    inp = synth.make_inputs(spec, seed=args.seed, device="cuda")
    g = inp.grid
    chan = SlabChannel(g, world, rank, device=local)
    k0, nzl = chan.s.k0, chan.s.nz_loc

    def zslice(f):
        extra = 1 if f.kind == "sz" else 0
        return Field(f.kind, f.hd, f.nx, f.ny, nzl, f.a[k0:k0 + nzl + extra + 2 * f.hd].clone())

    u = VField(*[zslice(f) for f in inp.u.components()])
    rho, pn, pnm1 = zslice(inp.rho), zslice(inp.psi_n), zslice(inp.psi_nm1)
    del inp
    torch.cuda.empty_cache()
    s_loc = Field("cl", 1, g.nx, g.ny, nzl, torch.zeros_like(pn.a))
    psi = Field("cl", 1, g.nx, g.ny, nzl, torch.zeros_like(pn.a))

    class _Eqn:  # the slab handle behind PoissonEqn's RHS and correction wrappers
        solver = chan
        rho0 = min(spec.rhol, spec.rhog)

    e = _Eqn()

    def step():
        PoissonEqn.compute_source(e, s_loc, pn, pnm1, rho, u, spec.dt, 1.0)
        chan.solve_fps(psi, s_loc, group)
        make_velocity_div_free(e, u, psi, pn, pnm1, rho, spec.dt, 1.0)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local)
    clk.start()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    chan.close()
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": g.ncells / (ms * 1e-3) / 1e9, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": spec.name, "cells": g.ncells, "precision": "fp64",
                   "parallelism": f"one channel in z/kx slabs x{world} (two all-to-alls per solve)",
                   "l2": "inputs larger than L2"},
        "e2e": None, "gpu_launches": 9 * args.steps, "clocks": clocks, "cpu_baseline": None,
        "note": "split RHS + solveFPS (forward x, all-to-all, z/y/z, all-to-all, inverse x, psi ghost planes) + "
                "correction per rank; synchronous library calls, events on the default stream",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.config == "c4":
        run_ensemble(args, world, rank, local)
        return
    if args.slabs:
        run_slabs(args, world, rank, local)
        return
    line = main_line(args, world, rank, local)
    if line is None:
        return
    if world == 1 and args.config == "c2" and not args.no_extra:
        import gc

        import torch

        gc.collect()
        torch.cuda.empty_cache()
        line.update(extra_legs(args))
    print(json.dumps(line), flush=True)


def main_line(args, world, rank, local):
    """The headline: one FP64 projection per step on the configured workload,
    with its stage times, the end-to-end host call, the accuracy checks and the
    other legs of the same channel.  Returns the JSON line on rank 0."""
    import torch
    import torch.distributed as dist

    from tbfsolver_b200 import synth
    from tbfsolver_b200._native import STAGES
    from tbfsolver_b200.fields import Field, VField
    from tbfsolver_b200.solver import PoissonEqn

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    spec = synth.CONFIGS[args.config]
    inp = synth.make_inputs(spec, seed=args.seed + rank, device="cuda")
    g = inp.grid
    stream = torch.cuda.Stream()
    eqn = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream, asynchronous=True, timing=True)
    dt, alpha = inp.dt, inp.alpha
    new = lambda: Field("cl", 1, g.nx, g.ny, g.nz, torch.zeros_like(inp.psi_n.a))  # noqa: E731
    u_in = inp.u
    u_out = VField(*[Field.like(f, torch.empty_like(f.a)) for f in u_in.components()])
    # calls 1 and 2 of the chain: builds psi^n, psi^{n-1} so the split term is active
    pn, pnm1 = inp.psi_n, inp.psi_nm1
    with torch.cuda.stream(stream):
        for _ in range(2):
            psi = new()
            eqn.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out, want_stats=False)
            pnm1, pn = pn, psi
    stream.synchronize()
    psi = new()

    def step():
        eqn.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out, want_stats=False)

    for _ in range(max(3, args.warmup)):
        step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    # per-stage device times (CUDA events recorded by the library between its launches)
    nstat = 5
    acc = [0.0] * 8
    last = None
    for _ in range(nstat):
        last = eqn.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out)
        for i in range(8):
            acc[i] += last.ms_stage[i] / nstat
    # the out-of-place path has no separate continuity stage (its two events are adjacent)
    stage_ms = {k: v for k, v in zip(STAGES, acc) if v > 0.01}
    # the FP64 result of this projection: the parity block and the mixed leg's errors
    psi64 = psi.a.clone()
    u64 = [f.a.clone() for f in u_out.components()]

    # accuracy of the FP64 path: ||s - L psi||/||s|| of the same projection (not timed)
    chk = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream, residual=True)
    chk_st = chk.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out)
    fp64_rel = chk_st.rel_residual
    chk.close()

    # mixed precision leg: FP32 spectrum + FP64 defect correction to 1e-10
    mixed = None
    if not args.no_mixed:
        mx = PoissonEqn(g, spec.rhol, spec.rhog, stream=stream.cuda_stream, precision="mixed", tol=1e-10,
                        max_iter=8)
        for _ in range(max(3, args.warmup)):
            mst = mx.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out)
        stream.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(args.steps):
            mx.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out, want_stats=False)
        m1.record(stream)
        stream.synchronize()
        mms = m0.elapsed_time(m1) / args.steps
        mst = mx.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, u_out=u_out)
        mixed = mixed_report(g, mms, mst, psi, u_out, psi64, u64)
        mx.close()

    # MG_MODE leg (config 5: FP64 PCG + FP32 V-cycles, 6 levels, 2+2 sweeps,
    # tolPCG 1e-10, tolMG 0.4) on the same input; psi starts from zero every step
    mgres = None
    if (args.mg or args.config == "c5") and not args.no_mg:
        from tbfsolver_b200.solver import PCG
        pcg = PCG(g, n_levels=6, n_pre=2, n_post=2, tol_mg=0.4, tol_pcg=1e-10, stream=stream.cuda_stream)
        mpsi = new()
        for _ in range(max(3, args.warmup)):
            mpsi.a.zero_()
            mst = pcg.projection(mpsi, inp.rho, u_in, dt, alpha, u_out=u_out)
        stream.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nmg = max(1, min(args.steps, 5))
        with torch.cuda.stream(stream):
            g0.record(stream)
            for _ in range(nmg):
                mpsi.a.zero_()
                mst = pcg.projection(mpsi, inp.rho, u_in, dt, alpha, u_out=u_out)
            g1.record(stream)
        stream.synchronize()
        gms = g0.elapsed_time(g1) / nmg
        mgres = {"value": g.ncells / (gms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": gms, "steps": nmg,
                 "pcg_iterations": mst.iterations, "v_cycles": int(mst.ms_stage[0]), "rel_residual": mst.rel_residual,
                 "max_div": mst.max_div, "fast_max_div": last.max_div,
                 "note": "variable-coefficient PCG (MG_MODE) on the FAST leg's input; max_div of both paths"}
        pcg.close()

    # material properties (updateMaterialProps + smoothVF) producing rho for the
    # projection, on the same channel; compulsory bytes: read c, write cs, rho, mu
    vofres = None
    if not args.no_vof:
        from tbfsolver_b200.solver import VOF
        vof = VOF(eqn.solver, rhol=spec.rhol, rhog=spec.rhog, mul=1e-3, mug=1e-3 * spec.rhog)
        vc = Field.like(inp.rho, inp.cs.a.clone())
        vcs, vrho, vmu = (Field.like(inp.rho, torch.empty_like(inp.rho.a)) for _ in range(3))
        for _ in range(max(3, args.warmup)):
            vof.update_material_props(vc, vcs, vrho, vmu)
        stream.synchronize()
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            v0.record(stream)
            for _ in range(args.steps):
                vof.update_material_props(vc, vcs, vrho, vmu)
            v1.record(stream)
        stream.synchronize()
        vms = v0.elapsed_time(v1) / args.steps
        vbytes = 32.0 * inp.rho.a.numel()
        pk0, _ = peaks()
        vofres = {"value": g.ncells / (vms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": vms,
                  "alg_bytes": vbytes, "alg_GBps": vbytes / (vms * 1e-3) / 1e9,
                  "frac": vbytes / (vms * 1e-3) / 1e9 / pk0, "launches_per_step": 2,
                  "note": "cs, rho, mu from the volume fraction (two cell-vertex-cell passes); bytes: read c, "
                          "write cs, rho, mu"}
        del vc, vcs, vrho, vmu

    # momentum predictor (solveMomentumEqn FAST, QUICK, AB2) on the same channel;
    # compulsory bytes of the in-place step: read u, c, mu, rho and the flux
    # history, write u and the new fluxes (15 FP64 values per cell)
    momres = None
    if not args.no_momentum:
        from tbfsolver_b200.solver import MomentumEqn
        mom = MomentumEqn(eqn.solver, scheme=2, gch=0.0, g=0.0)
        mu_ = Field.like(inp.rho, 1e-3 * (1.0 - inp.cs.a) + 1e-3 * spec.rhog * inp.cs.a)
        mu_u = VField(*[Field.like(f, f.a.clone()) for f in u_in.components()])
        for _ in range(max(3, args.warmup)):
            mom.predictor(mu_u, inp.cs, mu_, inp.rho, dt=dt, alpha=alpha, gamma=1.5, xi=-0.5, rho0=inp.rho0)
        stream.synchronize()
        t0m, t1m = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            t0m.record(stream)
            for _ in range(args.steps):
                mom.predictor(mu_u, inp.cs, mu_, inp.rho, dt=dt, alpha=alpha, gamma=1.5, xi=-0.5, rho0=inp.rho0)
            t1m.record(stream)
        stream.synchronize()
        mms_ = t0m.elapsed_time(t1m) / args.steps
        # the out-of-place form (update fused into the flux kernel) into a second buffer
        mu_o = VField(*[Field.like(f, torch.empty_like(f.a)) for f in u_in.components()])
        for _ in range(max(3, args.warmup)):
            mom.predictor(mu_u, inp.cs, mu_, inp.rho, dt=dt, alpha=alpha, gamma=1.5, xi=-0.5, rho0=inp.rho0,
                          u_out=mu_o)
        stream.synchronize()
        with torch.cuda.stream(stream):
            t0m.record(stream)
            for _ in range(args.steps):
                mom.predictor(mu_u, inp.cs, mu_, inp.rho, dt=dt, alpha=alpha, gamma=1.5, xi=-0.5, rho0=inp.rho0,
                              u_out=mu_o)
            t1m.record(stream)
        stream.synchronize()
        mms_out = t0m.elapsed_time(t1m) / args.steps
        del mu_o
        mbytes = 15 * 8.0 * g.ncells
        pk0, _ = peaks()
        momres = {"value": g.ncells / (mms_ * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": mms_,
                  "alg_bytes": mbytes, "alg_GBps": mbytes / (mms_ * 1e-3) / 1e9,
                  "frac": mbytes / (mms_ * 1e-3) / 1e9 / pk0, "launches_per_step": 3, "scheme": "QUICK",
                  "out_of_place_ms": mms_out,
                  "note": "convection + diffusion fluxes and the AB2 update of u in place; bytes: read u, c, mu, "
                          "rho, flux history, write u, fluxes"}
        del mu_, mu_u

    # surface tension from the sharp volume fraction (interface cells, height-function
    # curvature, face force), and the projection that reads it (st_n = st_nm1)
    stres = None
    if not args.no_st:
        from tbfsolver_b200.fields import field_shape
        from tbfsolver_b200.solver import compute_surface_tension
        stf = VField(*[Field(k, 1, g.nx, g.ny, g.nz, torch.zeros(field_shape(k, 1, g.nx, g.ny, g.nz),
                                                                dtype=torch.float64, device="cuda"))
                       for k in ("sx", "sy", "sz")])
        stn = list(stf.components())
        sigma = 5e-3  # channel_18/specs/parameters
        st_ms = _stream_timer(stream, lambda: compute_surface_tension(eqn.solver, inp.c, sigma, stf), args.steps,
                              args.warmup)
        pst_ms = _stream_timer(stream, lambda: eqn.projection(psi, pn, pnm1, inp.rho, u_in, dt, alpha, stn, stn,
                                                              u_out=u_out, want_stats=False),
                               args.steps, args.warmup)
        pk0, _ = peaks()
        sbytes = 32.0 * g.ncells  # read c, write the three face components
        stres = {"value": g.ncells / (st_ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": st_ms,
                 "alg_bytes": sbytes, "frac": sbytes / (st_ms * 1e-3) / 1e9 / pk0, "launches_per_step": 3,
                 "projection_with_st_ms": pst_ms,
                 "note": "interface cells, height-function curvature and st = sigma k_f grad c on every face "
                         "(200 bubbles); bytes: read c, write st; then one projection reading st at both levels"}
        del stf, stn

    # one whole FAST substep on the device (material properties, setPressGrad,
    # solveMomentumEqn, projection, updateBoundariesV, setFlowRate): what a
    # time step costs once u* stays on the GPU
    subres = None
    if not args.no_momentum:
        from tbfsolver_b200.solver import VOF, FlowControl, fast_substep
        svof = vof if not args.no_vof else VOF(eqn.solver, rhol=spec.rhol, rhog=spec.rhog, mul=1e-3,
                                                mug=1e-3 * spec.rhog)
        flow = FlowControl(eqn.solver, 1, ret=127.3)
        su = VField(*[Field.like(f, f.a.clone()) for f in u_in.components()])
        sc = Field.like(inp.rho, inp.cs.a.clone())
        scs, srho, smu = (Field.like(inp.rho, torch.empty_like(inp.rho.a)) for _ in range(3))
        spsi, spn, spm = new(), new(), new()
        sstar = VField(*[Field.like(f, f.a.clone()) for f in u_in.components()])
        mom.update_boundaries_v(su)
        for _ in range(max(3, args.warmup)):
            fast_substep(eqn, svof, mom, flow, sc, scs, srho, smu, su, spsi, spn, spm, dt, alpha, 1.5, -0.5,
                         want_stats=False, u_star=sstar)
        stream.synchronize()
        t0s, t1s = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            t0s.record(stream)
            for _ in range(args.steps):
                fast_substep(eqn, svof, mom, flow, sc, scs, srho, smu, su, spsi, spn, spm, dt, alpha, 1.5, -0.5,
                             want_stats=False, u_star=sstar)
                spn, spm, spsi = eqn.update_pressure(spsi, spn, spm)
            t1s.record(stream)
        stream.synchronize()
        sms = t0s.elapsed_time(t1s) / args.steps
        subres = {"value": g.ncells / (sms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": sms,
                  "note": "updateMaterialProps + setPressGrad + solveMomentumEqn (QUICK, AB2, into a second "
                          "velocity buffer) + projection (back into u) + updateBoundariesV + setFlowRate, "
                          "device-resident"}
        del su, sc, scs, srho, smu, spsi, spn, spm, sstar

    # end to end through the host entry point, pinned host buffers
    def pinned(f):
        h = torch.empty(f.a.shape, dtype=torch.float64, pin_memory=True)
        h.copy_(f.a)
        return Field.like(f, h.numpy())

    hu = VField(*[pinned(f) for f in u_in.components()])
    hrho, hpn, hpnm1 = pinned(inp.rho), pinned(pn), pinned(pnm1)
    hpsi = pinned(psi)
    hu0 = [f.a.copy() for f in hu.components()]
    h2d = sum(f.a.nbytes for f in (*hu.components(), hrho, hpn, hpnm1))
    d2h = sum(f.a.nbytes for f in (*hu.components(), hpsi))
    eqn.projection(hpsi, hpn, hpnm1, hrho, hu, dt, alpha, want_stats=False)  # warm the host path
    e2e_ms = []
    for _ in range(args.e2e_steps):
        for f, a0 in zip(hu.components(), hu0):
            f.a[...] = a0
        a0e, a1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0e.record(stream)
        eqn.projection(hpsi, hpn, hpnm1, hrho, hu, dt, alpha, want_stats=False)
        a1e.record(stream)
        stream.synchronize()
        e2e_ms.append(a0e.elapsed_time(a1e))
    e2e = statistics.median(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = float(t.item())

    N = g.ncells
    value = world * N / (ms * 1e-3) / 1e9
    e2e_value = world * N / (e2e * 1e-3) / 1e9
    pk, pk_kind = peaks()
    ab = alg_bytes(g.nx, g.ny, g.nz)
    dom = max(stage_ms, key=lambda k: stage_ms[k])
    achieved = ab[dom] / (stage_ms[dom] * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        try:
            with open(prof) as f:
                traffic = json.load(f).get(args.config, {}).get(dom)
        except Exception:
            traffic = None
    stages = {k: {"ms": round(v, 4), "alg_GBps": round(ab[k] / (v * 1e-3) / 1e9, 1),
                  "frac": round(ab[k] / (v * 1e-3) / 1e9 / pk, 3)} for k, v in stage_ms.items()}

    if mixed is not None:
        mixed["vs_fp64"] = mixed["value"] / (N / (ms * 1e-3) / 1e9)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    parity = None
    if not args.no_cpu_baseline and world == 1:
        arrays = [f.a.detach().cpu().numpy().copy() for f in (*u_in.components(), inp.rho, pn, pnm1)]
        sec, reps, thr, opsi, ou, omd = cpu_projection_timer(g, arrays, dt, alpha, inp.rho0, min_seconds=10.0)
        cpu = {"value": N / sec / 1e9, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"C/OpenMP oracle on the same {spec.name} inputs, {reps} projections, "
                         f"{sec * 1e3:.0f} ms each"}
        parity = parity_report(opsi, ou, omd, psi64, u64, u_out, last.max_div)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(spec, N, world),
        "solves_per_s": world * 1e3 / ms,
        "max_div": last.max_div, "cont_err": last.cont_err, "rel_residual": fp64_rel,
        "parity": parity,
        "mixed": mixed,
        "mg": mgres,
        "material_props": vofres,
        "momentum": momres,
        "substep": subres,
        "surface_tension": stres,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk, "unit": "GB/s",
                     "frac": achieved / pk, "traffic": traffic, "peak_kind": pk_kind,
                     "alg_bytes_per_launch": ab[dom]},
        "step_roofline": {"b_alg_bytes": ab["b_alg"], "achieved": ab["b_alg"] / (ms * 1e-3) / 1e9,
                          "frac": ab["b_alg"] / (ms * 1e-3) / 1e9 / pk},
        "stages": stages,
        "gpu_launches": 7 * args.steps,  # recip, rhs + x fwd, z fwd, y solve, z inv, x inv, correct
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    return line


if __name__ == "__main__":
    main()
