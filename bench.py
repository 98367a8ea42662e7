#!/usr/bin/env python
"""Benchmark: SCFT iterations/s (and triplets/s) of the AB-diblock BCC system on a
128^3 full grid with the PmmmDCT solver (64^3 physical grid), Ns = 200 (ds = 0.005),
fA = 0.25, chiN = 20, L = 4.2 Rg, lambda = 0.1.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|fp32] [--solver PMMM|3M|P1] [--grid 128]

A step is one SCFT iteration (400 triplets + Q, phi, energy, mixing).  N > 1 runs
independent replicas, one per GPU (a single instance does not shard); value is the
sum over ranks of K / (max over ranks of the device time).  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "SCFT iters/s & triplets/s at 128^3 BCC: FP64 vs FP32+polish at |dF/F|<=1e-8"
WORKLOAD = dict(fA=0.25, xN=20.0, ds=0.005, L=4.2, acc=0.1, phase="BCC")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--solver", choices=["PMMM", "3M", "P1"], default="PMMM")
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra-legs", action="store_true",
                    help="skip the batch and 256^3 legs of the default run")
    ap.add_argument("--workload", choices=["single", "batch"], default="single",
                    help="single: the 128^3 BCC system; batch: 64 seeded PMMM instances of mixed size")
    ap.add_argument("--instances", type=int, default=64)
    return ap.parse_args()


def workload_config(args, extra=None):
    n = args.grid
    phy = n if args.solver == "P1" else n // 2
    cfg = {
        "workload": (f"AB diblock {WORKLOAD['phase']} {n}^3 full grid, {args.solver} solver on {phy}^3, "
                     f"Ns=200 (ds={WORKLOAD['ds']}), fA={WORKLOAD['fA']}, chiN={WORKLOAD['xN']}, "
                     f"L={WORKLOAD['L']} Rg, simple mixing lambda={WORKLOAD['acc']}"),
        "solver": args.solver,
        "grid_log": [n, n, n],
        "grid_phy": [phy, phy, phy],
        "contour_steps": 200,
        "precision": args.precision,
        "parallelism": f"replicas x{args.gpus}",
        "l2": "inputs larger than L2: the stored contour (2 x 201 slices) is re-read each iteration",
    }
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.dev = device_index

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"]
        bus = self._bus_id()
        if bus:
            cmd += ["-i", bus]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def _bus_id(self):
        try:
            import torch

            p = torch.cuda.get_device_properties(self.dev)
            return f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        except Exception:
            return None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU: the reference (compiled as oracle/_ref) on the host cores
# ---------------------------------------------------------------------------
def reference_iterations(args, n_iter: int, threads: int | None = None):
    """Seconds per SCFT iteration of the reference solver on this workload."""
    import numpy as np

    from crysscft_sample_b200 import fields
    from oracle import ref

    n = args.grid
    if threads:
        ref.set_num_threads(threads)
    cores = ref.max_threads()
    wA, wB = fields.seed_fields((n, n, n), WORKLOAD["L"], WORKLOAD["phase"])
    a, b = fields.to_physical(args.solver, wA), fields.to_physical(args.solver, wB)
    R = ref.RefSolver(args.solver, (n, n, n))
    L = (WORKLOAD["L"],) * 3
    out = R.scft_run(WORKLOAD["fA"], WORKLOAD["ds"], WORKLOAD["xN"], L, WORKLOAD["acc"], n_iter, a, b)
    return out["wall_seconds"] / n_iter, cores, out


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for row in f:
                if row.startswith("model name"):
                    return row.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401

    from oracle import ref

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libscft_ref.so was not built"}))
        return 0
    # bounded sample: one untimed iteration, then min(K, cap) timed full iterations
    per_it, cores, _ = reference_iterations(args, 1)
    cap = max(1, int(120.0 / max(per_it, 1e-6)))
    k = max(1, min(args.steps, cap))
    t0 = time.perf_counter()
    per_it, cores, _ = reference_iterations(args, k)
    wall = time.perf_counter() - t0
    value = 1.0 / per_it
    U = 200
    line = {
        "metric": METRIC, "value": value, "unit": "iterations/s", "n_gpus": args.gpus, "steps": k,
        "warmup": 1, "ms_per_step": per_it * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded BCC fields)",
        "impl": "reference", "triplets_per_s": value * 2 * U,
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "iterations/s", "cores": cores, "kind": "reference",
                         "sample": (f"{k} full SCFT iteration(s) of the same workload ({2 * U} triplets each): "
                                    "the reference's C++ solvers and driver loop compiled with an FFTW-API "
                                    f"shim (FFTW absent), OpenMP {cores} threads, wall {wall:.1f} s"),
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def accuracy_protocol(run, ref_run, start, n_fp32: int, n_polish: int):
    """|dF/F| and max |dphi| after n_fp32 FP32 + n_polish FP64 iterations of `run` against
    n_fp32 + n_polish FP64 iterations of `ref_run`, both from the fields `start`."""
    import numpy as np

    run.set_fields(start["wA"], start["wB"])
    run.set_precision("fp32")
    run.iterate(n_fp32)
    run.set_precision("fp64")
    h = run.iterate(n_polish)
    got = run.get_fields()
    ref_run.set_fields(start["wA"], start["wB"])
    hr = ref_run.iterate(n_fp32 + n_polish)
    want = ref_run.get_fields()
    return {"dF_over_F": float(abs(h["F"][-1] - hr["F"][-1]) / abs(hr["F"][-1])),
            "phi_max_abs": float(max(np.abs(got["phiA"] - want["phiA"]).max(),
                                     np.abs(got["phiB"] - want["phiB"]).max()))}


def drop_in_triplets(solver, stream, M: int, n_dev: int = 400, n_host: int = 100):
    """Triplets/s through the per-triplet boundary the reference's driver calls
    (CrysPSSolverBase::diffusion, src/crysSCFT_sample.cpp:390): scft_solver_diffusion_device on
    a resident field (device-timed, back to back), and scft_solver_diffusion on the solver's
    pinned host iomat (copy in, triplet, copy out, synchronous; wall-timed like the
    reference's own loop)."""
    import numpy as np
    import torch

    rng = np.random.default_rng(5)
    q = torch.tensor(rng.random(M) + 0.5, dtype=torch.float64, device="cuda")
    for _ in range(5):
        solver.diffusion_device(q, stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n_dev):
        solver.diffusion_device(q, stream)  # the mean is kept (exp(-k^2 ds) = 1 at k = 0)
    e1.record(stream)
    e1.synchronize()
    dev_ms = e0.elapsed_time(e1)
    io = solver.get_iomat_for_diffusion()
    io[:] = rng.random(M) + 0.5
    for _ in range(3):
        solver.diffusion()
    t0 = time.perf_counter()
    for _ in range(n_host):
        solver.diffusion()
    host_s = time.perf_counter() - t0
    return {"device_triplets_per_s": n_dev / (dev_ms / 1e3),
            "host_iomat_triplets_per_s": n_host / host_s,
            "entry_points": "scft_solver_diffusion_device (device-timed), scft_solver_diffusion (host iomat, wall-timed, 2 x M x 8 bytes copied "
                            "per triplet)"}


def batch_leg(local: int, steps: int = 10):
    """The batching form on its configured workload (64 PMMM instances, reduced grids
    {16..64}^3, ds = 0.01): the contours of all instances in one persistent launch (form 4)
    and, for comparison, one contour kernel per instance (form 0).  Wall-timed around
    synchronous batch iterations (each ends with the per-instance history copies)."""
    import torch

    from crysscft_sample_b200 import batch

    cfg = batch.batch_config(64)
    B = batch.BatchSCFT("PMMM", cfg, ds=0.01, device=local)
    B.seed_fields()
    out = {"workload": "64 PMMM instances, reduced grids from {16,24,32,48,64}^3, chiN~U[14,30], "
                       "fA~U[0.2,0.35], L~U[3.8,5.5], ds=0.01, BCC or FCC (seeded)",
           "unit": "instance-iterations/s", "steps": steps}
    for form, ns, key in ((4, 4, "one_launch"), (0, 8, "per_instance_kernels")):
        B.configure(ns, form)
        B.iterate(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        B.iterate(steps)
        dt = time.perf_counter() - t0
        out[key] = {"value": len(cfg) * steps / dt, "ms_per_iteration": dt / steps * 1e3,
                    "launches_per_iteration": B.launches_per_iteration()}
        if form == 4:
            out[key]["plan"] = B.team_plan()
    out["speedup"] = out["one_launch"]["value"] / out["per_instance_kernels"]["value"]
    B.close()
    return out


def grid256_leg(local: int, stream, steps: int = 10):
    """The same BCC system on the 256^3 full grid (PmmmDCT on 128^3, Ns = 200), FP64 and FP32
    triplets, CUDA events on the library's stream around `steps` iterations each."""
    import torch

    from crysscft_sample_b200 import fields, scft, solvers

    n = 256
    N = (n, n, n)
    L = WORKLOAD["L"]
    G = solvers.make_solver("PMMM", N, precision="fp64", device=local)
    G.set_stream(stream)
    G.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(G, WORKLOAD["fA"], WORKLOAD["ds"], WORKLOAD["xN"], WORKLOAD["acc"])
    wA, wB = fields.seed_fields(N, L, WORKLOAD["phase"], seed=20261203)
    run.set_fields(fields.to_physical("PMMM", wA), fields.to_physical("PMMM", wB))
    out = {"workload": "AB diblock BCC 256^3 full grid, PMMM solver on 128^3, Ns=200 (ds=0.005)",
           "unit": "iterations/s", "steps": steps}
    for prec in ("fp64", "fp32"):
        run.set_precision(prec)
        run.iterate(3)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run.iterate(steps)
        e1.record(stream)
        e1.synchronize()
        out[prec] = {"value": steps / (e0.elapsed_time(e1) / 1e3)}
    out["fp32_speedup"] = out["fp32"]["value"] / out["fp64"]["value"]
    run.close()
    G.close()
    return out


def run_ours(args):
    import numpy as np
    import torch

    from crysscft_sample_b200 import fields, replicas, scft, solvers

    rank, world, local = replicas.dist_env()
    torch.cuda.set_device(local)
    dist = replicas.init("nccl", timeout_s=120)

    n = args.grid
    N = (n, n, n)
    L = WORKLOAD["L"]
    solver = solvers.make_solver(args.solver, N, precision="fp64", device=local)
    stream = torch.cuda.Stream()
    solver.set_stream(stream)
    solver.set_cell_para((L, L, L))
    run = scft.DiblockSCFT(solver, WORKLOAD["fA"], WORKLOAD["ds"], WORKLOAD["xN"], WORKLOAD["acc"])
    wA, wB = fields.seed_fields(N, L, WORKLOAD["phase"], seed=20261203 + rank)
    a, b = fields.to_physical(args.solver, wA), fields.to_physical(args.solver, wB)
    run.set_fields(a, b)
    M = solver.get_space_size_phy()
    U = run.NsA + run.NsB

    def barrier():
        replicas.barrier(dist)
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(dist, x)

    # ---- device-resident timed region ------------------------------------
    # precision form: K - P iterations with FP32 triplets, then P = K/10 FP64 polish iterations
    polish = max(1, args.steps // 10)
    run.set_precision("fp32")
    run.iterate(max(args.warmup, 3))
    run.set_precision("fp64")
    run.iterate(max(args.warmup, 3))  # both launch plans captured and warm before timing
    start_fields = run.get_fields()

    def timed(fn):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        barrier()
        return out, e0.elapsed_time(e1)

    def plain():
        run.set_fields(start_fields["wA"], start_fields["wB"])
        run.set_precision("fp64")
        return run.iterate(args.steps)

    def precision_form_run():
        run.set_fields(start_fields["wA"], start_fields["wB"])
        run.set_precision("fp32")
        h1 = run.iterate(args.steps - polish)
        run.set_precision("fp64")
        h2 = run.iterate(polish)
        return {k: np.concatenate([h1[k], h2[k]]) for k in h2}

    primary = precision_form_run if args.precision == "fp32" else plain
    secondary = plain if args.precision == "fp32" else precision_form_run
    clocks = ClockSampler(local)
    clocks.start()
    hist, ms = timed(primary)
    hist2, ms2 = timed(secondary)
    clk = clocks.stop()
    fp64_ms, prec_ms = (ms2, ms) if args.precision == "fp32" else (ms, ms2)
    href, hprec = (hist2, hist) if args.precision == "fp32" else (hist, hist2)
    dF_timed = abs(hprec["F"][-1] - href["F"][-1]) / abs(href["F"][-1])
    # accuracy on the precision form's protocol: 90 FP32 iterations and 10 FP64 polish
    # iterations against 100 FP64 iterations, both from the same fields
    ref_run = scft.DiblockSCFT(solver, WORKLOAD["fA"], WORKLOAD["ds"], WORKLOAD["xN"], WORKLOAD["acc"])
    acc = accuracy_protocol(run, ref_run, start_fields, 90, 10)
    ref_run.close()
    fp64_ms_all = max_over_ranks(fp64_ms)
    prec_ms_all = max_over_ranks(prec_ms)
    precision_form = {"fp32_iterations": args.steps - polish, "fp64_polish_iterations": polish,
                      "iterations_per_s": world * args.steps / (prec_ms_all / 1e3),
                      "triplets_per_s": world * args.steps / (prec_ms_all / 1e3) * 2 * U,
                      "fp64_plain_iterations_per_s": world * args.steps / (fp64_ms_all / 1e3),
                      "speedup_vs_fp64_plain": fp64_ms_all / prec_ms_all,
                      "protocol": "90 FP32 + 10 FP64 polish iterations vs 100 FP64 iterations, same start",
                      "dF_over_F": acc["dF_over_F"], "phi_max_abs": acc["phi_max_abs"],
                      "target": 1e-8, "meets_target": bool(acc["dF_over_F"] <= 1e-8),
                      "dF_over_F_timed_run": dF_timed,
                      "timed_run": (f"{args.steps - polish} FP32 + {polish} FP64 iterations vs {args.steps} FP64 "
                                    "iterations from the same fields (the target is stated on the protocol)"),
                      "device_ms": prec_ms_all}
    run.set_precision(args.precision)
    # the FP64 iterations with phi integrated in a separate pass over the stored contour
    # instead of inside the contour kernel (same fields, its own warmed-up graph)
    sep_run = scft.DiblockSCFT(solver, WORKLOAD["fA"], WORKLOAD["ds"], WORKLOAD["xN"], WORKLOAD["acc"])
    sep_run.set_phi_form(False)
    sep_run.set_fields(start_fields["wA"], start_fields["wB"])
    sep_run.iterate(max(args.warmup, 3))

    def separate_phi():
        sep_run.set_fields(start_fields["wA"], start_fields["wB"])
        return sep_run.iterate(args.steps)

    hsep, sep_ms = timed(separate_phi)
    sep_run.close()
    sep_ms = max_over_ranks(sep_ms)
    phi_form = {"fused_iterations_per_s": world * args.steps / (fp64_ms_all / 1e3),
                "separate_pass_iterations_per_s": world * args.steps / (sep_ms / 1e3),
                "F_rel_diff_last": float(abs(hsep["F"][-1] - href["F"][-1]) / abs(href["F"][-1])),
                "what": "FP64 iterations: phi summed inside the contour kernel (default) against the "
                        "separate integrate_phi pass over the stored contour"}
    ms = max_over_ranks(ms)
    value = world * args.steps / (ms / 1e3)
    launches = run.launches_per_iteration()
    if not np.all(np.isfinite(hist["F"])):
        raise RuntimeError("non-finite free energy in the timed region")

    # ---- phase timer: the triplet kernels' share (roofline) ---------------
    other = "fp32" if args.precision == "fp64" else "fp64"
    run.set_precision(other)
    phases_other = run.time_phases(10)
    run.set_precision(args.precision)
    phases = run.time_phases(10)
    chain_s = phases[1] / 1e3  # one launch of the contour kernel = all 2U triplets of an iteration
    b = 8 if args.precision == "fp64" else 4
    fp32_chain_s = (phases_other if args.precision == "fp64" else phases)[1] / 1e3
    fp32_bytes = 2 * U * 3 * M * 4
    precision_form["contour_kernel_fp32"] = {
        "launch_ms": fp32_chain_s * 1e3, "algorithmic_bytes_per_launch": fp32_bytes,
        "achieved_gbs": fp32_bytes / fp32_chain_s / 1e9,
        "phases_ms_per_iteration": dict(zip(("total", "triplets", "q_phi", "fields_energy"),
                                            phases_other if args.precision == "fp64" else phases))}

    # ---- the drop-in per-triplet boundary (CrysPSSolverBase::diffusion) ----
    drop_in = drop_in_triplets(solver, stream, M)
    # ---- the batching form and the 256^3 size on the default run -------------
    extra = {}
    if args.grid == 128 and args.solver == "PMMM" and not args.no_extra_legs:
        extra["batch_form"] = batch_leg(local)
        extra["grid256"] = grid256_leg(local, stream)
    # per triplet: read q(s), read exp(-w ds/2), write q(s+1); K generated on chip, not counted
    alg_bytes_launch = 2 * U * 3 * M * b
    achieved = alg_bytes_launch / chain_s / 1e9
    # FP64 multiply-adds the triplet kernels execute per point and axis: n/2 with the
    # even/odd operators, 3n/8 with two even/odd levels (PMMM, 64 or 128 points on every
    # axis), else n
    n_phy = solver.get_grid_size_phy()
    two_level = args.solver == "PMMM" and n_phy[0] in (64, 128) and all(v == n_phy[0] for v in n_phy)
    per_point = sum((3 * v // 8) if two_level else (v // 2) if (args.solver != "3M" and v % 16 == 0) else v
                    for v in n_phy)
    flops_launch = 2.0 * 2 * U * M * per_point
    import ctypes as _ct

    from crysscft_sample_b200 import _lib as _L

    simt, tens = _ct.c_double(), _ct.c_double()
    _L.check(_L.load().scft_measure_fp64_peak(local, _ct.byref(simt), _ct.byref(tens)))
    peak, peak_src = hbm_peak()
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        key = f"{args.solver}_{args.precision}_{n}"
        traffic = tj.get(key, {}).get("dram_bytes_per_launch")
    except Exception:
        pass

    # ---- end to end through the host-buffer ABI ---------------------------
    wA_h = torch.empty(M, dtype=torch.float64, pin_memory=True).numpy()
    wB_h = torch.empty(M, dtype=torch.float64, pin_memory=True).numpy()
    phiA_h = torch.empty(M, dtype=torch.float64, pin_memory=True).numpy()
    phiB_h = torch.empty(M, dtype=torch.float64, pin_memory=True).numpy()
    fA_, fB_ = run.get_fields()["wA"], run.get_fields()["wB"]
    wA_h[:] = fA_
    wB_h[:] = fB_
    k_e2e = max(10, args.steps // 5)
    run.iterate_host(wA_h, wB_h, 1, phiA_h, phiB_h)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(k_e2e):
        run.iterate_host(wA_h, wB_h, 1, phiA_h, phiB_h)
    e1.record(stream)
    e1.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = world * k_e2e / (e2e_ms / 1e3)

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32",
            "data": "synthetic (seeded BCC fields, no input file)",
            "triplets_per_s": value * 2 * U,
            "config": workload_config(args),
            "gpu_launches": launches * args.steps,
            "phases_ms_per_iteration": {"total": phases[0], "triplets": phases[1], "q_phi": phases[2],
                                        "fields_energy": phases[3]},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "contour kernel: one launch = the 2 x 200 triplets of one iteration",
                         "algorithmic_bytes_per_launch": alg_bytes_launch,
                         "launch_ms": chain_s * 1e3,
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                         else "fallback 6650 GB/s",
                         "fp64": {"achieved_tflops": flops_launch / chain_s / 1e12,
                                  "peak_tflops": tens.value, "peak_simt_tflops": simt.value,
                                  "frac": flops_launch / chain_s / 1e12 / tens.value,
                                  "flops_per_launch": flops_launch,
                                  "peak_source": "measured live (scft_measure_fp64_peak, FP64 m8n8k4 MMA)"}
                         if args.precision == "fp64" else None},
            "e2e": {"value": e2e_value, "unit": "iterations/s", "h2d_bytes_per_step": 2 * M * 8,
                    "d2h_bytes_per_step": 4 * M * 8 + 8 * 8},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
            "F_last": float(hist["F"][-1]),
            "precision_form": precision_form,
            "phi_form": phi_form,
            "drop_in": drop_in,
            **extra,
        }
    if dist is not None:
        dist.barrier()
    run.close()
    solver.close()
    if dist is not None:
        dist.destroy_process_group()

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            per_it, cores, _ = reference_iterations(args, 2)
            line["cpu_baseline"] = {
                "value": 1.0 / per_it, "unit": "iterations/s", "cores": cores, "kind": "reference",
                "sample": ("2 full SCFT iterations of the same workload: the reference's C++ solvers and "
                           "driver loop compiled with an FFTW-API shim (FFTW absent), OpenMP threads"),
                "cpu_model": cpu_model(),
            }
            # the reference's own setting (its driver calls omp_set_num_threads(1))
            per_1, _, _ = reference_iterations(args, 1, threads=1)
            from oracle import ref as _ref

            _ref.set_num_threads(cores)
            line["cpu_baseline"]["single_thread"] = {
                "value": 1.0 / per_1, "unit": "iterations/s", "cores": 1,
                "sample": "1 full SCFT iteration of the same workload, 1 OpenMP thread"}
        except Exception as e:  # the CPU baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "iterations/s", "cores": 0, "kind": "reference",
                                    "sample": f"unavailable: {e}"}
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_batch(args):
    """Batching form: `--instances` seeded PMMM instances (reduced grids {16..64}^3, random
    chiN, fA, L; ds = 0.01), one CUDA-graph launch per batch iteration; each rank runs its
    share of the instances (replicas.shard_instances).  A step is one batch iteration."""
    import numpy as np
    import torch

    from crysscft_sample_b200 import batch, replicas

    rank, world, local = replicas.dist_env()
    torch.cuda.set_device(local)
    dist = replicas.init("nccl", timeout_s=120)
    cfg = batch.batch_config(args.instances)
    ds = 0.01
    costs = [np.prod(c["N"]) / 8 * (int(c["fA"] / ds) + int((1 - c["fA"]) / ds)) for c in cfg]
    mine = [cfg[i] for i in replicas.shard_instances(costs, world)[rank]]
    B = batch.BatchSCFT("PMMM", mine, ds=ds, precision="fp64", device=local)
    B.seed_fields()
    tuned = B.autotune(2)
    plan = B.team_plan()  # the one-launch form's plan (grid 0 when another form was faster)
    B.iterate(max(args.warmup, 3))
    replicas.barrier(dist)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    h = B.iterate(args.steps)  # synchronous: ends with the per-instance history copies
    dt = time.perf_counter() - t0
    clk = clocks.stop()
    dt = replicas.max_over_ranks(dist, dt)
    n_inst = replicas.sum_over_ranks(dist, len(mine))
    trip = replicas.sum_over_ranks(dist, sum(2 * (int(c["fA"] / ds) + int((1 - c["fA"]) / ds)) for c in mine))
    alg = replicas.sum_over_ranks(dist, sum(2 * (int(c["fA"] / ds) + int((1 - c["fA"]) / ds)) * 3 * np.prod(c["N"]) / 8 * 8
                                            for c in mine))
    value = n_inst * args.steps / dt
    launches = int(replicas.sum_over_ranks(dist, B.launches_per_iteration() * args.steps))
    # end to end: fields of every instance copied in from page-locked host buffers and phi
    # and the new fields copied back out every step
    pinned = [[torch.empty(int(B.M[i]), dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
              for i in range(len(mine))]
    for i in range(len(mine)):
        B.get_fields(i, out=pinned[i])
    t0 = time.perf_counter()
    k_e2e = max(3, args.steps // 10)
    for _ in range(k_e2e):
        for i in range(len(mine)):
            B.set_fields(i, pinned[i][2], pinned[i][3])
        B.iterate(1)
        for i in range(len(mine)):
            B.get_fields(i, out=pinned[i])
    e2e_dt = replicas.max_over_ranks(dist, time.perf_counter() - t0)
    bytes_in = sum(2 * 8 * np.prod(c["N"]) / 8 for c in mine)
    peak, peak_src = hbm_peak()
    if rank == 0:
        achieved = alg / (dt / args.steps) / 1e9
        print(json.dumps({
            "metric": "SCFT instance-iterations/s, batch of 64 PMMM instances (reduced grids 16..64^3)",
            "value": value, "unit": "instance-iterations/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded BCC/FCC fields)",
            "triplets_per_s": trip * args.steps / dt,
            "config": {"workload": f"{args.instances} PMMM instances, reduced grids from {{16,24,32,48,64}}^3, "
                                   "chiN~U[14,30], fA~U[0.2,0.35], L~U[3.8,5.5], ds=0.01, BCC or FCC",
                       "autotuned": tuned, "team_plan": plan,
                       "parallelism": f"instances sharded over {world} GPU(s)",
                       "l2": "working set (all contour stores) larger than L2"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": "one batch iteration (graph of all instances)",
                         "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured"
                         else "fallback 6650 GB/s"},
            "e2e": {"value": n_inst * k_e2e / e2e_dt, "unit": "instance-iterations/s",
                    "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(2 * bytes_in)},
            "clocks": {"sm_mhz": clk["sm_mhz"], "sm_max_mhz": clk["sm_max_mhz"], "reasons": clk["reasons"],
                       "samples": clk["samples"]},
            "F_last_mean": float(np.mean(h["F"][-1])),
        }))
    B.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
