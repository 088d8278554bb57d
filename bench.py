#!/usr/bin/env python
"""Benchmark: MD ion-steps/s of the N=24,000 polarisable silica Nose-Hoover-chain step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision mixed|fp64] [--solver fused|cg|reference]
                    [--fp64-steps K64] [--fit-configs C] [--fit-evals E]

MD: a step is one MD step (src/md.c:229-241: prop_agate = NHC half-step, velocity-Verlet
drift, force evaluation with the induced-dipole solve, kick, NHC half-step; then
check_verletlist) of the seeded 24,000-ion system (8000 Si + 16000 O, beta-cristobalite
10^3 supercell with 0.05 Å displacements, 2.20 g/cm^3, L = 71.3 Å, MB velocities at
2500 K), Buckingham rc 7 Å, Ewald alpha 0.32, rc 10 Å, kmax 14, skin 1 Å, PIM with
ASPC order 4 and residual 1e-6.  `value` is the mixed-precision step (fused CG, each
step a CUDA graph); `fp64_plain` the FP64 step with the plain CG on the same system.
Fit (`fit`): one evaluation = force-matching loss + adjoint gradient over the seeded
set of 512 configurations (427k ions); metric config-gradients/s.

ours      : state resident on the GPU; each timed step is bracketed by CUDA events on
            the engine stream, with a 256 MB L2 flush between steps (not timed).
            `e2e` repeats the measurement through the C ABI with page-locked host
            arrays in the reference's per-component layout: positions and velocities
            uploaded, one step, positions, velocities and forces downloaded, every step,
            in one mdffgpu_md_steps_host call per step (one synchronisation).
reference : the reference's own CPU code (oracle/_ref, -O3 -Ofast -fopenmp) on all host
            cores, on a bounded sample of steps of the same system.
N > 1 GPUs: one process per GPU (torchrun).  MD: an independent replica per rank (the
path has no collective; weak scaling).  Fit: configurations sharded over the ranks,
one all-reduce of (loss, gradient) per evaluation.  Times = max over ranks.
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
from typing import Optional

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the fit keeps one stream per configuration in flight: let them map onto more than the
# default 8 hardware queues (read when the CUDA context is created)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "MD ion-steps/s & batched fit-gradients/s: mixed vs FP64 GPU at ≤1e-5 force err"
WORKLOAD = ("pim_silica_nvt_24000: 8000 Si + 16000 O, 2.20 g/cm^3, L=71.3 A, Buckingham rc 7 A, "
            "Ewald alpha 0.32 rc 10 A kmax 14, PIM alpha_O 1 A^3 TT-damped, SCF 1e-6 ASPC-4, NHC(3) 2500 K, "
            "dt 1 fs, skin 1 A")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--solver", choices=["cg", "fused", "reference"], default="fused")
    ap.add_argument("--fp64-steps", type=int, default=100, help="steps of the plain FP64 path timed beside")
    ap.add_argument("--force-check", type=int, default=1, help="mixed: force error against an FP64 evaluation")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--roof-kernel", default="k_rho,k_rec_ion",
                    help="kernel families timed for the roofline (the one with the larger share is `roofline`)")
    ap.add_argument("--drift-steps", type=int, default=1000,
                    help="H_tot drift of mixed and FP64 runs over this many steps from the same start (0: skip)")
    ap.add_argument("--named-configs", type=int, default=1, help="config 2 and config 3 lines (0: skip)")
    ap.add_argument("--tune", type=int, default=1,
                    help="mixed: pick the k-space launch shapes on this system first (mdffgpu_tune_launch)")
    ap.add_argument("--cpu-steps", type=int, default=20, help="reference CPU baseline: timed steps")
    ap.add_argument("--cpu-warmup", type=int, default=5, help="reference CPU baseline: untimed steps before")
    ap.add_argument("--profile-steps", type=int, default=3)
    ap.add_argument("--cells", type=int, default=10,
                    help="MD system: beta-cristobalite supercell edge (10: the 24000-ion bench system; smaller: "
                         "the same model on 24 cells^3 ions, e.g. for profiler captures)")
    ap.add_argument("--fit-configs", type=int, default=512, help="batched fit configurations (0: skip)")
    ap.add_argument("--fit-evals", type=int, default=3)
    ap.add_argument("--fit-threads", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms (read only)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self) -> dict:
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------- cpu baseline
def cpu_baseline(system, nsteps: int = 20, warm: int = 5) -> dict:
    """The reference's own code on the host cores: after its t=0 forces, `warm` untimed
    MD steps then `nsteps` timed ones (per-step wall clock inside the harness), step
    indices from 6 on so that the ASPC order is the configured one from the start."""
    from oracle import ref
    threads = os.cpu_count() or 1
    if ref.available("tim"):
        r = ref.run(system, "md", warm + nsteps, 0, 6, variant="tim", threads=threads, timeout=3600)
        wall = float(r["step_wall"][warm:warm + nsteps].sum())
        return {"value": system.nion * nsteps / wall, "unit": "ion-steps/s", "cores": threads,
                "kind": "reference",
                "sample": f"{nsteps} MD steps after {warm} untimed ones of the same {system.nion}-ion system, "
                          f"mdff20 C code -O3 -Ofast -fopenmp, OMP_NUM_THREADS={threads}, {wall:.2f} s timed"}
    from oracle.oracle import Oracle
    o = Oracle(system)
    o.gen_verletlist()
    o.engforce()
    for s in range(6, 6 + warm):
        o.md_step(s)
    t0 = time.perf_counter()
    for s in range(6 + warm, 6 + warm + nsteps):
        o.md_step(s)
    wall = time.perf_counter() - t0
    return {"value": system.nion * nsteps / wall, "unit": "ion-steps/s", "cores": os.cpu_count() or 1,
            "kind": "port",
            "sample": f"{nsteps} MD steps after {warm} untimed ones with the C restatement (OpenMP), {wall:.2f} s"}


# ---------------------------------------------------------------------------- arms
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def h_drift(th, nion: int) -> dict:
    """Conserved-quantity drift over recorded steps: H_tot = E_kin + U_lj + U_bh + U_coul
    + U_pol + e_nvt (info_thermo, src/thermo.c:12-35), thermo columns 0-5 (eV)."""
    import numpy as np
    h = th[:, 0] + th[:, 1] + th[:, 2] + th[:, 3] + th[:, 4] + th[:, 5]
    steps = max(1, len(h) - 1)
    return {"h_start_ev": float(h[0]), "h_end_ev": float(h[-1]),
            "ev_per_ion_per_step": float((h[-1] - h[0]) / (nion * steps)),
            "rel": float((h[-1] - h[0]) / abs(h[0])), "steps": int(len(h))}


def fit_cpu_baseline(sizes, sample: int = 4) -> dict:
    """The reference's own code computing force-matching gradients the only way it can:
    central finite differences, 2 x 10 + 1 force evaluations per configuration, on a
    sample of the configurations (every len/sample-th), all host cores."""
    from mdff20_b200 import fit
    from oracle import ref
    threads = os.cpu_count() or 1
    idx = list(range(0, len(sizes), max(1, len(sizes) // sample)))[:sample]
    if not ref.available("tim"):
        return {"value": None, "unit": "config-gradients/s", "error": "compiled reference not built"}
    t0 = time.perf_counter()
    for c in idx:
        s = fit.config4_one(c, sizes[c])
        th0 = fit.theta_of(s)
        for k in range(2 * fit.NPARAM + 1):
            th = th0.copy()
            if k:
                p = (k - 1) // 2
                th[p] += fit.fd_step(th0, p) * (1.0 if k % 2 else -1.0)
            ref.run(fit.with_theta(s, th), "engforce", variant="tim", threads=threads, timeout=600)
    wall = time.perf_counter() - t0
    return {"value": len(idx) / wall, "unit": "config-gradients/s", "cores": threads, "kind": "reference",
            "sample": f"configurations {idx} (ions {[sizes[c] for c in idx]}) of the set, each gradient by "
                      f"{2 * fit.NPARAM + 1} reference force evaluations (central differences), "
                      f"mdff20 -O3 -Ofast -fopenmp, OMP_NUM_THREADS={threads}, {wall:.1f} s"}


def run_fit(args, world, rank, dev, pg) -> Optional[dict]:
    """Batched force matching (config 4): loss + adjoint gradient over all configurations
    per evaluation, FP64 and mixed engines; configurations sharded over the ranks, one
    all-reduce of (loss, gradient) per evaluation."""
    import numpy as np
    import torch

    from mdff20_b200 import fit
    from mdff20_b200.engine import FP64, MIXED
    sizes = fit.config4_sizes(args.fit_configs)
    mine = fit.shard(sizes, world)[rank]
    t0 = time.perf_counter()
    systems = fit.config4(sizes=sizes, indices=mine, workers=min(16, os.cpu_count() or 1))
    gen_s = time.perf_counter() - t0
    th0 = fit.theta_of(systems[0])
    tht = fit.perturbed_theta(th0)
    b = fit.ForceMatchBatch(systems, None, device=dev, precision=FP64, threads=args.fit_threads, ntot=sum(sizes))
    b.set_targets(b.forces(tht))   # FP64 forces at the perturbed parameters
    # a fit moves theta every evaluation: a seeded sequence of distinct parameter vectors
    # (1% Gaussian steps), so no evaluation starts from dipoles converged at its own theta
    rng = np.random.default_rng(17)
    # (both precisions run the same sequence, so their last results compare)
    seq = [th0 * (1.0 + 0.01 * rng.standard_normal(len(th0))) for _ in range(args.fit_evals + 1)]
    res = {}
    for label, prec in (("fp64", FP64), ("mixed", MIXED)):
        b.set_precision(prec)
        b.loss_grad(seq[0])                    # warm-up (recording, first CG solves)
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for k in range(args.fit_evals):
            loss, grad = b.loss_grad(seq[1 + k])   # synchronous: every configuration's stream done
            if pg is not None:
                loss, grad = fit.allreduce_loss_grad(loss, grad)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t
        if pg is not None:
            tt = torch.tensor([dt], device=f"cuda:{dev}", dtype=torch.float64)
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
            dt = float(tt.item())
        res[label] = {"value": len(sizes) * args.fit_evals / dt, "ms_per_eval": 1000.0 * dt / args.fit_evals,
                      "loss": loss, "grad": [float(x) for x in grad]}
    b.close()
    g64, g32 = np.array(res["fp64"]["grad"]), np.array(res["mixed"]["grad"])
    out = {"metric": "batched fit-gradients/s", "unit": "config-gradients/s", "value": res["mixed"]["value"],
           "fp64": res["fp64"]["value"], "configs": len(sizes), "ions": int(sum(sizes)), "evals": args.fit_evals,
           "ms_per_eval_mixed": res["mixed"]["ms_per_eval"], "ms_per_eval_fp64": res["fp64"]["ms_per_eval"],
           "grad_max_rel_err_mixed_vs_fp64": float(np.max(np.abs(g32 - g64)) / np.max(np.abs(g64))),
           "loss_rel_err_mixed_vs_fp64": abs(res["mixed"]["loss"] - res["fp64"]["loss"]) / res["fp64"]["loss"],
           "params": list(fit.PARAM_NAMES), "host_threads": args.fit_threads, "setup_s": round(gen_s, 1),
           "timing": "host clock around the synchronous C-ABI evaluation (host parameters in, host loss and "
                     "gradient out), device synchronised on both sides, max over ranks; each evaluation at a new "
                     "theta (seeded 1% steps)",
           "path": "mdffgpu_fit_plan: each configuration's evaluation recorded once as a CUDA graph (device-side "
                   "CG loops, theta in a shared device buffer), all configurations replayed concurrently",
           "data": "synthetic: seeded random silica configurations, targets = FP64 forces at +-5% parameters"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = fit_cpu_baseline(sizes)
        except Exception as exc:  # reported, not fatal
            out["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    return out


def run_reference(args):
    world, rank, local, pg = dist_setup(args)
    from mdff20_b200 import synth
    if rank == 0:
        s = synth.config5()
        nsteps = max(1, min(args.steps, args.cpu_steps))
        warm = max(0, min(args.warmup, args.cpu_warmup))
        cb = cpu_baseline(s, nsteps, warm)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "ion-steps/s",
                "n_gpus": args.gpus, "steps": nsteps, "warmup": warm, "ms_per_step": 1000.0 * s.nion / cb["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic: seeded beta-cristobalite silica, MB velocities",
                "config": {"workload": WORKLOAD, "nion": s.nion, "parallelism": "host OpenMP"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "ion-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        if args.fit_configs > 0:
            from mdff20_b200 import fit
            fb = fit_cpu_baseline(fit.config4_sizes(args.fit_configs))
            line["fit"] = {"metric": "batched fit-gradients/s", "unit": "config-gradients/s",
                           "value": fb.get("value"), "cpu_baseline": fb}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def _events(n):
    import torch
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def _max_over_ranks(x: float, dev: int, pg) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], device=f"cuda:{dev}", dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def timed_md(eng, first: int, nsteps: int, flush, dev: int, pg):
    """nsteps MD steps, each one call of the C ABI (a CUDA graph replay), bracketed by
    CUDA events on the engine stream with the L2 flush written before each (untimed).
    Returns (device ms summed over the steps, max over ranks; thermo records)."""
    import numpy as np
    import torch
    st = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)
    evs = _events(nsteps)
    th = []
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    for k in range(nsteps):
        with torch.cuda.stream(st):
            flush.zero_()
        evs[k][0].record(st)
        th.append(eng.md_steps(first + k, 1)[0])
        evs[k][1].record(st)
    torch.cuda.synchronize()
    if pg is not None:
        pg.barrier()
    ms = float(sum(a.elapsed_time(b) for a, b in evs))
    return _max_over_ranks(ms, dev, pg), np.array(th)


def profile_kernel(eng, name: str, first: int, nsteps: int, flush, stream):
    """CUDA events around every launch of one kernel family over nsteps kernel-by-kernel
    steps: (ms, launches, algorithmic flops)."""
    import torch
    eng.profile(name)
    for k in range(nsteps):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.md_steps(first + k, 1)
    torch.cuda.synchronize()
    res = eng.profile_result()
    eng.profile(None)
    return res


# algorithmic flops per (ion, k-vector) of each k-space family, counted from the kernels'
# loop bodies (FMA = 2 flops), and the direct per-k evaluation they replace
ROOF_NOTES = {
    "k_rho": "flops counted on the paired-nz formulation: 8 per (ion, k) with dipoles, 4 without (a direct "
             "evaluation of (q + i k.mu) exp(i k.r) per k costs about 14 plus a sincos)",
    "k_rec_ion": "flops counted on the folded formulation: 8 per (ion, k) for the field, 12 with forces (a direct "
                 "per-k evaluation costs about 20 plus a sincos)",
}


def md_drift(s, pos, dev: int, nsteps: int) -> dict:
    """Conserved-quantity drift of the bench system over nsteps NHC steps from the same
    start, mixed (fused CG, the bench's form) and FP64 (plain CG), each step a graph."""
    import numpy as np

    from mdff20_b200.engine import FP64, MIXED, PIM_CG, PIM_CG_FUSED, Engine
    out = {"steps": nsteps}
    for label, prec, solver in (("mixed", MIXED, PIM_CG_FUSED), ("fp64", FP64, PIM_CG)):
        e = Engine(s, positions=pos, device=dev, precision=prec, pim_solver=solver)
        e.gen_verletlist()
        e.engforce()
        th = e.md_steps(1, nsteps)
        e.close()
        h = th[:, 0] + th[:, 1] + th[:, 2] + th[:, 3] + th[:, 4] + th[:, 5]
        t = np.arange(len(h), dtype=float)
        slope = float(np.polyfit(t, h, 1)[0])
        fluct = float(np.std(h - np.polyval(np.polyfit(t, h, 1), t))) / s.nion
        out[label] = {"ev_per_ion_per_step": (float(h[-1]) - float(h[0])) / (s.nion * (len(h) - 1)),
                      "fit_slope_ev_per_ion_per_step": slope / s.nion,
                      # the slope a residual of this size gives when it is correlated over
                      # the whole window, sqrt(12) sigma / T: the scale below which fitted
                      # slopes of two decorrelated trajectories cannot be told apart
                      "fit_slope_noise_ev_per_ion_per_step": float(np.sqrt(12.0)) * fluct / len(h),
                      "h_rms_fluct_ev_per_ion": fluct,
                      "h_start_ev": float(h[0]), "h_end_ev": float(h[-1]),
                      "scf_iter_mean": float(th[:, 10].mean()), "finite": bool(np.isfinite(th).all())}
    # end-to-end drift ratio (a ratio of fitted slopes divides by a slope near zero once
    # the two trajectories have decorrelated)
    out["ratio_mixed_over_fp64"] = out["mixed"]["ev_per_ion_per_step"] / out["fp64"]["ev_per_ion_per_step"]
    return out


def named_configs(dev: int, flush) -> dict:
    """Throughput of the other named systems: config 2 (3000-ion rigid-ion silica single
    points in FP64 and mixed) and config 3 (6000-ion polarisable silica single point, SCF
    to 1e-8 in FP64 and 1e-6 in mixed), device time with CUDA events."""
    import numpy as np
    import torch

    from mdff20_b200 import synth
    from mdff20_b200.cellmath import wrap_positions
    from mdff20_b200.engine import FP64, MIXED, PIM_CG, PIM_CG_FUSED, Engine
    out = {}
    s2 = synth.config2()
    p2 = wrap_positions(s2.cell, s2.pos)
    c2 = {"workload": "config2: 1000 Si + 2000 O rigid ions, L=35.7 A, Buckingham rc 7 A, Ewald alpha 0.32 rc 10 A "
                      "kmax 12; single points (energy, forces, stress): the seeded random packing falls into the "
                      "Buckingham short-range divergence within tens of MD steps, in the reference as here"}
    forces = {}
    for label, prec in (("fp64", FP64), ("mixed", MIXED)):
        e = Engine(s2, positions=p2, device=dev, precision=prec)
        e.gen_verletlist()
        e.engforce()
        st = torch.cuda.ExternalStream(e.stream_handle(), device=dev)
        reps = 10
        evs = _events(reps)
        for k in range(reps):
            with torch.cuda.stream(st):
                flush.zero_()
            evs[k][0].record(st)
            e.engforce()
            evs[k][1].record(st)
        torch.cuda.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in evs)) / reps
        forces[label] = e.forces()
        e.close()
        c2[label] = {"ms_per_single_point": ms, "ion_evals_per_s": s2.nion * 1000.0 / ms}
    c2["force_rms_rel_err_mixed_vs_fp64"] = _rms_rel(forces["mixed"], forces["fp64"])
    c2["speedup_mixed_vs_fp64"] = c2["fp64"]["ms_per_single_point"] / c2["mixed"]["ms_per_single_point"]
    out["config2"] = c2
    s3 = synth.config3()
    p3 = wrap_positions(s3.cell, s3.pos)
    c3 = {"workload": "config3: 2000 Si + 4000 O polarisable, L=44.9 A, kmax 14, TT-damped, single point (energy, "
                      "forces, stress, induced dipoles from zero), SCF 1e-8 (FP64) / 1e-6 (mixed)"}
    res = {}
    for label, prec, tol in (("fp64", FP64, 1e-8), ("mixed", MIXED, 1e-6)):
        s3.conv_tol_ind = tol
        e = Engine(s3, positions=p3, device=dev, precision=prec, pim_solver=PIM_CG_FUSED if prec else PIM_CG)
        e.gen_verletlist()
        zero = np.zeros((s3.nion, 6, 3))
        st = torch.cuda.ExternalStream(e.stream_handle(), device=dev)
        e.engforce()
        reps = 5
        evs = _events(reps)
        for k in range(reps):
            e.set_dipole_history(zero)
            with torch.cuda.stream(st):
                flush.zero_()
            evs[k][0].record(st)
            e.engforce()
            evs[k][1].record(st)
        torch.cuda.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in evs)) / reps
        th = e.thermo()
        res[label] = (e.forces(), e.dipole_history()[:, 0, :], th)
        e.close()
        c3[label] = {"ms_per_single_point": ms, "single_points_per_s": 1000.0 / ms,
                     "ion_evals_per_s": s3.nion * 1000.0 / ms, "scf_iter": th["scf_iter"], "scf_tol": tol}
    (f64, m64, t64), (f32, m32, t32) = res["fp64"], res["mixed"]
    c3["errors_mixed_vs_fp64"] = {
        "force_rms_rel": _rms_rel(f32, f64), "dipole_rms_rel": _rms_rel(m32, m64),
        "u_coul_rel": abs(t32["u_coul"] - t64["u_coul"]) / abs(t64["u_coul"]),
        "u_pol_rel": abs(t32["u_pol"] - t64["u_pol"]) / abs(t64["u_pol"]),
        "tau_coul_rel": float(np.abs(t32["tau_coul"] - t64["tau_coul"]).max() / np.abs(t64["tau_coul"]).max())}
    c3["speedup_mixed_vs_fp64"] = c3["fp64"]["ms_per_single_point"] / c3["mixed"]["ms_per_single_point"]
    out["config3"] = c3
    return out


def _rms_rel(a, b) -> float:
    import numpy as np
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, 1))) / np.sqrt(np.mean(np.sum(b ** 2, 1))))


def run_ours(args):
    import numpy as np
    import torch

    from mdff20_b200 import synth
    from mdff20_b200.engine import FP64, MIXED, PIM_CG, PIM_CG_FUSED, PIM_REFERENCE, Engine, fma_peak_tflops
    from mdff20_b200.cellmath import wrap_positions

    world, rank, local, pg = dist_setup(args)
    dev = local
    torch.cuda.set_device(dev)
    s = synth.config5(cells=args.cells)
    pos = wrap_positions(s.cell, s.pos)
    prec = MIXED if args.precision == "mixed" else FP64
    solver = {"cg": PIM_CG, "fused": PIM_CG_FUSED, "reference": PIM_REFERENCE}[args.solver]
    eng = Engine(s, positions=pos, device=dev, precision=prec, pim_solver=solver)
    eng.gen_verletlist()
    eng.engforce()                                    # forces at t=0 (src/md.c:209)
    force_err = None
    if prec == MIXED and args.force_check:
        # relative RMS force error of the mixed path against the FP64 path at t=0
        ref = Engine(s, positions=pos, device=dev, precision=FP64, pim_solver=solver)
        ref.gen_verletlist()
        ref.engforce()
        force_err = _rms_rel(eng.forces(), ref.forces())
        ref.close()
    tuning = None
    if prec == MIXED and args.tune and s.polit is not None:
        tuning = eng.tune_launch(10)                  # untimed: launch shapes for this system
    istep = 1
    if args.warmup > 0:
        eng.md_steps(istep, args.warmup)
        istep += args.warmup
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{dev}")   # 256 MB > L2
    peak = fma_peak_tflops(dev, prec)

    # ------------------------------------------------ device-resident timed region
    l0 = eng.launch_count()
    clocks = ClockSampler(dev)
    clocks.start()
    total_ms, th = timed_md(eng, istep, args.steps, flush, dev, pg)
    clk = clocks.stop()
    istep += args.steps
    launches = eng.launch_count() - l0
    value = world * s.nion * args.steps / (total_ms / 1000.0)
    # the two k-space kernel families timed with CUDA events around each launch, over a few
    # more steps issued kernel by kernel (events inside the step; L2 flushed before each)
    roofs = []
    for name in args.roof_kernel.split(","):
        kms, kcount, kflops = profile_kernel(eng, name, istep, args.profile_steps, flush, stream)
        istep += args.profile_steps
        achieved = (kflops / (kms / 1000.0) / 1e12) if kms > 0 else None
        roofs.append({"kernel": name, "bound": "fp64" if prec == FP64 else "fp32", "achieved": achieved,
                      "peak": peak, "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                      "flops_note": ROOF_NOTES.get(name), "launches": kcount,
                      "ms_per_launch": (kms / kcount) if kcount else None,
                      "ms_per_step": kms / max(1, args.profile_steps),
                      "share_of_step": (kms / max(1, args.profile_steps)) / (total_ms / args.steps)
                      if world == 1 else None,
                      "peak_source": "measured by mdffgpu_fma_peak (independent FMA chains) on this GPU"})

    # ------------------------------------------------ FP64 arms on the same system
    def fp64_arm(solver64, label):
        e64 = Engine(s, positions=pos, device=dev, precision=FP64, pim_solver=solver64)
        e64.gen_verletlist()
        e64.engforce()
        if args.warmup > 0:
            e64.md_steps(1, args.warmup)
        ms64, th64 = timed_md(e64, 1 + args.warmup, args.fp64_steps, flush, dev, pg)
        e64.close()
        return {"value": world * s.nion * args.fp64_steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.fp64_steps,
                "steps": args.fp64_steps, "precision": "fp64", "pim_solver": label, "graph": True,
                "scf_iter_mean": float(th64[:, 10].mean()), "h_tot_drift": h_drift(th64, s.nion)}

    fp64_plain = fp64_fused = None
    if prec == MIXED and args.fp64_steps > 0:
        fp64_plain = fp64_arm(PIM_CG, "cg")
        # the same algorithm as the mixed arm (fused CG, polarisable-ion subsets of the CG
        # fields, polynomial predictor) in FP64: what precision alone buys
        fp64_fused = fp64_arm(PIM_CG_FUSED, "fused")

    # ------------------------------------------------ end to end through the C ABI
    # page-locked host arrays in the reference's per-component layout (rx[], ry[], ...):
    # positions and velocities in, positions, velocities and forces out, every step (one
    # C-ABI call: the copies are queued with the step and share its synchronisation)
    nE = max(1, args.e2e_steps)
    host = [torch.empty(s.nion, dtype=torch.float64).pin_memory().numpy() for _ in range(9)]
    eng.state_soa(*host)
    e_evs = _events(nE)
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    for k in range(nE):
        with torch.cuda.stream(stream):
            flush.zero_()
        e_evs[k][0].record(stream)
        eng.md_steps_host(istep, 1, host[0:6], host)
        e_evs[k][1].record(stream)
        istep += 1
    torch.cuda.synchronize()
    e2e_ms = _max_over_ranks(float(sum(a.elapsed_time(b) for a, b in e_evs)), dev, pg)
    e2e_value = world * s.nion * nE / (e2e_ms / 1000.0)
    n = s.nion
    h2d = 2 * n * 3 * 8
    d2h = 3 * n * 3 * 8 + 12 * 8
    eng.close()

    line = None
    if rank == 0:
        traffic = {}
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            traffic = json.load(open(tpath))
        for r_ in roofs:
            r_["traffic"] = traffic.get(f"{r_['kernel']}:{args.precision}")
        dominant = max(roofs, key=lambda x: x["ms_per_step"]) if roofs else None
        line = {
            "metric": METRIC, "value": value, "unit": "ion-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == FP64 else "f32+f64",
            "data": "synthetic: seeded beta-cristobalite silica, MB velocities",
            "config": {"workload": WORKLOAD if args.cells == 10 else f"{WORKLOAD} -- reduced to {n} ions "
                                                                          f"({args.cells}^3 cells)",
                       "nion": n, "kmax": 14, "nk": int(s.nk()),
                       "precision": args.precision, "pim_solver": args.solver,
                       "l2": "256 MB written between timed steps (untimed)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "ion-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": nE, "ms_per_step": e2e_ms / nE},
            "roofline": dict(dominant, dominant_of=[x["kernel"] for x in roofs]) if dominant else None,
            "roofline_kernels": roofs,
            "clocks": clk,
            "gpu_launches": launches,
            "launch_tuning": tuning,
            "force_rms_rel_err_vs_fp64": force_err,
            "h_tot_drift": h_drift(th, n),
            "fp64_plain": fp64_plain,
            "fp64_fused": fp64_fused,
            "speedup_vs_fp64_plain": (value / fp64_plain["value"]) if fp64_plain else None,
            "speedup_vs_fp64_fused": (value / fp64_fused["value"]) if fp64_fused else None,
            "scf_iter_mean": float(th[:, 10].mean()),
            "list_rebuilds": int(th[-1, 9] - th[0, 9]) + 1,
            "finite": bool(np.isfinite(th).all()),
        }
        if world == 1 and args.drift_steps > 0:
            line["h_tot_drift_long"] = md_drift(s, pos, dev, args.drift_steps)
        if world == 1 and args.named_configs:
            line["named_configs"] = named_configs(dev, flush)
        if world == 1 and not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = cpu_baseline(s, args.cpu_steps, args.cpu_warmup)
            except Exception as exc:  # reported, not fatal
                line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    fit_line = run_fit(args, world, rank, dev, pg) if args.fit_configs > 0 else None
    if rank == 0:
        if fit_line is not None:
            line["fit"] = fit_line
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
