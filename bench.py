#!/usr/bin/env python
"""Residual + Jacobian evaluations per second on the ternary spline EAM workload.

Workload (one "step"): one residual + analytic Jacobian + JᵀJ/Jᵀr evaluation
over 500 periodic configurations × 256 atoms (Zr/Cu/Al random packings at
0.060 Å⁻³), 6 φ + 3 ρ + 3 F makima splines × 20 knots (D = 240),
w_e = 1, w_s = 0.1 — rows = 388,000.  FP32 compute, FP64 sums.

  value     device-timed throughput (CUDA events on the library's stream,
            inputs resident in HBM, L2 flushed between timed steps)
  e2e       the same step through the C ABI with host buffers: x uploaded
            (H2D) and JᵀJ, Jᵀr, ‖F‖² read back (D2H) every step
  roofline  the dominant kernel's algorithmic bytes (or FLOPs) ÷ its measured
            per-launch time, against MEASURED_PEAKS.json
  cpu_baseline  the oracle (FP64 CPU restatement of the reference path,
            OpenMP over configurations) running the reference's own method —
            a residual plus a central-difference Jacobian, 1 + 2·D residual
            evaluations — once over a sample of the configurations, scaled
            by configuration count; beside it the best CPU method (the
            analytic Jacobian restated on the CPU, every configuration)

`--impl reference` times that CPU path alone as the reference arm: each
step is one complete central-difference evaluation over 125 of the 500
configurations.

Two more legs ride in the same JSON line (one GPU, rank 0): `de`, the
batched DE population objective on 200 configurations of 32-512 atoms with
NP = 15 D, and `surrogate`, the wall time surrogate-screened DE needs to reach
plain device DE's final objective (within 1 %) against plain DE's own time.
With the CPU leg on, `sw` (Stillinger-Weber Si, 1000 configurations) and
`al99_fit` (the Al fcc LM fit, device-driven against oracle-driven) are added.
Multi-GPU (torchrun): every rank evaluates its own 500-configuration shard
(weak scaling) and the normal equations are summed over ranks with one
NCCL all-reduce per step (the exchange an LM step needs).
"""
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

import numpy as np  # noqa: E402

W_E, W_S = 1.0, 0.1
N_CFG, N_ATOMS = 500, 256
WORKLOAD = "ternary Zr-Cu-Al makima-spline EAM, 500 configs x 256 atoms, D=240, w_e=1, w_s=0.1"
METRIC = "residual+Jacobian evals/s (ternary EAM, 500x256 atoms, D=240)"
L2_FLUSH_BYTES = 256 << 20
SURROGATE_SEEDS = (11, 12, 13)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--e2e-steps", type=int, default=50)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-sample", type=int, default=50,
                   help="configurations in the CPU central-difference sample of cpu_baseline")
    p.add_argument("--small", action="store_true", help="small case for profiler captures")
    p.add_argument("--leg", default="all", choices=["all", "de", "lmbtr"],
                   help="de: only the DE and surrogate legs; lmbtr: only the LMBTR leg (profiler captures "
                        "of their kernels)")
    p.add_argument("--surrogate-seeds", type=int, default=len(SURROGATE_SEEDS),
                   help="seeds of the surrogate comparison (the first N of 11, 12, 13)")
    p.add_argument("--de-generations", type=int, default=200,
                   help="generations of the DE and surrogate-screened DE legs (0: skip them)")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d["hbm_gbs"], d["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def workload(rank=0, small=False):
    from forcesmith_b200 import synth
    # the small case (profiler captures): 200 configurations, J = 149 MB > L2
    n_cfg, n_at = (200, 256) if small else (N_CFG, N_ATOMS)
    ds = synth.packing(np.full(n_cfg, n_at, np.int32), seed=20261204 + 7919 * rank)
    true = synth.ternary_true_model(20)
    start = synth.perturb(true, 0.95, 1.05, seed=7)
    return ds, true, start


def label_on_gpu(ds, true, device):
    from forcesmith_b200.gpu import GpuSession
    g = GpuSession(device, "fp64")
    g.upload(ds)
    g.set_model(true)
    out = g.eval(W_E, W_S, want=("forces", "energy", "stress"))
    g.close()
    return ds.with_labels(out["forces"], out["energy"], out["stress"])


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic(g, phase, M, D, P, N, ndens=60):
    """Algorithmic bytes (or FLOPs) of one launch of each phase's main kernel."""
    if phase == "residual":
        # 4-B (j, image) word per directed pair, per-atom position/type/ref force in
        # and force out, per-row residual out
        return "hbm", P * 4 + N * (24 + 4 + 24 + 24) + M * 8
    if phase == "jac_forces":
        # column-major FP32 J written once, pairs and ∂ρ/∂y rows read once
        return "hbm", M * D * 4 + P * 4 + N * ndens * 4 + N * 40
    if phase == "jac_atoms":
        return "hbm", P * 4 + N * (ndens * 4 + 40) + 2 * D * 8
    # JᵀJ: 2·m·D² FLOPs (dense contraction), plus Jᵀr
    return "tensor", 2.0 * M * D * D + 2.0 * M * D


def traffic_from_profiles(kernel):
    """DRAM bytes per full-size launch of `kernel`, from the committed ncu
    summary (a line `traffic_bytes_per_launch[kernel]: N`), else None."""
    import glob
    import re
    pat = re.compile(r"traffic_bytes_per_launch\[" + re.escape(kernel) + r"\]:\s*([0-9.eE+]+)")
    for f in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(f) as fh:
            m = pat.search(fh.read())
        if m:
            return float(m.group(1))
    return None


def fp64_leg(local, ds, start, steps=10):
    """The same step in an FP64 context (every kernel in FP64): device-timed
    residual + Jacobian + JtJ/Jtr per second, to show what FP32 compute buys."""
    import torch
    from forcesmith_b200 import gpu as G
    g = G.GpuSession(local, "fp64")
    g.upload(ds)
    g.set_model(start)
    tune = g.autotune(W_E, W_S)
    for _ in range(3):
        g.jacobian_async(W_E, W_S)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        a.record(stream)
    for _ in range(steps):
        g.jacobian_async(W_E, W_S)
    with torch.cuda.stream(stream):
        b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    g.close()
    return {"value": 1000.0 / ms, "unit": "evals/s", "ms_per_step": ms, "steps": steps,
            "schedule": {"lanes_per_atom": tune["lanes_per_atom"], "jac_forces_warps": tune["k2_warps"]},
            "note": "J (745 MB FP64) exceeds L2, no flush needed"}


def jacobian_to_host_leg(g, x, M, D, steps=5):
    """The drop-in path that hands the full Jacobian to the host, as the
    reference's solvers take it (Eigen column-major FP64 fjac): per step
    fs_gpu_set_params from pinned memory and fs_gpu_eval_jacobian with J, F,
    JtJ, Jtr and the objective returned into pageable host arrays."""
    import ctypes as C
    from forcesmith_b200.abi import _dp
    J = np.empty((D, M))  # column-major M × D
    F = np.empty(M)
    JtJ, Jtr, obj = np.zeros((D, D)), np.zeros(D), C.c_double()
    J.fill(0.0)  # touch every page once, outside the timed steps
    times = []
    for k in range(steps + 1):
        t0 = time.perf_counter()
        g.set_params(x)
        rc = g._lib.fs_gpu_eval_jacobian(g._h, W_E, W_S, _dp(F), _dp(J), _dp(JtJ), _dp(Jtr), C.byref(obj))
        assert rc == 0
        if k > 0:
            times.append(time.perf_counter() - t0)
    s_step = float(np.median(times))
    return {"value": 1.0 / s_step, "unit": "evals/s", "ms_per_step_median": s_step * 1e3, "steps": steps,
            "h2d_bytes_per_step": D * 8, "d2h_bytes_per_step": (M * D + M + D * D + D + 1) * 8,
            "path": "fs_gpu_set_params + fs_gpu_eval_jacobian with J (FP64 column-major, widened and "
                    "transposed on the device) and F into pageable host memory"}


def de_legs(local, generations, seeds=SURROGATE_SEEDS, cpu=True):
    """Batched DE on the 200-configuration set (32-512 atoms, NP = 15 D):
    throughput of the population objective, then the surrogate comparison -
    wall time of plain device DE over `generations` generations against the
    wall time surrogate-screened DE needs to reach plain DE's final best
    objective within 1 %."""
    import torch
    from forcesmith_b200 import gpu as G, solvers, synth
    ds = synth.de_geometry()
    true = synth.ternary_true_model(20)
    start = synth.perturb(true, 0.95, 1.05, seed=7)
    ds = label_on_gpu(ds, true, local)
    g = G.GpuSession(local, "fp32")
    g.upload(ds)
    g.set_model(start)
    tune = g.autotune(1.0, 0.0)
    x = g.gather_params()
    D, P = x.size, g.num_pairs()
    NP = 15 * D
    # finite knot box x0 ± 10 % (the reference keeps finite bounds as given)
    lb, ub = solvers.de_box(x, x - 0.1 * np.abs(x) - 1e-3, x + 0.1 * np.abs(x) + 1e-3)
    g.de_init(lb, ub, x0=x, NP=NP, seed=11)
    g.de_run(3, use_graph=True)  # warm-up (graph capture)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.ExternalStream(g.stream)
    n_t = 10
    with torch.cuda.stream(stream):
        ev0.record(stream)
    g.de_run(n_t, use_graph=True)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    ms_gen = ev0.elapsed_time(ev1) / n_t
    flops = 60.0 * P * NP / (ms_gen * 1e-3)
    sm_mhz = 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6  # FP32 CUDA-core FMA rate at the max SM clock (nominal)
    de = {"workload": f"DE population objective, {ds.n_cfg} configs x 32-512 atoms ({ds.n_atoms} atoms, "
                      f"{P} pairs), NP={NP}, D={D}, F=0.65, CR=0.5, box x0 +/- 10%",
          "ms_per_generation": ms_gen, "pair_trials_per_s": P * NP / (ms_gen * 1e-3),
          "schedule": {"population_waves": tune["pop_waves"], "chosen_by": "fs_gpu_autotune"},
          "roofline": {"bound": "fp32", "achieved": flops / 1e12, "peak": fp32_peak / 1e12,
                       "unit": "TFLOP/s", "frac": flops / fp32_peak, "peak_source": "nominal",
                       "algorithmic": "60 FLOP per pair-trial"}}
    if generations <= 0 or not seeds:
        g.close()
        return de, None
    runs = []
    for seed in seeds:
        # plain DE, device-resident, graph replay: wall time of `generations`
        # generations, with the best objective after each one
        g.de_init(lb, ub, x0=x, NP=NP, seed=seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        best_plain, _, hist = g.de_run(generations, use_graph=True, history=True)
        torch.cuda.synchronize()
        t_plain = time.perf_counter() - t0
        target = 1.01 * best_plain
        # plain DE's own time to reach its target: every plain generation does
        # the same work, so the time scales with the generation count
        g_plain = int(np.argmax(np.asarray(hist) <= target)) + 1
        t_plain_target = t_plain * g_plain / generations
        # surrogate-screened DE from the same start, in chunks until the target
        g.de_init(lb, ub, x0=x, NP=NP, seed=seed)
        g.surrogate_init(seed=seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done, gens, best_s, screened = 0, 0, float("inf"), 0
        chunk = 1  # the target is checked after every generation
        while gens < generations:
            b, _, info = g.de_run_screened(min(chunk, generations - gens))
            gens += min(chunk, generations - gens)
            screened += int(info["screened"].sum())
            best_s = b
            if b <= target:
                done = 1
                break
        torch.cuda.synchronize()
        t_scr = time.perf_counter() - t0
        runs.append({"seed": seed, "plain_final_objective": best_plain, "plain_wall_s": t_plain,
                     "plain_generations_to_target": g_plain, "plain_wall_s_to_target": t_plain_target,
                     "screened_reached": bool(done), "screened_generations": gens,
                     "screened_generations_screened": screened, "screened_best_objective": best_s,
                     "screened_wall_s": t_scr, "wall_ratio": t_scr / t_plain,
                     "wall_ratio_vs_plain_time_to_target": t_scr / t_plain_target})
    pop = g.de_population()[0]
    g.close()
    sur = {"plain_generations": generations, "target": "plain final objective x 1.01",
           "seeds": list(seeds),
           "wall_ratio": float(np.median([r["wall_ratio"] for r in runs])),
           "wall_ratio_vs_plain_time_to_target": float(np.median(
               [r["wall_ratio_vs_plain_time_to_target"] for r in runs])),
           "all_reached": all(r["screened_reached"] for r in runs), "runs": runs,
           "model": "BF16 MLP D->256->256->1 (GELU, Adam lr 1e-3), 4 candidates per member, "
                    "warm start 5 generations, Spearman gate 0.8 on a 10% held-out slice"}
    if cpu:
        de["cpu_baseline"] = cpu_de_generation(ds, start, pop)
    return de, sur


def cpu_de_generation(ds, start, pop):
    """The reference's DE on the host: BoostDESolver evaluates the population
    serially (threads = 1) with each objective parallel over configurations.
    One generation (NP objective evaluations of the oracle, OpenMP over
    configurations) is timed; 200 generations are extrapolated from it."""
    from oracle.api import Oracle, set_threads
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds)
    o.set_model(start)
    o.eval(1.0, 0.0, want=("obj",))
    t0 = time.perf_counter()
    o.eval_population(pop, 1.0, 0.0)
    t_gen = time.perf_counter() - t0
    return {"s_per_generation": t_gen, "s_200_generations_extrapolated": 200.0 * t_gen,
            "objective_evals_per_s": pop.shape[0] / t_gen, "cores": threads, "kind": "port",
            "sample": f"one generation timed ({pop.shape[0]} serial objective evaluations over {ds.n_cfg} "
                      "configurations); the 200-generation time is extrapolated"}


def three_body_leg(local, which, steps=20):
    """Tersoff or Angular on diamond Si: 1000 configurations of 64, 216 or 512
    atoms (sigma = 0.15 A, volumetric strain U[0.95, 1.05]).  Device: FP32
    residuals per second (CUDA events, 20 evaluations), and the FP64
    central-difference Jacobian (the reference's method for these families:
    2 D + 1 residuals) per second, the median of 5 host-timed calls that each
    end with the normal equations read back.  CPU: the oracle (16 threads, FP64), one
    residual timed, the Jacobian extrapolated as (2 D + 1) residuals."""
    import numpy as np
    import torch
    from forcesmith_b200 import gpu as G, synth
    from forcesmith_b200.abi import FS_FAMILY_ANGULAR, FS_FAMILY_TERSOFF, Model, Table
    from oracle.api import Oracle, set_threads
    ds = synth.diamond(1000)
    if which == "tersoff":
        def model(s):
            return Model(FS_FAMILY_TERSOFF, 1, [Table.tersoff(
                3264.7 * s, 95.373, 3.2394, 1.3258, 0.33675, 22.956, 4.8381, 2.0417, 0.0, 3.0, 3.2)])
        name = "Tersoff Si (1988 parameter set, R = 3.0, S = 3.2 A), D = 11"
    else:
        r = np.linspace(2.0, 3.8, 12)
        c = np.linspace(-1.0, 1.0, 9)
        def model(s):
            return Model(FS_FAMILY_ANGULAR, 1, [
                Table.spline(2.0, 3.8, s * 2.0 * (np.exp(-3 * (r - 2.35)) - 2 * np.exp(-1.5 * (r - 2.35))) * (1 - (r / 3.8) ** 4)),
                Table.spline(2.0, 3.8, s * np.exp(-1.2 * (r - 2.35)) * (1 - (r / 3.8) ** 3)),
                Table.spline(-1.0, 1.0, s * 1.5 * (c + 1.0 / 3.0) ** 2)])
        name = "Angular Si (12-knot pair and radial splines, 9-knot angular spline), D = 33"
    ds = label_on_gpu(ds, model(1.0), local)
    start = model(1.05)
    out = {"workload": f"{name}, {ds.n_cfg} configs x 64/216/512 atoms ({ds.n_atoms} atoms), w_e=1, w_s=0.1"}
    g = G.GpuSession(local, "fp32")
    g.upload(ds)
    g.set_model(start)
    for _ in range(3):
        g.eval(W_E, W_S, want=("obj",))
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(steps):
        g._lib.fs_gpu_eval(g._h, W_E, W_S, None, None, None, None, None, None)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    res_ms = ev0.elapsed_time(ev1) / steps
    P = g.num_pairs()
    g.close()
    g = G.GpuSession(local, "fp64")
    g.upload(ds)
    g.set_model(start)
    D = g.D
    g.jacobian_async(W_E, W_S)
    g.normal_equations()
    times = []
    for _ in range(5):
        t0 = time.perf_counter()
        g.jacobian_async(W_E, W_S)
        g.normal_equations()
        times.append(time.perf_counter() - t0)
    jac_s = float(np.median(times))
    g.close()
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds)
    o.set_model(start)
    o.eval(W_E, W_S, want=("obj",))
    t0 = time.perf_counter()
    o.eval(W_E, W_S, want=("F",))
    t_res = time.perf_counter() - t0
    out.update({"pairs": P, "D": D,
                "residual_fp32": {"value": 1000.0 / res_ms, "unit": "evals/s", "ms_per_eval": res_ms},
                "jacobian_fp64_fd": {"value": 1.0 / jac_s, "unit": "evals/s", "s_per_eval": jac_s,
                                     "method": "central differences, 2 D + 1 device residuals"},
                "cpu_baseline": {"residual": {"value": 1.0 / t_res, "unit": "evals/s"},
                                 "jacobian_fd": {"value": 1.0 / (t_res * (2 * D + 1)), "unit": "evals/s"},
                                 "cores": threads, "kind": "port",
                                 "sample": f"one FP64 residual ({t_res * 1e3:.0f} ms); the Jacobian as 2 D + 1 of them"}})
    return out


def acsf_leg(local, steps=20):
    """ACSF descriptors (G1, 4 G2, G3, 2 G4, G5; rcut 4.2 A) with a linear head
    on diamond Si, 1000 configurations.  Device FP32: residuals per second,
    and residual + exact Jacobian + JtJ per second.  CPU: the oracle's
    residual (16 threads, FP64); the reference forms this Jacobian from
    cached descriptor gradients, which the oracle does not restate, so no CPU
    Jacobian rate is given."""
    import numpy as np
    import torch
    from forcesmith_b200 import gpu as G, synth
    from forcesmith_b200.abi import FS_FAMILY_ACSF, Model, Table, acsf_size
    from oracle.api import Oracle, set_threads
    spec = Table.acsf(4.2, g1=1, g2=[(0.5, 2.3), (1.0, 3.0), (2.0, 3.8), (0.3, 0.0)], g3=[1.1],
                      g4=[(0.05, 1.0, 1.0), (0.05, 2.0, -1.0)], g5=[(0.08, 1.5, 1.0)])
    S = acsf_size(spec, 1)
    rng = np.random.default_rng(4)

    def model(w):
        return Model(FS_FAMILY_ACSF, 1, [spec, Table.linear_head(w, -4.0)])
    w_true = rng.normal(0, 0.3, S)
    ds = label_on_gpu(synth.diamond(1000), model(w_true), local)
    start = model(w_true * (1 + 0.1 * rng.normal(size=S)))
    g = G.GpuSession(local, "fp32")
    g.upload(ds)
    g.set_model(start)
    for _ in range(3):
        g.jacobian_async(W_E, W_S)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
        for _ in range(steps):
            fn()
        with torch.cuda.stream(stream):
            b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps
    res_ms = timed(lambda: g._lib.fs_gpu_eval(g._h, W_E, W_S, None, None, None, None, None, None))
    jac_ms = timed(lambda: g.jacobian_async(W_E, W_S))
    P = g.num_pairs()
    g.close()
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds)
    o.set_model(start)
    o.eval(W_E, W_S, want=("obj",))
    t0 = time.perf_counter()
    o.eval(W_E, W_S, want=("F",))
    t_res = time.perf_counter() - t0
    return {"workload": f"ACSF + linear head (S = {S}), Si, {ds.n_cfg} configs x 64/216/512 atoms "
                        f"({ds.n_atoms} atoms, {P} pairs), w_e=1, w_s=0.1",
            "residual_fp32": {"value": 1000.0 / res_ms, "unit": "evals/s", "ms_per_eval": res_ms},
            "jacobian_fp32": {"value": 1000.0 / jac_ms, "unit": "evals/s", "ms_per_eval": jac_ms,
                              "method": "exact (linear head): residual + J + JtJ + Jtr"},
            "cpu_baseline": {"residual": {"value": 1.0 / t_res, "unit": "evals/s"}, "cores": threads,
                             "kind": "port", "sample": f"one FP64 residual ({t_res * 1e3:.0f} ms)"}}


def lmbtr_leg(local, steps=10, n_cfg=1000, cpu_cfgs=4):
    """LMBTR descriptors at the reference's defaults (rcut 6 A, weight scale
    3 A, k2 grid 0-6 A x 50 bins, sigma 0.3; k3 grid cos 0 in [-1, 1] x 50
    bins, sigma 0.1; L2 normalised) with a linear head on diamond Si,
    n_cfg configurations of 64/216/512 atoms.  Device FP32: residuals per
    second (forces from the exact descriptor derivative), and residual +
    exact head Jacobian + JtJ per second.  CPU: the oracle's residual (all
    host threads, FP64), whose forces are the reference's central
    differences of the whole descriptor (6 descriptors per neighbour of
    every atom); timed on the first cpu_cfgs configurations and scaled to
    n_cfg by atom count."""
    import numpy as np
    import torch
    from forcesmith_b200 import gpu as G, synth
    from forcesmith_b200.abi import FS_FAMILY_LMBTR, Model, Table, lmbtr_size
    from oracle.api import Oracle, set_threads
    spec = Table.lmbtr()
    S = lmbtr_size(spec, 1)
    rng = np.random.default_rng(6)

    def model(w):
        return Model(FS_FAMILY_LMBTR, 1, [spec, Table.linear_head(w, -4.0)])
    w_true = rng.normal(0, 0.3, S)
    ds = label_on_gpu(synth.diamond(n_cfg), model(w_true), local)
    start = model(w_true * (1 + 0.1 * rng.normal(size=S)))
    g = G.GpuSession(local, "fp32")
    g.upload(ds)
    g.set_model(start)
    for _ in range(3):
        g.jacobian_async(W_E, W_S)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream)

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
        for _ in range(steps):
            fn()
        with torch.cuda.stream(stream):
            b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps
    res_ms = timed(lambda: g._lib.fs_gpu_eval(g._h, W_E, W_S, None, None, None, None, None, None))
    jac_ms = timed(lambda: g.jacobian_async(W_E, W_S))
    P = g.num_pairs()
    g.close()
    threads = set_threads(os.cpu_count() or 1)
    sub = ds.subset(range(cpu_cfgs))
    o = Oracle()
    o.upload(sub)
    o.set_model(start)
    t0 = time.perf_counter()
    o.eval(W_E, W_S, want=("F",))
    t_sub = time.perf_counter() - t0
    t_res = t_sub * ds.n_atoms / sub.n_atoms
    return {"workload": f"LMBTR (reference defaults, S = {S}) + linear head, Si, {ds.n_cfg} configs x "
                        f"64/216/512 atoms ({ds.n_atoms} atoms, {P} pairs), w_e=1, w_s=0.1",
            "residual_fp32": {"value": 1000.0 / res_ms, "unit": "evals/s", "ms_per_eval": res_ms},
            "jacobian_fp32": {"value": 1000.0 / jac_ms, "unit": "evals/s", "ms_per_eval": jac_ms,
                              "method": "exact (linear head): residual + J + JtJ + Jtr"},
            "cpu_baseline": {"residual": {"value": 1.0 / t_res, "unit": "evals/s"}, "cores": threads,
                             "kind": "port",
                             "sample": f"one FP64 residual of the first {sub.n_cfg} configurations "
                                       f"({sub.n_atoms} atoms, {t_sub:.2f} s), scaled by atom count"}}


def sw_leg(local, steps=20):
    """Stillinger-Weber Si: 1000 diamond configurations of 64, 216 or 512
    atoms (sigma = 0.15 A, volumetric strain U[0.95, 1.05]), 7 perturbed SW
    parameters; FP32 residual + analytic parameter Jacobian + normal
    equations per second, against the oracle (16 threads, FP64) running the
    reference's central differences for SW (2 D + 1 residual evaluations),
    timed on one residual and extrapolated."""
    import torch
    from forcesmith_b200 import gpu as G, synth
    from oracle.api import Oracle, set_threads
    ds = synth.diamond(1000)
    true, start = synth.sw_model(), synth.sw_start_model()
    ds = label_on_gpu(ds, true, local)
    g = G.GpuSession(local, "fp32")
    g.upload(ds)
    g.set_model(start)
    D = g.D
    for _ in range(3):
        g.jacobian_async(W_E, W_S)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(g.stream)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(steps):
        g.jacobian_async(W_E, W_S)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    P = g.num_pairs()
    g.close()
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds)
    o.set_model(start)
    o.eval(W_E, W_S, want=("obj",))
    t0 = time.perf_counter()
    o.eval(W_E, W_S, want=("F",))
    t_res = time.perf_counter() - t0
    cpu = 1.0 / (t_res * (2 * D + 1))
    return {"workload": f"Stillinger-Weber Si, {ds.n_cfg} configs x 64/216/512 atoms ({ds.n_atoms} atoms, "
                        f"{P} pairs), D={D}, w_e=1, w_s=0.1, FP32 residual + analytic Jacobian + JtJ",
            "value": 1000.0 / ms, "unit": "evals/s", "ms_per_eval": ms,
            "cpu_baseline": {"value": cpu, "unit": "evals/s", "cores": threads, "kind": "port",
                             "sample": f"one FP64 residual ({t_res*1e3:.0f} ms) x (2 D + 1) central-difference "
                                       "evaluations"}}


def al99_leg(local):
    """Al fcc LM fit (20 x 108 atoms, three 15-knot splines, D = 45,
    max_iter 200, w_e = 1, w_s = 0; labels from the Al99 setfl fixture): wall
    time of the device-driven LM against the same solver driven by the oracle
    (16 threads, FP64, analytic Jacobian). Each arm first runs one untimed
    evaluation at x0."""
    import numpy as np
    from forcesmith_b200 import gpu as G, solvers
    from forcesmith_b200.abi import Dataset, Model, Table, FS_FAMILY_EAM
    from oracle import api as O
    z = np.load(os.path.join(ROOT, "tests", "golden", "al99_c1.npz"))
    ds = Dataset(z["natoms"], z["box9"], z["pos"], z["type"], z["forces"], z["energy"], z["stress9"])
    start = Model(FS_FAMILY_EAM, 1, [Table.spline(float(lo), float(hi), z["start_knots"][k])
                                     for k, (lo, hi) in enumerate(z["start_domains"])])

    class OracleSteps(O.Oracle):
        def jacobian_async(self, w_e=1.0, w_s=0.0):
            F = self.eval(w_e, w_s, want=("F",))["F"]
            self._ne = O.normal_equations(self.jacobian_analytic(w_e, w_s), F) + (float(F @ F),)

        def normal_equations(self):
            return self._ne

        def lm_step(self, lam, mode=0):
            return O.lm_step(self._ne[0], self._ne[1], lam, mode)

    out = {"workload": "Al fcc, 20 configs x 108 atoms, 3 x 15-knot splines (D=45), LM max_iter 200, "
                       "labels: Al99 setfl"}
    for name, make in (("gpu_fp64", lambda: G.GpuSession(local, "fp64")), ("cpu_oracle", O.Oracle)):
        sess = OracleSteps() if name == "cpu_oracle" else make()
        sess.upload(ds)
        sess.set_model(start)
        x0 = sess.gather_params()
        # one untimed evaluation at x0 (first kernel loads, first-call buffers)
        sess.jacobian_async(1.0, 0.0)
        sess.normal_equations()
        sess.lm_step(1.0)
        sess.eval_population(np.stack([x0, x0, x0]), 1.0, 0.0)
        t0 = time.perf_counter()
        _, x, info = solvers.LMSolver(max_iter=200).minimize(sess, x0)
        out[name] = {"wall_s": time.perf_counter() - t0, "iterations": info["iterations"],
                     "final_objective": info["obj"][-1], "start_objective": info["obj"][0]}
    out["speedup"] = out["cpu_oracle"]["wall_s"] / out["gpu_fp64"]["wall_s"]
    return out


REF_SAMPLE_CFGS = 125  # configurations per reference-arm step (a quarter of the workload)


def cpu_fd_step(o, D):
    """One residual + Jacobian evaluation by the reference's method for spline
    tables: the residual (ForcesmithFunctor::operator()) and a central-difference
    Jacobian of 2·D residual evaluations, h = 1e-5 (opt::fd_jacobian)."""
    t0 = time.perf_counter()
    o.eval(W_E, W_S, want=("F",))
    o.jacobian_fd(W_E, W_S)
    return time.perf_counter() - t0


def cpu_baseline(ds, start, n_sample):
    """The reference's CPU path on the host, measured (no extrapolation over
    columns): (i) its own method, one complete central-difference evaluation
    over the first n_sample configurations, scaled to the workload by
    configuration count; (ii) the best CPU method, the analytic Jacobian
    restated on the CPU plus JtJ/Jtr, over every configuration."""
    from oracle.api import Oracle, set_threads
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds.subset(list(range(n_sample))))
    o.set_model(start)
    D = o.D
    o.eval(W_E, W_S, want=("obj",))  # warm
    t_fd = cpu_fd_step(o, D)
    frac = n_sample / ds.n_cfg
    o = Oracle()
    o.upload(ds)
    o.set_model(start)
    o.eval(W_E, W_S, want=("obj",))
    t0 = time.perf_counter()
    F = o.eval(W_E, W_S, want=("F",))["F"]
    J = o.jacobian_analytic(W_E, W_S)
    JtJ, Jtr = J.T @ J, J.T @ F
    t_an = time.perf_counter() - t0
    del J, JtJ, Jtr
    return {"value": frac / t_fd, "unit": "evals/s", "cores": threads, "kind": "port",
            "method": "central-difference Jacobian (2 D residuals, h=1e-5) + residual, the reference's "
                      "method for spline tables",
            "sample": f"one complete evaluation over {n_sample} of {ds.n_cfg} configurations "
                      f"({t_fd:.2f} s), scaled by configuration count",
            "best_cpu_analytic": {"value": 1.0 / t_an, "unit": "evals/s", "cores": threads,
                                  "sample": f"all {ds.n_cfg} configurations: residual + analytic Jacobian "
                                            f"(oracle restatement, FP64) + JtJ/Jtr (numpy BLAS), {t_an:.2f} s"}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ds, true, start = workload(0, args.small)
    from oracle.api import Oracle, set_threads
    threads = set_threads(os.cpu_count() or 1)
    o = Oracle()
    o.upload(ds)
    o.set_model(true)
    lab = o.eval(W_E, W_S)
    ds = ds.with_labels(lab["forces"], lab["energy"], lab["stress"])
    n_s = min(REF_SAMPLE_CFGS, ds.n_cfg)
    o = Oracle()
    o.upload(ds.subset(list(range(n_s))))
    o.set_model(start)
    D = o.D
    for _ in range(args.warmup):
        cpu_fd_step(o, D)
    t = [cpu_fd_step(o, D) for _ in range(args.steps)]
    t_step = float(np.mean(t))
    frac = n_s / ds.n_cfg
    v = frac / t_step
    sample = (f"per step one complete residual + central-difference Jacobian (1 + 2 D = {2 * D + 1} "
              f"residual evaluations, h=1e-5) over {n_s} of {ds.n_cfg} configurations; value = "
              f"({n_s}/{ds.n_cfg}) / step time")
    line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "method": "central-difference Jacobian, h=1e-5",
                       "threads": threads, "configs_per_step": n_s,
                       "ms_per_full_evaluation": t_step / frac * 1e3,
                       "step_ms_min_max": [min(t) * 1e3, max(t) * 1e3]},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_de_only(args):
    """The DE and surrogate legs alone on one GPU (profiler captures)."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    seeds = SURROGATE_SEEDS[:max(0, args.surrogate_seeds)]
    de, sur = de_legs(local, args.de_generations, seeds, cpu=not args.no_cpu_baseline)
    print(json.dumps({"de": de, "surrogate": sur}))
    return 0


def run_lmbtr_only(args):
    """The LMBTR leg alone on one GPU (profiler captures): at most 10 timed
    calls of each kind; --small: 100 configurations instead of 1000."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    steps = max(1, min(args.steps, 10))
    print(json.dumps({"lmbtr": lmbtr_leg(local, steps=steps, n_cfg=100 if args.small else 1000)}))
    return 0


def run_ours(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    from forcesmith_b200 import gpu as G

    ds, true, start = workload(rank, args.small)
    ds = label_on_gpu(ds, true, local)
    g = G.GpuSession(local, args.precision)
    g.upload(ds)
    g.set_model(start)
    tune = g.autotune(W_E, W_S)  # launch shapes timed on this workload (outside the timed region)
    M, D, P, N = g.residual_count(W_S), g.D, g.num_pairs(), ds.n_atoms
    stream = torch.cuda.ExternalStream(g.stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    ne = torch.empty(D * D + D + 1, dtype=torch.float64, device=f"cuda:{local}")

    def step():
        g.jacobian_async(W_E, W_S)
        if dist is not None:
            G.copy_normal_equations(g, ne.data_ptr())
            with torch.cuda.stream(stream):
                dist.all_reduce(ne)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    G.set_profiling(g, args.steps)
    l0 = G.launch_count(g)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush between timed steps, outside the step events
            ev[k][0].record(stream)
        step()
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t_wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    launches = G.launch_count(g) - l0
    phases, nprof = G.phase_times(g)
    G.set_profiling(g, 0)
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * 1000.0 / ms

    # e2e through the C ABI with host buffers (x in pinned memory)
    x = torch.from_numpy(g.gather_params()).pin_memory().numpy()
    JtJ, Jtr = np.zeros((D, D)), np.zeros(D)
    import ctypes as C
    from forcesmith_b200.abi import _dp
    obj = C.c_double()
    for _ in range(3):
        g.set_params(x)
        g._lib.fs_gpu_eval_jacobian(g._h, W_E, W_S, None, None, _dp(JtJ), _dp(Jtr), C.byref(obj))
    if dist is not None:
        dist.barrier()
    # each step timed on the host clock; the median step is the value (host
    # contention on a shared machine shows up as outliers, kept in the line)
    e2e_steps = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        g.set_params(x)
        rc = g._lib.fs_gpu_eval_jacobian(g._h, W_E, W_S, None, None, _dp(JtJ), _dp(Jtr), C.byref(obj))
        e2e_steps.append(time.perf_counter() - t0)
        assert rc == 0
    e2e_s = float(np.median(e2e_steps))
    if dist is not None:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    assert np.isfinite(obj.value) and np.all(np.isfinite(JtJ))
    j_host = None
    if rank == 0 and world == 1 and not args.small:
        j_host = jacobian_to_host_leg(g, x, M, D)

    hbm, bf16, src = peaks()
    per = {k: v / max(nprof, 1) for k, v in phases.items()}
    dom = max(per, key=per.get)
    bound, alg = algorithmic(g, dom, M, D, P, N)
    t_dom = per[dom] * 1e-3
    if bound == "hbm":
        achieved, peak, unit = alg / t_dom / 1e9, hbm, "GB/s"
    else:
        # the JtJ kernel issues tcgen05 kind::tf32 MMAs: its dense peak is half
        # the BF16 rate
        achieved, peak, unit = alg / t_dom / 1e12, bf16 / 2.0, "TFLOP/s"
        src = src + " (TF32 = half the BF16 burst)"
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": args.precision.replace("fp", "f") + "+f64acc",
        "data": "synthetic (seeded packings; labels from a seeded true model in FP64)",
        "config": {"workload": WORKLOAD, "rows": M, "params": D, "pairs": P, "atoms": N,
                   "parallelism": f"weak dp{world}" if world > 1 else "1 GPU",
                   "l2": "flushed by a 256 MiB write between timed steps",
                   "schedule": {"lanes_per_atom": tune["lanes_per_atom"], "jac_forces_warps": tune["k2_warps"],
                                "chosen_by": "fs_gpu_autotune"},
                   "wall_s_timed": t_wall},
        "e2e": {"value": world / e2e_s, "unit": "evals/s", "h2d_bytes_per_step": D * 8,
                "d2h_bytes_per_step": (D * D + D + 1) * 8, "steps": args.e2e_steps,
                "ms_per_step_median": e2e_s * 1e3, "ms_per_step_mean": float(np.mean(e2e_steps)) * 1e3,
                "ms_per_step_max": float(np.max(e2e_steps)) * 1e3,
                "path": "fs_gpu_set_params (x from pinned host memory) + fs_gpu_eval_jacobian "
                        "(JtJ, Jtr, objective to host)"},
        "gpu_launches": int(launches),
        "phases_ms": {k: round(v, 5) for k, v in per.items()},
        "phases_note": "stream-ordered phase boundaries of one step; the residual runs on a side stream "
                       "beside jac_atoms, so its time falls inside jac_atoms / jac_forces",
        "roofline": {"kernel": dom, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": achieved / peak, "peak_source": src, "traffic": None,
                     "algorithmic": alg},
        "clocks": clk,
    }
    line["roofline"]["traffic"] = traffic_from_profiles(dom)
    if j_host is not None:
        line["e2e_jacobian_to_host"] = j_host
    if rank == 0 and world == 1 and not args.small and args.precision == "fp32":
        line["fp64"] = fp64_leg(local, ds, start)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ds, start, min(args.cpu_sample, ds.n_cfg))
    if rank == 0 and world == 1 and not args.small and not args.no_cpu_baseline:
        line["sw"] = sw_leg(local)
        line["tersoff"] = three_body_leg(local, "tersoff")
        line["angular"] = three_body_leg(local, "angular")
        line["acsf"] = acsf_leg(local)
        line["lmbtr"] = lmbtr_leg(local)
        line["al99_fit"] = al99_leg(local)
    if rank == 0 and world == 1 and not args.small and args.de_generations >= 0:
        de, sur = de_legs(local, args.de_generations, SURROGATE_SEEDS[:max(0, args.surrogate_seeds)])
        line["de"] = de
        if sur is not None:
            line["surrogate"] = sur
    if dist is not None:
        dist.barrier()
    g.close()
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.leg == "de":
        return run_de_only(args)
    if args.leg == "lmbtr":
        return run_lmbtr_only(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
