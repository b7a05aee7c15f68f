#!/usr/bin/env python
"""Headline benchmark: simulated days per second of the 2048 x 2048 x 2-layer wind-driven
double gyre (rigid lid, AB3, FP64 state, multigrid pressure), one model step per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm runs the CUDA path through the C ABI (``pawsim_b200``). ``value`` is device-timed
throughput with the state resident in HBM; ``e2e`` is the same metric through the public
API with the initial state uploaded from pinned host memory, the per-step solve report read
back every step and the final state read back, all inside the timed region. The roofline
object times the dominant kernel (the fused tendency + AB3 kernel) alone with CUDA events.
The reference arm (``--impl reference``) times the reference's own serial build of the same
step (``oracle/_ref/ref_harness``, built from the reference sources) on the host cores.

Multi-GPU runs (torchrun, one rank per GPU) advance independent replicas: the model does not
shard in this build, so there is no data-path collective; only the timing uses a MAX
all-reduce. Inputs are seeded synthetic fields of the headline configuration; dt is 50 s:
120 s blows up at once, 60 s (near the AB3 gravity-wave limit of this grid, about 64 s) before
step 2250 as the gyre spins up, 50 s runs 6000 steps (3.5 days) with the state bounded.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

# the ensemble sub-line runs 81 streams; more hardware work queues than the default 8 keep
# unrelated members' kernels from queueing behind one another (read when the CUDA context is
# created, so it is set before torch or the library touch the GPU)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sim-days/s at 2048^2 2-layer (double gyre, rigid lid, AB3, MG pressure)"
N_GRID = int(os.environ.get("PAWSIM_BENCH_N", "2048"))
DT = 50.0
TOL = 1e-10
# Stable steps of the other configurations. The channel's biharmonic 1e10 m^4/s on 3.9 km
# cells limits AB3 to about 200 s (dt 900 s grows without bound); on the 977 m cells of the
# 4096^2 gyre a biharmonic 5e9 m^4/s would need dt below 2 s and the internal wave limits dt to
# about 80 s, so that case runs with 1e8 m^4/s and 50 s.
FULL_WS_SPIN = 100
FULL_WS_EPOCHS = 5
CHANNEL_DT = 150.0
FULL_DT = 50.0
FULL_A4 = 1e8
# grid spacing of the ensemble's jets members: at dt = 600 s the AB3 limit of the internal
# gravity wave (about 3 m/s) needs dx above about 7 km
ENS_DX = 10e3
# untimed ensemble steps: the AB start-up, the multigrid's first (tuning) solves and the capture
# of the six step graphs
ENS_WARMUP = 12
FP32_INNER = 4   # FP32 V-cycles per FP64 defect-correction step in the mixed-precision solves


def max_over_ranks(x, dist=None):
    """The largest of each rank's x (a CPU all-reduce over the replica group; x itself
    without one)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def job_throughput(world, steps, seconds):
    """Whole-job sim-days/s: every replica advances `steps` steps of DT in `seconds`."""
    return world * steps * DT / 86400.0 / seconds


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def tendency_traffic():
    """DRAM bytes per launch of the tendency kernel from the committed ncu summary of the same
    workload (one ncu capture; ncu cannot run inside the timed benchmark)."""
    p = os.path.join(ROOT, "profiles", f"tendency_kernel_gyre{N_GRID}x{N_GRID}x2.txt")
    if os.path.exists(p):
        for line in open(p):
            if line.startswith("dram_bytes_per_launch:"):
                return int(line.split()[1])
    return None


def make_inputs(d):
    from pawsim_b200 import inputs
    return inputs.gyre(d, N=N_GRID, dt=DT, Nt=1000, solver=1, tol=TOL, seed=0)


class Clocks:
    """nvidia-smi samples during the timed region (median SM clock, throttle reasons)."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def _lines(self):
        with open(self.out.name) as fh:
            return fh.read().count("\n")

    def __enter__(self):
        # the sampler is running (its first line written) before the timed region starts;
        # rows from the last one before the region onwards are kept
        self.first = 0
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return self
        t0 = time.time()
        while time.time() - t0 < 10 and self.p.poll() is None and self._lines() == 0:
            time.sleep(0.01)
        self.first = max(self._lines() - 1, 0)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.out.flush()
        rows = []
        with open(self.out.name) as fh:
            for line in fh.readlines()[self.first:]:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 6:
                    rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[2 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# the reference arm times at most this many steps (about 4 s each at 2048^2 on one core), so
# that a run with many --steps still ends within a few minutes; the line states the count
REF_MAX_STEPS = 40


def cpu_reference(param, warmup, steps):
    """Run the reference's serial step with ref_harness for warmup + steps steps after its
    set-up; returns (seconds of each of the last `steps` steps, sample text)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(exe):
        return None, "oracle/_ref/ref_harness not built"
    r = subprocess.run([exe, param, str(warmup + steps)], capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        return None, "ref_harness failed: " + r.stderr.strip()[-200:]
    rows = [json.loads(l) for l in r.stdout.splitlines() if '"phase": "step"' in l]
    timed = [row for row in rows if row["n"] > warmup]
    if len(timed) != steps:
        return None, f"ref_harness timed {len(timed)} of {steps} steps"
    first, last = timed[0]["n"], timed[-1]["n"]
    return ([row["seconds"] for row in timed],
            f"steps {first}..{last} of the {N_GRID}x{N_GRID}x2 gyre (after {warmup} untimed steps and the "
            f"set-up; steps 1-3 are the AB1/AB2 start-up), reference serial build, 1 thread")


def bench_config(world, mg_fp32=0):
    return {"workload": f"double gyre {N_GRID}x{N_GRID}x2, dt={DT} s, MG tol={TOL}",
            "pressure": "GPU multigrid, " + ("FP32 V-cycles in FP64 defect correction"
                                             if mg_fp32 else "FP64 V-cycles"),
            "l2": "inputs larger than L2 (state 201 MB + history 403 MB)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def run_reference_arm(args, rank, world):
    """The reference's own serial build of the same step (oracle/_ref/ref_harness, built from
    the reference sources) on rank 0's host cores: exactly --warmup untimed steps, then
    --steps timed steps (at most REF_MAX_STEPS; "steps" states the count timed). The reference
    has no threaded build and no MPI compiler exists on these hosts, so it runs on one core."""
    if rank != 0:
        return
    steps = min(args.steps, REF_MAX_STEPS)
    with tempfile.TemporaryDirectory() as d:
        param = make_inputs(d)
        secs, sample = cpu_reference(param, args.warmup, steps)
    line = {"metric": METRIC, "unit": "sim-days/s", "impl": "reference", "n_gpus": world,
            "steps": steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded double-gyre inputs of the headline configuration)",
            "config": bench_config(world, args.mg_fp32)}
    if steps != args.steps:
        line["steps_requested"] = args.steps
    if secs is None:
        line.update({"unavailable": sample})
    else:
        per = float(np.mean(secs))
        v = DT / 86400.0 / per
        line.update({"value": v, "ms_per_step": per * 1e3,
                     "cpu_baseline": {"value": v, "unit": "sim-days/s", "cores": 1,
                                      "kind": "reference", "sample": sample},
                     "e2e": {"value": v, "unit": "sim-days/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
    print(json.dumps(line), flush=True)


def tracer_timing(cfg, stream, reps):
    """Device time of the tracer kernel per step: integrator steps of the same set-up with and
    without a passive tracer (CUDA events on the model's stream), the difference."""
    import tempfile as _tf
    import pawsim_b200
    import torch
    out = []
    with _tf.TemporaryDirectory() as d:
        for tracer in (False, True):
            p = pawsim_b200.inputs.gyre(d + f"/t{int(tracer)}", N=N_GRID, solver=1, dt=DT)
            if tracer:
                pawsim_b200.inputs.add_tracer(p, scheme=2, relax_days=100.0, K2=100.0)
            c = pawsim_b200.inputs.read_config(p)
            m = pawsim_b200.Model(c)
            m.set_stream(stream.cuda_stream)
            with torch.cuda.stream(stream):
                m.prelim()
                for n in range(1, 4):
                    m.integrator_step(n)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for n in range(4, 4 + reps):
                    m.integrator_step(n)
                e1.record(stream)
                torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / reps)
            m.close()
    return out[1] - out[0]


def budget_timing(stream, reps):
    """Device time per step of the budget build of the tendency kernel with the u, v,
    thickness and energy budgets on (savefreqUMom/VMom/Thic/Energy), against the plain
    kernel: integrator steps of the same set-up with and without budgets, the difference."""
    import tempfile as _tf
    import pawsim_b200
    import torch
    out = []
    with _tf.TemporaryDirectory() as d:
        for bud in (False, True):
            extra = dict(savefreqUMom=3600.0, savefreqVMom=3600.0, savefreqThic=3600.0,
                         savefreqEnergy=3600.0) if bud else None
            p = pawsim_b200.inputs.gyre(d + f"/b{int(bud)}", N=N_GRID, solver=1, dt=DT, extra=extra)
            m = pawsim_b200.Model(pawsim_b200.inputs.read_config(p))
            m.set_stream(stream.cuda_stream)
            with torch.cuda.stream(stream):
                m.prelim()
                for n in range(1, 4):
                    m.integrator_step(n)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for n in range(4, 4 + reps):
                    m.integrator_step(n)
                e1.record(stream)
                torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / reps)
            m.close()
    return out


def config_timing(kind, steps, warmup, stream, peak):
    """The other stated configurations at their full sizes: steps/s and sim-days/s of the
    plain FP64 multigrid and of FP32 V-cycles in FP64 defect correction (device-timed runs with
    the state resident, CUDA events on the model's stream), the fused kernel's time inside
    complete steps, and whether the state stayed finite.
      channel: 1024 x 512 x 3 zonally periodic channel with a ridge, biharmonic 1e10
      full: 4096 x 4096 x 4 closed gyre, random bathymetry, 200 km sponge restoring the
            interfaces over 30 days, w_dia 1e-7 m/s, biharmonic viscosity
    The time steps are the largest the AB3 scheme keeps stable on these grids (CHANNEL_DT,
    FULL_DT, FULL_A4 below)."""
    import tempfile as _tf
    import pawsim_b200
    import torch
    out = {}
    with _tf.TemporaryDirectory() as d:
        if kind == "channel":
            p = pawsim_b200.inputs.channel(d + "/c", Nx=1024, Ny=512, dt=CHANNEL_DT, A4=1e10, solver=1, tol=TOL)
            desc = f"1024 x 512 x 3 channel (x-periodic, ridge), biharmonic 1e10 m^4/s, dt {CHANNEL_DT:g} s, AB3"
        else:
            p = pawsim_b200.inputs.full_physics(d + "/f", N=4096, dt=FULL_DT, A4=FULL_A4, solver=1, tol=TOL)
            desc = ("4096 x 4096 x 4 closed gyre, bathymetry, sponge restoring, w_dia 1e-7 m/s, "
                    f"biharmonic {FULL_A4:g} m^4/s, dt {FULL_DT:g} s, AB3")
        cfg = pawsim_b200.inputs.read_config(p)
        fields = pawsim_b200.inputs.load_fields(cfg)
        out["workload"] = desc
        L, ncell = cfg.Nlay, cfg.Nx * cfg.Ny
        dt = cfg.dt
        variants = [("fp64_mg", 0, False), ("fp32_in_fp64_mg", 1, False)]
        if kind == "full":
            # the learned warm start at this size: pairs collected over FULL_WS_SPIN steps,
            # FULL_WS_EPOCHS epochs on the GPU (untimed)
            variants.append(("learned_fp32_in_fp64_mg", 1, True))
        for label, fp32, learn in variants:
            inner = FP32_INNER if fp32 else 1
            m = pawsim_b200.Model(cfg, fields, mg_fp32=fp32, mg_fp32_inner=inner, check_nonfinite=1)
            m.set_stream(stream.cuda_stream)
            with torch.cuda.stream(stream):
                spin = FULL_WS_SPIN if learn else warmup
                if learn:
                    m.nn_setup(collect=True, use=False, max_pairs=spin, batch=8, seed=7)
                m.prelim()
                n = 1
                for _ in range(spin):
                    m.step(n)
                    n += 1
                extra = {}
                if learn:
                    loss = m.nn_train(epochs=FULL_WS_EPOCHS, lr=1e-3)
                    extra = {"train_pairs": m.nn_pairs(), "train_epochs": FULL_WS_EPOCHS, "train_loss": loss}
                    m.nn_setup(collect=False, use=True)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                finite = True
                iters, used = [], 0
                try:
                    if learn:   # the guess is formed and checked on the host's schedule: per-step calls
                        for q in range(steps):
                            st = m.step(n + q)
                            iters.append(st["iters"])
                            used += st["warm_start"] == 1
                    else:
                        m.run(n, steps)
                        iters = list(m.run_iterations())
                except pawsim_b200.PawsimError:
                    finite = False
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                n += steps
                res = {"ms_per_step": ms / steps, "sim_days_per_s": steps * dt / 86400.0 / (ms / 1e3),
                       "gpl_updates_per_s": steps * ncell * L / (ms / 1e3), "finite": finite, **extra}
                if learn:
                    res["guess_used_steps"] = int(used)
                if finite:
                    res["vcycles_per_step"] = float(np.mean(iters)) * inner
                    k_ms = 0.0
                    for _ in range(5):
                        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        k0.record(stream)
                        m.integrator_step(n)
                        k1.record(stream)
                        m.pressure_correct(True)
                        n += 1
                        torch.cuda.synchronize()
                        k_ms += k0.elapsed_time(k1) / 5
                    alg = ncell * (120 * L + 24)
                    res["tendency_kernel_ms"] = k_ms
                    res["tendency_frac_of_measured_hbm"] = alg / (k_ms / 1e3) / 1e9 / peak
                out[label] = res
            m.close()
    out["tendency_bytes_note"] = ("algorithmic bytes N (120 L + 24): state, AB history and outputs; the "
                                  "feature inputs (restoring fields, w_dia, bathymetry) are not counted")
    return out


def ensemble_timing(steps, warmup, peak):
    """The batched uneven ensemble: 64 members at 256 x 256 and 16 at 512 x 512 of the
    doubly periodic 2-layer jets set-up (dx = 10 km, dt = 600 s, distinct noise seeds, plain
    FP64 multigrid), advanced together (one fused-kernel launch per step over all members'
    tiles, each member's correction on its own stream), against the same members from the same
    start advanced one after another with their own runs. Times are host clocks around
    synchronised runs (the ensemble's streams are its own); the kernel time is CUDA events on
    the launch stream."""
    import tempfile as _tf
    import pawsim_b200
    import torch
    specs = [(256, 1000 + i) for i in range(64)] + [(512, 2000 + i) for i in range(16)]
    dt = 600.0
    with _tf.TemporaryDirectory() as d:
        cfgs = []
        for i, (N, seed) in enumerate(specs):
            p = pawsim_b200.inputs.jets(f"{d}/m{i}", N=N, Ly=N * ENS_DX, dt=dt, seed=seed, solver=1, tol=TOL)
            c = pawsim_b200.inputs.read_config(p)
            cfgs.append((c, pawsim_b200.inputs.load_fields(c)))

        def fresh():
            ms = []
            for c, f in cfgs:
                m = pawsim_b200.Model(c, f, check_nonfinite=1)
                m.prelim()
                ms.append(m)
            return ms

        # the members one after another, each with its own run (its own launch sequence)
        alone = fresh()
        for m in alone:
            m.run(1, warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for m in alone:
            m.run(1 + warmup, steps)
        torch.cuda.synchronize()
        sec_alone = time.perf_counter() - t0
        iters_alone = np.concatenate([m.run_iterations() for m in alone])
        for m in alone:
            m.close()
        # the same members from the same start, advanced together; the warm-up also captures
        # the step graphs (one per arrangement of the state buffers, period 6), untimed
        members = fresh()
        ens = pawsim_b200.Ensemble(members)
        ens.run(1, warmup)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.run(1 + warmup, steps)
        sec = time.perf_counter() - t0
        graph_steps = ens.graph_steps()
        iters = np.concatenate([m.run_iterations() for m in members])
        # the batched launch's device time, from a few stream-mode steps after the timed run
        ens.set_graphs(False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.run(1 + warmup + steps, 10)
        sec_streams = (time.perf_counter() - t0) / 10
        k_ms = ens.kernel_ms()
        ens.close()
        for m in members:
            m.close()
    L = 2
    cells = sum(N * N for N, _ in specs)
    alg = cells * (120 * L + 24)
    ach = alg / (k_ms / 1e3) / 1e9
    return {
        "workload": "64 x 256^2 + 16 x 512^2 jets members, 2 layers, dt 600 s, AB3, FP64 multigrid 1e-10",
        "members": len(specs), "steps": steps, "warmup": warmup,
        "ms_per_step": sec / steps * 1e3,
        "member_steps_per_s": len(specs) * steps / sec,
        "sim_days_per_s_all_members": len(specs) * steps * dt / 86400.0 / sec,
        "gpl_updates_per_s": steps * cells * L / sec,
        "vcycles_per_step": float(np.mean(iters)),
        "same_vcycles_as_alone": bool(np.array_equal(iters, iters_alone)),
        "graph_steps": graph_steps,
        "stream_mode_ms_per_step": sec_streams * 1e3,
        "alone_ms_per_step": sec_alone / steps * 1e3,
        "speedup_vs_members_alone": sec_alone / sec,
        "timing": "host clock around synchronised runs; inputs (80 x 2 x 3 state planes) above L2",
        "roofline": {"bound": "hbm", "kernel": "tendency_batch_kernel + tendency_batch_exact_kernel",
                     "kernel_ms": k_ms, "algorithmic_bytes": alg, "achieved": ach, "peak": peak,
                     "unit": "GB/s", "frac": ach / peak},
    }


def pressure_comparison(cfg, fields, stream, spin, steps, epochs, pairs):
    """Pressure ms/step and V-cycles/step of the plain FP64 multigrid (started from the
    previous pressure, as the reference's solver is) against FP32 V-cycles in FP64 defect
    correction (2 or FP32_INNER cycles per FP64 defect step), and against the same with the
    learned guess. Every variant runs the same `spin` untimed steps (the learned one collecting
    a training pair per step), the network is trained on the GPU (untimed), then `steps` steps
    of each are timed with CUDA events. vcycles_per_step counts every V-cycle (defect steps x
    cycles per step); guess_used_steps counts the steps whose solve started from the guess."""
    import torch
    import pawsim_b200
    res = {}
    variants = (("plain_fp64", 0, 1, False), ("fp32_inner2", 1, 2, False), (f"fp32_inner{FP32_INNER}", 1, FP32_INNER, False),
                ("learned_fp32_inner2", 1, 2, True))
    for name, fp32, inner, learn in variants:
        m = pawsim_b200.Model(cfg, fields, mg_fp32=fp32, mg_fp32_inner=inner, check_nonfinite=1)
        m.set_stream(stream.cuda_stream)
        with torch.cuda.stream(stream):
            if learn:
                m.nn_setup(collect=True, use=False, max_pairs=pairs, batch=8, seed=7)
            m.prelim()
            m.run(1, spin)   # the learned variant's solves synchronise (pairs are collected after each)
            n = spin + 1
            extra = {}
            if learn:
                t0 = time.perf_counter()
                loss = m.nn_train(epochs=epochs, lr=1e-3)
                torch.cuda.synchronize()
                extra = {"train_pairs": m.nn_pairs(), "train_epochs": epochs, "train_s": time.perf_counter() - t0,
                         "train_loss": loss, "params": m.nn_net().param_count}
                m.nn_setup(collect=False, use=True)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            iters, solve, used = [], [], 0
            e0.record(stream)
            for _ in range(steps):
                st = m.step(n)
                iters.append(st["iters"])
                solve.append(st["solve_ms"])
                used += st["warm_start"] == 1
                n += 1
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms = e0.elapsed_time(e1) / steps
        res[name] = {"pressure_ms_per_step": float(np.mean(solve)),
                     "vcycles_per_step": float(np.mean(iters)) * inner,
                     "defect_steps_per_step": float(np.mean(iters)) if fp32 else None,
                     "ms_per_step": step_ms, "sim_days_per_s": DT / 86400.0 / (step_ms / 1e3), **extra}
        if learn:
            res[name]["guess_used_steps"] = int(used)
        m.close()
    res["window"] = f"steps {spin + 1}..{spin + steps} after prelim, dt {DT:g} s"
    res["pressure_speedup"] = res["plain_fp64"]["pressure_ms_per_step"] / res["learned_fp32_inner2"]["pressure_ms_per_step"]
    res["fp32_speedup"] = res["plain_fp64"]["pressure_ms_per_step"] / min(
        res["fp32_inner2"]["pressure_ms_per_step"], res[f"fp32_inner{FP32_INNER}"]["pressure_ms_per_step"])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mg-fp32", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-warm-start", action="store_true", help="skip the learned+FP32 pressure comparison")
    ap.add_argument("--ws-spin", type=int, default=5000, help="spin-up steps that collect training pairs")
    ap.add_argument("--ws-epochs", type=int, default=8)
    ap.add_argument("--ws-steps", type=int, default=200, help="timed steps of the pressure comparison")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched ensemble sub-line")
    ap.add_argument("--no-configs", action="store_true", help="skip the channel and full-physics sub-lines")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    import pawsim_b200
    from pawsim_b200 import inputs

    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    tmp = tempfile.TemporaryDirectory()
    param = make_inputs(tmp.name)
    cfg = inputs.read_config(param)
    fields = inputs.load_fields(cfg)
    model = pawsim_b200.Model(cfg, fields, mg_fp32=args.mg_fp32)
    model.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        model.prelim()
        n = 1
        for _ in range(args.warmup):
            model.step(n)
            n += 1
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        launches0 = model.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        iters = []
        solve_ms = []
        with Clocks(local) as clk:
            # the steps are enqueued back to back (pawsim_gpu_run: no host synchronisation per
            # step; each step's V-cycle count is read from the device once at the end)
            e0.record(stream)
            model.run(n, args.steps)
            e1.record(stream)
            torch.cuda.synchronize()
        iters = [int(x) for x in model.run_iterations()]
        n += args.steps
        launches = model.launch_count() - launches0
        ms = e0.elapsed_time(e1)
        # the solve's own device time, sampled on a few synchronous steps after the timed region
        for _ in range(5):
            solve_ms.append(model.step(n)["solve_ms"])
            n += 1

        # roofline of the dominant kernel: the fused tendency + AB3 kernel (with its exact pass
        # over flagged tiles, an early-exit launch when none is), timed inside complete steps
        # (integrator step, then the rigid-lid correction) with CUDA events on the model's stream
        reps = 10
        k_ms = 0.0
        for _ in range(reps):
            k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0.record(stream)
            model.integrator_step(n)
            k1.record(stream)
            model.pressure_correct(True)
            n += 1
            torch.cuda.synchronize()
            k_ms += k0.elapsed_time(k1)
        k_ms /= reps

        # the online-average accumulation (savefreqAvg), which runs once per step when a set-up
        # asks for averages; not part of the headline step
        model.accumulate_averages(1.0)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(reps):
            model.accumulate_averages(1.0)
        a1.record(stream)
        torch.cuda.synchronize()
        avg_ms = a0.elapsed_time(a1) / reps

        # the energy and enstrophy sums of one EZdiags.dat line (savefreqEZ): the terms kernel
        # with per-block partials, the final tree and the read of KE, PE, Z_k; per call
        model.energy()
        ez_ms = 0.0
        for _ in range(reps):
            z0, z1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            z0.record(stream)
            model.energy()
            z1.record(stream)
            torch.cuda.synchronize()
            ez_ms += z0.elapsed_time(z1)
        ez_ms /= reps

    ms_max = max_over_ranks(ms, dist)
    sec = ms_max / 1e3
    value = job_throughput(world, args.steps, sec)

    # e2e through the public API: upload the state from pinned host memory, step, read the
    # per-step report, download the final state -- all inside the timed region
    L = cfg.Nlay
    pinned = {k: torch.from_numpy(np.ascontiguousarray(fields[k])).pin_memory() for k in ("u", "v", "h")}
    pinned_out = {k: torch.empty((L, cfg.Ny, cfg.Nx), dtype=torch.float64).pin_memory() for k in ("u", "v", "h")}
    pinned_out["pi"] = torch.empty((cfg.Ny, cfg.Nx), dtype=torch.float64).pin_memory()
    model2 = pawsim_b200.Model(cfg, fields, mg_fp32=args.mg_fp32)
    model2.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        model2.prelim()
        # the same untimed warm-up as the device-timed leg (one-time set-up of the solver:
        # shape tuning, the smoother-weight choice, graph capture); the timed region then
        # uploads the whole state again
        for w in range(args.warmup):
            model2.step(w + 1)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for k in range(L):
            for name in ("u", "v", "h"):
                model2.set(name, k, pinned[name][k].numpy())
        h2d = 3 * L * cfg.Nx * cfg.Ny * 8
        model2.run(1, args.steps)
        rep = model2.run_iterations()
        for name in ("u", "v", "h"):
            for k in range(L):
                model2.get(name, k, out=pinned_out[name][k].numpy())
        model2.get("pi", 0, out=pinned_out["pi"].numpy())
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    # the final state and pi, and the run's per-step report (an iteration count and a stopping
    # measure per step, read once)
    d2h = sum(t.numel() * 8 for t in pinned_out.values()) + args.steps * (4 + 8)
    e2e_value = job_throughput(world, args.steps, max_over_ranks(e2e_s, dist))

    # the sub-lines after the headline run on rank 0 only (its JSON line carries them; the
    # other ranks' replicas add nothing to them)
    extras = rank == 0
    ws = None
    if extras and not args.no_warm_start:
        ws = pressure_comparison(cfg, fields, stream, args.ws_spin, args.ws_steps, args.ws_epochs, args.ws_spin)

    peak, peak_kind = peaks()
    ncell = cfg.Nx * cfg.Ny
    alg_bytes = ncell * (120 * L + 24)
    achieved = alg_bytes / (k_ms / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "sim-days/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded double-gyre inputs of the headline configuration)",
        "config": bench_config(world, args.mg_fp32),
        "pressure_ms_per_step": float(np.mean(solve_ms)),
        "pressure_ms_sampled": "solve device time of 5 synchronous steps after the timed region",
        "vcycles_per_step": float(np.mean(iters)),
        "gpu_launches": int(launches),
        # the secondary throughput of the metric: grid-point-layer updates per second, all ranks
        "gpl_updates_per_s": world * args.steps * ncell * cfg.Nlay / sec,
        "e2e": {"value": e2e_value, "unit": "sim-days/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": tendency_traffic(),
                     "kernel": "tendency_kernel (fused tendency + AB3) + tendency_exact_kernel (empty list)", "kernel_ms": k_ms,
                     "algorithmic_bytes": alg_bytes, "peak_kind": peak_kind},
        "clocks": clk.summary(),
    }
    # the passive tracer (a set-up with useTracer: KT00 advection, K2, relaxation) on the same
    # grid, not part of the headline step
    tr = tracer_timing(cfg, stream, args.steps) if extras else None
    # bytes per cell: read u, v, h and pi, hhb, w_dia; read and write the 10 L + 2 sums
    avg_bytes = ncell * (24 * L + 8 * (L + 3) + 16 * (10 * L + 2))
    line["averages"] = {"kernel": "accumulate_averages_kernel", "ms_per_step": avg_ms,
                        "algorithmic_bytes": avg_bytes,
                        "achieved_gbs": avg_bytes / (avg_ms / 1e3) / 1e9,
                        "frac": avg_bytes / (avg_ms / 1e3) / 1e9 / peak}
    # bytes per cell: read u, v, h per layer (the thickness for eta is h under the rigid
    # lid), hhb and Coriolis
    ez_bytes = ncell * (24 * L + 16)
    line["energy"] = {"kernel": "ez_partial_kernel + ez_final_kernel", "ms_per_call": ez_ms,
                      "algorithmic_bytes": ez_bytes, "achieved_gbs": ez_bytes / (ez_ms / 1e3) / 1e9,
                      "frac": ez_bytes / (ez_ms / 1e3) / 1e9 / peak}
    if extras:
        bt = budget_timing(stream, min(args.steps, 20))
        # budget sums read and written once per step: 16 + 16 + 2 + 15 terms per layer; the
        # kernel itself as in the roofline line
        bud_bytes = ncell * L * 16 * (16 + 16 + 2 + 15)
        line["budgets"] = {"kernel": "tendency_kernel budget build (32 x 8 tiles)",
                           "families": "UMom VMom Thic Energy",
                           "ms_per_step": bt[1], "plain_ms_per_step": bt[0], "extra_ms": bt[1] - bt[0],
                           "budget_bytes": bud_bytes,
                           "budget_gbs": bud_bytes / ((bt[1] - bt[0]) / 1e3) / 1e9 if bt[1] > bt[0] else None}
    if tr is not None:
        tr_bytes = ncell * L * 88   # read u, v, h, b, bRelax, bTime, f1, f2, w_dia; write b, f
        line["tracer"] = {"kernel": "tracer_tile_kernel (KT00, K2, relaxation)", "ms_per_step": tr,
                          "algorithmic_bytes": tr_bytes, "achieved_gbs": tr_bytes / (tr / 1e3) / 1e9,
                          "frac": tr_bytes / (tr / 1e3) / 1e9 / peak}
    if ws is not None:
        line["pressure_learned_fp32_vs_plain_fp64"] = ws
    if extras and not args.no_ensemble:
        line["ensemble"] = ensemble_timing(min(args.steps, 100), max(args.warmup, ENS_WARMUP), peak)
    if extras and not args.no_configs:
        line["channel_1024x512x3"] = config_timing("channel", min(args.steps, 100), args.warmup, stream, peak)
        line["full_physics_4096x4096x4"] = config_timing("full", min(args.steps, 20), args.warmup, stream, peak)
    if rank == 0 and not args.no_cpu_baseline:
        # a bounded sample in steady state: steps 4 and 5 (after the AB1/AB2 start-up)
        secs, sample = cpu_reference(param, 3, 2)
        if secs is not None:
            line["cpu_baseline"] = {"value": DT / 86400.0 / float(np.mean(secs)), "unit": "sim-days/s",
                                    "cores": 1, "kind": "reference", "sample": sample}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "sim-days/s", "cores": 1,
                                    "kind": "reference", "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    model.close()
    model2.close()
    tmp.cleanup()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
