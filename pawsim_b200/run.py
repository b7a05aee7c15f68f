"""Run a seeded synthetic set-up through the library (quick runs, profiling, timing).

    python -m pawsim_b200.run --setup gyre --N 1024 --steps 4 [--integrator-only]
                              [--solver 0|1] [--mg-fp32] [--mg-tile K] [--mg-omega W]
                              [--mg-pre P] [--mg-post Q] [--pi-guess G] [--dt 60] [--param FILE]
                              [--ws-collect S --ws-epochs E] [--tracer SCHEME]
                              [--averages] [--energy] [--budgets]

``--run`` advances with one ``pawsim_gpu_run`` call (steps enqueued without a host
synchronisation). ``--integrator-only`` advances with ``pawsim_gpu_integrator_step`` alone (one fused tendency
kernel per step, no pressure correction), which isolates the tendency kernel for a profiler.
``--param`` runs an existing AWSIM parameter file instead of a synthetic set-up.
``--ws-collect S`` first runs S steps that collect warm-start training pairs, trains the
network for ``--ws-epochs`` epochs on the GPU, then runs ``--steps`` steps whose solves start
from the network's guess (this exercises the tcgen05 convolution kernels).
``--tracer SCHEME`` adds a passive tracer (0 AL81, 1 UP3, 2 KT00; K2 = 100, relaxation over
100 days). ``--averages`` accumulates the online averages after every step; ``--energy``
computes the energy and enstrophy sums after every step; ``--budgets`` turns on the u, v,
thickness and energy budgets (the budget build of the fused kernel).
``--ensemble 64x256,16x512`` advances a batched ensemble of jets members instead (count x grid
size per group, dx 10 km, dt 600 s unless ``--dt``, distinct noise seeds, ``--solver``) for
``--steps`` steps after 12 warm-up steps; ``--no-graphs`` keeps every step on streams (the
batched launch is then a kernel of its own for a profiler).
"""
from __future__ import annotations

import argparse
import json
import tempfile
import time

from . import Ensemble, Model, inputs

SETUPS = {"gyre": inputs.gyre, "channel": inputs.channel, "jets": inputs.jets,
          "full": inputs.full_physics}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--setup", default="gyre", choices=sorted(SETUPS))
    ap.add_argument("--param", default=None)
    ap.add_argument("--N", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--solver", type=int, default=1)
    ap.add_argument("--mg-fp32", action="store_true")
    ap.add_argument("--pi-guess", type=int, default=0, help="1: extrapolated first guess of the solves")
    ap.add_argument("--fp32-inner", type=int, default=1, help="FP32 V-cycles per defect-correction step")
    ap.add_argument("--mg-tile", type=int, default=0, help="0 autotune, 1..4 force a tile shape, 5 strips")
    ap.add_argument("--mg-omega", type=float, default=-1.0, help="red-black weight; negative: chosen by the solver")
    ap.add_argument("--mg-pre", type=int, default=1)
    ap.add_argument("--mg-post", type=int, default=1)
    ap.add_argument("--integrator-only", action="store_true")
    ap.add_argument("--run", action="store_true", help="advance with one pawsim_gpu_run call (no per-step sync)")
    ap.add_argument("--ws-collect", type=int, default=0)
    ap.add_argument("--ws-epochs", type=int, default=2)
    ap.add_argument("--tracer", type=int, default=-1, help="tracer scheme 0..2; negative: no tracer")
    ap.add_argument("--averages", action="store_true")
    ap.add_argument("--energy", action="store_true")
    ap.add_argument("--budgets", action="store_true")
    ap.add_argument("--ensemble", default=None, help="COUNTxN[,COUNTxN...]: a batched jets ensemble")
    ap.add_argument("--no-graphs", action="store_true", help="ensemble steps on streams, not graph replays")
    a = ap.parse_args(argv)
    if a.ensemble:
        return run_ensemble(a)
    with tempfile.TemporaryDirectory() as d:
        if a.param:
            cfg = inputs.read_config(a.param)
        else:
            kw = {"solver": a.solver}
            if a.setup == "channel":
                kw.update(Nx=a.N, Ny=max(a.N // 2, 4))
            else:
                kw["N"] = a.N
            if a.budgets:
                kw["extra"] = dict(savefreqUMom=86400.0, savefreqVMom=86400.0, savefreqThic=86400.0,
                                   savefreqEnergy=86400.0)
            if a.dt:
                kw["dt"] = a.dt
            elif a.setup == "gyre":
                kw["dt"] = 50.0 * 2048 / a.N if a.N <= 2048 else 50.0
            p = SETUPS[a.setup](d, **kw)
            if a.tracer >= 0:
                inputs.add_tracer(p, scheme=a.tracer, relax_days=100.0, K2=100.0)
            cfg = inputs.read_config(p)
        m = Model(cfg, mg_fp32=int(a.mg_fp32), mg_tile=a.mg_tile, mg_omega=a.mg_omega, mg_pre=a.mg_pre,
                  mg_post=a.mg_post, pi_guess=a.pi_guess, mg_fp32_inner=a.fp32_inner)
        t0 = time.perf_counter()
        def diagnostics():
            if a.averages:
                m.accumulate_averages(1.0)
            if a.energy:
                m.energy()

        if a.integrator_only:
            for n in range(1, a.steps + 1):
                m.integrator_step(n)
                diagnostics()
            m.synchronize()
            rep = {}
        else:
            n0 = 1
            ws = {}
            if a.ws_collect:
                m.nn_setup(collect=True, use=False, max_pairs=a.ws_collect, batch=8)
            m.prelim()
            if a.ws_collect:
                for n0 in range(1, a.ws_collect + 1):
                    m.step(n0)
                n0 += 1
                ws["loss"] = m.nn_train(epochs=a.ws_epochs)
                ws["pairs"] = m.nn_pairs()
                m.nn_setup(collect=False, use=True)
            rep = {}
            iters, used = [], 0
            if a.run:
                rep = m.run(n0, a.steps)
                iters = [int(x) for x in m.run_iterations()]
            else:
                for n in range(n0, n0 + a.steps):
                    rep = m.step(n)
                    diagnostics()
                    iters.append(rep["iters"])
                    used += rep["warm_start"] == 1
            rep["iters_per_step"] = iters
            if ws:
                rep["warm_start_used"] = used
                rep["warm_start_training"] = ws
        m.synchronize()
        dt = time.perf_counter() - t0
        print(json.dumps({"setup": a.param or a.setup, "N": [cfg.Nx, cfg.Ny, cfg.Nlay], "steps": a.steps,
                          "seconds": dt, "last": rep}))
        m.close()


def run_ensemble(a):
    groups = []
    for part in a.ensemble.split(","):
        count, n = part.lower().split("x")
        groups.append((int(count), int(n)))
    dt = a.dt or 600.0
    members = []
    with tempfile.TemporaryDirectory() as d:
        seed = 1000
        for count, n in groups:
            for _ in range(count):
                p = inputs.jets(f"{d}/m{seed}", N=n, Ly=n * 10e3, dt=dt, seed=seed, solver=a.solver)
                m = Model(inputs.read_config(p))
                m.prelim()
                members.append(m)
                seed += 1
    ens = Ensemble(members)
    ens.set_graphs(not a.no_graphs)
    # untimed: the AB start-up, the multigrid's first solves, the capture of the step graphs
    ens.run(1, 12)
    t0 = time.perf_counter()
    ens.run(13, a.steps)
    sec = time.perf_counter() - t0
    print(json.dumps({"ensemble": a.ensemble, "members": len(members), "steps": a.steps, "seconds": sec,
                      "graph_steps": ens.graph_steps(), "kernel_ms": ens.kernel_ms(),
                      "iters_member0": [int(x) for x in members[0].run_iterations()]}))
    ens.close()
    for m in members:
        m.close()


if __name__ == "__main__":
    main()
