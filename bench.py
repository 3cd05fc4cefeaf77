#!/usr/bin/env python
"""Benchmark of the B200 pseudo-time iteration: wall-seconds per physical time
step (dual time stepping to a 1e-6 drop of the pseudo-time update, capped at
the case's itmax), one replica per GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--case channel|cavity]
                  [--impl ours|reference]

ours:       value = device-timed seconds per physical step of the product
            configuration (MIXED precision: FP64 state, residual and update,
            FP32 line-sweep work; linear-extrapolation initial guess), state
            resident in HBM.  e2e = the same step through the C ABI with the
            state copied from pinned host memory and back every step.  The
            plain FP64 path (q^n guess, as the reference) is timed too, and
            predictor_ab compares the three initial guesses (q^n, linear
            extrapolation, the learned network) by iterations and seconds per
            physical step to an absolute tolerance on the laminar cavity, and
            alm gives the cost of the actuator-line forcing, outlet that
            of the characteristics outlet on an open wake box,
            wall_functions that of the log-law wall functions, and
            batched_blocks steps eight uneven blocks one after another and
            together.
reference:  the CPU oracle (C++ restatement of the reference, FP32 like the
            reference's own build, its loops on every host thread) on the same
            case; a bounded sample of pseudo-iterations scaled to one physical
            step.

Under torchrun each rank runs an independent replica on its own GPU
(the path does not shard: no collective in the data path); times are the max
over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "des-alm_b200"))

from desalm import abi, cases  # noqa: E402

METRIC = "wall-s per physical step to 1e-6 residual drop: learned+mixed vs plain FP64 GPU"
UNIT = "s/step"

# Algorithmic bytes per interior node of each kernel class: every distinct
# array element the kernel must read or write once, at its stored precision
# (T = state bytes, W = line-sweep work bytes).  Halo re-reads and the
# line-solve scratch are not algorithmic.
def alg_bytes(kind, T, W, coarse):
    pk = 4 * T if coarse else 0
    return {
        "resid": 24 * T + 11 * W + pk,    # q4 qn3 qnm1-3 metrics9 aj 1/aj nut dtau | wk4 sigma tc3 hc3, diss1
        "recalc": 26 * T + pk,            # q4 qn3 qnm1-3 metrics9 aj 1/aj nut diss1 | rh4
        "sweep_i": 10 * W,                # line solve: wk4 in/out, tc, hc
        "sweep_j": 10 * W,
        "sweep_k": 10 * W,
        "xform_i": 15 * W,                # wk4 in/out, sigma, csi3, eta3 (metrics stored in W; j-face rows: not counted)
        "xform_j": 15 * W,                # wk4 in/out, sigma, eta3, zet3
        "xform_k": 8 * W + 8 * T,         # wk4, sigma, zet3 | q4 in/out
        "dtau": 4 * T,                    # nut, the two metric parts | dtau
        "norm": 15 * T,                   # q5 qold5 | qold5
        "rsmooth": (20 * W + 8 * T) / 3,  # dq4 in/out in W; the k direction reads dq4 and updates q4 (mean of 3)
        "prolong": 4 * W,                 # dq4 out in W (coarse reads amortised)
        "sa_rhs": 22 * 8 + 10 * W,        # q5 qn5 qnm1-5, U/J 3, metrics9, aj, 1/aj, wd, wo, dtev | rh, ADI rows 9
        "sa_sweep": 5 * W + 8,            # ADI row 3, rh in/out; k sweep: q5 in/out, dtev (1/3 each)
    }.get(kind)


def build_case(name, precision, predictor):
    if name == "cavity":
        case, grid, state = cases.cavity(n=65, itmax=200)
        desc = "laminar lid-driven cavity Re=1000, 65^3 perturbed cube, 3-level FAS, 200 pseudo-iterations/step"
    elif name == "channel":
        case, grid, state = cases.channel()
        desc = "SA RANS channel Re_tau=395, 129x97x65 tanh-stretched, periodic i/k, 3-level FAS"
    elif name == "wake":
        case, grid, state = cases.wake(im=129, jm=97, km=65, turbulence=1, itmax=200)
        desc = "SA wake box 129x97x65, uniform inflow, characteristics outlet, 3-level FAS"
    else:
        raise SystemExit("unknown case " + name)
    case.precision_mode = precision
    case.predictor = predictor
    case.use_graph = 1      # each physical step replays one CUDA graph (device-side while loop)
    return case, grid, state, desc


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        out, _ = self.p.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def over_ranks(x, op, dist, device="cuda"):
    """Reduce one timing over the replicas (op = "max" or "sum"); the only
    cross-rank step of the benchmark (the data path has no collective)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def run_ours(args, rank, world, dist):
    import torch
    from desalm.solver import Solver

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    torch.cuda.init()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return over_ranks(x, "max", dist)

    def sum_over_ranks(x):
        return over_ranks(x, "sum", dist)

    def predictor_ab(n_steps=24, skip=10):
        """The three initial guesses on the laminar cavity 65^3 (MIXED, graph
        path), each physical step run to an absolute tolerance of the
        pseudo-time update: log10 mean |dq| of u, v, w below -7 (the
        reference's eo_min test; its relative er_min test is switched off,
        because it measures the drop from the guess's own first update and so
        asks more of a better guess).  Steps skip+1 .. n_steps (after the lid's
        start-up); seconds per step by CUDA events around mg_driver, training
        of the network included."""
        res = {"workload": "laminar lid-driven cavity Re=1000, 65^3, MIXED, steps %d-%d of dt=0.05, "
                           "tolerance log10 mean|dq(u,v,w)| < -7, itmax 200" % (skip + 1, n_steps)}
        for P, name, mask in ((abi.PRED_QN, "qn", None), (abi.PRED_LINEAR, "linear", None),
                              (abi.PRED_LEARNED, "learned", None), (abi.PRED_LEARNED, "learned_all_fields", 0x1f)):
            case, grid, state = cases.cavity(n=65, itmax=200)
            case.precision_mode = abi.MIXED
            case.predictor = P
            case.use_graph = 1
            case.er_min = -100.0
            case.eo_min = -7.0
            S = Solver(case)
            S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
            S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
            if mask is not None:
                S.lp_fields(mask)
            stream = torch.cuda.ExternalStream(S.stream())
            its, secs = [], []
            for k in range(n_steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                S.sync()
                e0.record(stream)
                r = S.mg_driver()
                e1.record(stream)
                S.sync()
                torch.cuda.synchronize()
                if k >= skip:
                    its.append(r["iterations"])
                    secs.append(e0.elapsed_time(e1) / 1e3)
            entry = {"iterations_per_step": its, "mean_iterations": float(np.mean(its)),
                     "s_per_step": float(np.mean(secs))}
            if P == abi.PRED_LEARNED:
                entry["network"] = S.lp_report()
                entry["fields_corrected"] = "p, u, v, w, nu_tilde" if mask == 0x1f else "p, nu_tilde (default)"
                lin = res["linear"]["iterations_per_step"]
                d = np.array(its, float) - np.array(lin, float)
                entry["vs_linear_paired"] = {"mean_iteration_difference": float(d.mean()),
                                             "standard_error": float(d.std(ddof=1) / np.sqrt(len(d))),
                                             "steps_with_fewer_iterations": int((d < 0).sum()), "steps": len(d)}
            res[name] = entry
            del S
        return res

    def option_cost(case, grid, state, variants, kernel_class, rounds=3, steps=1):
        """Seconds per physical step of one case under several options, each
        variant a (setup(solver), case edit) pair on its own solver.  The
        variants are timed in turn, rounds times, and each keeps its fastest
        round, so that a drift of the box between runs does not pose as the
        option's cost.  One profiled (eager) step of the last variant gives
        kernel_class's time per pseudo-iteration."""
        solvers = {}
        for name, (setup, edit) in variants.items():
            c = case.copy()
            edit(c)
            S = Solver(c)
            S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
            S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
            setup(S)
            S.mg_driver()
            solvers[name] = S
        best = {}
        for _ in range(rounds):
            for name, S in solvers.items():
                sec, reps = timed_steps(S, steps, S.mg_driver)
                its = float(np.mean([r["iterations"] for r in reps]))
                if name not in best or sec < best[name]["s_per_step"]:
                    best[name] = {"s_per_step": sec, "pseudo_iterations_per_step": its,
                                  "ms_per_iteration": 1e3 * sec / its}
        S = solvers[list(variants)[-1]]
        S.profile(True)
        r = S.mg_driver()
        stats, _ = S.kernel_stats()
        S.profile(False)
        ms = sum(v[0] for v in stats.get(kernel_class, {}).values())
        best["kernel_ms_per_iteration"] = ms / max(1, r["iterations"])
        best["method"] = "fastest of %d alternating rounds of %d step(s) per variant" % (rounds, steps)
        solvers.clear()
        return best

    def alm_cost():
        """Actuator-line forcing (rhs_lines) on the SA channel 129x97x65 (MIXED,
        graph path) with three seeded synthetic rotors, with and without the
        forcing; the forcing kernels' time per pseudo-iteration."""
        case, grid, state, spec = cases.channel_alm(im=129, jm=97, km=65, n_tur=3, itmax=400)
        case.precision_mode = abi.MIXED
        case.predictor = abi.PRED_LINEAR
        case.use_graph = 1
        res = option_cost(case, grid, state, {"without": (lambda S: None, lambda c: None),
                                               "with": (lambda S: S.alm_set(spec), lambda c: None)}, "alm")
        res["workload"] = ("SA channel 129x97x65, MIXED, 3 synthetic rotors (3 blades x 12 elements, %d kernel nodes)"
                           % sum(len(T["ker_index"]) for T in spec["turbines"]))
        return res

    def outlet_cost():
        """Characteristics outlet (btype 5) on the SA wake box 129x97x65 (MIXED,
        graph path), against a first-order extrapolation exit (btype 3) on the
        same grid and state; the outlet kernel's time per pseudo-iteration."""
        case, grid, state = cases.wake(im=129, jm=97, km=65, turbulence=1, itmax=200)
        case.precision_mode = abi.MIXED
        case.predictor = abi.PRED_LINEAR
        case.use_graph = 1

        def exit_as(bt):
            def edit(c):
                c.btype[1] = bt
            return edit
        res = option_cost(case, grid, state, {"extrapolation_exit": (lambda S: None, exit_as(abi.BC_FREESTREAM)),
                                              "outlet": (lambda S: None, exit_as(abi.BC_OUTLET))}, "outlet")
        res["workload"] = "SA wake box 129x97x65, MIXED, uniform inflow, outlet at i = im, itmax 200"
        return res

    def wallfn_cost():
        """Wall functions (wf_eta after every fine DAF step) on the SA channel
        129x97x65 with a first wall spacing of 0.08 (layer 2 in the log law),
        MIXED, graph path, with and without them; the kernel's time per
        pseudo-iteration."""
        case, grid, state = cases.channel(im=129, jm=97, km=65, wall_first=0.08, itmax=200)
        case.precision_mode = abi.MIXED
        case.predictor = abi.PRED_LINEAR
        case.use_graph = 1

        def wf(on):
            def edit(c):
                c.wall_functions = on
            return edit
        res = option_cost(case, grid, state, {"without": (lambda S: None, wf(0)), "with": (lambda S: None, wf(1))},
                          "wallfn")
        res["workload"] = "SA channel 129x97x65, first wall spacing 0.08, MIXED, itmax 200"
        return res

    def batched_blocks(rounds=3):
        """Eight independent blocks of uneven sizes (33^3, 2 x 49x49x33,
        65x49x49, 2 x 97x65x65, 129x65x65, 161x97x65: 2,730,248 nodes), each
        an open wake box with 5% seeded inflow noise, SA, MIXED, graph path,
        itmax 100: wall-seconds for one physical step of all blocks, stepped
        one after another (desalm_mg_driver each) and together
        (desalm_mg_driver_batch).  Fastest of alternating rounds; each
        round's blocks start from the same state."""
        from desalm.solver import mg_driver_batch
        shapes = [(33, 33, 33), (49, 49, 33), (49, 49, 33), (65, 49, 49), (97, 65, 65), (97, 65, 65),
                  (129, 65, 65), (161, 97, 65)]
        built = []
        for b, (im, jm, km) in enumerate(shapes):
            case, grid, state = cases.wake(im=im, jm=jm, km=km, turbulence=1, seed=b, itmax=100, noise=0.05)
            case.precision_mode = abi.MIXED
            case.predictor = abi.PRED_LINEAR
            case.use_graph = 1
            built.append((case, grid, state))

        def fresh():
            out = []
            for case, grid, state in built:
                S = Solver(case)
                S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
                S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
                out.append(S)
            return out
        seq, bat = fresh(), fresh()
        for S in seq:          # graph capture and warm-up, outside the timing
            S.mg_driver()
        mg_driver_batch(bat)
        best = {"one_after_another": None, "batched": None}
        its = None
        for _ in range(rounds):
            for group in (seq, bat):
                for S, (_, _, st) in zip(group, built):
                    S.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
            t0 = time.perf_counter()
            reps = [S.mg_driver() for S in seq]
            t1 = time.perf_counter()
            repb = mg_driver_batch(bat)
            t2 = time.perf_counter()
            its = [r["iterations"] for r in repb]
            assert [r["iterations"] for r in reps] == its
            for name, t in (("one_after_another", t1 - t0), ("batched", t2 - t1)):
                if best[name] is None or t < best[name]:
                    best[name] = t
        nodes = sum(a * b * c for a, b, c in shapes)
        return {"workload": "8 wake blocks %s, %d nodes, SA, MIXED, itmax 100" % (shapes, nodes),
                "s_per_step_one_after_another": best["one_after_another"],
                "s_per_step_batched": best["batched"],
                "speedup": best["one_after_another"] / best["batched"],
                "pseudo_iterations_per_block": its,
                "timing": "host wall clock around the whole step of all blocks (each call ends synchronised); "
                          "fastest of %d alternating rounds" % rounds}

    def timed_steps(S, K, body):
        """K calls of body(), bracketed by barrier + synchronize, CUDA events
        on the library's stream; returns seconds per call (max over ranks)."""
        stream = torch.cuda.ExternalStream(S.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        S.sync()
        torch.cuda.synchronize()
        e0.record(stream)
        reps = []
        for _ in range(K):
            reps.append(body())
        e1.record(stream)
        S.sync()
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3 / K), reps

    # ---- product configuration: MIXED + linear extrapolation
    case, grid, state, desc = build_case(args.case, abi.MIXED, abi.PRED_LINEAR)
    nint = (case.im - 2) * (case.jm - 2) * (case.km - 2)
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    widths = S.sweep_widths()[:case.ng].tolist()
    for _ in range(args.warmup):
        S.mg_driver()
    clk = Clocks(dev)
    clk.start()
    S.profile(False)
    S.profile(False)  # resets the launch counter
    sec, reps = timed_steps(S, args.steps, S.mg_driver)
    clocks = clk.stop()
    _, launches = S.kernel_stats()
    iters = [r["iterations"] for r in reps]
    conv = [r["converged"] for r in reps]

    # ---- e2e through the C ABI with host buffers (pinned), H2D + D2H per step
    N = case.im * case.jm * case.km
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    hq, hqn, hqnm1, hnut = pin(5 * N), pin(5 * N), pin(5 * N), pin(N)
    st = S.get_state()
    hq[:], hqn[:], hqnm1[:], hnut[:] = st["q"], st["qn"], st["qnm1"], st["nut"]
    import ctypes as C
    L = S.L
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))

    def e2e_step():
        S._ck(L.desalm_set_state(S.ctx, P(hq), P(hqn), P(hqnm1), P(hnut)), "set_state")
        r = S.mg_driver()
        S._ck(L.desalm_get_state(S.ctx, P(hq), P(hqn), P(hqnm1), P(hnut)), "get_state")
        return r

    e2e_sec, _ = timed_steps(S, args.steps, e2e_step)
    h2d = (3 * 5 * N + N) * 8
    d2h = (3 * 5 * N + N) * 8

    # ---- per-kernel CUDA-event timing over the same workload (roofline)
    S.profile(True)
    for _ in range(args.steps):
        S.mg_driver()
    stats, _ = S.kernel_stats()
    S.profile(False)
    T = {1: 8, 2: 8, 3: 8, 4: 8}      # MIXED: FP64 state on every level
    W = {1: 4, 2: 4, 3: 4, 4: 4}      # FP32 line-sweep work
    best = None
    for kind, per in stats.items():
        ms = sum(v[0] for v in per.values())
        if best is None or ms > best[1]:
            best = (kind, ms, per)
    kind, ms_tot, per = best
    # roofline of the dominant class on its fine-level launches (the ones the
    # ncu traffic figures in profiles/ describe)
    ms_sum, nlaunch, nodes = per[1]
    byts = (alg_bytes(kind, T[1], W[1], False) or 0) * nodes
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = byts / (ms_sum / 1e3) / 1e9 if ms_sum > 0 else 0.0
    share = {k: round(sum(v[0] for v in p.values()) / max(1e-9, sum(sum(w[0] for w in q.values()) for q in stats.values())), 4)
             for k, p in stats.items()}
    # every class with an algorithmic-byte count, on its fine-level launches
    by_kernel = {}
    for k, p in stats.items():
        b1 = alg_bytes(k, T[1], W[1], False)
        if not b1 or 1 not in p or p[1][0] <= 0:
            continue
        ms1, n1, nodes1 = p[1]
        gbs = b1 * nodes1 / (ms1 / 1e3) / 1e9
        by_kernel[k] = {"achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
                        "avg_launch_us": round(1e3 * ms1 / max(1, n1), 2), "alg_bytes_per_node": b1}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get(args.case, {}).get(kind)
    del S

    # ---- plain FP64 GPU path (q^n guess, as the reference's mg_driver)
    case64, grid, state, _ = build_case(args.case, abi.FP64, abi.PRED_QN)
    S64 = Solver(case64)
    S64.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S64.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    for _ in range(args.warmup):
        S64.mg_driver()
    sec64, reps64 = timed_steps(S64, args.steps, S64.mg_driver)
    iters64 = [r["iterations"] for r in reps64]
    st64 = S64.get_state()
    del S64

    # ---- per-field error of the mixed path against the FP64 path: MIXED with
    # the same q^n guess, the same number of physical steps from the same state
    caseq, _, _, _ = build_case(args.case, abi.MIXED, abi.PRED_QN)
    SQ = Solver(caseq)
    SQ.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    SQ.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    for _ in range(args.warmup + args.steps):
        SQ.mg_driver()
    stq = SQ.get_state()
    del SQ
    a = np.asarray(stq["q"]).reshape(-1, 5)
    b = np.asarray(st64["q"]).reshape(-1, 5)
    names = ["p", "u", "v", "w", "nu_tilde"] if case.turbulence else ["p", "u", "v", "w"]
    field_err = {nm: float(np.linalg.norm(a[:, m] - b[:, m]) / max(1e-300, np.linalg.norm(b[:, m])))
                 for m, nm in enumerate(names)}

    # one-GPU characterisations (initial guesses, option costs, batching):
    # run once, not on every replica of a multi-GPU run
    extra = not args.no_ab and world == 1
    ab = predictor_ab() if extra else None
    alm = alm_cost() if extra else None
    outlet = outlet_cost() if extra else None
    wallfn = wallfn_cost() if extra else None
    batched = batched_blocks() if extra else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.case, max(1, int(np.mean(iters64))))

    cell_updates = nint * float(np.mean(iters)) / sec
    out = {
        "metric": METRIC, "value": sec, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded numpy generator; the reference ships no grids or solutions)",
        "impl": "ours",
        "config": {"workload": desc, "case": args.case, "grid": [case.im, case.jm, case.km],
                   "interior_nodes": nint, "precision": "mixed (FP64 state, residual, restriction, update and norm on every level; FP32 line-sweep work, modal transforms and SA ADI)",
                   "predictor": "linear extrapolation",
                   "learned_predictor": "built (predictor DESALM_PRED_LEARNED); compared in predictor_ab",
                   "pseudo_iterations_per_step": iters, "converged": conv,
                   "l2": "working set of every level > 126 MB L2 for the channel; no flush between steps",
                   "parallelism": "replicas only (%d independent replicas)" % world,
                   "sweep_lines_per_cta": {"levels_x_ijk": widths,
                                           "how": "timed per level and direction when the grid is set "
                                                  "(0 = shared-memory rule, DESALM_AUTOTUNE=0)"}},
        "fp64_plain": {"value": sec64, "unit": UNIT, "pseudo_iterations_per_step": iters64,
                       "speedup_mixed_vs_fp64": sec64 / sec},
        "mixed_vs_fp64_rel_l2": {"fields": field_err,
                                 "how": "relative L2 over all nodes of the state after %d physical steps from the same "
                                        "initial state, both with the q^n guess" % (args.warmup + args.steps)},
        "cell_updates_per_s": sum_over_ranks(cell_updates),
        "predictor_ab": ab,
        "alm": alm,
        "outlet": outlet,
        "wall_functions": wallfn,
        "batched_blocks": batched,
        "e2e": {"value": e2e_sec, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": kind, "level": "fine", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": byts / max(1, nlaunch), "launches": nlaunch,
                     "avg_launch_ms": ms_sum / max(1, nlaunch),
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"},
        "kernel_time_share": share,
        "roofline_by_kernel": by_kernel,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    return out


def cpu_baseline(case_name, iters_per_step, budget_s=20.0):
    """The CPU oracle in FP32 (the reference's precision) on every host
    thread its OpenMP loops can use: a bounded sample of pseudo-iterations,
    scaled to one physical step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    case, grid, state, _ = build_case(case_name, abi.FP64, abi.PRED_QN)
    o = oracle.OracleSolver(case, 4)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    o.begin_step()
    t0 = time.perf_counter()
    k = 0
    while True:
        o.pseudo_iteration()
        k += 1
        if time.perf_counter() - t0 > budget_s or k >= iters_per_step:
            break
    per_it = (time.perf_counter() - t0) / k
    nth = oracle.threads()
    return {"value": per_it * iters_per_step, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": "%d pseudo-iterations of the first physical step (%.2f s each, FP32 oracle, %d threads), "
                      "scaled by the %d pseudo-iterations the FP64 GPU path needed per step"
                      % (k, per_it, nth, iters_per_step)}


def run_reference(args):
    """--impl reference: the oracle (CPU port of the reference) on this case."""
    iters = {"cavity": 200}.get(args.case)
    if iters is None:
        iters = REF_ITERS.get(args.case, 200)
    vals = []
    for _ in range(args.warmup + args.steps):
        cb = cpu_baseline(args.case, iters, budget_s=max(5.0, 60.0 / max(1, args.steps + args.warmup)))
        vals.append(cb)
    v = float(np.mean([c["value"] for c in vals[args.warmup:]]))
    cb = vals[-1]
    cb["value"] = v
    _, _, _, desc = build_case(args.case, abi.FP64, abi.PRED_QN)
    # n_gpus: the N this arm was launched with, as the arm it is compared
    # with; the work runs on rank 0's host cores
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "case": args.case, "device": "host cores of rank 0 (no GPU)"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# pseudo-iterations per physical step of the FP64 path (q^n guess) on each
# case, as measured on the GPU path whose iterates follow the oracle's
# (used only to scale the reference arm's bounded CPU sample)
REF_ITERS = {"cavity": 200, "channel": 400}


def ncu_workload(case_name, precision, learned=False):
    """A short, eager run for Nsight Compute captures: the case's setup, the
    start of a physical step and one pseudo-iteration, without CUDA graphs
    (so every kernel is a separate, capturable launch).  learned: instead,
    four physical steps of two pseudo-iterations with the learned guess, so
    that steps 2-4 train the network and steps 3-4 start from its guess."""
    from desalm.solver import Solver
    case, grid, state, _ = build_case(case_name, precision, abi.PRED_LEARNED if learned else abi.PRED_LINEAR)
    case.use_graph = 0
    if learned:
        case.itmax = 2
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    if learned:
        for _ in range(4):
            S.mg_driver()
    else:
        S.begin_step()
        S.pseudo_iteration()
    S.sync()
    print(json.dumps({"ncu_workload": case_name, "precision": precision, "learned": learned}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--case", default="channel", choices=["cavity", "channel", "wake"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ab", action="store_true", help="skip the initial-guess and forcing sections")
    ap.add_argument("--ncu-workload", action="store_true",
                    help="run one eager pseudo-iteration of --case for an ncu capture and exit")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--learned", action="store_true", help="with --ncu-workload: learned-guess steps")
    args = ap.parse_args()
    if args.ncu_workload:
        ncu_workload(args.case, abi.MIXED if args.precision == "mixed" else abi.FP64, args.learned)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as td
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = td
    out = run_ours(args, rank, world, dist)
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
