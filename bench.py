#!/usr/bin/env python
"""Benchmark of the B200 pseudo-time iteration: wall-seconds per physical time
step of dual time stepping, each step run to the convergence test of the
reference's mg_ck_conver, one replica per GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--case turbine|channel|cavity]
                  [--model kw|sa] [--impl ours|reference] [--extras]

Workload (default): the actuator-line turbine box of 385 x 193 x 193 nodes
(10 D x 5 D x 5 D, sinh-clustered at the rotor; a 3-blade rotor of D = 1, TSR
7, Gaussian projection eps = 0.05 D, seeded synthetic polars; uniform inflow,
characteristics outlet, symmetry side faces), Re_D = 1e5, dt = 0.005 D/U,
3-level FAS, with the k-omega model (--model kw; --model sa for
Spalart-Allmaras).  The rotor advances by omega dt between physical steps.

Convergence test (mg_ck_conver, src/mg_driver.F90:372-398): after it_min = 7
pseudo-iterations, stop when the largest of the u, v, w updates has dropped
by 6 decades from the step's first update (er_min = -6, the 1e-6 drop) or is
below 10^-7.5 in absolute terms (eo_min = -7.5, the reference's own input
deck, ind3dmg.dat:4); at most 400 pseudo-iterations.  On this method the
relative drop slows to about 0.15 decades per 100 iterations after the first
ones (the CPU oracle shows the same rate), so the absolute test is the one
that ends the steps; the line reports which test ended each step.

ours:       value = device-timed seconds per physical step of the learned,
            mixed-precision path (FP64 state, residual, restriction, update and
            norm; FP32 line sweeps, modal transforms and turbulence ADI; the
            network's initial guess), state resident in HBM, K steps after W
            warm-up steps.  On the same physical steps: the plain FP64 path
            (linear extrapolation, the plain guess) and FP64 with the
            reference's q^n guess, and MIXED with linear extrapolation (what
            the network adds).  e2e = the learned mixed step through the C ABI
            with the state copied from pinned host memory and back every step.
reference:  the CPU oracle (C++ restatement of the reference, FP64, its loops
            on every host thread), the reference's own method (q^n guess), on
            the same workload: one whole physical step, run to the same
            convergence test.

Under torchrun each rank runs an independent replica on its own GPU (the
path does not shard: no collective in the data path); times are the max
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
CRITERION = {"it_min": 7, "er_min": -6.0, "eo_min": -7.5, "itmax": 400}
SECONDARY_STEPS = 3     # timed steps of each comparison variant (after the same W warm-up steps)


# Algorithmic bytes per interior node of each kernel class: every distinct
# array element the kernel must read or write once, at its stored precision
# (T = state bytes, W = line-sweep work bytes).  Halo re-reads and the
# line-solve scratch are not algorithmic.
def alg_bytes(kind, T, W, coarse, model="sa"):
    pk = 4 * T if coarse else 0
    turb_rhs = (22 * 8 + 10 * W) if model == "sa" else (27 * 8 + 20 * W)
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
        # SA: q5 qn5 qnm1-5, U/J 3, metrics9, aj, 1/aj, wd, wo, dtev | rh, ADI rows 9
        # k-omega: k w kn km1 wn wm1 u v w U/J3 metrics9 aj nut ptke As Ac Bs dtev | rh2 rows18
        "sa_rhs": turb_rhs,
        "sa_sweep": 5 * W + 8,            # ADI row 3, rh in/out; k sweep: scalar in/out, dtev (1/3 each)
    }.get(kind)


def build_case(name, precision, predictor, model="kw", small=False):
    """(case, grid, state, omega, alm spec, rotor rate, description); small:
    the turbine box at 193 x 97 x 97 (profiler captures)."""
    omega, spec, rate = None, None, 0.0
    if name == "turbine":
        dims = dict(im=193, jm=97, km=97) if small else {}
        case, grid, state, spec, rate = cases.turbine(itmax=CRITERION["itmax"], **dims)
        desc = ("actuator-line turbine box 385x193x193 (10Dx5Dx5D, sinh-clustered), 3-blade rotor D=1, TSR 7, "
                "eps=0.05D, seeded polars, inflow/characteristics outlet/symmetry, Re_D=1e5, dt=0.005 D/U, "
                "3-level FAS, %s" % ("k-omega (Wilcox 1994)" if model == "kw" else "Spalart-Allmaras"))
        if model == "kw":
            case, grid, state, omega = cases.with_kw(case, grid, state)
    elif name == "cavity":
        case, grid, state = cases.cavity(n=65, itmax=200)
        desc = "laminar lid-driven cavity Re=1000, 65^3 perturbed cube, 3-level FAS"
    elif name == "channel":
        case, grid, state = cases.channel()
        desc = "SA RANS channel Re_tau=395, 129x97x65 tanh-stretched, periodic i/k, 3-level FAS"
    elif name == "ogrid":
        case, grid, state = cases.ogrid()
        desc = ("SA-DES cylinder O-grid 257x129x65 (radial geometric stretching to 20D, span pi D), Re=3900, "
                "dt=0.005 D/U, impulsive start, 3-level FAS")
    else:
        raise SystemExit("unknown case " + name)
    case.it_min = CRITERION["it_min"]
    case.er_min = CRITERION["er_min"]
    case.eo_min = CRITERION["eo_min"]
    case.itmax = CRITERION["itmax"]
    case.precision_mode = precision
    case.predictor = predictor
    case.use_graph = 1      # each physical step replays one CUDA graph (device-side while loop)
    return case, grid, state, omega, spec, rate, desc


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


def which_test(rep):
    """Which mg_ck_conver test ended a step: 'drop' (er_min), 'absolute'
    (eo_min), or 'cap' (itmax reached unconverged)."""
    r = np.array(rep["residual"])
    r0 = np.array(rep["init_residual"])
    if not rep["converged"]:
        return "cap"
    if (r - r0)[1:4].max() < CRITERION["er_min"]:
        return "drop"
    return "absolute"


class Workload:
    """One solver on the bench workload, with the rotor advanced between
    physical steps (src/main.F90:42-50)."""

    def __init__(self, name, precision, predictor, model, lp_mask=None):
        from desalm.solver import Solver
        (self.case, grid, state, omega, self.spec, self.rate, self.desc) = build_case(name, precision, predictor, model)
        self.S = Solver(self.case)
        self.S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        self.S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        if omega is not None:
            self.S.set_omega(omega["omega"], omega["omega_n"], omega["omega_nm1"])
        if lp_mask is not None:
            self.S.lp_fields(lp_mask)
        self.angle = None
        if self.spec is not None:
            self.S.alm_set(self.spec)
            self.angle = self.spec["turbines"][0]["angle"]
        self.nint = (self.case.im - 2) * (self.case.jm - 2) * (self.case.km - 2)

    def step(self):
        r = self.S.mg_driver()
        if self.angle is not None:
            self.angle += self.rate * self.case.delti
            self.S.alm_set_angle(1, self.angle)
        return r

    def close(self):
        self.S.close()


def timed(S, K, body, barrier, max_over_ranks):
    """K calls of body(), bracketed by barrier + synchronize, CUDA events on
    the library's stream around each; returns (seconds per call over the K
    calls, max over ranks; the calls' results; per-call seconds)."""
    import torch
    stream = torch.cuda.ExternalStream(S.stream())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    barrier()
    S.sync()
    torch.cuda.synchronize()
    ev[0].record(stream)
    reps = []
    for k in range(K):
        reps.append(body())
        ev[k + 1].record(stream)
    S.sync()
    torch.cuda.synchronize()
    barrier()
    per = [ev[k].elapsed_time(ev[k + 1]) / 1e3 for k in range(K)]
    return max_over_ranks(sum(per) / K), reps, per


def steps_summary(reps, per):
    return {"pseudo_iterations_per_step": [r["iterations"] for r in reps],
            "ended_by": [which_test(r) for r in reps],
            "drop_reached": [round(float((np.array(r["residual"]) - np.array(r["init_residual"]))[1:4].max()), 3)
                             for r in reps],
            "s_per_step_each": [round(p, 4) for p in per],
            "pivot_rows": int(sum(r["pivots"] for r in reps)),
            "pivot_line_systems": int(sum(r.get("pivot_lines", 0) for r in reps))}


def run_ours(args, rank, world, dist):
    import torch

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

    K, W = args.steps, max(1, args.warmup)
    KS = min(K, SECONDARY_STEPS)

    # ---- the learned, mixed-precision path (the headline)
    wl = Workload(args.case, abi.MIXED, abi.PRED_LEARNED, args.model)
    S = wl.S
    for _ in range(W):
        wl.step()
    clk = Clocks(dev)
    clk.start()
    S.profile(False)  # resets the launch counter
    sec, reps, per = timed(S, K, wl.step, barrier, max_over_ranks)
    clocks = clk.stop()
    _, launches = S.kernel_stats()
    lp = S.lp_report()
    head = steps_summary(reps, per)

    # ---- per-kernel CUDA-event timing of one more step (eager, profiled)
    S.profile(True)
    rprof = wl.step()
    stats, _ = S.kernel_stats()
    S.profile(False)
    case = wl.case
    wl.close()
    torch.cuda.empty_cache()

    # ---- e2e through the C ABI with host buffers (pinned), H2D + D2H per
    # step, on a second instance of the same path over the comparison steps
    # (W warm-up steps, then KS timed)
    wl = Workload(args.case, abi.MIXED, abi.PRED_LEARNED, args.model)
    S = wl.S
    for _ in range(W):
        wl.step()
    # ---- e2e through the C ABI with host buffers (pinned), H2D + D2H per step
    import ctypes as C
    N = case.im * case.jm * case.km
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    # one pinned host array per field (q, q^n, q^{n-1} of the five components,
    # nu_t): desalm_set_field / desalm_get_field move the state without
    # touching the learned guess's history, so the network keeps training as
    # in the headline run (desalm_set_state would start a new history)
    bases = (abi.F_Q, abi.F_QN, abi.F_QNM1)
    hf = [[pin(N) for _ in range(5)] for _ in bases]
    for a, fb in enumerate(bases):
        for m in range(5):
            hf[a][m][:] = S.get_field(1, fb + m)
    hnut = pin(N)
    hnut[:] = S.get_field(1, abi.F_NUT)
    kw = case.turbulence == 2
    hw = [pin(N) for _ in range(3)] if kw else None
    if kw:
        om = S.get_omega()
        hw[0][:], hw[1][:], hw[2][:] = om["omega"], om["omega_n"], om["omega_nm1"]
    L = S.L
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))

    copy_s = []

    def e2e_step():
        t0 = time.perf_counter()
        for a, fb in enumerate(bases):
            for m in range(5):
                S._ck(L.desalm_set_field(S.ctx, 1, fb + m, P(hf[a][m])), "set_field")
        S._ck(L.desalm_set_field(S.ctx, 1, abi.F_NUT, P(hnut)), "set_field")
        if kw:
            S._ck(L.desalm_set_omega(S.ctx, P(hw[0]), P(hw[1]), P(hw[2])), "set_omega")
        t1 = time.perf_counter()
        r = wl.step()
        S.sync()
        t2 = time.perf_counter()
        for a, fb in enumerate(bases):
            for m in range(5):
                S._ck(L.desalm_get_field(S.ctx, 1, fb + m, P(hf[a][m])), "get_field")
        S._ck(L.desalm_get_field(S.ctx, 1, abi.F_NUT, P(hnut)), "get_field")
        if kw:
            S._ck(L.desalm_get_omega(S.ctx, P(hw[0]), P(hw[1]), P(hw[2])), "get_omega")
        t3 = time.perf_counter()
        copy_s.append((t1 - t0) + (t3 - t2))
        return r

    e2e_sec, e2e_reps, e2e_per = timed(S, KS, e2e_step, barrier, max_over_ranks)
    nbytes = (3 * 5 * N + N + (3 * N if kw else 0)) * 8

    wl.close()
    torch.cuda.empty_cache()

    T = {1: 8, 2: 8, 3: 8, 4: 8}      # MIXED: FP64 state on every level
    Wb = {1: 4, 2: 4, 3: 4, 4: 4}     # FP32 line-sweep work
    best = None
    for kind_, per_ in stats.items():
        ms = sum(v[0] for v in per_.values())
        if best is None or ms > best[1]:
            best = (kind_, ms, per_)
    kind, ms_tot, perk = best
    ms_sum, nlaunch, nodes = perk[1]
    byts = (alg_bytes(kind, T[1], Wb[1], False, args.model) or 0) * nodes
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = byts / (ms_sum / 1e3) / 1e9 if ms_sum > 0 else 0.0
    tot_ms = sum(sum(w[0] for w in q.values()) for q in stats.values())
    share = {k: round(sum(v[0] for v in p.values()) / max(1e-9, tot_ms), 4) for k, p in stats.items()}
    by_kernel = {}
    for k, p in stats.items():
        b1 = alg_bytes(k, T[1], Wb[1], False, args.model)
        if not b1 or 1 not in p or p[1][0] <= 0:
            continue
        ms1, n1, nodes1 = p[1]
        gbs = b1 * nodes1 / (ms1 / 1e3) / 1e9
        by_kernel[k] = {"achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4),
                        "avg_launch_us": round(1e3 * ms1 / max(1, n1), 2), "alg_bytes_per_node": b1}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        traffic = json.load(open(tfile)).get("%s_%s" % (args.case, args.model), {}).get(kind)

    # ---- the comparison paths on the same physical steps (W warm-up, KS timed)
    variants = {}
    finals = {}
    for name, prec, pred, mask in (("fp64_plain", abi.FP64, abi.PRED_LINEAR, None),
                                   ("fp64_qn", abi.FP64, abi.PRED_QN, None),
                                   ("mixed_linear", abi.MIXED, abi.PRED_LINEAR, None),
                                   ("learned_p_corrected", abi.MIXED, abi.PRED_LEARNED, 1)):
        v = Workload(args.case, prec, pred, args.model, lp_mask=mask)
        _, wreps, wper = timed(v.S, W, v.step, barrier, max_over_ranks)
        vsec, vreps, vper = timed(v.S, KS, v.step, barrier, max_over_ranks)
        variants[name] = dict({"value": vsec, "unit": UNIT, "steps": "%d-%d" % (W + 1, W + KS)}, **steps_summary(vreps, vper))
        variants[name]["step1"] = {"s": wper[0], "pseudo_iterations": wreps[0]["iterations"],
                                   "ended_by": which_test(wreps[0])}
        if name in ("fp64_plain", "mixed_linear"):
            finals[name] = v.S.get_state()["q"]
        v.close()
        torch.cuda.empty_cache()
    variants["fp64_plain"]["guess"] = "linear extrapolation (the plain guess)"
    variants["fp64_qn"]["guess"] = "q^n (the reference's mg_driver)"
    variants["mixed_linear"]["guess"] = "linear extrapolation"
    variants["learned_p_corrected"]["guess"] = ("learned, the network's correction applied to p (desalm_lp_fields(1)) "
                                                "with the automatic blend")
    a = np.asarray(finals["mixed_linear"]).reshape(-1, 5)
    b = np.asarray(finals["fp64_plain"]).reshape(-1, 5)
    names = ["p", "u", "v", "w", "k" if kw else "nu_tilde"]
    field_err = {nm: float(np.linalg.norm(a[:, m] - b[:, m]) / max(1e-300, np.linalg.norm(b[:, m])))
                 for m, nm in enumerate(names)}

    extra = args.extras and world == 1
    extras = run_extras(barrier, max_over_ranks) if extra else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.case, args.model, max(1, variants["fp64_qn"]["step1"]["pseudo_iterations"]))

    same = float(np.mean(per[:KS]))   # the headline path on the comparison steps
    mean_its = float(np.mean(head["pseudo_iterations_per_step"]))
    cell_updates = wl.nint * mean_its / sec
    out = {
        "metric": METRIC, "value": sec, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": sec * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
        "data": "synthetic (seeded numpy generator; the reference ships no grids or solutions)",
        "impl": "ours",
        "config": {"workload": wl.desc, "case": args.case, "model": args.model, "grid": [case.im, case.jm, case.km],
                   "interior_nodes": wl.nint,
                   "precision": "mixed (FP64 state, residual, restriction, update and norm on every level; FP32 line "
                                "sweeps, modal transforms and turbulence ADI)",
                   "predictor": "learned: 3D conv network trained online on the GPU (its Adam steps overlapped with "
                                "the physical step); the guess is linear extrapolation plus the blended correction "
                                "of the fields in the library's default mask, which is none (every correction "
                                "measured raised the pseudo-iterations: see learned_p_corrected)",
                   "convergence": "mg_ck_conver: after it_min=7, u,v,w update drop below 1e-6 of the step's first "
                                  "(er_min=-6) or below 10^-7.5 absolute (eo_min=-7.5, the reference deck "
                                  "ind3dmg.dat:4); itmax 400",
                   "steps_timed": "%d-%d" % (W + 1, W + K),
                   "l2": "working set of every level > 126 MB L2; no flush between steps",
                   "parallelism": "replicas only (%d independent replicas)" % world,
                   "batching": "one block (the overset blocks of the reference exchange donor data; not built)"},
        "steps_detail": head,
        "network": lp,
        "fp64_plain": variants["fp64_plain"],
        "fp64_qn": variants["fp64_qn"],
        "mixed_linear": variants["mixed_linear"],
        "learned_p_corrected": variants["learned_p_corrected"],
        "learned_mixed_on_comparison_steps": {"value": same, "unit": UNIT, "steps": "%d-%d" % (W + 1, W + KS),
                                              "pseudo_iterations_per_step": head["pseudo_iterations_per_step"][:KS]},
        "speedup_vs_fp64_plain": variants["fp64_plain"]["value"] / same,
        "speedup_how": "plain FP64 over the learned mixed path on the same physical steps %d-%d" % (W + 1, W + KS),
        "mixed_vs_fp64_rel_l2": {"fields": field_err,
                                 "how": "relative L2 over all nodes after %d physical steps from the same state, "
                                        "MIXED and FP64 both with linear extrapolation (the FP64 GPU path equals "
                                        "the FP64 oracle to 1e-10 at this size: tests/test_gpu_fullsize.py)" % (W + KS)},
        "cell_updates_per_s": sum_over_ranks(cell_updates),
        "e2e": {"value": e2e_sec, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                "steps": "%d-%d" % (W + 1, W + KS), "pseudo_iterations_per_step": [r["iterations"] for r in e2e_reps],
                "copy_s_per_step": float(np.mean(copy_s)) if copy_s else None,
                "note": "a second instance of the learned mixed path (W warm-up steps, then these), the state moved "
                        "field by field (desalm_set_field / desalm_get_field from pinned host arrays) so that the "
                        "network keeps its history and trains on every step, as in the headline run"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": kind, "level": "fine", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "alg_bytes_per_launch": byts / max(1, nlaunch), "launches": nlaunch,
                     "avg_launch_ms": ms_sum / max(1, nlaunch),
                     "measured_over": "one eager profiled step (%d pseudo-iterations)" % rprof["iterations"],
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback 6650 GB/s"},
        "kernel_time_share": share,
        "roofline_by_kernel": by_kernel,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "extras": extras,
    }
    return out


def run_extras(barrier, max_over_ranks):
    """One-GPU characterisations of the options (--extras): the initial
    guesses on the laminar cavity, and what the actuator-line forcing, the
    characteristics outlet, the wall functions and block batching cost."""
    import torch
    from desalm.solver import Solver, mg_driver_batch

    def predictor_ab(n_steps=24, skip=10):
        res = {"workload": "laminar lid-driven cavity Re=1000, 65^3, MIXED, steps %d-%d of dt=0.05, "
                           "tolerance log10 mean|dq(u,v,w)| < -7, itmax 200" % (skip + 1, n_steps)}
        for P, name, mask in ((abi.PRED_QN, "qn", None), (abi.PRED_LINEAR, "linear", None),
                              (abi.PRED_LEARNED, "learned", None)):
            case, grid, state = cases.cavity(n=65, itmax=200)
            case.precision_mode = abi.MIXED
            case.predictor = P
            case.use_graph = 1
            case.er_min = -100.0
            case.eo_min = -7.0
            S = Solver(case)
            S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
            S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
            its, secs = [], []
            for k in range(n_steps):
                s, reps, _ = timed(S, 1, S.mg_driver, barrier, max_over_ranks)
                if k >= skip:
                    its.append(reps[0]["iterations"])
                    secs.append(s)
            res[name] = {"iterations_per_step": its, "mean_iterations": float(np.mean(its)),
                         "s_per_step": float(np.mean(secs))}
            S.close()
        return res

    def option_cost(case, grid, state, variants, rounds=3):
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
                sec, reps, _ = timed(S, 1, S.mg_driver, barrier, max_over_ranks)
                its = float(reps[0]["iterations"])
                if name not in best or sec < best[name]["s_per_step"]:
                    best[name] = {"s_per_step": sec, "ms_per_iteration": 1e3 * sec / its}
        for S in solvers.values():
            S.close()
        best["method"] = "fastest of %d alternating rounds of one step per variant" % rounds
        return best

    out = {"predictor_ab": predictor_ab()}
    case, grid, state, spec = cases.channel_alm(im=129, jm=97, km=65, n_tur=3, itmax=400)
    case.precision_mode, case.predictor, case.use_graph = abi.MIXED, abi.PRED_LINEAR, 1
    out["alm"] = option_cost(case, grid, state, {"without": (lambda S: None, lambda c: None),
                                                 "with": (lambda S: S.alm_set(spec), lambda c: None)})
    case, grid, state = cases.wake(im=129, jm=97, km=65, turbulence=1, itmax=200)
    case.precision_mode, case.predictor, case.use_graph = abi.MIXED, abi.PRED_LINEAR, 1

    def exit_as(bt):
        def edit(c):
            c.btype[1] = bt
        return edit
    out["outlet"] = option_cost(case, grid, state, {"extrapolation_exit": (lambda S: None, exit_as(abi.BC_FREESTREAM)),
                                                    "outlet": (lambda S: None, exit_as(abi.BC_OUTLET))})
    shapes = [(33, 33, 33), (49, 49, 33), (49, 49, 33), (65, 49, 49), (97, 65, 65), (97, 65, 65),
              (129, 65, 65), (161, 97, 65)]
    built = []
    interior = [(im - 2) * (jm - 2) * (km - 2) for im, jm, km in shapes]
    for b, (im, jm, km) in enumerate(shapes):
        c, g, s = cases.wake(im=im, jm=jm, km=km, turbulence=1, seed=b, itmax=100)
        c.precision_mode, c.predictor, c.use_graph = abi.MIXED, abi.PRED_LINEAR, 1
        # uniform inflow plus 5% synthetic turbulence (the random flow generator)
        built.append((c, g, s, cases.rfg_inflow(c, intensity=0.05, length_scale=0.2, nmodes=1000, seed=100 + b)))

    def fresh():
        out_ = []
        for c, g, s, r in built:
            S = Solver(c)
            S.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
            S.set_state(s["q"], s["qn"], s["qnm1"], s["nut"])
            S.rfg_set(r)
            out_.append(S)
        return out_
    seq, bat = fresh(), fresh()
    for S in seq:
        S.rfg_inlet(built[0][0].delti)
        S.mg_driver()
    for S in bat:
        S.rfg_inlet(built[0][0].delti)
    mg_driver_batch(bat)
    bestb = {"one_after_another": None, "batched": None}
    its = {"one_after_another": None, "batched": None}
    for rnd in range(3):
        t_in = (rnd + 2) * built[0][0].delti
        for group in (seq, bat):
            for S, (_, _, s, _) in zip(group, built):
                S.set_state(s["q"], s["qn"], s["qnm1"], s["nut"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        reps_seq = []
        for S in seq:
            S.rfg_inlet(t_in)
            reps_seq.append(S.mg_driver())
        t1 = time.perf_counter()
        for S in bat:
            S.rfg_inlet(t_in)
        reps_bat = mg_driver_batch(bat)
        t2 = time.perf_counter()
        for nm, t, reps in (("one_after_another", t1 - t0, reps_seq), ("batched", t2 - t1, reps_bat)):
            if bestb[nm] is None or t < bestb[nm]:
                bestb[nm] = t
                its[nm] = [r["iterations"] for r in reps]
    for S in seq + bat:
        S.close()
    out["batched_blocks"] = {"workload": "8 wake blocks %s, SA, MIXED, itmax 100, inflow u = 1 plus 5%% "
                                         "synthetic turbulence (1000 modes)" % (shapes,),
                             "s_per_step_one_after_another": bestb["one_after_another"],
                             "s_per_step_batched": bestb["batched"],
                             "speedup": bestb["one_after_another"] / bestb["batched"],
                             "pseudo_iterations_per_block": its,
                             # interior-node pseudo-iterations per second of all blocks together, against the
                             # single 129x97x65 SA channel block of the "alm" comparison ("without")
                             "ns_per_node_iteration": {
                                 nm: 1e9 * bestb[nm] / sum(n_in * k for n_in, k in zip(interior, its[nm]))
                                 for nm in its}}
    ch = out["alm"]["without"]
    out["batched_blocks"]["ns_per_node_iteration"]["single_block_channel129x97x65"] = \
        1e6 * ch["ms_per_iteration"] / (127 * 95 * 63)
    return out


def run_guesses(args):
    """The initial guesses of a physical step on one workload (MIXED, each step
    to the convergence criterion): q^n (the reference's), linear
    extrapolation, the learned guess with the library's defaults (no field
    corrected), and the learned guess correcting p and nu_tilde (mask 17).
    Each runs from the same seeded start on its own context; steps after the
    first --warmup are reported (pseudo-iterations and device seconds)."""
    from desalm.solver import DesalmError, Solver

    def noop():
        pass
    res = {"section": "initial_guesses", "criterion": dict(CRITERION), "steps": args.guesses,
           "reported_from_step": args.warmup + 1}
    for name, pred, mask in (("qn", abi.PRED_QN, None), ("linear", abi.PRED_LINEAR, None),
                             ("learned", abi.PRED_LEARNED, None), ("learned_p_nut", abi.PRED_LEARNED, 17)):
        case, grid, state, omega, spec, rate, desc = build_case(args.case, abi.MIXED, pred, args.model)
        res["workload"] = desc
        S = Solver(case)
        S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        if omega is not None:
            S.set_omega(omega["omega"], omega["omega_n"], omega["omega_nm1"])
        if mask is not None:
            S.lp_fields(mask)
        its, secs, failed, reps = [], [], None, None
        for k in range(args.guesses):
            try:
                sec, reps, _ = timed(S, 1, S.mg_driver, noop, lambda x: x)
            except DesalmError as e:   # e.g. a non-finite norm: the step's failure is the result
                failed = {"step": k + 1, "error": str(e)}
                break
            its.append(reps[0]["iterations"])
            secs.append(sec)
        w = args.warmup
        res[name] = {"iterations_per_step": its,
                     "mean_iterations": float(np.mean(its[w:])) if len(its) > w else None,
                     "s_per_step": float(np.mean(secs[w:])) if len(secs) > w else None,
                     "ended_by_last": which_test(reps[0]) if reps else None, "failed": failed}
        if pred == abi.PRED_LEARNED:
            res[name]["network"] = S.lp_report()
        S.close()
    return res


def _oracle_solver(case_name, model, real_bytes, predictor):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    case, grid, state, omega, spec, rate, desc = build_case(case_name, abi.FP64, predictor, model)
    o = oracle.OracleSolver(case, real_bytes)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    if omega is not None:
        o.set_omega(omega["omega"], omega["omega_n"], omega["omega_nm1"])
    if spec is not None:
        o.alm_set(spec)
    return o, oracle, desc


def cpu_baseline(case_name, model, iters_per_step, budget_s=20.0):
    """The CPU oracle in FP64 on every host thread its OpenMP loops can use:
    a bounded sample of pseudo-iterations of physical step 1, scaled by the
    pseudo-iterations the FP64 GPU path (whose iterates follow the oracle's)
    needed for that step with the same q^n guess."""
    o, oracle, _ = _oracle_solver(case_name, model, 8, abi.PRED_QN)
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
            "sample": "%d pseudo-iterations of physical step 1 (%.2f s each, FP64 oracle, %d threads), "
                      "scaled by the %d pseudo-iterations that step needs (FP64 GPU path, q^n guess, measured "
                      "in this run)" % (k, per_it, nth, iters_per_step)}


def run_reference(args):
    """--impl reference: the oracle (CPU restatement of the reference, FP64,
    every host thread), the reference's own method (q^n guess), one whole
    physical step of the workload from the seeded state, run to the same
    convergence test.  It times what it reports: steps = 1, warmup = 0."""
    o, oracle, desc = _oracle_solver(args.case, args.model, 8, abi.PRED_QN)
    t0 = time.perf_counter()
    rep = o.mg_driver()
    sec = time.perf_counter() - t0
    nth = oracle.threads()
    cb = {"value": sec, "unit": UNIT, "cores": nth, "kind": "port",
          "sample": "physical step 1 of the workload, whole, %d pseudo-iterations to the convergence test (%s), "
                    "FP64 oracle, q^n guess, %d threads" % (rep["iterations"], which_test(rep), nth)}
    # n_gpus: the N this arm was launched with, as the arm it is compared
    # with; the work runs on rank 0's host cores
    return {"metric": METRIC, "value": sec, "unit": UNIT, "n_gpus": args.gpus, "steps": 1, "warmup": 0,
            "ms_per_step": sec * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": desc, "case": args.case, "model": args.model, "device": "host cores of rank 0 (no GPU)",
                       "pseudo_iterations": rep["iterations"], "ended_by": which_test(rep),
                       "requested_steps_warmup": [args.steps, args.warmup]},
            "cpu_baseline": cb,
            "e2e": {"value": sec, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def ncu_workload(case_name, precision, model, learned=False, small=False):
    """A short, eager run for Nsight Compute captures: the case's setup, the
    start of a physical step and one pseudo-iteration, without CUDA graphs
    (so every kernel is a separate, capturable launch).  learned: instead,
    four physical steps of two pseudo-iterations with the learned guess, so
    that steps 2-4 train the network and steps 3-4 start from its guess."""
    from desalm.solver import Solver
    case, grid, state, omega, spec, rate, _ = build_case(
        case_name, precision, abi.PRED_LEARNED if learned else abi.PRED_LINEAR, model, small)
    case.use_graph = 0
    if learned:
        case.itmax = 2
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    if omega is not None:
        S.set_omega(omega["omega"], omega["omega_n"], omega["omega_nm1"])
    if spec is not None:
        S.alm_set(spec)
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
    ap.add_argument("--case", default="turbine", choices=["turbine", "cavity", "channel", "ogrid"])
    ap.add_argument("--model", default="kw", choices=["kw", "sa"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--extras", action="store_true", help="add the option-cost and initial-guess sections")
    ap.add_argument("--ncu-workload", action="store_true",
                    help="run one eager pseudo-iteration of --case for an ncu capture and exit")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--learned", action="store_true", help="with --ncu-workload: learned-guess steps")
    ap.add_argument("--small", action="store_true", help="with --ncu-workload: the turbine box at 193x97x97")
    ap.add_argument("--guesses", type=int, default=0, metavar="STEPS",
                    help="instead of the bench line: the initial guesses on --case (MIXED), each from the seeded "
                         "start for STEPS physical steps, the first --warmup of them untimed")
    args = ap.parse_args()
    if args.guesses:
        print(json.dumps(run_guesses(args)))
        return
    if args.ncu_workload:
        ncu_workload(args.case, abi.MIXED if args.precision == "mixed" else abi.FP64, args.model, args.learned,
                     args.small)
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
