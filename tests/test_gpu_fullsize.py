"""Parity of the CUDA path with the FP64 oracle at the full sizes of the
benchmark workloads: the laminar cavity 65^3 (3-level FAS), the SA channel
129x97x65, the SA cylinder O-grid 257x129x65 and the actuator-line turbine box
385x193x193.

For each workload the library and the threaded oracle go through identical
call sequences:
- one fine-level solver_daf without and with the recalculated residual, then
  mg_nlevel and one coarse-level solver_daf (FP64: relative L2 <= 1e-12 per
  field);
- three whole pseudo-iterations (FP64: <= 1e-10 per field);
- three MIXED pseudo-iterations (FP32 line sweeps and transforms) against the
  same FP64 oracle, at the tolerance stated per workload.
The line solves' would-swap counter (rows where SGTSV's partial pivoting
would interchange) is read after the pseudo-iterations; it must stay 0 on
these workloads, whose DAF systems are diagonally dominant.

The turbine box at full size (14.3 M nodes) runs only the pseudo-iteration
checks: its oracle needs about 12 GB of host memory and a few seconds per
pseudo-iteration on the host threads.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu

Q4 = [abi.F_Q + m for m in range(4)]


def _build(name):
    if name == "cavity65":
        case, grid, state = cases.cavity(n=65, seed=0)
        return case, grid, state, None
    if name == "channel129":
        case, grid, state = cases.channel()
        return case, grid, state, None
    if name == "ogrid257":
        case, grid, state = cases.ogrid()
        return case, grid, state, None
    if name == "turbine385":
        case, grid, state, spec, _ = cases.turbine()
        return case, grid, state, spec
    raise ValueError(name)


def _pair(name, precision, oracle_mod):
    from desalm.solver import Solver
    case, grid, state, spec = _build(name)
    case.precision_mode = precision
    g = Solver(case)
    o = oracle_mod.OracleSolver(case, 8)
    for s in (g, o):
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        if spec is not None:
            s.alm_set(spec)
    return case, g, o


def _fields(case):
    return Q4 + ([abi.F_Q + 4, abi.F_NUT] if case.turbulence else [])


def _worst(g, o, n, fields):
    return max(rel_l2(g.get_field(n, f), o.get_field(n, f)) for f in fields)


# The raw recalculated residual rh and the coarse forcing pk of the O-grid
# are sums of terms much larger than themselves near the wall (wall-normal
# spacing 8e-4 against 20 D: metric products up to 1e6).  Measured on a
# B200: rh(u) 2.2e-11 fine and 1.0e-10 coarse, pk(u) 1.0e-11, while q and
# dtau agree to 1e-15.  Their tolerance is stated per workload.
RH_TOL = {"cavity65": 1e-12, "channel129": 1e-12, "ogrid257": 5e-10}


@pytest.mark.parametrize("name", ["cavity65", "channel129", "ogrid257"])
def test_solver_daf_full_size(name, oracle_mod):
    case, g, o = _pair(name, abi.FP64, oracle_mod)
    try:
        for s in (g, o):
            s.begin_step()
            s.solver_daf(1, 0, 1)
        errs = {"fine q%d" % m: rel_l2(g.get_field(1, abi.F_Q + m), o.get_field(1, abi.F_Q + m)) for m in range(4)}
        errs["fine dtau"] = rel_l2(g.get_field(1, abi.F_DTAU), o.get_field(1, abi.F_DTAU))
        for s in (g, o):
            s.solver_daf(1, 1, 1)
        for m in range(4):
            errs["recalc q%d" % m] = rel_l2(g.get_field(1, abi.F_Q + m), o.get_field(1, abi.F_Q + m))
            errs["recalc rh%d" % m] = rel_l2(g.get_field(1, abi.F_RH + m), o.get_field(1, abi.F_RH + m))
        for s in (g, o):
            s.mg_nlevel(2)
            s.solver_daf(2, 1, 1)
        for m in range(4):
            for nm, f in (("q", abi.F_Q), ("pk", abi.F_PK), ("rh", abi.F_RH)):
                errs["coarse %s%d" % (nm, m)] = rel_l2(g.get_field(2, f + m), o.get_field(2, f + m))
        print(name, {k: "%.2e" % v for k, v in errs.items()})
        bad = {k: v for k, v in errs.items() if v > (RH_TOL[name] if ("rh" in k or "pk" in k) else 1e-12)}
        assert not bad, bad
    finally:
        g.close()


# MIXED against the FP64 oracle after three pseudo-iterations: the FP32
# preconditioner's rounding, relative L2 per field
MIXED_TOL = {"cavity65": 2e-5, "channel129": 5e-5, "ogrid257": 5e-5, "turbine385": 5e-5}


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
@pytest.mark.parametrize("name", ["cavity65", "channel129", "ogrid257", "turbine385"])
def test_pseudo_iterations_full_size(name, precision, oracle_mod):
    case, g, o = _pair(name, precision, oracle_mod)
    try:
        g.begin_step()
        o.begin_step()
        pivots = 0
        for it in range(3):
            rg = g.pseudo_iteration()
            o.pseudo_iteration()
            pivots += rg["pivots"]
        tol = 1e-10 if precision == abi.FP64 else MIXED_TOL[name]
        errs = {f: rel_l2(g.get_field(1, f), o.get_field(1, f)) for f in _fields(case)}
        print("%s precision %d: worst field rel L2 %.3e, would-swap rows %d" %
              (name, precision, max(errs.values()), pivots))
        assert max(errs.values()) <= tol, errs
        assert pivots == 0, pivots
    finally:
        g.close()
