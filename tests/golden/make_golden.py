"""Regenerate the golden fixtures in this directory from the CPU oracle.

The reference cannot be built here (Fortran 90 + MPI, no compiler) and ships
no golden data, so these fixtures are regression pins of the oracle itself:
they freeze the oracle's output on small seeded cases so that any later
change to the restatement shows up.  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "des-alm_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from desalm import abi, cases  # noqa: E402
import oracle  # noqa: E402


def run_rfg():
    """The random flow generator's oracle: mode tables of a seed and the
    inflow plane of a small wake box with per-node anisotropic tensors."""
    import rfg_oracle
    case, grid, state = cases.wake(im=9, jm=13, km=11, turbulence=0, seed=5)
    tab = rfg_oracle.modes(200, 77)
    spec = cases.rfg_inflow(case, tables=tab)
    rng = np.random.default_rng(78)
    uij = np.zeros((case.km, case.jm, 6))
    for k in range(case.km):
        for j in range(case.jm):
            B = rng.normal(size=(3, 3))
            R = (B @ B.T + 0.5 * np.eye(3)) * 1e-3
            uij[k, j] = (R[0, 0], R[0, 1], R[0, 2], R[1, 1], R[1, 2], R[2, 2])
    spec["uij"] = uij
    spec["t_ts"] = rng.uniform(0.1, 0.5, size=(case.km, case.jm))
    spec["t_ls"] = rng.uniform(0.1, 0.4, size=(case.km, case.jm))
    q = state["q"].reshape(case.km, case.jm, case.im, 5).copy()
    q = rfg_oracle.inlet_forcing(q, grid, (case.im, case.jm, case.km), 0.3, spec)
    return {"p": tab["p"], "q": tab["q"], "k": tab["k"], "omega": tab["omega"], "plane": q[1:-1, 1:-1, 0, 1:4]}


def run(name):
    if name == "rfg":
        return run_rfg()
    if name == "cavity17":
        case, grid, state = cases.cavity(n=17, seed=123, itmax=5)
    else:
        case, grid, state = cases.channel(im=17, jm=17, km=17, seed=321, itmax=4)
    o = oracle.OracleSolver(case, 8)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    out = {}
    o.solver_daf(1, 1, 1)
    out["daf_q"] = o.get_state()["q"]
    out["daf_rh"] = np.stack([o.get_field(1, abi.F_RH + m) for m in range(4)])
    o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    rep = o.mg_driver()
    out["step_q"] = o.get_state()["q"]
    out["step_nut"] = o.get_state()["nut"]
    out["step_residual"] = np.array(rep["residual"])
    out["step_iterations"] = np.array(rep["iterations"])
    return out


def main():
    for name in ("cavity17", "channel17", "rfg"):
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **run(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
