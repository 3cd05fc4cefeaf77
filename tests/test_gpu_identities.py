"""The oracle's known-answer identities (tests/test_oracle_identities.py) on
the GPU path, through the C ABI: the CUDA kernels must give the analytic
residual of linear and quadratic fields (QUICK, pressure, continuity, the
full-stress viscous term, the coarse levels' upwind), the BDF2 term, the
local pseudo-time step, bcond_fm's face rows, the SA closure, the convergence
norm and the exact prolongation of a linear correction, each to the same
tolerance as the oracle.  These pin the kernels to the reference's formulas
directly, not only through the oracle.

Both precision modes: MIXED keeps the state, residual, dtau, boundary rows
and norm in FP64, and these identities either make the DAF update zero
(dtau = 0) or do not reach it, so they hold to the FP64 tolerance there too.
The prolongation's correction is FP32 in MIXED, so that identity runs in FP64
only."""
import pytest

import test_oracle_identities as ident
from desalm import abi

pytestmark = pytest.mark.gpu

CHECKS = [
    "uniform_flow_has_zero_residual",
    "linear_velocity_residual_is_exact",
    "quadratic_velocity_residual_is_exact",
    "coarse_levels_convect_first_order_upwind",
    "bdf2_term_of_a_uniform_accelerating_flow",
    "local_pseudo_time_step",
    "boundary_extrapolation_and_walls",
    "sa_eddy_viscosity_closure",
    "residual_norm_definition",
    "prolongation_of_linear_correction_is_exact",
]


def _params():
    for name in CHECKS:
        yield pytest.param(name, abi.FP64, id=name + "-fp64")
        if name != "prolongation_of_linear_correction_is_exact":
            yield pytest.param(name, abi.MIXED, id=name + "-mixed")


@pytest.mark.parametrize("name,precision", list(_params()))
def test_identity_on_gpu(name, precision):
    from desalm.solver import Solver

    def make(case):
        c = case.copy()
        c.precision_mode = precision
        return Solver(c)

    getattr(ident, "check_" + name)(make)
