"""The oracle's known-answer identities (tests/test_oracle_identities.py) on
the GPU path, through the C ABI: the CUDA kernels must give the analytic
residual of linear and quadratic fields (QUICK, pressure, continuity, the
full-stress viscous term, the coarse levels' upwind), the BDF2 term, the
local pseudo-time step, bcond_fm's face rows, the SA closure, the convergence
norm and the exact prolongation of a linear correction, each to the same
tolerance as the oracle (FP64 path).  These pin the kernels to the reference's
formulas directly, not only through the oracle."""
import pytest

import test_oracle_identities as ident

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


@pytest.mark.parametrize("name", CHECKS)
def test_identity_on_gpu(name):
    from desalm.solver import Solver
    getattr(ident, "check_" + name)(Solver)
