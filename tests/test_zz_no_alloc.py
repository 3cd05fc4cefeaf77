"""desalm_mg_residual_noalloc: the convergence norm for callers that cannot
allocate device memory (for example while a CUDA stream is being captured
into a graph, or when a Fortran host's device memory belongs to another
allocator).  It must give the same five log10 values as the context's
desalm_mg_residual on the same q and qold, call after call, while the
library allocates nothing for it (its scratch is a fixed device array).

This file is collected last on purpose; it runs alone or after the others.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    from desalm.solver import lib
    L = lib()
    f = L.desalm_mg_residual_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


def test_noalloc_residual_matches_context_residual():
    import torch
    from desalm import abi, cases
    from desalm.solver import Solver
    case, grid, state = cases.cavity(n=33, seed=7)
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"])
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    S.begin_step()                     # qold_mg <- q
    f = _noalloc_fn()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        S.solver_daf(1, 0, 1)          # q moves away from qold_mg
        want = S.mg_residual(1)        # context path (cudaMalloc'd scratch)
        q = torch.tensor(np.concatenate([S.get_field(1, abi.F_Q + m) for m in range(5)]), device="cuda")
        qold = torch.tensor(np.concatenate([S.get_field(1, abi.F_QOLD + m) for m in range(5)]), device="cuda")
        torch.cuda.synchronize()
        got = (C.c_double * 5)()
        rc = f(q.data_ptr(), qold.data_ptr(), case.im, case.jm, case.km, got, stream)
        assert rc == 0, rc
        got = np.array(got)
        finite = np.isfinite(want)
        assert np.array_equal(finite, np.isfinite(got))
        assert np.allclose(got[finite], want[finite], rtol=0, atol=1e-12), (call, got, want)


def test_noalloc_rejects_oversized_grid():
    """1026^3 nodes (1024^3 interior) is beyond the fixed scratch: rejected
    with DESALM_ENOMEM on the host.  The arrays passed are null, so nothing
    could be launched even if the size check were wrong (that would return
    DESALM_EINVAL instead)."""
    f = _noalloc_fn()
    got = (C.c_double * 5)()
    rc = f(None, None, 1026, 1026, 1026, got, None)
    assert rc == -2
