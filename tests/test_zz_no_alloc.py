"""desalm_mg_residual_noalloc: the convergence norm for callers that cannot
allocate device memory (a Fortran host whose device arrays belong to another
runtime or pool allocator, or a process held to a fixed device-memory
budget).  It must give the same five log10 values as the context's
desalm_mg_residual on the same q and qold, call after call, while the
library allocates nothing for it (its scratch is a fixed device array).

This file is collected last on purpose; it runs alone or after the others.
The argument checks run on the host only and need no GPU.
"""
import ctypes as C

import numpy as np
import pytest


def _noalloc_fn():
    from desalm.solver import lib
    L = lib()
    f = L.desalm_mg_residual_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.c_void_p]
    f.restype = C.c_int
    return f


@pytest.mark.gpu
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
    S.close()


def _nblk(im, jm, km):
    return -(-((im - 2) * (jm - 2) * (km - 2)) // 2048)


def test_noalloc_size_limit_and_null_arrays():
    """The size check comes first, then the pointers, both on the host before
    any CUDA call, so null arrays make every case here launch-free.
    514^3 nodes (512^3 interior, exactly 65,536 partials) fit the scratch:
    with null arrays that is DESALM_EINVAL.  514 x 514 x 515 and 1026^3 do
    not fit: DESALM_ENOMEM.  A small valid grid with null arrays: EINVAL."""
    assert _nblk(514, 514, 514) == 65536 and _nblk(514, 514, 515) > 65536
    f = _noalloc_fn()
    got = (C.c_double * 5)()
    assert f(None, None, 514, 514, 514, got, None) == -1
    assert f(None, None, 514, 514, 515, got, None) == -2
    assert f(None, None, 1026, 1026, 1026, got, None) == -2
    assert f(None, None, 17, 17, 17, got, None) == -1
    assert f(None, None, 2, 17, 17, got, None) == -1
