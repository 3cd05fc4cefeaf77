"""The C-ABI library loads (no GPU needed) and exports every symbol that
include/desalm.h declares; the case validation runs on the host."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "desalm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(desalm_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("desalm_init", "desalm_solver_daf", "desalm_mg_nlevel", "desalm_mg_prolong",
              "desalm_mg_residual", "desalm_bcond_fm", "desalm_des_eddy", "desalm_mg_driver"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from desalm.solver import LIB_PATH, build
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_invalid_case_is_rejected_without_gpu():
    """check_case runs before any CUDA call: an even extent with full
    coarsening must give DESALM_EINVAL and a message."""
    from desalm import cases
    from desalm.solver import Solver, DesalmError
    case, _, _ = cases.cavity(n=17)
    case.im = 18
    with pytest.raises(DesalmError) as e:
        Solver(case)
    assert "odd extents" in str(e.value)
    case.im = 17
    case.ifix = 18
    with pytest.raises(DesalmError) as e:
        Solver(case)
    assert "pressure reference node" in str(e.value)
    case.ifix = 1
    case.wall_functions = 2
    with pytest.raises(DesalmError) as e:
        Solver(case)
    assert "wall_functions" in str(e.value)


def test_entry_points_reject_null_arguments_without_gpu():
    """Host-side argument checks that return before any CUDA call."""
    from desalm import abi
    from desalm.solver import lib
    L = lib()
    assert L.desalm_mg_driver_batch(None, 1, None) == abi.DESALM_EINVAL
    ctxs = (C.c_void_p * 2)(None, None)
    assert L.desalm_mg_driver_batch(ctxs, 2, None) == abi.DESALM_EINVAL
    assert L.desalm_mg_driver_batch(ctxs, -1, None) == abi.DESALM_EINVAL
    assert L.desalm_mg_driver_batch(ctxs, 0, None) == 0          # nothing to step
    out = (C.c_int * 12)()
    assert L.desalm_sweep_widths(None, out) == abi.DESALM_EINVAL
    assert L.desalm_wall_functions(None) == abi.DESALM_EINVAL
    assert L.desalm_lp_fields(None, 1) == abi.DESALM_EINVAL
