"""The oracle reproduces its committed golden fixtures (regression pins of
the CPU restatement; generated by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["cavity17", "channel17", "rfg"])
def test_oracle_matches_golden(name, oracle_mod):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    want = np.load(os.path.join(HERE, "golden", name + ".npz"))
    got = mg.run(name)
    for k in want.files:
        a, b = np.asarray(got[k], dtype=np.float64), want[k]
        if k == "step_residual":
            fin = np.isfinite(b)
            assert np.array_equal(np.isfinite(a), fin)
            assert np.allclose(a[fin], b[fin], rtol=0, atol=1e-12), k
        else:
            assert np.allclose(a, b, rtol=1e-13, atol=1e-15), k
