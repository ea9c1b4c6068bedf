"""FP32-compensated treecode at the full bump-on-tail size: three species of
1025 x 2049 points (6,300,675 points), theta 0.7, degree 8, leaf 2000,
eps 0.02, after two steps of the FP32c session.

* FP32c treecode against the FP64 treecode on all 6.3M targets: <= 1e-6
  relative L2 (the FP32 near field's rounding; the far field is FP64 in both).
* Both against the plain FP64 direct sum (the reference arithmetic, rescaled by
  the treecode kernel's normalisation sqrt(L^2 + 4 eps^2) / L,
  src/FieldStructure.cpp:949 vs :150) on 4096 evenly spaced targets: the
  treecode's own approximation error, which FP32c leaves unchanged to 1e-7."""
import numpy as np
import pytest

import multi_species_b200 as M
from multi_species_b200 import decks

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_treecode32c_full_size_accuracy():
    d = decks.bump_on_tail(h=9, ph=1, steps=50)
    sim = M.Simulation(d, "treecode32c")
    assert sim.n == 6300675
    sim.step(2)
    st = sim.state()
    sim.close()
    L, eps = d["xmax"] - d["xmin"], d["greens_epsilon"]
    x, q = st["xs"], st["q_ws"]
    args = (L, eps, d["mac"], d["degree"], d["max_source"])
    t32 = M.E_MQ_Treecode_B200(*args, precision="fp32c")
    t64 = M.E_MQ_Treecode_B200(*args, precision="fp64")
    e32, e64 = t32.evaluate(x, x, q), t64.evaluate(x, x, q)
    t32.close()
    t64.close()
    err_fp32c = rel(e32, e64)
    assert err_fp32c <= 1e-6
    idx = np.linspace(0, len(x) - 1, 4096).astype(np.int64)
    f = M.E_MQ_DirectSum_B200(L, eps, "fp64")
    ed = f.evaluate(x[idx], x, q) * np.sqrt(L * L + 4 * eps * eps) / L
    f.close()
    tree_err64 = rel(e64[idx], ed)
    tree_err32 = rel(e32[idx], ed)
    print(f"fp32c vs fp64 treecode {err_fp32c:.2e}; vs direct sum (4096 targets): fp64 tree {tree_err64:.2e}, "
          f"fp32c tree {tree_err32:.2e}")
    assert tree_err64 < 1e-3
    assert abs(tree_err32 - tree_err64) <= 1e-6 + 0.01 * tree_err64
