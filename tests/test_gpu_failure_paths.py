"""Failure paths driven without a GPU fault: the bounds of the device waits are
lowered through the test hook fs_debug_set_wait_limits so that a bounded wait
runs out, the call returns its error status, and the next call on the same
object works.  Nothing traps and no wait is unbounded: with zero polls every
tile wait gives up at once, and the kernel still lets its own copies land
(bounded) before its CTAs exit."""
import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M
from multi_species_b200 import decks

pytestmark = pytest.mark.gpu

FS_ERR_WALK, FS_ERR_TIMEOUT = 4, 6


@pytest.fixture(autouse=True)
def _default_limits():
    yield
    M.debug_set_wait_limits(0)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_pair_kernel_wait_timeout_then_recovers():
    rng = np.random.default_rng(3)
    L = 4 * np.pi
    x = rng.uniform(-L, 2 * L, 20000)
    q = rng.normal(size=20000) * 1e-3
    f = M.E_MQ_DirectSum_B200(L, 0.05, "fp32c")
    ref = O.direct_sum(L, 0.05, x, x, q)
    assert rel(f.evaluate(x, x, q), ref) < 1e-6
    M.debug_set_wait_limits(0, mbar_polls=0)
    with pytest.raises(M.FsError) as e:
        f.evaluate(x, x, q)
    assert e.value.code == FS_ERR_TIMEOUT
    M.debug_set_wait_limits(0)
    for _ in range(2):
        assert rel(f.evaluate(x, x, q), ref) < 1e-6
    f.close()


def test_session_fp32c_timeout_is_reported():
    """A session step whose field wait runs out returns FS_ERR_TIMEOUT; a new
    session on the same device then steps normally."""
    d = decks.two_stream(h=4, ph=1, steps=4, remesh_period=5)
    g = M.Simulation(d, "direct32c")
    M.debug_set_wait_limits(0, mbar_polls=0)
    with pytest.raises(M.FsError) as e:
        g.step(1)
    assert e.value.code == FS_ERR_TIMEOUT
    M.debug_set_wait_limits(0)
    g.close()
    a, b = M.Simulation(d, "direct32c"), M.Simulation(d, "direct64")
    a.step(2)
    b.step(2)
    assert rel(a.state()["es"], b.state()["es"]) < 1e-6


def test_remesh_walk_limit_then_recovers():
    """The step that remeshes fails with FS_ERR_WALK when walks may visit only
    one panel; the state is left as the step's RK4 made it, and a remesh with
    the default bound on the same session gives the state of an undisturbed
    session bit for bit."""
    d = decks.two_stream(h=4, ph=1, steps=10, remesh_period=5)
    g, ref = M.Simulation(d, "direct64"), M.Simulation(d, "direct64")
    g.step(4)
    ref.step(5)
    M.debug_set_wait_limits(0, walk_panels=1)
    with pytest.raises(M.FsError) as e:
        g.step(1)
    assert e.value.code == FS_ERR_WALK
    st = g.state()
    assert not np.array_equal(st["xs"], ref.state()["xs"])  # not remeshed: still the moved points
    M.debug_set_wait_limits(0)
    g.remesh()
    a, b = g.state(), ref.state()
    for k in ("xs", "ps", "fs", "q_ws", "es"):
        assert np.array_equal(a[k], b[k]), k
    g.step(2)
    ref.step(2)
    for k in ("xs", "ps", "fs", "q_ws", "es"):
        assert np.array_equal(g.state()[k], ref.state()[k]), k
