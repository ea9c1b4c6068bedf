"""GPU field kernels vs the reference (through the C ABI)."""
import glob
import os

import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL32 = 1e-6  # relative L2 bound on E for the FP32-compensated kernel


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "field_direct_*.npz"))))
def test_direct64_bit_identical_to_reference_golden(path):
    g = np.load(path)
    f = M.E_MQ_DirectSum_B200(float(g["L"]), float(g["eps"]), "fp64")
    e = f.evaluate(g["targets"], g["sources"], g["q"])
    assert np.array_equal(e, g["es"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "field_direct_*.npz"))))
def test_direct32c_reference_golden(path):
    g = np.load(path)
    f = M.E_MQ_DirectSum_B200(float(g["L"]), float(g["eps"]), "fp32c")
    e = f.evaluate(g["targets"], g["sources"], g["q"])
    assert rel_l2(e, g["es"]) < TOL32


def test_drop_in_call_signature_fills_es():
    rng = np.random.default_rng(3)
    L = 4 * np.pi
    x = rng.uniform(0, L, 333)
    q = rng.normal(size=333)
    es = np.full(333, np.nan)
    f = M.E_MQ_DirectSum_B200(L, 0.05)
    f(es, x.copy(), 333, x.copy(), q, 333)
    assert np.array_equal(es, O.direct_sum(L, 0.05, x, x, q))


@pytest.mark.parametrize("n", [1, 2, 31, 513, 16770])
def test_direct64_sizes_vs_oracle(n):
    rng = np.random.default_rng(n)
    L = 4 * np.pi
    x = rng.uniform(-L, 2 * L, n)
    q = rng.normal(size=n) * 1e-3
    e = M.E_MQ_DirectSum_B200(L, 0.05, "fp64").evaluate(x, x, q)
    assert np.array_equal(e, O.direct_sum(L, 0.05, x, x, q))


@pytest.mark.parametrize("n,spread", [(1000, 1.0), (20000, 1.0), (20000, 3.0), (70000, 0.05)])
def test_direct32c_vs_direct64(n, spread):
    rng = np.random.default_rng(n + int(spread * 10))
    L = 10 * np.pi
    x = rng.uniform(-spread * L, spread * L, n) + L / 3
    q = -np.abs(rng.normal(size=n)) * (L / n)
    e64 = M.E_MQ_DirectSum_B200(L, 0.02, "fp64").evaluate(x, x, q)
    e32 = M.E_MQ_DirectSum_B200(L, 0.02, "fp32c").evaluate(x, x, q)
    assert rel_l2(e32, e64) < TOL32


def test_direct32c_lattice_two_stream_scale():
    """Full two-stream lattice (525,825 points), the precision form's workload:
    FP32c vs the bit-exact FP64 GPU path."""
    from multi_species_b200 import decks
    d = decks.two_stream()
    m = M.mesh(8, 1, 0.0, d["xmax"], -8.0, 8.0, q=-1.0, quadrature=0)
    k = 2 * np.pi / d["xmax"]
    f0 = (1 + 0.005 * np.cos(k * m["xs"])) * m["ps"] ** 2 * np.exp(-m["ps"] ** 2 / 2) / np.sqrt(2 * np.pi)
    q = m["base_weights"] * f0
    x = m["xs"] + 0.2 * m["ps"]  # one step of streaming
    e64 = M.E_MQ_DirectSum_B200(d["xmax"], 0.02, "fp64").evaluate(x, x, q)
    e32 = M.E_MQ_DirectSum_B200(d["xmax"], 0.02, "fp32c").evaluate(x, x, q)
    assert rel_l2(e32, e64) < TOL32


def test_empty_and_disjoint_sets():
    L = 2.0
    f32 = M.E_MQ_DirectSum_B200(L, 0.1, "fp32c")
    f64 = M.E_MQ_DirectSum_B200(L, 0.1, "fp64")
    t = np.linspace(0, 2, 7)
    assert np.array_equal(f64.evaluate(t, np.zeros(0), np.zeros(0)), np.zeros(7))
    assert np.array_equal(f32.evaluate(t, np.zeros(0), np.zeros(0)), np.zeros(7))
    assert f32.evaluate(np.zeros(0), t, np.ones(7)).shape == (0,)
    s = np.array([0.1, 0.5, 1.7])
    qs = np.array([1.0, -2.0, 0.5])
    assert rel_l2(f32.evaluate(t, s, qs), O.direct_sum(L, 0.1, t, s, qs)) < TOL32


def test_uniform_lattice_field_vanishes():
    """A uniform charge lattice has E = 0 at its points by symmetry; the FP32
    kernel's residue is bounded relative to the field scale sum|q|/2 = 0.5."""
    L = 2 * np.pi
    x = np.arange(4096) * (L / 4096)
    q = np.full(4096, 1.0 / 4096)
    e = M.E_MQ_DirectSum_B200(L, 0.05, "fp32c").evaluate(x, x, q)
    assert np.max(np.abs(e)) < 1e-8 * 0.5
    e64 = M.E_MQ_DirectSum_B200(L, 0.05, "fp64").evaluate(x, x, q)
    assert np.max(np.abs(e64)) < 1e-13


# ------------------------------------------------------------------ treecode
def test_treecode64_reference_golden():
    g = np.load(os.path.join(GOLD, "field_treecode.npz"))
    f = M.E_MQ_Treecode_B200(float(g["L"]), float(g["eps"]), float(g["mac"]), int(g["degree"]),
                             int(g["max_source"]), precision="fp64")
    e = f.evaluate(g["sources"], g["sources"], g["q"])
    assert rel_l2(e, g["es"]) < 1e-12


@pytest.mark.parametrize("n,leaf,mac,deg", [(1, 2000, 0.7, 8), (50, 2000, 0.7, 8), (3000, 200, 0.7, 8),
                                            (20000, 500, 0.5, 6), (40000, 2000, 0.7, 8)])
def test_treecode64_vs_oracle(n, leaf, mac, deg):
    rng = np.random.default_rng(n + leaf)
    L = 20 * np.pi
    x = rng.uniform(-L / 2, 1.5 * L, n)
    q = rng.normal(size=n) * 1e-4
    ref = O.treecode(L, 0.02, mac, deg, leaf, x, q)
    e = M.E_MQ_Treecode_B200(L, 0.02, mac, deg, leaf, precision="fp64").evaluate(x, x, q)
    if n == 1:
        assert np.array_equal(e, ref)
    else:
        assert rel_l2(e, ref) < 1e-12


@pytest.mark.parametrize("n,leaf", [(3000, 200), (40000, 2000)])
def test_treecode32c_vs_oracle(n, leaf):
    rng = np.random.default_rng(7 * n)
    L = 20 * np.pi
    x = rng.uniform(-L / 2, 1.5 * L, n)
    q = -np.abs(rng.normal(size=n)) * (L / n)
    ref = O.treecode(L, 0.02, 0.7, 8, leaf, x, q)
    e = M.E_MQ_Treecode_B200(L, 0.02, 0.7, 8, leaf, precision="fp32c").evaluate(x, x, q)
    assert rel_l2(e, ref) < TOL32


def test_treecode_rejects_distinct_targets():
    f = M.E_MQ_Treecode_B200(1.0, 0.1, 0.7, 8, 100)
    with pytest.raises(M.FsError):
        f.evaluate(np.zeros(3), np.zeros(4), np.zeros(4))


def test_open_boundary_plugin_bit_identical_to_reference_golden():
    g = np.load(os.path.join(GOLD, "field_open.npz"))
    f = M.E_MQ_DirectSum_openbcs_B200(float(g["eps"]))
    e = f.evaluate(g["targets"], g["sources"], g["q"])
    assert np.array_equal(e, g["es"])


@pytest.mark.parametrize("n", [1, 1000, 20000])
def test_open_boundary_plugin_vs_oracle(n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-10.0, 30.0, n)
    q = rng.normal(size=n) * 1e-3
    f = M.E_MQ_DirectSum_openbcs_B200(0.02)
    assert np.array_equal(f.evaluate(x, x, q), O.direct_sum_open(0.02, x, x, q))


def test_fp32c_persistent_launch_is_deterministic_whatever_the_item_order():
    """200,000 clustered points: the one-simulation pair launch takes its
    (target block, source chunk) items in a device-computed order (band-heavy
    items spread over the queue) and from an atomic counter, so which CTA runs
    which item changes from launch to launch; every item writes its own
    partials and the chunks are summed in a fixed order, so E is bit-identical
    across launches and objects, and within 1e-6 of the FP64 sum."""
    rng = np.random.default_rng(11)
    L = 2 * np.pi
    n = 200_000
    x = np.concatenate([rng.normal(1.0, 0.05, n // 2), rng.uniform(0, L, n - n // 2)]) % L
    q = rng.normal(size=n) * 1e-5 + 1.0 / n
    f = M.E_MQ_DirectSum_B200(L, 0.05, "fp32c")
    e1 = f.evaluate(x, x, q)
    e2 = f.evaluate(x, x, q)
    e3 = M.E_MQ_DirectSum_B200(L, 0.05, "fp32c").evaluate(x, x, q)
    assert np.array_equal(e1, e2) and np.array_equal(e1, e3)
    e64 = M.E_MQ_DirectSum_B200(L, 0.05, "fp64").evaluate(x, x, q)
    assert rel_l2(e1, e64) < TOL32


def test_fp32c_treecode_is_deterministic():
    """The FP32c treecode's exact linear and sign terms come from prefix sums of
    the sorted charges, taken with a fixed association: 1.5 million points
    evaluate bit-identically on repeated calls and in a fresh object."""
    rng = np.random.default_rng(12)
    L = 20 * np.pi
    n = 1_500_000
    x = rng.uniform(0, L, n)
    q = rng.normal(size=n) * 1e-7 + 1.0 / n
    f = M.E_MQ_Treecode_B200(L, 0.02, 0.7, 8, 2000, precision="fp32c")
    e1 = f.evaluate(x, x, q)
    e2 = f.evaluate(x, x, q)
    e3 = M.E_MQ_Treecode_B200(L, 0.02, 0.7, 8, 2000, precision="fp32c").evaluate(x, x, q)
    assert np.array_equal(e1, e2) and np.array_equal(e1, e3)


def test_fp32c_treecode_session_is_deterministic():
    """Two FP32c treecode sessions of the same bump-on-tail deck (three species,
    about 400,000 points) agree bit for bit after three steps."""
    from multi_species_b200 import decks
    d = decks.bump_on_tail(h=7, ph=1, steps=10)
    out = []
    for _ in range(2):
        s = M.Simulation(d, "treecode32c")
        s.step(3)
        out.append(s.state())
        s.close()
    for k in ("xs", "ps", "es"):
        assert np.array_equal(out[0][k], out[1][k]), k
