"""The oracle pinned against the reference: its own field solvers and
simulation compiled from the reference sources (oracle/_ref) and the golden
fixtures they produced."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from multi_species_b200 import decks

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "field_direct_*.npz"))))
def test_direct_sum_matches_reference_golden_bitwise(path):
    g = np.load(path)
    e = O.direct_sum(float(g["L"]), float(g["eps"]), g["targets"], g["sources"], g["q"])
    assert np.array_equal(e, g["es"])


def test_open_boundary_sum_matches_reference_golden_bitwise():
    g = np.load(os.path.join(GOLD, "field_open.npz"))
    e = O.direct_sum_open(float(g["eps"]), g["targets"], g["sources"], g["q"])
    assert np.array_equal(e, g["es"])


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_drive_fields_match_reference_golden_bitwise(kind):
    g = np.load(os.path.join(GOLD, "drive_fields.npz"))
    for t, ref in zip(g["times"], g[f"es_{kind}"]):
        e = O.external_field(kind, float(g["Am"]), float(g["k"]), float(g["omega"]), np.zeros_like(g["x"]),
                             g["x"], float(t))
        assert np.array_equal(e, ref), t


def test_drive_field_in_the_session():
    """The oracle session adds the drive at every evaluation, at the
    evaluation's time: after a step, E is the field at the new positions plus
    the drive at t = dt on them, and the trajectory differs from the undriven one."""
    d = decks.landau_two_species(h=3, ph=1, steps=4)
    d["remesh_period"] = 100
    d2 = dict(d, external_field={"use_external_field": 1, "external_type": 1, "Am": 0.4, "k": 0.5, "omega": 0.37})
    s0, s1 = O.Sim(d), O.Sim(d2)
    s0.step(1)
    s1.step(1)
    a, b = s0.state(), s1.state()
    assert not np.array_equal(a["xs"], b["xs"])
    L = d["xmax"] - d["xmin"]
    field = O.direct_sum(L, d["greens_epsilon"], b["xs"], b["xs"], b["q_ws"])
    drive = O.external_field(1, 0.4, 0.5, 0.37, np.zeros(len(b["xs"])), b["xs"], d["dt"])
    assert np.max(np.abs(b["es"] - field - drive)) <= 4e-16 * np.max(np.abs(field))


def test_treecode_matches_reference_golden_bitwise():
    g = np.load(os.path.join(GOLD, "field_treecode.npz"))
    e = O.treecode(float(g["L"]), float(g["eps"]), float(g["mac"]), int(g["degree"]), int(g["max_source"]),
                   g["sources"], g["q"])
    assert np.array_equal(e, g["es"])


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("n,spread,seed", [(1, 1.0, 0), (2, 1.0, 1), (257, 3.0, 2), (1500, 0.01, 3)])
def test_direct_sum_live_reference(n, spread, seed):
    rng = np.random.default_rng(seed)
    L = 10 * np.pi
    x = rng.uniform(-spread * L, spread * L, n)
    x[: n // 3] = x[0]  # coincident points (z == 0 skipped)
    q = rng.normal(size=n)
    assert np.array_equal(O.direct_sum(L, 0.02, x, x, q), O.ref_direct_sum(L, 0.02, x, x, q))


@pytest.mark.skipif(not O.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("n,leaf,mac,deg", [(50, 2000, 0.7, 8), (3000, 200, 0.7, 8), (4000, 100, 0.5, 4)])
def test_treecode_live_reference(n, leaf, mac, deg):
    rng = np.random.default_rng(n)
    L = 4 * np.pi
    x = rng.uniform(-L, 2 * L, n)
    q = rng.normal(size=n) * 1e-3
    assert np.array_equal(O.treecode(L, 0.05, mac, deg, leaf, x, q), O.ref_treecode(L, 0.05, mac, deg, leaf, x, q))


def test_treecode_normalisation_vs_direct():
    """The reference treecode's kernel is the direct kernel times sqrt(L^2+4eps^2)/L."""
    rng = np.random.default_rng(5)
    L, eps = 4 * np.pi, 0.05
    x = rng.uniform(0, L, 6000)
    q = rng.normal(size=6000) * 1e-3
    d = O.direct_sum(L, eps, x, x, q) * np.sqrt(L * L + 4 * eps * eps) / L
    t = O.treecode(L, eps, 0.7, 8, 400, x, q)
    assert np.linalg.norm(t - d) / np.linalg.norm(d) < 1e-5


def _adaptive_two_stream():
    d = decks.two_stream(h=3, ph=1, steps=6, remesh_period=3)
    d["species_list"][0].update(do_adaptively_refine=True, max_height=5, amr_epsilons=[0.02])
    return d


def _bump_on_tail_treecode():
    d = decks.bump_on_tail(h=3, ph=1, steps=6)
    d["max_source"] = 200
    d["remesh_period"] = 3
    return d


SIM_FIXTURES = {
    "sim_landau_h3.npz": decks.landau_two_species(h=3, ph=1, steps=6),
    "ref_sim_two_stream_h4.npz": decks.two_stream(h=4, ph=1, steps=8, remesh_period=3),
    "ref_sim_adaptive_two_stream_h3.npz": _adaptive_two_stream(),
    "ref_sim_bump_on_tail_h3.npz": _bump_on_tail_treecode(),
}


@pytest.mark.parametrize("fixture", sorted(SIM_FIXTURES))
def test_sim_trajectory_matches_reference_golden_bitwise(fixture):
    """Trajectories of the reference's AMRSimulation (remeshes, adaptive
    refinement and the treecode included) against the restatement's session."""
    g = np.load(os.path.join(GOLD, fixture))
    s = O.Sim(SIM_FIXTURES[fixture])
    for k in [int(i) for i in g["iters"]]:
        s.step(k - s.iter)
        st = s.state()
        for key in ("xs", "ps", "fs", "q_ws", "es"):
            assert np.array_equal(st[key], g[f"{key}_{k}"]), (k, key)
