"""Invariants of the remesh / mesh restatement; its parity with the
reference's own AMRStructure code is in tests/test_oracle_reference_sim.py."""
import numpy as np
import pytest

import oracle as O
from multi_species_b200 import decks


def landau(x, p):
    return (1 + 0.01 * np.cos(0.5 * x)) * np.exp(-p * p / 2) / np.sqrt(2 * np.pi)


@pytest.mark.parametrize("h,ph", [(2, 0), (3, 1), (5, 1)])
def test_mesh_sizes_and_links(h, ph):
    L = 4 * np.pi
    m = O.Mesh(h, ph, 0.0, L, -6.0, 6.0)
    npx, npp = 2 ** h, 2 ** (h + ph)
    assert m.npoints == (2 * npx + 1) * (2 * npp + 1)
    assert m.nleaves == npx * npp
    lv = m.panels[m.leaves]
    assert (lv[:, 13:17] == -1).sum() == 0          # every leaf link resolved
    assert (lv[:, 14] == -2).sum() == npx and (lv[:, 16] == -2).sum() == npx
    assert len(np.unique(m.ps)) == 2 * npp + 1
    w = m.base_weights(-1.0, 0)
    assert abs(w.sum() + L * 12.0) < 1e-12 * L * 12
    ws = m.base_weights(-1.0, 1)
    assert abs(ws.sum() + L * 12.0) < 1e-12 * L * 12


def test_identity_remesh_reproduces_nodes():
    m = O.Mesh(4, 1, 0.0, 4 * np.pi, -6.0, 6.0)
    f = landau(m.xs, m.ps)
    nf, leaf, _ = m.remesh(m.xs, m.ps, f, 0.0)
    inside = leaf != 0
    assert np.max(np.abs(nf[inside] - f[inside])) < 1e-7
    assert np.all(m.ps[~inside] == 6.0)              # only the top row is beyond (half-open top edge)


def test_quadratic_reproduced_exactly_under_shear():
    """f = a + b x + c p + d x^2 + e x p + ... lies in the fit space: remesh is exact."""
    m = O.Mesh(4, 1, 0.0, 4 * np.pi, -6.0, 6.0)
    t = 0.3
    ox, op = m.xs + m.ps * t, m.ps.copy()
    of = 1.0 + 0.2 * m.ps + 0.01 * m.ps ** 2     # depends on p only: invariant under x-shear
    nf, leaf, _ = m.remesh(ox, op, of, 0.0)
    exact = 1.0 + 0.2 * m.ps + 0.01 * m.ps ** 2
    ok = leaf != 0
    assert np.max(np.abs(nf[ok] - exact[ok])) < 1e-9


@pytest.mark.parametrize("t", [0.5, 2.5, 5.0])
def test_free_streaming_remesh_accuracy(t):
    m = O.Mesh(5, 1, 0.0, 4 * np.pi, -6.0, 6.0)
    ox, op = m.xs + m.ps * t, m.ps.copy()
    nf, leaf, fx = m.remesh(ox, op, landau(m.xs, m.ps), 0.0)
    ok = leaf != 0
    exact = landau(m.xs - m.ps * t, m.ps)
    assert np.max(np.abs(nf[ok] - exact[ok])) < 1e-6


def test_reduce_matches_numpy_unique():
    rng = np.random.default_rng(0)
    x = np.round(rng.uniform(0, 5, 400), 1)
    q = rng.normal(size=400)
    rx, rw, inv = O.reduce(x, q)
    ux = np.unique(x)
    assert np.array_equal(rx, ux)
    assert np.allclose(rw, [q[x == u].sum() for u in ux], rtol=1e-14, atol=1e-14)
    assert np.array_equal(rx[inv], x)


def test_field_energy_formula():
    L = 2 * np.pi
    x = np.linspace(0, L, 65)[:-1]
    e = np.sin(x)
    assert abs(O.field_energy(x, e, L) - 0.5 * np.pi) < 1e-12


def test_adaptive_session_start_and_remesh():
    """The oracle session with adaptive refinement: its initial state is the
    adaptive mesh builder's (f0 at every point, new ones included), and it
    steps through two remeshes, refining again at each."""
    d = decks.two_stream(h=3, ph=1, steps=6, remesh_period=3)
    d["species_list"][0].update(do_adaptively_refine=True, max_height=5, amr_epsilons=[0.02])
    sp = d["species_list"][0]
    xs, ps, f, _, _ = O.adaptive_mesh(3, 1, d["xmin"], d["xmax"], sp["pmin"], sp["pmax"],
                                      (sp["ics_type"], sp["pth"], sp["pstr"], sp["amp"], 1.0), [0.02], 5)
    s = O.Sim(d)
    st = s.state()
    assert len(st["xs"]) == len(xs) > 17 * 33
    assert np.array_equal(st["xs"], xs) and np.array_equal(st["ps"], ps) and np.array_equal(st["fs"], f)
    for _ in range(6):
        s.step()
        st = s.state()
        assert len(st["xs"]) > 17 * 33 and np.all(np.isfinite(st["fs"])) and np.all(np.isfinite(st["es"]))


def test_relativistic_push_respects_the_speed_limit():
    """With the opt-in relativistic push every point moves less than c dt per
    step (|v| = |p|/sqrt(1 + p^2) < 1 for m = 1); without it points with
    |p| > 1 move further."""
    d = decks.relativistic_two_stream(h=3, ph=1, steps=1)
    s = O.Sim(d)
    x0 = s.state()["xs"]
    s.step()
    assert np.max(np.abs(s.state()["xs"] - x0)) < d["dt"]
    d["relativistic_push"] = 0
    n = O.Sim(d)
    n.step()
    assert np.max(np.abs(n.state()["xs"] - x0)) > 2 * d["dt"]
