"""Device-resident simulation vs the oracle restatement (through the C ABI)."""
import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M
from multi_species_b200 import decks

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_initial_state_bit_identical():
    d = decks.landau_two_species(h=4, ph=1)
    g, o = M.Simulation(d), O.Sim(d)
    a, b = g.state(), o.state()
    for k in ("xs", "ps", "fs", "q_ws", "es"):
        assert np.array_equal(a[k], b[k]), k


def test_rk4_steps_bit_identical_before_remesh():
    d = decks.landau_two_species(h=4, ph=1)
    g, o = M.Simulation(d), O.Sim(d)
    for _ in range(4):
        g.step()
        o.step()
        a, b = g.state(), o.state()
        for k in ("xs", "ps", "q_ws", "es"):
            assert np.array_equal(a[k], b[k]), k


def test_remesh_step_matches_oracle():
    d = decks.landau_two_species(h=4, ph=1)
    g, o = M.Simulation(d), O.Sim(d)
    g.step(5)
    o.step(5)
    a, b = g.state(), o.state()
    assert np.array_equal(a["xs"], b["xs"]) and np.array_equal(a["ps"], b["ps"])
    assert rel(a["fs"], b["fs"]) < 1e-12
    assert rel(a["q_ws"], b["q_ws"]) < 1e-12
    assert rel(a["es"], b["es"]) < 1e-11


def test_remesh_with_long_walks_matches_oracle():
    """A long-box Landau deck (L = 20.5, |v| up to 6, 5 steps of 0.25 before the
    remesh) whose point location walks visit many panels before revisiting one;
    every visited panel has to be remembered, as the reference's set does."""
    d = decks.landau_batch(count=2, seed=29, steps=10)[1]
    for s in d["species_list"]:
        s["initial_height"], s["p_height"] = min(s["initial_height"], 5), min(s["p_height"], 1)
    g, o = M.Simulation(d, "direct64"), O.Sim(d)
    g.step(6)
    o.step(6)
    a, b = g.state(), o.state()
    assert rel(a["fs"], b["fs"]) < 1e-12
    assert rel(a["xs"], b["xs"]) < 1e-12
    assert rel(a["es"], b["es"]) < 1e-11


def test_remesh_only_matches_oracle_interpolation():
    """Remesh of a streamed two-stream state, species by species."""
    d = decks.two_stream(h=5, ph=1, remesh_period=1000)
    g, o = M.Simulation(d), O.Sim(d)
    g.step(3)
    o.step(3)
    st = o.state()
    m = O.Mesh(5, 1, d["xmin"], d["xmax"], -8.0, 8.0)
    fmin = float(np.min(O.Sim(d).state()["fs"]))
    nf, leaf, _ = m.remesh(st["xs"], st["ps"], st["fs"], fmin)
    g.remesh()
    a = g.state()
    assert rel(a["fs"], nf) < 1e-12
    assert np.array_equal(a["xs"], m.xs)


def test_fp32c_session_field_error():
    d = decks.two_stream(h=6, ph=1, remesh_period=5)
    g64, g32 = M.Simulation(d, "direct64"), M.Simulation(d, "direct32c")
    e0 = g64.state()["es"]
    assert rel(g32.state()["es"], e0) < 1e-6
    g64.step(2)
    g32.step(2)
    assert rel(g32.state()["es"], g64.state()["es"]) < 1e-6


def test_field_energy_drift_fp32c_vs_fp64():
    """Two-stream at reduced size (65 x 129 points), 100 steps with remesh every 5:
    FP32c field energy within 1e-5 of the FP64 path over the whole run."""
    d = decks.two_stream(h=5, ph=1, steps=100, remesh_period=5)
    a, b = M.Simulation(d, "direct64"), M.Simulation(d, "direct32c")
    L = d["xmax"]
    wa, wb = [], []
    for _ in range(100):
        a.step()
        b.step()
        sa, sb = a.state(), b.state()
        wa.append(O.field_energy(sa["xs"], sa["es"], L))
        wb.append(O.field_energy(sb["xs"], sb["es"], L))
    wa, wb = np.array(wa), np.array(wb)
    assert np.max(np.abs(wb - wa)) / np.max(wa) < 1e-5


def test_pair_count_and_launches():
    d = decks.landau_two_species(h=3, ph=1)
    n0 = M.kernel_launches()
    g = M.Simulation(d)
    g.step(1)
    assert M.kernel_launches() > n0
    n = g.n
    assert g.pair_count() > 4 * n * n


def test_treecode_simulation_matches_oracle():
    """Bump-on-tail at reduced size (3 species, 33 x 65 points each, leaf 300):
    device treecode session vs the oracle's treecode session."""
    d = decks.bump_on_tail(h=4, ph=1)
    d["max_source"] = 300
    g, o = M.Simulation(d, "treecode64"), O.Sim(d)
    a, b = g.state(), o.state()
    assert rel(a["es"], b["es"]) < 1e-12
    for _ in range(5):
        g.step()
        o.step()
    a, b = g.state(), o.state()
    for k in ("xs", "ps"):
        assert rel(a[k], b[k]) < 1e-11, k
    assert rel(a["fs"], b["fs"]) < 1e-9
    assert rel(a["es"], b["es"]) < 1e-9


def test_treecode32c_simulation_field_error():
    d = decks.bump_on_tail(h=5, ph=1)
    g64, g32 = M.Simulation(d, "treecode64"), M.Simulation(d, "treecode32c")
    g64.step(2)
    g32.step(2)
    assert rel(g32.state()["es"], g64.state()["es"]) < 1e-6


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_drive_field_session_matches_oracle(kind):
    """Drive fields (tanh / sine / logistic) added at every evaluation with the
    stage times of rk4_step; 24 steps of 0.5 cross the logistic switch-on at
    t = 10 and include four remeshes.  The device sine differs from the host's
    by at most an ulp, so the bound is a rounding-level one."""
    d = decks.landau_two_species(h=3, ph=1, steps=24)
    d["species_list"] = d["species_list"][:1]  # electrons: the cold ions of this coarse mesh tangle by step 20
    d["external_field"] = {"use_external_field": 1, "external_type": kind, "Am": 0.4, "k": 0.5, "omega": 0.37}
    g, o = M.Simulation(d, "direct64"), O.Sim(d)
    for step in range(24):
        g.step()
        o.step()
        a, b = g.state(), o.state()
        for k in ("xs", "ps", "es"):
            assert rel(a[k], b[k]) < 1e-11, (step, k)
    d.pop("external_field")
    und = O.Sim(d)
    und.step(24)
    assert rel(g.state()["es"], und.state()["es"]) > 1e-6  # the drive acted


def test_drive_field_fp32c_session():
    """FP32c session with a sine drive: after 3 steps its E minus the drive at
    t = 3 dt is the FP64 field at its own positions, within the FP32c bound
    (relative to the field: the drive is added exactly in FP64)."""
    d = decks.two_stream(h=6, ph=1, remesh_period=5)
    d["external_field"] = {"use_external_field": 1, "external_type": 1, "Am": 0.4, "k": 0.2, "omega": 0.37}
    g32 = M.Simulation(d, "direct32c")
    g32.step(3)
    st = g32.state()
    L = d["xmax"] - d["xmin"]
    field = M.E_MQ_DirectSum_B200(L, d["greens_epsilon"], "fp64").evaluate(st["xs"], st["xs"], st["q_ws"])
    drive = O.external_field(1, 0.4, 0.2, 0.37, np.zeros(len(st["xs"])), st["xs"], 3 * d["dt"])
    assert np.max(np.abs(drive)) > 1e-3
    assert rel(st["es"] - drive, field) < 1e-6


def _adaptive_two_stream(steps=6, remesh_period=3):
    d = decks.two_stream(h=4, ph=1, steps=steps, remesh_period=remesh_period)
    d["species_list"][0].update(do_adaptively_refine=True, max_height=7, amr_epsilons=[0.02])
    return d


def test_adaptive_initial_mesh_bit_identical_to_oracle():
    """generate_mesh at the initial step with adaptive refinement: f0 on the
    uniform mesh, panels whose f spread exceeds 0.02 split 2x2 up to level 7."""
    d = _adaptive_two_stream()
    g, o = M.Simulation(d, "direct64"), O.Sim(d)
    a, b = g.state(), o.state()
    assert len(a["xs"]) == len(b["xs"]) > 33 * 65
    for k in ("xs", "ps", "fs", "q_ws", "es"):
        assert np.array_equal(a[k], b[k]), k


def test_adaptive_remesh_matches_oracle():
    """Remesh with adaptive refinement: the lattice interpolated by the walk,
    refinement passes whose new points are interpolated from the previous mesh
    (root search + fit), the state laid out again with the new point count."""
    d = _adaptive_two_stream(steps=7, remesh_period=3)
    g, o = M.Simulation(d, "direct64"), O.Sim(d)
    for step in range(7):
        g.step()
        o.step()
        a, b = g.state(), o.state()
        assert len(a["xs"]) == len(b["xs"]), step
        assert np.array_equal(a["xs"], b["xs"]) or rel(a["xs"], b["xs"]) < 1e-12, step
        assert rel(a["fs"], b["fs"]) < 1e-11, step
        assert rel(a["es"], b["es"]) < 1e-10, step


def test_adaptive_fp32c_session_runs_with_refinement():
    d = _adaptive_two_stream(steps=6, remesh_period=3)
    g64, g32 = M.Simulation(d, "direct64"), M.Simulation(d, "direct32c")
    g64.step(4)
    g32.step(4)
    a, b = g32.state(), g64.state()
    assert len(a["xs"]) == len(b["xs"])
    assert rel(a["es"], b["es"]) < 1e-5


def test_relativistic_push_steps_bit_identical():
    """The opt-in relativistic push (relativistic_momentum_push's velocity
    (p/m)/sqrt(1 + (p/m)^2) in every RK4 stage) on the two-species Landau deck:
    device steps equal the oracle's bit for bit before the first remesh, and
    the push changes the trajectory."""
    d = decks.landau_two_species(h=4, ph=1)
    d["relativistic_push"] = 1
    g, o = M.Simulation(d), O.Sim(d)
    for _ in range(4):
        g.step()
        o.step()
        a, b = g.state(), o.state()
        for k in ("xs", "ps", "q_ws", "es"):
            assert np.array_equal(a[k], b[k]), k
    d["relativistic_push"] = 0
    n = O.Sim(d)
    n.step(4)
    assert rel(g.state()["xs"], n.state()["xs"]) > 1e-6


def test_relativistic_two_stream_session_matches_oracle():
    """ics 7 (boosted Maxwell-Juttner pair) with the relativistic push through
    two remeshes.  The initial f equals the library's host f0 at the mesh
    points bit for bit; against the oracle, whose K_1 is its own quadrature,
    it agrees to 1e-14, and so the trajectory agrees to rounding."""
    d = decks.relativistic_two_stream(h=4, ph=1, steps=12)
    g, o = M.Simulation(d, "direct64"), O.Sim(d)
    a, b = g.state(), o.state()
    assert np.array_equal(a["xs"], b["xs"]) and np.array_equal(a["ps"], b["ps"])
    assert np.array_equal(a["fs"], M.initial_f0(d, 0, a["xs"], a["ps"]))
    assert rel(a["fs"], b["fs"]) < 1e-14
    for step in range(12):
        g.step()
        o.step()
        a, b = g.state(), o.state()
        for k in ("xs", "ps", "fs", "es"):
            assert rel(a[k], b[k]) < 1e-11, (step, k)
    assert np.max(np.abs(np.diff(a["xs"]))) > 0 and np.max(np.abs(a["ps"])) > 1.0


@pytest.mark.parametrize("ics,keys,dom", [
    (5, {"pth": 0.5, "amp": 0.02}, (-0.001, 0.001)),
    (6, {"mu": 2.0, "amp": 0.01}, (0.0, 4 * np.pi)),
    (8, {"amp": 1.3, "wave_beta": 0.8, "pth": 0.3}, (0.0, 5.0)),
])
def test_boost_initial_conditions_in_session(ics, keys, dom):
    """Friedman beam, Maxwell-Juttner and travelling-wave initial conditions
    build a session whose initial f is the host f0 at its mesh points, and
    which steps."""
    d = dict(xmin=dom[0], xmax=dom[1], dt=0.05, greens_epsilon=0.05, remesh_period=5, quadrature=0,
             species_list=[dict(name="e", ics_type=ics, q=-1.0, m=1.0, initial_height=4, p_height=1,
                                pmin=-3.0, pmax=3.0, **keys)])
    g = M.Simulation(d, "direct64")
    a = g.state()
    assert np.array_equal(a["fs"], M.initial_f0(d, 0, a["xs"], a["ps"]))
    assert np.array_equal(a["fs"], O.initial_f0(d, 0, a["xs"], a["ps"])) or ics != 5
    g.step(2)
    assert np.all(np.isfinite(g.state()["xs"]))
    g.close()


def test_two_species_landau_config_reports_the_reference_shift_failure():
    """At the step-20 remesh of the two-species Landau configuration the
    reference throws "too many shifts!" (tests/test_oracle_reference_sim.py);
    the device session returns FS_ERR_SHIFT at that step, after 19 steps that
    match the restatement."""
    d = decks.landau_two_species(h=5, ph=1, steps=20)
    g = M.Simulation(d, "direct64")
    g.step(19)
    o = O.Sim(d)
    o.step(19)
    a, b = g.state(), o.state()
    assert rel(a["fs"], b["fs"]) < 1e-11 and rel(a["xs"], b["xs"]) < 1e-11
    with pytest.raises(M.FsError) as e:
        g.step(1)
    assert e.value.code == 5  # FS_ERR_SHIFT
    g.close()
