"""Diagnostic and restart files of a device-resident session in the
reference's formats (AMRStructure_io.cpp, AMRStructure_restart.cpp,
AMRSimulation_field.cpp), written asynchronously while the steps run."""
import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M
from multi_species_b200 import decks

pytestmark = pytest.mark.gpu


def _read(path, dtype=np.float64):
    return np.fromfile(str(path), dtype=dtype)


def test_dump_files_match_state_and_mesh(tmp_path):
    d = decks.landau_two_species(h=3, ph=1, steps=6)
    g = M.Simulation(d, "direct64")
    g.set_output(str(tmp_path), diag_period=5, diag_phase_space_period=2)
    states = {0: g.state()}
    for it in range(1, 7):
        g.step()
        states[it] = g.state()
    g.flush_output()
    out = tmp_path / "simulation_output"
    starts = np.concatenate([[0], np.cumsum(g.species_points)])
    names = [sp["name"] for sp in d["species_list"]]
    for it in range(7):
        for k, name in enumerate(names):
            a, b = starts[k], starts[k + 1]
            xs = out / name / "xs" / f"xs_{it}"
            if it % 2:
                assert not xs.exists()
                continue
            assert np.array_equal(_read(xs), states[it]["xs"][a:b])
            assert np.array_equal(_read(out / name / "ps" / f"ps_{it}"), states[it]["ps"][a:b])
            assert np.array_equal(_read(out / name / "fs" / f"fs_{it}"), states[it]["fs"][a:b])
    # panels: the uniform mesh of the restatement (bit-identical to the library's host mesh)
    sp0 = d["species_list"][0]
    m = O.Mesh(3, 1, d["xmin"], d["xmax"], sp0["pmin"], sp0["pmax"])
    inds = _read(out / names[0] / "panels" / "leaf_point_inds_4", np.int32).reshape(-1, 9)
    assert np.array_equal(inds, m.panels[m.leaves, :9])
    raw = (out / names[0] / "panels" / "full_tree_4").read_bytes()
    assert np.frombuffer(raw[:8], dtype=np.int64)[0] == m.npanels
    assert len(raw) == 8 + 80 * m.npanels
    rec = np.frombuffer(raw[8:], dtype=np.uint8).reshape(m.npanels, 80)
    ints = rec[:, :72].copy().view(np.int32).reshape(m.npanels, 18)
    assert np.array_equal(ints[:, 0], np.arange(m.npanels))
    assert np.array_equal(ints[:, 1], m.panels[:, 9])       # level
    assert np.array_equal(ints[:, 2], m.panels[:, 10])      # parent
    assert np.array_equal(ints[:, 3], m.panels[:, 11])      # which child
    assert np.array_equal(ints[:, 4:13], m.panels[:, :9])   # point indices
    assert np.array_equal(ints[:, 13:17], m.panels[:, 13:17])  # left, top, right, bottom
    assert np.array_equal(ints[:, 17], m.panels[:, 12])     # first child
    flags = m.panels[:, 17]
    assert np.array_equal(rec[:, 72], (flags & 1 > 0).astype(np.uint8))
    assert np.array_equal(rec[:, 73], (flags & 2 > 0).astype(np.uint8))
    assert np.array_equal(rec[:, 74], (flags & 4 > 0).astype(np.uint8))
    assert np.array_equal(rec[:, 75], (flags & 8 > 0).astype(np.uint8))
    # reduced grid at the start (iteration 0) and at the remesh (5)
    L = d["xmax"] - d["xmin"]
    rxs, rws = [], []
    for k in range(2):
        a, b = starts[k], starts[k + 1]
        rx, rw, _ = O.reduce(states[0]["xs"][a:b], states[0]["q_ws"][a:b])
        rxs.append(rx)
        rws.append(rw)
    rx, rw = np.concatenate(rxs), np.concatenate(rws)
    assert np.array_equal(_read(out / "reduce_xs" / "xs_0"), rx)
    assert np.array_equal(_read(out / "reduced_es" / "es_0"), O.direct_sum(L, d["greens_epsilon"], rx, rx, rw))
    assert _read(out / "reduced_es" / "es_5").size == rx.size
    assert not (out / "reduced_es" / "es_2").exists()
    g.close()


def test_dump_errors_are_reported(tmp_path):
    blocker = tmp_path / "simulation_output"
    blocker.write_text("a file where the output directory should be")
    g = M.Simulation(decks.landau_two_species(h=3, ph=1))
    g.set_output(str(tmp_path), 1, 1)
    with pytest.raises(M.FsError):
        g.flush_output()
    g.close()


def test_dumps_follow_adaptive_meshes(tmp_path):
    """With adaptive refinement the point count changes at each remesh; each
    dump carries the mesh and the sizes of its own iteration."""
    d = decks.two_stream(h=4, ph=1, steps=6, remesh_period=3)
    d["species_list"][0].update(do_adaptively_refine=True, max_height=6, amr_epsilons=[0.05])
    g = M.Simulation(d, "direct64")
    g.set_output(str(tmp_path), diag_period=3, diag_phase_space_period=3)
    sizes = {0: g.state()["xs"].size}
    for it in range(1, 7):
        g.step()
        if it % 3 == 0:
            sizes[it] = g.state()["xs"].size
    g.flush_output()
    out = tmp_path / "simulation_output" / d["species_list"][0]["name"]
    for it, n in sizes.items():
        assert _read(out / "xs" / f"xs_{it}").size == n
        tree = (out / "panels" / f"full_tree_{it}").read_bytes()
        npan = int(np.frombuffer(tree[:8], dtype=np.int64)[0])
        assert len(tree) == 8 + 80 * npan
        inds = _read(out / "panels" / f"leaf_point_inds_{it}", np.int32)
        assert inds.max() == n - 1
    g.close()


@pytest.mark.parametrize("adaptive", [False, True])
def test_restart_from_dumps_continues_the_run(tmp_path, adaptive):
    """Dump at iteration 4 (a remesh iteration), restart a fresh session from
    the files: the loaded state equals the original, t = 4 dt, and three more
    steps follow the original within rounding (the restart recomputes E on the
    reduced grid).  Like the reference, the restart recomputes the weights from
    the loaded leaves, which equals the carried weights when the dump was
    taken right after a remesh."""
    d = decks.two_stream(h=4, ph=1, steps=7, remesh_period=4)
    if adaptive:
        d["species_list"][0].update(do_adaptively_refine=True, max_height=6, amr_epsilons=[0.05])
    g = M.Simulation(d, "direct64")
    g.set_output(str(tmp_path), diag_period=2, diag_phase_space_period=2)
    g.step(4)
    g.flush_output()
    ref4 = g.state()
    r = M.Simulation(d, "direct64")
    r.restart(str(tmp_path), 4)
    it, t = r.iteration()
    assert it == 4 and t == pytest.approx(4 * d["dt"], rel=1e-15)
    got = r.state()
    for k in ("xs", "ps", "fs", "q_ws"):
        assert np.array_equal(got[k], ref4[k]), k
    assert np.linalg.norm(got["es"] - ref4["es"]) <= 1e-12 * np.linalg.norm(ref4["es"])
    g.step(3)
    r.step(3)
    a, b = r.state(), g.state()
    assert len(a["xs"]) == len(b["xs"])
    for k in ("xs", "ps", "fs", "es"):
        assert np.linalg.norm(a[k] - b[k]) <= 1e-10 * np.linalg.norm(b[k]), k
    g.close()
    r.close()


def test_restart_rejects_missing_or_corrupt_files(tmp_path):
    d = decks.two_stream(h=4, ph=1, steps=2)
    g = M.Simulation(d, "direct64")
    with pytest.raises(M.FsError):
        g.restart(str(tmp_path), 0)  # nothing written yet
    g.set_output(str(tmp_path), 1, 1)
    g.flush_output()
    tree = tmp_path / "simulation_output" / "electrons" / "panels" / "full_tree_0"
    raw = bytearray(tree.read_bytes())
    raw[8 + 80 * 3 + 52:8 + 80 * 3 + 56] = np.int32(10 ** 6).tobytes()  # a neighbour far outside the tree
    tree.write_bytes(bytes(raw))
    before = g.state()
    with pytest.raises(M.FsError):
        g.restart(str(tmp_path), 0)
    after = g.state()
    for k in before:
        assert np.array_equal(before[k], after[k]), k  # the session is unchanged
    g.close()
