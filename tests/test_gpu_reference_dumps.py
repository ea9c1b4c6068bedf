"""Diagnostic / restart files and restart loading against the reference's own
code (oracle/_ref/libamr_ref.so: AMRStructure_io.cpp, AMRStructure_restart.cpp,
AMRSimulation_field.cpp, AMRSimulation.cpp's restart branch).

* The session writes the same files as the reference, under the same names:
  leaf_point_inds and full_tree byte for byte, particle files bit for bit
  before the first remesh and within 1e-12 after it (the remesh fit rounds
  differently, see tests/test_gpu_reference_trajectories.py), reduced-grid
  files likewise.
* Restarts cross: the reference restarts from the session's files and the
  session from the reference's, and both continue as the uninterrupted run."""
import os
import shutil

import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M
from multi_species_b200 import decks

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.amr_ref_available(), reason="reference simulation library not built")]


def _deck():
    d = decks.landau_two_species(h=3, ph=1, steps=8)
    d["diag_period"] = 1
    d["diag_phase_space_period"] = 1
    return d


def _files(root):
    out = {}
    for dirpath, _, names in os.walk(os.path.join(root, "simulation_output")):
        for n in names:
            p = os.path.join(dirpath, n)
            out[os.path.relpath(p, root)] = p
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_dump_files_match_the_reference_writers(tmp_path):
    d = _deck()
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "ours"
    ref = O.RefSim(d, sim_dir=str(ref_dir))
    ref.step(7)
    ref.close()
    g = M.Simulation(d, "direct64")
    g.set_output(str(our_dir))
    g.step(7)
    g.flush_output()
    g.close()
    rf, of = _files(str(ref_dir)), _files(str(our_dir))
    assert set(rf) == set(of), sorted(set(rf) ^ set(of))[:10]
    assert any("full_tree_5" in k for k in rf)
    for k in sorted(rf):
        a, b = open(rf[k], "rb").read(), open(of[k], "rb").read()
        it = int(k.rsplit("_", 1)[1])
        if "/panels/" in k or "reduce_xs" in k or it < 5:
            assert a == b, k  # panels, unique x, and every file before the first remesh
        else:
            x, y = np.frombuffer(a, np.float64), np.frombuffer(b, np.float64)
            assert len(x) == len(y) and rel(y, x) < 1e-11, k


@pytest.mark.parametrize("writer", ["reference", "session"])
def test_restart_crosses_between_reference_and_session(tmp_path, writer):
    """A dump taken right after the remesh at step 5, by either side, is loaded
    by both; both continue to step 8 as the uninterrupted reference run."""
    d = _deck()
    src = tmp_path / "src"
    if writer == "reference":
        r = O.RefSim(d, sim_dir=str(src))
        r.step(5)
        r.close()
    else:
        g = M.Simulation(d, "direct64")
        g.set_output(str(src))
        g.step(5)
        g.flush_output()
        g.close()
    full = O.RefSim(d)
    full.step(8)
    want = full.state()
    full.close()
    # the reference restarting (its constructor loads the files when the deck says so)
    rdir = tmp_path / "ref_restart"
    shutil.copytree(src, rdir)
    rd = dict(d, restart=True, restart_iter=5)
    r2 = O.RefSim(rd, sim_dir=str(rdir))
    assert r2.iter == 5
    r2.step(3)
    got_ref = r2.state()
    r2.close()
    # the session restarting
    sdir = tmp_path / "ses_restart"
    shutil.copytree(src, sdir)
    s2 = M.Simulation(d, "direct64")
    s2.restart(str(sdir), 5)
    s2.step(3)
    got_ses = s2.state()
    s2.close()
    for k in ("xs", "ps", "fs", "q_ws", "es"):
        assert rel(got_ref[k], want[k]) < 1e-11, ("reference", k)
        assert rel(got_ses[k], want[k]) < 1e-11, ("session", k)
