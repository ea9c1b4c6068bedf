"""Batched stepping of many simulations (fs_batch_*): results against each
member stepped alone (fs_sim_step), graph replay against launch-by-launch
stepping, membership changes, and members of other field kinds."""
import numpy as np
import pytest

import multi_species_b200 as fs
from field_error import fp32c_bound
from multi_species_b200 import decks

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _small_decks(count, seed):
    out = []
    for d in decks.landau_batch(count=count, seed=seed, steps=10):
        for s in d["species_list"]:  # keep the members small: 1k-17k points each
            s["initial_height"] = min(s["initial_height"], 5)
            s["p_height"] = min(s["p_height"], 1)
        out.append(d)
    return out


def _alone(deck, steps, backend="direct32c"):
    sim = fs.Simulation(deck, backend)
    sim.step(steps)
    st = sim.state()
    sim.close()
    return st


def test_batch_matches_members_alone():
    ds = _small_decks(4, seed=3)
    b = fs.Batch()
    ids = [b.add(d) for d in ds]
    sims = [fs.Simulation(d, "direct32c") for d in ds]
    ref64 = [fs.Simulation(d, "direct64") for d in ds]
    b.step(4)  # steps 2-4 from a graph
    for s in sims + ref64:
        s.step(4)
    for i, s in zip(ids, sims):
        got, ref = b.state(i), s.state()
        assert b.info(i)["iter"] == 4
        # the members' FP32 pair sums are split into chunks differently alone
        # (tiles per item), so E differs at FP32 rounding level and the
        # positions integrate it
        assert _rel(got["es"], ref["es"]) <= 1e-6
        assert _rel(got["xs"], ref["xs"]) <= 1e-8 and _rel(got["ps"], ref["ps"]) <= 1e-8
    b.step(3)  # remesh at step 5, graph replays after it
    for s in sims + ref64:
        s.step(3)
    st = b.stats()
    assert st["graph_steps"] >= 4 and st["plain_steps"] >= 2, st
    for i, d in zip(ids, ds):
        # every evaluation of a member in the mix is within 1e-6 of the FP64
        # field of the member's own state (after the remesh E comes from the
        # reduced grid, which equals the field at every point)
        got = b.state(i)
        e64 = _fp64_field(d, got)
        assert np.linalg.norm(got["es"] - e64) <= fp32c_bound(got["xs"], got["q_ws"], d["xmax"] - d["xmin"],
                                                               d["greens_epsilon"], e64)
    b.close()


def _fp64_field(deck, st):
    L = deck["xmax"] - deck["xmin"]
    f = fs.E_MQ_DirectSum_B200(L, deck["greens_epsilon"], "fp64")
    e = f.evaluate(st["xs"], st["xs"], st["q_ws"])
    f.close()
    return e


def _electron_decks(count, seed):
    """Members without the cold ion species: lattice points of a well-resolved
    distribution do not sit on old panel edges, so rounding-level position
    differences do not change the remesh's point location."""
    out = _small_decks(count, seed)
    for d in out:
        d["species_list"] = d["species_list"][:1]
    return out


def test_autotuned_batch_matches_members_alone_through_remesh():
    ds = _electron_decks(4, seed=3)
    b = fs.Batch()
    ids = [b.add(d) for d in ds]
    b.step(7)  # one remesh at step 5
    for i, d in zip(ids, ds):
        alone = _alone(d, 7)
        got = b.state(i)
        e64 = _fp64_field(d, got)
        tol = fp32c_bound(got["xs"], got["q_ws"], d["xmax"] - d["xmin"], d["greens_epsilon"], e64)
        for k in ("fs", "xs", "ps"):
            assert _rel(got[k], alone[k]) <= 1e-6, k
        assert np.linalg.norm(got["es"] - alone["es"]) <= tol
        assert np.linalg.norm(got["es"] - e64) <= tol
    b.close()


def test_batch_fp32c_against_fp64():
    ds = _small_decks(3, seed=5)
    b = fs.Batch()
    ids = [b.add(d) for d in ds]
    b.step(1)
    for i, d in zip(ids, ds):
        ref = _alone(d, 1, "direct64")
        assert _rel(b.state(i)["es"], ref["es"]) <= 1e-6
    b.close()


def test_graphs_replay_bit_identical():
    ds = _small_decks(3, seed=7)
    out = []
    for graphs in (True, False):
        b = fs.Batch(graphs=graphs, tuning=(4, 8))
        ids = [b.add(d) for d in ds]
        b.step(6)
        out.append([b.state(i) for i in ids])
        st = b.stats()
        assert (st["graph_steps"] > 0) == graphs
        b.close()
    for a, c in zip(*out):
        for k in a:
            assert np.array_equal(a[k], c[k]), k


def test_member_alone_and_in_mix_bit_identical():
    ds = _small_decks(5, seed=11)
    b1 = fs.Batch(tuning=(4, 16))
    i1 = b1.add(ds[0])
    b1.step(6)
    alone = b1.state(i1)
    b2 = fs.Batch(tuning=(4, 16))
    ids = [b2.add(d) for d in ds]
    b2.step(6)
    mixed = b2.state(ids[0])
    for k in alone:
        assert np.array_equal(alone[k], mixed[k]), k
    b1.close()
    b2.close()


def test_membership_changes_and_phases():
    ds = _small_decks(4, seed=13)
    b = fs.Batch(tuning=(8, 32))
    a = b.add(ds[0])
    c = b.add(ds[1])
    b.step(3)
    b.remove(c)
    d = b.add(ds[2])  # joins at iteration 0 while `a` is at 3: remeshes fall on different steps
    b.step(4)
    assert b.info(a)["iter"] == 7 and b.info(d)["iter"] == 4
    assert b.stats()["graph_steps"] > 0
    with pytest.raises(fs.FsError):
        b.info(c)
    for sid, deck, steps in ((a, ds[0], 7), (d, ds[2], 4)):
        ref = _alone(deck, steps)
        got = b.state(sid)
        assert _rel(got["es"], ref["es"]) <= 1e-6
        assert _rel(got["xs"], ref["xs"]) <= 1e-8
    b.close()


def test_other_field_kinds_join_bit_identical():
    ds = _small_decks(2, seed=17)
    b = fs.Batch()
    i64 = b.add(ds[0], "direct64")
    i32 = b.add(ds[1])
    b.step(6)
    ref = _alone(ds[0], 6, "direct64")
    got = b.state(i64)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
    assert _rel(b.state(i32)["es"], _alone(ds[1], 6)["es"]) <= 1e-6
    b.close()


def test_batch_argument_errors():
    b = fs.Batch()
    with pytest.raises(fs.FsError):
        b.set_tuning(3, 8)
    with pytest.raises(fs.FsError):
        b.remove(12345)
    b.step(0)
    b.step(2)  # empty batch: nothing to do
    b.close()


def test_profile_counts_graph_replayed_launches():
    ds = _small_decks(2, seed=19)
    b = fs.Batch(tuning=(4, 16))
    for d in ds:
        b.add(d)
    fs.profile_reset()
    fs.profile_enable(True)
    try:
        b.step(4)  # step 1 launch by launch, step 2 captured, 3-4 replayed
    finally:
        fs.profile_enable(False)
    n, ms, w = fs.profile_read("k_pairs32_batched")
    assert b.stats()["graph_steps"] == 3
    assert n == 16 and ms > 0
    assert w == pytest.approx(b.pair_count(), rel=1e-12)
    b.close()


def test_adaptive_member_alone_and_in_batch_bit_identical():
    """A member whose mesh refines adaptively (its point count changes at each
    remesh) steps in a batch exactly as alone; the batch is not graph-captured."""
    ad = decks.two_stream(h=4, ph=1, steps=7, remesh_period=3)
    ad["species_list"][0].update(do_adaptively_refine=True, max_height=6, amr_epsilons=[0.05])
    other = _small_decks(1, seed=53)[0]
    b1 = fs.Batch(tuning=(4, 16))
    i1 = b1.add(ad)
    b1.step(7)
    alone = b1.state(i1)
    b2 = fs.Batch(tuning=(4, 16))
    i2 = b2.add(ad)
    b2.add(other)
    b2.step(7)
    mixed = b2.state(i2)
    assert b2.stats()["graph_steps"] == 0
    for k in alone:
        assert np.array_equal(alone[k], mixed[k]), k
    b1.close()
    b2.close()


def test_relativistic_member_alone_and_in_batch_bit_identical():
    """A member with the relativistic push (positions move with p/sqrt(1+p^2))
    steps in a batch, graph-captured, exactly as alone; its push does not leak
    into the other members."""
    rd = decks.relativistic_two_stream(h=4, ph=1, steps=7)
    others = _small_decks(2, seed=59)
    b1 = fs.Batch(tuning=(4, 16))
    i1 = b1.add(rd)
    b1.step(7)
    alone = b1.state(i1)
    b2 = fs.Batch(tuning=(4, 16))
    i2 = b2.add(rd)
    io = [b2.add(d) for d in others]
    b2.step(7)
    assert b2.stats()["graph_steps"] > 0
    for k in alone:
        assert np.array_equal(alone[k], b2.state(i2)[k]), k
    b3 = fs.Batch(tuning=(4, 16))
    io3 = [b3.add(d) for d in others]
    b3.step(7)
    for a, c in zip(io, io3):
        for k in ("xs", "ps", "es"):
            assert np.array_equal(b2.state(a)[k], b3.state(c)[k]), k
    for b in (b1, b2, b3):
        b.close()


def test_band_pairs_of_the_last_evaluation():
    """fs_batch_band_pairs: the FP32c members' last evaluation counts n^2 pairs
    each, of which the band |d| <= 16 eps (evaluated in FP64) is close to its
    share 32 eps / L of a near-uniform Landau density; an FP64 member counts
    none."""
    ds = _small_decks(3, seed=5)
    b = fs.Batch()
    ids = [b.add(d) for d in ds]
    b.add(ds[0], "direct64")
    b.step(1)  # no remesh: the last evaluation is a full one
    band, pairs = b.band_pairs()
    ns = [b.info(i)["n"] for i in ids]
    b.close()
    assert pairs == float(sum(n * n for n in ns))
    want = sum(n * n * 32 * d["greens_epsilon"] / (d["xmax"] - d["xmin"]) for n, d in zip(ns, ds))
    assert 0 < band < pairs
    assert abs(band / want - 1) < 0.3, (band, want)


def test_large_members_take_the_ordered_launch_bit_identical_and_accurate():
    """Members of 70k-200k points with 8 tiles per item give each batched launch
    far more items than the persistent grid has CTAs, so the items are taken in
    the device-computed order (band-heavy ones spread over the queue), which
    depends on the whole mix.  A member's results are still bit-identical alone
    and in the mix, and its field is within the error model of the FP64 sum."""
    ds = [d for d in decks.landau_batch(count=64, seed=0, steps=10) if decks.deck_points(d) >= 70_000][:3]
    assert len(ds) == 3
    b1 = fs.Batch(tuning=(4, 8))
    i1 = b1.add(ds[0])
    b1.step(2)
    alone = b1.state(i1)
    b1.close()
    b2 = fs.Batch(tuning=(4, 8))
    ids = [b2.add(d) for d in ds]
    b2.step(2)
    mixed = [b2.state(i) for i in ids]
    b2.close()
    for k in alone:
        assert np.array_equal(alone[k], mixed[0][k]), k
    for d, st in zip(ds, mixed):
        L = d["xmax"] - d["xmin"]
        e64 = fs.E_MQ_DirectSum_B200(L, d["greens_epsilon"], "fp64").evaluate(st["xs"], st["xs"], st["q_ws"])
        assert np.linalg.norm(st["es"] - e64) <= fp32c_bound(st["xs"], st["q_ws"], L, d["greens_epsilon"], e64)
