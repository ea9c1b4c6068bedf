"""The synthetic workloads the benchmark runs: point counts of the named
configurations, and the stated distributions of the uneven Landau batch and of
the serving request stream.  Host only."""
import math

import numpy as np

from multi_species_b200 import decks


def test_configuration_sizes():
    assert decks.deck_points(decks.landau_two_species(h=5, ph=1)) == 2 * 65 * 129 == 16770
    assert decks.deck_points(decks.two_stream(h=8, ph=1)) == 513 * 1025 == 525825
    assert decks.deck_points(decks.bump_on_tail(h=9, ph=1)) == 3 * 1025 * 2049 == 6300675


def test_bump_on_tail_splits_density_with_fixed_charge_to_mass():
    sl = decks.bump_on_tail(h=4, ph=1)["species_list"]
    assert [s["name"] for s in sl] == ["bulk", "beam", "ions"]
    assert math.isclose(sl[0]["q"] + sl[1]["q"], -1.0)
    assert sl[0]["q"] / sl[0]["m"] == sl[1]["q"] / sl[1]["m"] == -1.0


def test_landau_batch_stated_ranges_and_determinism():
    ds = decks.landau_batch(count=64, seed=0)
    assert len(ds) == 64
    for d in ds:
        n = decks.deck_points(d)
        assert 2000 <= n <= 200000
        k = 2 * math.pi / (d["xmax"] - d["xmin"])
        assert 0.3 <= k <= 0.6
        assert 1 <= len(d["species_list"]) <= 3
        assert 0.001 <= d["species_list"][0]["amp"] <= 0.1
        assert (d["greens_epsilon"], d["dt"], d["remesh_period"]) == (0.05, 0.25, 5)
        hs = {(s["initial_height"], s["p_height"]) for s in d["species_list"]}
        assert len(hs) == 1  # every species of an instance shares the mesh
    sizes = [decks.deck_points(d) for d in ds]
    assert max(sizes) / min(sizes) > 20  # uneven
    assert sizes == [decks.deck_points(d) for d in decks.landau_batch(count=64, seed=0)]


def test_serving_stream_stated_distribution():
    reqs = decks.serving_requests(rate=20.0, seconds=60.0, seed=0)
    assert abs(len(reqs) - 1200) < 4 * math.sqrt(1200)  # Poisson count
    t = [r[0] for r in reqs]
    assert t == sorted(t) and 0 < t[0] and t[-1] < 60.0
    kinds = {r[1] for r in reqs}
    assert kinds == {"landau", "two_stream", "bump_on_tail"}
    backend = {"landau": "direct32c", "two_stream": "direct32c", "bump_on_tail": "treecode32c"}
    pts = []
    for _, kind, d, steps in reqs:
        assert 10 <= steps <= 100 and d["num_steps"] == steps
        assert d["field_backend"] == backend[kind]
        n = decks.deck_points(d)
        assert 10000 <= n <= 2000000
        pts.append(n)
    assert 5e4 < float(np.median(pts)) < 2e5  # log-normal median 1e5, quantised
