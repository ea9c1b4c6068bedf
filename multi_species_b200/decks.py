"""Synthetic decks (deck.json keys) for the workloads of the benchmark configs.

They stand in for the reference's run decks: the reference ships no decks for
these configurations, so the values below restate the configuration text
(shapes, parameters); all inputs are generated from them."""
import math

ION_PTH = math.sqrt(1.0 / 1836.0)


def landau_two_species(h=5, ph=1, steps=20):
    """Two-species Landau damping on [0, 4 pi), v in [-6, 6], eps 0.05, dt 0.5,
    remesh every 5 steps, trapezoid quadrature (32 x 64 panels per species at h=5)."""
    L = 4 * math.pi
    sp = dict(initial_height=h, p_height=ph, pmin=-6.0, pmax=6.0, normalized_wavenumber=1.0, pstr=0.0)
    return dict(xmin=0.0, xmax=L, pmin=-6.0, pmax=6.0, bcs=0, greens_epsilon=0.05, dt=0.5, num_steps=steps,
                remesh_period=5, use_treecode=0, quadrature=0,
                species_list=[dict(sp, name="electrons", ics_type=1, pth=1.0, amp=0.01, q=-1.0, m=1.0),
                              dict(sp, name="ions", ics_type=1, pth=ION_PTH, amp=0.0, q=1.0, m=1836.0)])


def two_stream(h=8, ph=1, steps=100, remesh_period=5):
    """Strong two-stream instability on [0, 10 pi), v in [-8, 8], eps 0.02, dt 0.2,
    electrons only (the kernel's per-source background neutralises);
    256 x 512 panels (525,825 points) at h=8."""
    L = 10 * math.pi
    return dict(xmin=0.0, xmax=L, pmin=-8.0, pmax=8.0, bcs=0, greens_epsilon=0.02, dt=0.2, num_steps=steps,
                remesh_period=remesh_period, use_treecode=0, quadrature=0,
                species_list=[dict(name="electrons", ics_type=3, pth=1.0, pstr=0.0, amp=0.005,
                                   normalized_wavenumber=1.0, q=-1.0, m=1.0, initial_height=h, p_height=ph,
                                   pmin=-8.0, pmax=8.0)])


def bump_on_tail(h=9, ph=1, steps=50, amp=0.04):
    """Three-species bump-on-tail on [0, 20 pi), v in [-10, 10], treecode
    (degree 8, theta 0.7, leaf 2000), eps 0.02, dt 0.1.  The 0.9 / 0.1 density
    split of the bulk and beam electrons is carried by q and m with q/m = -1."""
    L = 20 * math.pi
    sp = dict(initial_height=h, p_height=ph, pmin=-10.0, pmax=10.0, normalized_wavenumber=1.0, amp=amp)
    return dict(xmin=0.0, xmax=L, pmin=-10.0, pmax=10.0, bcs=0, greens_epsilon=0.02, dt=0.1, num_steps=steps,
                remesh_period=5, use_treecode=1, mac=0.7, degree=8, max_source=2000, max_target=2000,
                quadrature=0,
                species_list=[dict(sp, name="bulk", ics_type=9, pth=1.0, pstr=0.0, q=-0.9, m=0.9),
                              dict(sp, name="beam", ics_type=9, pth=0.5, pstr=4.5, q=-0.1, m=0.1),
                              dict(sp, name="ions", ics_type=9, pth=ION_PTH, pstr=0.0, amp=0.0, q=1.0, m=1836.0)])


def relativistic_two_stream(h=5, ph=1, steps=20, mu=25.0, pstr=1.0, amp=0.01, push=True, remesh_period=5):
    """Relativistic two-stream (ics 7: two boosted Maxwell-Juttner beams at
    +-pstr with inverse temperature mu) on [0, 4 pi), p in [-4, 4], eps 0.05,
    dt 0.2, electrons only; positions move with the relativistic velocity
    p / sqrt(1 + p^2) when `push` is set."""
    L = 4 * math.pi
    return dict(xmin=0.0, xmax=L, pmin=-4.0, pmax=4.0, bcs=0, greens_epsilon=0.05, dt=0.2, num_steps=steps,
                remesh_period=remesh_period, use_treecode=0, quadrature=0, relativistic_push=1 if push else 0,
                species_list=[dict(name="electrons", ics_type=7, mu=mu, pstr=pstr, amp=amp,
                                   normalized_wavenumber=1.0, q=-1.0, m=1.0, initial_height=h, p_height=ph,
                                   pmin=-4.0, pmax=4.0)])


def _quantized_mesh(target_per_species, nsp, lo=2000, hi=200000):
    """(h, ph) with h in 4..8, ph in 0..2 whose point count (2*2^h+1)*(2*2^(h+ph)+1)
    is closest in log to the per-species target, with the instance total in
    [lo, hi] (panel counts must be powers of two)."""
    best = None
    for h in range(4, 9):
        for ph in range(0, 3):
            n = (2 * 2 ** h + 1) * (2 * 2 ** (h + ph) + 1)
            if not lo <= n * nsp <= hi:
                continue
            d = abs(math.log(n / target_per_species))
            if best is None or d < best[0]:
                best = (d, h, ph)
    return best[1], best[2]


def landau_batch(count=64, seed=0, steps=40):
    """Independent Landau-damping instances of uneven size: amplitude
    alpha ~ U[0.001, 0.1], k ~ U[0.3, 0.6] (L = 2 pi / k), 1-3 species
    (electrons; ions of mass 1836; a 10% electron beam at v = 2), total points
    log-uniform in [2k, 200k] quantised to power-of-two panel counts;
    eps 0.05, dt 0.25, remesh every 5 steps, FP32-compensated direct sum."""
    import numpy as np

    rng = np.random.default_rng(seed)
    decks = []
    for _ in range(count):
        alpha = float(rng.uniform(0.001, 0.1))
        k = float(rng.uniform(0.3, 0.6))
        nsp = int(rng.integers(1, 4))
        total = float(np.exp(rng.uniform(math.log(2000), math.log(200000))))
        h, ph = _quantized_mesh(total / nsp, nsp)
        L = 2 * math.pi / k
        sp = dict(initial_height=h, p_height=ph, pmin=-6.0, pmax=6.0, normalized_wavenumber=1.0, pstr=0.0)
        species = [dict(sp, name="electrons", ics_type=1, pth=1.0, amp=alpha, q=-1.0, m=1.0)]
        if nsp >= 2:
            species.append(dict(sp, name="ions", ics_type=1, pth=ION_PTH, amp=0.0, q=1.0, m=1836.0))
        if nsp >= 3:
            species.append(dict(sp, name="beam", ics_type=9, pth=0.5, pstr=2.0, amp=alpha, q=-0.1, m=0.1))
        decks.append(dict(xmin=0.0, xmax=L, pmin=-6.0, pmax=6.0, bcs=0, greens_epsilon=0.05, dt=0.25,
                          num_steps=steps, remesh_period=5, use_treecode=0, quadrature=0,
                          field_backend="direct32c", species_list=species))
    return decks


def deck_points(deck):
    """Total panel points of a uniform deck."""
    return sum((2 * 2 ** s["initial_height"] + 1) * (2 * 2 ** (s["initial_height"] + s["p_height"]) + 1)
               for s in deck["species_list"])


def _quantized_heights(total, nsp, lo, hi):
    """(h, ph) per species, h in 4..10, ph in 0..2, with nsp species of that
    mesh totalling in [lo, hi] and closest in log to `total`."""
    best = None
    for h in range(4, 11):
        for ph in range(0, 3):
            n = nsp * (2 * 2 ** h + 1) * (2 * 2 ** (h + ph) + 1)
            if not lo <= n <= hi:
                continue
            d = abs(math.log(n / total))
            if best is None or d < best[0]:
                best = (d, h, ph)
    return best[1], best[2]


def serving_requests(rate=20.0, seconds=60.0, seed=0, sigma=1.0):
    """Poisson arrivals at `rate` per second for `seconds`; each request is a
    Landau (two species, direct FP32c), two-stream (one species, direct FP32c)
    or bump-on-tail (three species, FP32c treecode) deck with the parameters
    of those workloads, total points log-normal with median 100k and log-sd
    `sigma`, clipped to [10k, 2M] and quantised to power-of-two panel counts,
    and 10-100 steps.  Returns [(arrival_s, kind, deck, steps)]."""
    import numpy as np

    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= seconds:
            return out
        kind = ("landau", "two_stream", "bump_on_tail")[int(rng.integers(0, 3))]
        total = float(np.clip(np.exp(rng.normal(math.log(1e5), sigma)), 1e4, 2e6))
        steps = int(rng.integers(10, 101))
        nsp = {"landau": 2, "two_stream": 1, "bump_on_tail": 3}[kind]
        h, ph = _quantized_heights(total, nsp, 10000, 2000000)
        if kind == "landau":
            d = landau_two_species(h=h, ph=ph, steps=steps)
            d["field_backend"] = "direct32c"
        elif kind == "two_stream":
            d = two_stream(h=h, ph=ph, steps=steps)
            d["field_backend"] = "direct32c"
        else:
            d = bump_on_tail(h=h, ph=ph, steps=steps)
            d["field_backend"] = "treecode32c"
        out.append((t, kind, d, steps))
