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
