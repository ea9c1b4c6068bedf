"""Initial distributions of every ics_type (make_f0_return_ptr,
AMRSimulation_load.cpp:139-225; initial_distributions.cpp:11-460) on the host:
the oracle's special functions against SciPy and against the normalisation the
distributions carry, and the library's host f0 (fs_initial_f0) against the
oracle.  The reference evaluates K_1 and the incomplete elliptic integrals with
Boost.Math, which is absent here; the library uses the C++17 standard library's
versions and the oracle its own quadrature and Carlson forms."""
import math

import numpy as np
import pytest
from scipy import special

import oracle as O
import multi_species_b200 as M


def _deck(sp, xmin, xmax):
    sp = dict(dict(pmin=-4.0, pmax=4.0, initial_height=3, p_height=1, q=-1.0, m=1.0), **sp)
    return {"xmin": xmin, "xmax": xmax, "dt": 0.1, "greens_epsilon": 0.05, "species_list": [sp]}


def _points(n, xr, pr, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(*xr, n), rng.uniform(*pr, n)


@pytest.mark.parametrize("x", [0.01, 0.05, 0.5, 1.0, 2.0, 10.0, 50.0, 300.0, 700.0])
def test_oracle_bessel_k1(x):
    assert O.bessel_k1(x) == pytest.approx(special.k1(x), rel=1e-14)


def test_oracle_elliptic_integrals():
    """F(k, phi) and E(k, phi) including |phi| > pi/2 (the travelling wave's
    orbit parameter runs over [-pi/2, 5 pi/2])."""
    for k in (0.0, 0.07, 0.3, 0.7, 0.95):
        for phi in (-3.0, -math.pi / 2, 0.3, 1.2, math.pi / 2, 2.0, 4.0, 2.5 * math.pi, 7.0):
            assert O.ellint_1(k, phi) == pytest.approx(special.ellipkinc(phi, k * k), rel=1e-14, abs=1e-15)
            assert O.ellint_2(k, phi) == pytest.approx(special.ellipeinc(phi, k * k), rel=1e-14, abs=1e-15)


def test_relativistic_distributions_are_normalised():
    """Maxwell-Juttner: int exp(-mu gamma) dp = 2 K_1(mu), so f integrates to 1
    in p; the boosted pair of the relativistic two-stream integrates to
    gamma_str = sqrt(1 + pstr^2) (a Lorentz boost of the rest-frame density)."""
    p = np.linspace(-40, 40, 400001)
    mj = _deck({"ics_type": 6, "mu": 2.5, "amp": 0.0}, 0.0, 1.0)
    f = O.initial_f0(mj, 0, np.zeros_like(p), p)
    assert np.trapezoid(f, p) == pytest.approx(1.0, rel=1e-10)
    r2 = _deck({"ics_type": 7, "mu": 20.0, "pstr": 1.5, "amp": 0.0}, 0.0, 1.0)
    f = O.initial_f0(r2, 0, np.zeros_like(p), p)
    assert np.trapezoid(f, p) == pytest.approx(math.sqrt(1 + 1.5 ** 2), rel=1e-10)


CASES = [
    # name, species keys, domain, p range, library vs oracle bound (0 = bit-identical)
    ("friedman_beam", {"ics_type": 5, "pth": 0.5, "amp": 0.02}, (-0.001, 0.001), (-3, 3), 0.0),
    ("friedman_beam_wide", {"ics_type": 5, "pth": 1.0, "amp": 0.05}, (-2.0, 2.0), (-3, 3), 0.0),
    ("maxwell_juttner", {"ics_type": 6, "mu": 2.0, "amp": 0.01}, (0.0, 4 * math.pi), (-8, 8), 1e-14),
    ("relativistic_two_stream", {"ics_type": 7, "mu": 30.0, "pstr": 1.0, "amp": 0.01}, (0.0, 4 * math.pi),
     (-4, 4), 1e-14),
    ("travelling_wave", {"ics_type": 8, "amp": 1.3, "wave_beta": 0.8, "pth": 0.3}, (0.0, 5.0), (-1.5, 1.5),
     1e-13),
    ("landau", {"ics_type": 1, "pth": 1.0, "amp": 0.05}, (0.0, 4 * math.pi), (-6, 6), 0.0),
    ("colder_two_stream", {"ics_type": 4, "pth": 0.5, "pstr": 2.0, "amp": 0.05}, (0.0, 4 * math.pi), (-6, 6), 0.0),
]


@pytest.mark.parametrize("name,sp,xr,pr,bound", CASES, ids=[c[0] for c in CASES])
def test_library_f0_matches_oracle(name, sp, xr, pr, bound):
    d = _deck(sp, *xr)
    x, p = _points(3000, xr, pr, seed=len(name))
    a, b = M.initial_f0(d, 0, x, p), O.initial_f0(d, 0, x, p)
    assert np.all(np.isfinite(a)) and np.max(b) > 0
    if bound == 0.0:
        assert np.array_equal(a, b)
    else:
        assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)) <= bound


def test_unknown_ics_type_is_landau():
    """make_f0_return_ptr's default branch builds F0_LD."""
    x, p = _points(200, (0, 4 * math.pi), (-6, 6), seed=3)
    ld = _deck({"ics_type": 1, "pth": 1.0, "amp": 0.05}, 0.0, 4 * math.pi)
    unk = _deck({"ics_type": 11, "pth": 1.0, "amp": 0.05}, 0.0, 4 * math.pi)
    assert np.array_equal(M.initial_f0(unk, 0, x, p), M.initial_f0(ld, 0, x, p))


@pytest.mark.parametrize("sp,xr,x", [
    ({"ics_type": 8, "amp": 0.9, "wave_beta": 0.8}, (0.0, 5.0), 1.0),     # max gamma below 1
    ({"ics_type": 8, "amp": 2.0, "wave_beta": 0.8}, (0.0, 5.0), 1.0),     # particles faster than the wave
    ({"ics_type": 8, "amp": 1.3, "wave_beta": 0.8}, (0.0, 50.0), 40.0),   # beyond the tabulated orbit
    ({"ics_type": 5, "amp": 0.02}, (-0.01, 0.001), -0.009),               # beyond the density table
    ({"ics_type": 6, "mu": 0.0}, (0.0, 1.0), 0.5),                        # K_1(0) undefined
    ({"ics_type": 7, "mu": -1.0}, (0.0, 1.0), 0.5),
])
def test_invalid_initial_conditions_are_rejected(sp, xr, x):
    """Where the reference throws (check_gamma) or reads past its tables, the
    library returns FS_ERR_ARG and the oracle raises."""
    d = _deck(sp, *xr)
    with pytest.raises(M.FsError) as e:
        M.initial_f0(d, 0, np.array([x]), np.array([0.1]))
    assert e.value.code == 1
    with pytest.raises(ValueError):
        O.initial_f0(d, 0, np.array([x]), np.array([0.1]))


def test_stateless_oracle_helpers_refuse_tabulated_forms():
    for ics in (5, 6, 7, 8):
        with pytest.raises(ValueError):
            O.f0(ics, 1.0, 0.0, 0.5, 0.01, [0.1], [0.2])
    assert O.f0(1, 1.0, 0.0, 0.5, 0.01, [0.1], [0.2])[0] > 0
