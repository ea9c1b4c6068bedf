"""Host-side product code and the C ABI boundary (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import multi_species_b200 as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "fs_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:fs_status|const char\*|int|long long)\s+(fs_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(M.LIB_PATH)
    syms = header_symbols()
    assert syms and sorted(M.EXPORTS) == syms
    for s in syms:
        assert hasattr(lib, s), s


@pytest.mark.parametrize("h,ph,pmin,pmax", [(1, 0, -1.0, 1.0), (2, 1, -6.0, 6.0), (3, 2, -8.0, 8.0),
                                            (5, 1, -6.0, 6.0), (6, 2, -10.0, 10.0)])
@pytest.mark.parametrize("quad", [0, 1])
def test_host_mesh_bit_identical_to_oracle(h, ph, pmin, pmax, quad):
    L = 10 * np.pi
    a = O.Mesh(h, ph, 0.0, L, pmin, pmax)
    b = M.mesh(h, ph, 0.0, L, pmin, pmax, q=-0.9, quadrature=quad)
    assert np.array_equal(a.xs, b["xs"]) and np.array_equal(a.ps, b["ps"])
    assert np.array_equal(a.panels, b["panels"])
    assert np.array_equal(a.leaves, b["leaves"])
    assert np.array_equal(a.base_weights(-0.9, quad), b["base_weights"])


def test_argument_errors_are_reported():
    with pytest.raises(M.FsError) as ei:
        M.mesh(0, 0, 0.0, 1.0, 0.0, 1.0)
    assert ei.value.code == 1
    with pytest.raises(M.FsError) as ei:
        M.E_MQ_DirectSum_B200(-1.0, 0.1)
    assert ei.value.code == 1
    with pytest.raises(M.FsError) as ei:
        M.sim_params(dict(bcs=1, species_list=[{}]))
    assert ei.value.code == 8


def test_no_cpu_fallback_without_library(tmp_path, monkeypatch):
    monkeypatch.setattr(M, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(M, "_lib", None)
    with pytest.raises(ImportError):
        M.E_MQ_DirectSum_B200(1.0, 0.1)


def test_pool_estimate_grows_with_points_and_rejects_bad_params():
    from multi_species_b200 import decks
    fs = M
    small = fs.estimate_bytes(decks.landau_two_species(h=4, ph=0))
    big = fs.estimate_bytes(decks.landau_two_species(h=7, ph=1))
    assert 0 < small < big
    # 2 species x 257 x 513 points at about 1.1 kB each
    assert big == pytest.approx(2 * 257 * 513 * 1100 + 8 * 1024 * 1024)
    tree = fs.estimate_bytes(decks.bump_on_tail(h=5, ph=1), "treecode32c")
    assert tree > fs.estimate_bytes(decks.bump_on_tail(h=5, ph=1), "direct32c")
    for kw in (dict(max_live=0), dict(hbm_budget=0.0), dict(tuning=(3, 8)), dict(tuning=(4, 0))):
        with pytest.raises(fs.FsError):
            fs.Pool(**kw)


def test_session_rejects_open_boundaries_and_bad_drive():
    from multi_species_b200 import decks
    d = decks.landau_two_species(h=3, ph=1)
    with pytest.raises(M.FsError) as e:
        M.Simulation(d, "direct64_open")
    assert e.value.code == 8  # FS_ERR_UNSUPPORTED: field plugin only
    d2 = dict(d, external_field={"use_external_field": 1, "external_type": 7, "Am": 0.1, "k": 0.5, "omega": 0.3})
    with pytest.raises(M.FsError) as e:
        M.Simulation(d2)
    assert e.value.code == 1


def test_bench_host_rk4_caller_is_the_references_step():
    """The end-to-end leg of bench.py emulates AMRSimulation::rk4_step calling
    the field plugin with host arrays; with the oracle's direct sum as the
    plugin it reproduces the oracle's step bit for bit."""
    import importlib.util
    import pathlib

    import oracle as O
    from multi_species_b200 import decks
    spec = importlib.util.spec_from_file_location("bench", pathlib.Path(__file__).resolve().parents[1] / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    d = decks.landau_two_species(h=3, ph=1)
    d["remesh_period"] = 100
    o = O.Sim(d)
    st = o.state()
    L = d["xmax"] - d["xmin"]
    counts = o.species_points
    qm = np.concatenate([np.full(c, sp["q"] / sp["m"]) for c, sp in zip(counts, d["species_list"])])

    def field(es, t, nt, s, q, ns):
        es[:] = O.direct_sum(L, d["greens_epsilon"], t[:nt], s[:ns], q[:ns])

    xs, ps, es = bench.host_rk4_step(field, st["xs"], st["ps"], st["es"], st["q_ws"], qm, d["dt"])
    o.step()
    b = o.state()
    assert np.array_equal(xs, b["xs"]) and np.array_equal(ps, b["ps"]) and np.array_equal(es, b["es"])
