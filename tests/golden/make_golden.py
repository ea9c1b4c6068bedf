"""Generate the golden fixtures in tests/golden/.

    python tests/golden/make_golden.py

field_*.npz, drive_fields.npz -- inputs and outputs of the REFERENCE's own
    E_MQ_DirectSum, E_MQ_DirectSum_openbcs, E_MQ_Treecode and drive fields
    (ExternalTanh / ExternalSine / ExternalLogistic) (src/FieldStructure.cpp),
    run through oracle/_ref/libfs_ref.so (built from the reference sources by
    oracle/Makefile).  These pin the field.
sim_landau_h3.npz, ref_sim_*.npz -- trajectories of the REFERENCE's own
    AMRSimulation (constructor from the deck, then step(); src/simulation_files,
    src/structure_files, src/FieldStructure.cpp) run through
    oracle/_ref/libamr_ref.so, built from the reference sources by
    oracle/Makefile: the state (xs, ps, fs, q_ws, es, species concatenated) at
    the listed iterations.  These pin RK4, step control, the remesh, the
    reduced grid, adaptive refinement and the treecode session.

Inputs are seeded; every array is float64.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from multi_species_b200 import decks  # noqa: E402


def field_cases():
    rng = np.random.default_rng(20261203)
    L = 4 * np.pi
    cases = {}
    # random sources spread over three periods (unwrapped positions, as the
    # reference never wraps x), mixed-sign weights
    x = rng.uniform(-L, 2 * L, 700)
    q = rng.normal(size=700) * 1e-3
    cases["random"] = dict(L=L, eps=0.05, targets=x, sources=x, q=q)
    # separate target set, exact half-period and coincident offsets
    t = np.concatenate([rng.uniform(0, L, 300), x[:20], x[:10] + L / 2, x[:10] + L])
    cases["targets"] = dict(L=L, eps=0.05, targets=t, sources=x, q=q)
    # lattice of a small mesh (duplicate x columns, many exact coincidences)
    m = O.Mesh(2, 1, 0.0, 10 * np.pi, -8.0, 8.0)
    w = m.base_weights(-1.0, 0)
    f = O.f0(3, 1.0, 0.0, 0.2, 0.005, m.xs, m.ps)
    cases["lattice"] = dict(L=10 * np.pi, eps=0.02, targets=m.xs, sources=m.xs, q=w * f)
    return cases


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libfs_ref.so missing: run `make -C oracle` where the reference sources exist")
    for name, c in field_cases().items():
        e = O.ref_direct_sum(c["L"], c["eps"], c["targets"], c["sources"], c["q"])
        np.savez_compressed(os.path.join(HERE, f"field_direct_{name}.npz"), L=c["L"], eps=c["eps"],
                            targets=c["targets"], sources=c["sources"], q=c["q"], es=e)
    # open boundaries (E_MQ_DirectSum_openbcs): separate targets, coincident points
    rng = np.random.default_rng(11)
    src = rng.uniform(-3.0, 9.0, 600)
    tgt = np.concatenate([rng.uniform(-4.0, 10.0, 250), src[:25]])
    qo = rng.normal(size=600) * 1e-3
    e = O.ref_direct_sum_open(0.05, tgt, src, qo)
    np.savez_compressed(os.path.join(HERE, "field_open.npz"), eps=0.05, targets=tgt, sources=src, q=qo, es=e)
    # drive fields (ExternalTanh / Sine / Logistic) at times across their switches
    x = rng.uniform(-5.0, 30.0, 200)
    times = np.array([0.0, 3.0, 9.75, 10.0, 49.0, 60.0, 70.0, 120.0, 175.0, 205.0, 300.0])
    drive = {}
    for kind in (0, 1, 2):
        out = []
        for t in times:
            e0 = np.zeros_like(x)
            out.append(O.ref_external_field(kind, 0.3, 0.26, 0.37, e0, x, float(t)))
        drive[f"es_{kind}"] = np.array(out)
    np.savez_compressed(os.path.join(HERE, "drive_fields.npz"), x=x, times=times, Am=0.3, k=0.26, omega=0.37,
                        **drive)
    rng = np.random.default_rng(7)
    L = 20 * np.pi
    x = rng.uniform(-L / 2, 1.5 * L, 5000)
    q = np.abs(rng.normal(size=5000)) * 1e-4 - 5e-5
    e = O.ref_treecode(L, 0.02, 0.7, 8, 300, x, q)
    np.savez_compressed(os.path.join(HERE, "field_treecode.npz"), L=L, eps=0.02, mac=0.7, degree=8,
                        max_source=300, sources=x, q=q, es=e)
    if not O.amr_ref_available():
        raise SystemExit("oracle/_ref/libamr_ref.so missing: run `make -C oracle REF=<reference checkout>`")
    save_trajectory("sim_landau_h3.npz", decks.landau_two_species(h=3, ph=1, steps=6), range(7))
    for name, (deck, iters) in REF_TRAJECTORIES.items():
        save_trajectory(f"ref_sim_{name}.npz", deck, iters)
    print("golden fixtures written to", HERE)


def _adaptive_two_stream():
    d = decks.two_stream(h=3, ph=1, steps=6, remesh_period=3)
    d["species_list"][0].update(do_adaptively_refine=True, max_height=5, amr_epsilons=[0.02])
    return d


def _bump_on_tail_treecode():
    d = decks.bump_on_tail(h=3, ph=1, steps=6)
    d["max_source"] = 200
    d["remesh_period"] = 3
    return d


# name -> (deck, iterations whose state is stored)
REF_TRAJECTORIES = {
    "two_stream_h4": (decks.two_stream(h=4, ph=1, steps=8, remesh_period=3), (0, 2, 3, 6, 8)),
    "adaptive_two_stream_h3": (_adaptive_two_stream(), (0, 2, 3, 6)),
    "bump_on_tail_h3": (_bump_on_tail_treecode(), (0, 2, 3, 6)),
}


def save_trajectory(fname, deck, iters):
    """The reference's state at each iteration of `iters` (increasing)."""
    r = O.RefSim(deck)
    out = {"iters": np.array(list(iters), dtype=np.int32)}
    for k in iters:
        r.step(k - r.iter)
        st = r.state()
        for key in ("xs", "ps", "fs", "q_ws", "es"):
            out[f"{key}_{k}"] = st[key]
    r.close()
    np.savez_compressed(os.path.join(HERE, fname), **out)


if __name__ == "__main__":
    main()
