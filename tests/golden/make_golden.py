"""Generate the golden fixtures in tests/golden/.

    python tests/golden/make_golden.py

field_*.npz, drive_fields.npz -- inputs and outputs of the REFERENCE's own
    E_MQ_DirectSum, E_MQ_DirectSum_openbcs, E_MQ_Treecode and drive fields
    (ExternalTanh / ExternalSine / ExternalLogistic) (src/FieldStructure.cpp),
    run through oracle/_ref/libfs_ref.so (built from the reference sources by
    oracle/Makefile).  These pin the field.
sim_landau_h3.npz -- a short two-species trajectory (3 panels deep, 6 steps,
    one remesh) of the C oracle restatement (oracle/liboracle.so).  The
    reference's simulation driver cannot be compiled here, so this fixture
    records the restatement (parity unpinned) and guards it against drift.

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
    deck = decks.landau_two_species(h=3, ph=1, steps=6)
    s = O.Sim(deck)
    traj = {}
    for k in range(7):
        st = s.state()
        for key in ("xs", "ps", "fs", "q_ws", "es"):
            traj[f"{key}_{k}"] = st[key]
        if k < 6:
            s.step()
    np.savez_compressed(os.path.join(HERE, "sim_landau_h3.npz"), **traj)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
