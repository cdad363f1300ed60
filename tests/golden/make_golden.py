"""Generates the golden fixtures in tests/golden/ by running the reference's own
functions (oracle/_ref/libdelta_ref.so, built from the reference sources by
oracle/Makefile) on seeded inputs.

    python tests/golden/make_golden.py

The fixtures pin the oracle restatement (tests/test_oracle.py) on machines where the
reference sources are absent.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from delta_b200.scenarios import narrowphase_pairs, sphere_mesh  # noqa: E402
from oracle.oracle import CONTACT_DTYPE, Reference  # noqa: E402

OUT = Path(__file__).resolve().parent


def edge_case_pairs():
    """Hand-made pairs: KAT-1 (multiscale/dem/tests/CollisionTest.cpp:32-86), identical,
    coplanar-overlapping, parallel edges, shared vertex, degenerate (zero-area) triangles."""
    A0 = np.array([[0, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    cases = [
        (A0, A0 + [0.2, 0, 0]),                                     # KAT-1
        (A0, A0.copy()),                                            # identical
        (A0, A0 + [0, 0.3, 0.3]),                                   # coplanar, overlapping
        (A0, A0 + [0.0, 1.5, 0.0]),                                 # coplanar, apart
        (A0, A0[[0, 2, 1]] + [0.1, 0.0, 0.0]),                      # reversed winding
        (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
         np.array([[0.2, 0.2, 0.5], [0.8, 0.2, 0.5], [0.2, 0.8, 0.5]], float)),  # parallel planes
        (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
         np.array([[0.25, -1, 0.3], [0.25, 1, 0.3], [0.25, 0, 1.0]], float)),    # edge over face
        (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
         np.array([[0, 0, 0], [-1, 0, 0], [0, -1, 0.5]], float)),   # shared vertex
        (np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0]], float),
         np.array([[0, 1, 0], [1, 1, 0], [0, 2, 1]], float)),       # degenerate A (collinear)
        (np.array([[0, 0, 0], [1, 1, 1], [1, 1, 1]], float),
         np.array([[3, 0, 0], [3, 1, 0], [3, 0, 1]], float)),       # degenerate A (repeated vertex)
        (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
         np.array([[0.3, 0.3, -0.5], [0.3, 0.3, 0.5], [0.9, 0.9, 0.0]], float)),  # piercing
        (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float),
         np.array([[0.5, 0.5, 1e-9], [0.9, 0.5, 1e-9], [0.5, 0.9, 1e-9]], float)),  # touching above edge
    ]
    a = np.stack([c[0].reshape(9) for c in cases], 1)
    b = np.stack([c[1].reshape(9) for c in cases], 1)
    return a, b


def main():
    ref = Reference("par")
    # ---- pair list: microbenchmark draw + edge cases --------------------------------------
    a, b, dtrue, cls = narrowphase_pairs(384, seed=20240601)
    ea, eb = edge_case_pairs()
    a = np.concatenate([a, ea], 1)
    b = np.concatenate([b, eb], 1)
    max_error = 1e-3
    res = {"a": a, "b": b, "max_error": np.float64(max_error)}
    for m, name in enumerate(["bf", "penalty", "penalty_iter", "gjk", "hybrid"]):
        p, q, d, fl = ref.pairs(m, a, b, max_error=max_error, nthreads=1)
        res[f"{name}_p"], res[f"{name}_q"], res[f"{name}_d"], res[f"{name}_flags"] = p, q, d, fl
    np.savez_compressed(OUT / "pairs.npz", **res)

    # ---- particle-pair drivers on two perturbed sphere meshes -------------------------------
    rng = np.random.default_rng(7)
    VA, FA = sphere_mesh(20, rng, radius=0.05, perturb=(0.9, 1.1))
    VB, FB = sphere_mesh(20, rng, radius=0.05, perturb=(0.9, 1.1))
    A = VA[FA].reshape(-1, 3).T.copy()
    B = (VB[FB].reshape(-1, 3) + [0.078, 0.01, 0.0]).T.copy()
    nA, nB = FA.shape[0], FB.shape[0]
    drv = {"A": A, "B": B, "nA": nA, "nB": nB, "eps": np.float64(0.004)}
    for d_ in range(7):
        c, st = ref.detect(d_, A, nA, 0.004, 1, 3, B, nB, 0.004, 1, 8, stats=True)
        drv[f"contacts_{d_}"] = c
        drv[f"hist_{d_}"] = np.array(list(st.newton_hist), np.int64)
        drv[f"fails_{d_}"] = np.array([st.penalty_fails, st.batch_fails], np.int64)
    np.savez_compressed(OUT / "drivers.npz", **drv)

    # ---- forces and dynamics (forces.cpp constants SPRING 1e4, DAMPER 0.5, FRICTION 0.5) ---
    dyn = {}
    c = np.zeros(6, CONTACT_DTYPE)
    c["x"] = rng.random((6, 3)) * 0.1
    nrm = rng.normal(size=(6, 3))
    c["normal"] = nrm / np.linalg.norm(nrm, axis=1, keepdims=True)
    c["depth"] = rng.random(6) * 1e-3
    c["friction"] = [1, 0, 1, 0, 1, 1]
    state = [rng.random(3) * 0.1, rng.normal(size=3), rng.normal(size=3), 0.02,
             rng.random(3) * 0.1, rng.normal(size=3), rng.normal(size=3), 0.05]
    F, T = ref.contacts_forces(c, *state)
    dyn.update(forces_contacts=c, forces_state=np.array([*state[0], *state[1], *state[2], state[3], *state[4],
                                                         *state[5], *state[6], state[7]]), forces_F=F, forces_T=T)
    om = np.concatenate([rng.normal(size=(8, 3)) * 0.05, rng.normal(size=(4, 3))])  # small and large angles
    dyn["expmap_in"] = om
    dyn["expmap_out"] = np.stack([ref.expmap(o) for o in om])
    np.savez_compressed(OUT / "dynamics.npz", **dyn)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
