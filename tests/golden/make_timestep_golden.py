"""Generates the time-step fixtures tests/golden/timestep_{lattice_1000,hopper_2000}.json by
running the reference-driven time step (oracle/ref_sim.cpp over the reference's own bf(),
getContactsForces, updateAngular, updateRotationMatrix and updateVertices, built by
oracle/Makefile into oracle/_ref/libdelta_ref.so without FMA contraction) for the full
length of two configurations:

    python tests/golden/make_timestep_golden.py [lattice|hopper ...]

- lattice: 256 icospheres (80 triangles) on an 8x4x8 lattice over a 2-triangle floor
  (delta_b200.scenarios.lattice_scene(seed=2024)), dt 1e-5, 1000 steps;
- hopper: 10,000 spheres of 40-320 triangles over a 2,048-triangle cone
  (hopper_scene(10000, seed=7)), dt 5e-6, 2000 steps.

Gravity (0, -9.81, 0); the force constants are those compiled into forces.cpp (spring 1e4,
damper 0.5, friction 0.5).  A fixture holds the contacts of every step and the SHA-256 of
every state array after the last step (positions, velocities, angular velocities,
rotations, vertices), so the GPU test compares the whole state bit for bit without
storing it.
"""
from __future__ import annotations

import hashlib
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from delta_b200.scenarios import hopper_scene, lattice_scene  # noqa: E402
from oracle.oracle import Reference  # noqa: E402

OUT = Path(__file__).resolve().parent
STATE = ("pos", "vel", "ang", "ref_ang", "rot", "x", "y", "z")
CASES = {
    "lattice": dict(scene=lambda: lattice_scene(seed=2024), dt=1e-5, steps=1000, name="timestep_lattice_1000.json"),
    "hopper": dict(scene=lambda: hopper_scene(10000, seed=7), dt=5e-6, steps=2000, name="timestep_hopper_2000.json"),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float64).tobytes()).hexdigest()


def main(names):
    ref = Reference("par")
    for name in names:
        c = CASES[name]
        t0 = time.time()
        state, cps = ref.simulate(c["scene"](), c["dt"], (0.0, -9.81, 0.0), c["steps"])
        out = {"case": name, "dt": c["dt"], "steps": c["steps"], "gravity": [0.0, -9.81, 0.0],
               "material": {"spring": 1e4, "damper": 0.5, "friction": 0.5},
               "contacts_per_step": [int(x) for x in cps],
               "sha256": {k: digest(state[k]) for k in STATE},
               "pos_first_bodies": np.asarray(state["pos"][:24], np.float64).tolist(),
               "seconds": round(time.time() - t0, 1)}
        (OUT / c["name"]).write_text(json.dumps(out, indent=1) + "\n")
        print(name, out["seconds"], "s")


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
