"""Seeded inputs for the zoltan/ code path tests: a whole SoA system of bodies and
triangles (zoltan/dynamics.h layouts) and per-master contact lists (zoltan/forces.h)."""
import numpy as np


def _rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([1 - 2 * (y * y + z * z), 2 * (x * y + z * w), 2 * (x * z - y * w),
                  2 * (x * y - z * w), 1 - 2 * (x * x + z * z), 2 * (y * z + x * w),
                  2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)])  # column-major rows
    return R


def system(nb=64, tris_per_body=20, seed=0, omega=1.0):
    """Bodies (arrays (k, nb)) and their triangles t (6, 3, nt) with owner pid."""
    rng = np.random.default_rng(seed)
    position = np.zeros((6, nb))
    position[:3] = rng.uniform(-1, 1, (3, nb))
    position[3:] = position[:3] + rng.normal(0, 0.01, (3, nb))
    angular = np.zeros((6, nb))
    angular[:3] = rng.normal(0, omega, (3, nb))
    angular[3:] = rng.normal(0, omega, (3, nb))
    linear = rng.normal(0, 1, (3, nb))
    rotation = _rotations(rng, nb)
    d = rng.uniform(0.5, 2.0, (3, nb))
    inertia = np.zeros((9, nb)); inverse = np.zeros((9, nb))
    inertia[[0, 4, 8]] = d
    inverse[[0, 4, 8]] = 1.0 / d
    inertia[[1, 3]] = inertia[[3, 1]] = 0.01 * d[0] * d[1]
    mass = rng.uniform(0.5, 3.0, nb)
    force = rng.normal(0, 1, (3, nb)); torque = rng.normal(0, 0.1, (3, nb))
    nt = nb * tris_per_body
    pid = np.repeat(np.arange(nb, dtype=np.int32), tris_per_body)
    rng.shuffle(pid)
    t = np.zeros((6, 3, nt))
    t[3:] = position[3:6, pid][None] + rng.normal(0, 0.05, (3, 3, nt))
    t[:3] = t[3:] + rng.normal(0, 1e-3, (3, 3, nt))
    return dict(t=t, pid=pid, angular=angular, linear=linear, rotation=rotation, position=position,
                inertia=inertia, inverse=inverse, mass=mass, force=force, torque=torque)


def contacts(nb=64, per_master=(0, 6), seed=0):
    """Contacts grouped by master body: offset (nb+1), slave, point (3, n), normal, depth."""
    rng = np.random.default_rng(seed + 1000)
    counts = rng.integers(per_master[0], per_master[1] + 1, nb)
    offset = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    n = int(offset[-1])
    master = np.repeat(np.arange(nb), counts)
    slave = (master + rng.integers(1, nb, n)) % nb
    point = rng.uniform(-1, 1, (3, n))
    normal = rng.normal(size=(3, n))
    depth = rng.uniform(-1e-3, 1e-2, n)
    return dict(offset=offset, slave=slave.astype(np.int32), point=point, normal=normal, depth=depth)
