"""Sphere model on the GPU (delta_sphere_contacts, delta_sphere_mesh_contacts,
delta_sphere_overlap) against the oracle (pinned to sphere.cpp/point.cpp): bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["x", "normal", "depth", "P", "Q", "friction", "eps_total", "master", "slave", "penetration", "tri_a",
          "tri_b"]


def _cloud(rng, n):
    centre = rng.uniform(0, 0.06, (3, n))
    diameter = rng.uniform(0.008, 0.02, n)
    eps = rng.uniform(5e-4, 2e-3, n)
    fric = (rng.random(n) < 0.5).astype(np.uint8)
    ids = np.arange(n, dtype=np.int32) * 3 + 1
    return centre, diameter, eps, fric, ids


def test_sphere_contacts_match_oracle(ctx, oracle):
    from delta_b200.detection import Spheres, sphere

    from oracle.oracle import CONTACT_DTYPE

    rng = np.random.default_rng(0)
    n = 300
    centre, diameter, eps, fric, ids = _cloud(rng, n)
    pa, pb = np.triu_indices(n, 1)
    pa, pb = pa.astype(np.int32), pb.astype(np.int32)
    got = sphere(ctx, Spheres(centre, diameter, eps, fric, ids), pa, pb, capacity=16).to_numpy()
    ref = [oracle.sphere(centre[:, a], diameter[a], eps[a], fric[a], ids[a], centre[:, b], diameter[b], eps[b],
                         fric[b], ids[b]) for a, b in zip(pa, pb)]
    ref = np.concatenate(ref) if ref else np.zeros(0, CONTACT_DTYPE)
    assert len(got) == len(ref) > 100
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f], equal_nan=True), f


@pytest.mark.parametrize("sphere_is_b", [0, 1])
def test_sphere_mesh_contacts_match_oracle(ctx, oracle, sphere_is_b):
    from delta_b200.detection import Meshes, Spheres, sphereWithBarrierAB, sphereWithBarrierBA
    from delta_b200.scenarios import sphere_mesh

    from oracle.oracle import CONTACT_DTYPE

    rng = np.random.default_rng(10 + sphere_is_b)
    bodies = []
    for k, nt in enumerate((80, 160, 40)):
        V, F = sphere_mesh(nt, rng, 0.03, (0.9, 1.1))
        bodies.append((V[F].reshape(-1, 3) + np.array([0.07 * k, 0, 0])).T.copy())
    meshes = Meshes.from_bodies(bodies, np.array([1e-3, 2e-3, 1.5e-3]), np.array([1, 0, 1], np.uint8),
                                np.array([100, 101, 102]))
    centre, diameter, eps, fric, ids = _cloud(rng, 60)
    centre[0] *= 2.5
    sidx = np.repeat(np.arange(60, dtype=np.int32), 3)
    bidx = np.tile(np.arange(3, dtype=np.int32), 60)
    fn = sphereWithBarrierBA if sphere_is_b else sphereWithBarrierAB
    got = fn(ctx, Spheres(centre, diameter * 3, eps, fric, ids), meshes, sidx, bidx, capacity=8).to_numpy()
    ref = []
    for s, bd in zip(sidx, bidx):
        ref.append(oracle.sphere_mesh(sphere_is_b, centre[:, s], diameter[s] * 3, eps[s], fric[s], ids[s],
                                      bodies[bd], bodies[bd].shape[1] // 3, meshes.eps[bd].item(),
                                      int(meshes.friction[bd].item()), int(meshes.id[bd].item())))
    ref = np.concatenate(ref) if ref else np.zeros(0, CONTACT_DTYPE)
    assert len(got) == len(ref) > 20
    for f in FIELDS:
        assert np.array_equal(got[f], ref[f], equal_nan=True), f


def test_sphere_overlap_matches_oracle(ctx, oracle):
    from delta_b200.detection import isSphereOverlayInContact

    rng = np.random.default_rng(3)
    n = 500
    centre = rng.normal(size=(3, n))
    radius = rng.uniform(0, 1.5, n)
    pa = rng.integers(0, n, 20000).astype(np.int32)
    pb = rng.integers(0, n, 20000).astype(np.int32)
    got = isSphereOverlayInContact(ctx, centre, radius, pa, pb).cpu().numpy()
    ref = np.array([oracle.sphere_overlay(centre[:, a], radius[a], centre[:, b], radius[b]) for a, b in zip(pa, pb)])
    assert np.array_equal(got, ref)
    assert 0 < got.sum() < got.size


def test_sphere_empty_inputs(ctx):
    from delta_b200.detection import Spheres, isSphereOverlayInContact, sphere

    rng = np.random.default_rng(4)
    s = Spheres(*_cloud(rng, 4))
    assert sphere(ctx, s, [], []).count == 0
    assert isSphereOverlayInContact(ctx, rng.normal(size=(3, 4)), np.ones(4), [], []).numel() == 0
