"""Scene construction (host only)."""
import numpy as np

from delta_b200.scenarios import lattice_scene, mass_properties, sphere_mesh


def test_sphere_mesh_counts_and_closure():
    rng = np.random.default_rng(0)
    for nt in (20, 40, 80, 160, 320, 500):
        V, F = sphere_mesh(nt, rng, 1.0)
        assert F.shape == (nt, 3)
        # closed 2-manifold: every edge shared by exactly two triangles
        e = np.sort(np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]), 1)
        _, cnt = np.unique(e, axis=0, return_counts=True)
        assert np.all(cnt == 2)


def test_mass_properties_of_a_fine_sphere():
    V, F = sphere_mesh(1280, None, 0.5)
    m, c, J = mass_properties(V, F, 2.0)
    exact = 2.0 * 4.0 / 3.0 * np.pi * 0.5 ** 3
    assert abs(m - exact) / exact < 0.02
    assert np.allclose(c, 0.0, atol=1e-12)
    assert np.allclose(J, np.eye(3) * J[0, 0], atol=1e-3 * J[0, 0])
    assert abs(J[0, 0] - 0.4 * m * 0.25) / (0.4 * m * 0.25) < 0.02


def test_mass_properties_translation_invariant():
    V, F = sphere_mesh(80, np.random.default_rng(1), 0.01, (0.8, 1.2))
    a = mass_properties(V, F, 2500.0)
    b = mass_properties(V + [0.3, -0.2, 5.0], F, 2500.0)
    assert np.isclose(a[0], b[0]) and np.allclose(a[1] + [0.3, -0.2, 5.0], b[1]) and np.allclose(a[2], b[2])


def test_lattice_scene_shape():
    s = lattice_scene(0)
    assert s["n_bodies"] == 257 and s["obstacle"].sum() == 1
    assert s["tri_offset"][-1] == 256 * 80 + 2
    assert np.all(s["mass"][:256] > 0) and np.isinf(s["mass"][256])
    assert np.all(s["radius"][:256] < 0.014)
