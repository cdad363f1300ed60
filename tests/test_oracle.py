"""The oracle restatement (oracle/delta_oracle.c) against the reference's own outputs:
committed golden fixtures (always) and the reference build in oracle/_ref (when present)."""
import numpy as np
import pytest

from oracle.oracle import CONTACT_DTYPE, Reference

PAIR_METHODS = ["bf", "penalty", "penalty_iter", "gjk", "hybrid"]
CONTACT_FIELDS = ["x", "normal", "depth", "P", "Q", "friction", "eps_total", "master", "slave", "penetration"]


@pytest.mark.parametrize("m", range(5))
def test_pairs_match_golden_bitwise(oracle, golden, m):
    g = golden["pairs"]
    name = PAIR_METHODS[m]
    p, q, d, fl = oracle.pairs(m, g["a"], g["b"], max_error=float(g["max_error"]), nthreads=1)
    assert np.array_equal(p, g[f"{name}_p"])
    assert np.array_equal(q, g[f"{name}_q"])
    assert np.array_equal(d, g[f"{name}_d"])
    assert np.array_equal(fl, g[f"{name}_flags"])


def test_kat1_collision_test_geometry(oracle):
    """KAT-1 of multiscale/dem/tests/CollisionTest.cpp:32-86: A = {(0,0,0),(0,1,0),(0,0,1)},
    B = A shifted to x = 0.2; no contact at eps_total 0.1, one at 0.25."""
    A = np.array([[0, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    B = A + [0.2, 0, 0]
    p, q, d, _ = oracle.pairs(0, A.reshape(9, 1), B.reshape(9, 1))
    assert np.allclose(p[:, 0], [0, 0, 0]) and np.allclose(q[:, 0], [0.2, 0, 0]) and d[0] == pytest.approx(0.2)
    c, _ = oracle.detect(0, A.T.copy(), 1, 0.05, 0, 0, B.T.copy(), 1, 0.05, 0, 1)
    assert len(c) == 0
    c, _ = oracle.detect(0, A.T.copy(), 1, 0.125, 0, 0, B.T.copy(), 1, 0.125, 0, 1)
    assert len(c) == 1
    assert np.allclose(c["x"][0], [0.1, 0, 0]) and np.allclose(c["normal"][0], [-1, 0, 0])
    assert c["depth"][0] == pytest.approx(0.05)


@pytest.mark.parametrize("drv", range(7))
def test_drivers_match_golden(oracle, golden, drv):
    g = golden["drivers"]
    c, st = oracle.detect(drv, g["A"], int(g["nA"]), float(g["eps"]), 1, 3, g["B"], int(g["nB"]), float(g["eps"]),
                          1, 8, stats=True)
    ref = g[f"contacts_{drv}"]
    assert len(c) == len(ref)
    for f in CONTACT_FIELDS:
        assert np.array_equal(c[f], ref[f]), f
    if drv == 2:
        assert list(st.newton_hist) == list(g["hist_2"])
    if drv in (5, 6):
        assert [st.penalty_fails, st.batch_fails] == list(g[f"fails_{drv}"])


def test_forces_and_expmap_match_golden(oracle, golden):
    g = golden["dynamics"]
    s = g["forces_state"]
    F, T = oracle.contacts_forces(g["forces_contacts"], 1.0, s[0:3], s[3:6], s[6:9], s[9], s[10:13], s[13:16],
                                  s[16:19], s[19], 1e4, 0.5, 0.5)
    assert np.array_equal(F, g["forces_F"]) and np.array_equal(T, g["forces_T"])
    for o, L in zip(g["expmap_in"], g["expmap_out"]):
        out = oracle.expmap(o)
        if np.dot(o, o) < 3.0461741978671e-02:
            assert np.array_equal(out, L)  # Taylor branch: pure arithmetic
        else:
            assert np.allclose(out, L, rtol=0, atol=1e-15)  # libm sin/cos


needs_ref = pytest.mark.skipif(not Reference.available(), reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("m", range(5))
def test_pairs_match_reference_build(oracle, m):
    from delta_b200.scenarios import narrowphase_pairs

    ref = Reference()
    a, b, _, _ = narrowphase_pairs(20000, seed=11)
    r = ref.pairs(m, a, b, max_error=2e-4)
    o = oracle.pairs(m, a, b, max_error=2e-4)
    for x, y in zip(r, o):
        assert np.array_equal(x, y)


@needs_ref
@pytest.mark.parametrize("drv", range(7))
def test_drivers_match_reference_build(oracle, drv):
    from delta_b200.scenarios import sphere_mesh

    ref = Reference()
    rng = np.random.default_rng(100 + drv)
    for nt in (20, 40):
        VA, FA = sphere_mesh(nt, rng, 0.05, (0.85, 1.15))
        VB, FB = sphere_mesh(nt, rng, 0.05, (0.85, 1.15))
        A = VA[FA].reshape(-1, 3).T.copy()
        B = (VB[FB].reshape(-1, 3) + rng.normal(size=3) * 0.02 + [0.08, 0, 0]).T.copy()
        r, _ = ref.detect(drv, A, nt, 0.003, 1, 1, B, nt, 0.003, 0, 2)
        o, _ = oracle.detect(drv, A, nt, 0.003, 1, 1, B, nt, 0.003, 0, 2)
        assert len(r) == len(o)
        for f in CONTACT_FIELDS:
            assert np.array_equal(r[f], o[f]), f


@needs_ref
def test_forces_match_reference_build(oracle):
    ref = Reference()
    rng = np.random.default_rng(5)
    c = np.zeros(40, CONTACT_DTYPE)
    c["x"] = rng.random((40, 3))
    n = rng.normal(size=(40, 3))
    c["normal"] = n / np.linalg.norm(n, axis=1, keepdims=True)
    c["depth"] = rng.random(40) * 1e-3
    c["friction"] = rng.integers(0, 2, 40)
    st = (rng.random(3), rng.normal(size=3), rng.normal(size=3), 0.3, rng.random(3), rng.normal(size=3),
          rng.normal(size=3), 0.7)
    F1, T1 = oracle.contacts_forces(c, 1.0, *st, 1e4, 0.5, 0.5)
    F2, T2 = ref.contacts_forces(c, *st)
    assert np.array_equal(F1, F2) and np.array_equal(T1, T2)


def test_time_step_equals_the_reference_driven_step(oracle):
    """The oracle's time step (dor_sim_run) against a time step driven by the reference's
    own bf(), getContactsForces, updateAngular, updateRotationMatrix and updateVertices
    (oracle/ref_sim.cpp), with forces.cpp's compiled constants: bit for bit."""
    from oracle.oracle import Reference

    if not Reference.available("par"):
        pytest.skip("oracle/_ref not built (the reference sources are absent)")
    from delta_b200.scenarios import lattice_scene

    sc = lattice_scene(seed=7, nx=4, ny=2, nz=4, friction=True)
    dt, g = 1e-5, (0.0, -9.81, 0.0)
    o_state, o_cps, _ = oracle.simulate(sc, dt, g, 1e4, 0.5, 0.5, 4)
    r_state, r_cps = Reference("par").simulate(sc, dt, g, 4)
    assert list(o_cps) == list(r_cps) and o_cps[-1] > 0
    for k in ("pos", "vel", "ang", "ref_ang", "rot", "x", "y", "z"):
        assert np.array_equal(o_state[k], r_state[k]), k
