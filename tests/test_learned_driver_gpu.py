"""The learned FP32 hybrid as a particle driver (DELTA_DRV_LEARNED) and in the time step,
against FP64 bf (the oracle's contact set and trajectory).

Bounds: every contact's distance within 1e-6 relative of FP64 bf's for the same
triangle pair; the contact set equal to FP64 bf's except for triangle pairs whose FP64
distance lies within 1e-6 (relative) of the threshold; over 40 time steps of the
256-icosphere lattice the positions stay within 1e-12 m and the velocities within 1e-9 m/s
of the oracle's FP64 trajectory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = dict(dt=1e-5, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0)


def _scene(seed, sizes=(20, 40, 80, 20, 40, 80, 160), eps=0.003):
    from delta_b200.scenarios import sphere_mesh

    rng = np.random.default_rng(seed)
    bodies = []
    for k, nt in enumerate(sizes):
        V, F = sphere_mesh(nt, rng, 0.05, (0.85, 1.15))
        c = np.array([0.085 * k, 0.004 * rng.normal(), 0.004 * rng.normal()])
        bodies.append((V[F].reshape(-1, 3) + c).T.copy())
    n = len(sizes)
    pa = list(range(n - 1)) + list(range(n - 2))
    pb = [i + 1 for i in range(n - 1)] + [i + 2 for i in range(n - 2)]
    return bodies, pa, pb, np.full(n, eps), np.zeros(n, np.uint8), np.arange(n) * 10 + 3


def _key(c):
    return list(zip(c["master"].tolist(), c["slave"].tolist(), c["tri_a"].tolist(), c["tri_b"].tolist()))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_learned_driver_contacts_vs_fp64_bf(ctx, seed):
    from delta_b200.detection import DRV_BF, DRV_LEARNED, Meshes, detect

    bodies, pa, pb, eps_b, fric, ids = _scene(seed)
    m = Meshes.from_bodies(bodies, eps_b, fric, ids)
    ref = detect(ctx, DRV_BF, m, pa, pb)[0].to_numpy()
    got = detect(ctx, DRV_LEARNED, m, pa, pb)[0].to_numpy()
    assert len(ref) > 0
    thr = ref["eps_total"][0]
    kr, kg = _key(ref), _key(got)
    dr = thr - ref["depth"]
    dg = thr - got["depth"]
    # the same triangle pairs, except ones whose FP64 distance sits in the band
    only_ref = set(kr) - set(kg)
    only_got = set(kg) - set(kr)
    for k in only_ref:
        d = dr[kr.index(k)]
        assert abs(d - thr) <= 1e-6 * thr, (k, d)
    assert not only_got or all(abs(dg[kg.index(k)] - thr) <= 2e-6 * thr for k in only_got)
    # distances of the common contacts within 1e-6 relative; most are bit-identical
    idx = {k: i for i, k in enumerate(kg)}
    common = [(i, idx[k]) for i, k in enumerate(kr) if k in idx]
    ir, ig = np.array(common).T
    rel = np.abs(dg[ig] - dr[ir]) / dr[ir]
    assert rel.max() <= 1e-6
    # where the FP32 search named bfSolver's own feature the points are bfSolver's bit for
    # bit; elsewhere another feature within 1e-6 of the minimum was taken
    same = np.all(got["P"][ig] == ref["P"][ir], axis=1) & np.all(got["Q"][ig] == ref["Q"][ir], axis=1)
    assert same.mean() >= 0.75, same.mean()


@pytest.mark.parametrize("graph", [False, True])
def test_learned_driver_trajectory_close_to_oracle(ctx, oracle, graph):
    from delta_b200.detection import DRV_LEARNED
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.scenarios import lattice_scene

    scene = lattice_scene(seed=3)
    steps = 40
    p = PARAMS
    o_state, o_cps, _ = oracle.simulate(scene, p["dt"], p["gravity"], p["spring"], p["damper"], p["friction"], steps)
    sim = Simulation(ctx, scene, DRV_LEARNED)
    cps = sim.step(steps, StepParams.make(**p), graph=graph)
    st = sim.state()
    sim.close()
    assert np.max(np.abs(np.asarray(cps) - np.asarray(o_cps))) <= 2
    assert np.max(np.abs(st["pos"] - o_state["pos"])) <= 1e-12
    assert np.max(np.abs(st["vel"] - o_state["vel"])) <= 1e-9
    print("learned trajectory: max |dpos|", np.max(np.abs(st["pos"] - o_state["pos"])),
          "max |dvel|", np.max(np.abs(st["vel"] - o_state["vel"])),
          "contacts/step equal:", np.mean(np.asarray(cps) == np.asarray(o_cps)))
