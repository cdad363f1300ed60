"""Time step on the GPU against the oracle's time step (oracle/delta_oracle.c dor_sim_run):
same update order, FP64 reference arithmetic, deterministic summation order, so the
trajectory (positions, velocities, rotations, angular velocities, vertices) and the
contact lists must agree bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = dict(dt=1e-5, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0)
STATE = ("pos", "vel", "ang", "ref_ang", "rot", "x", "y", "z")
FIELDS = ["x", "normal", "depth", "P", "Q", "friction", "eps_total", "master", "slave", "tri_a", "tri_b"]


@pytest.fixture(scope="module")
def scene():
    from delta_b200.scenarios import lattice_scene

    return lattice_scene(seed=3)


def _oracle(oracle, scene, steps, friction_flag=False):
    p = PARAMS
    return oracle.simulate(scene, p["dt"], p["gravity"], p["spring"], p["damper"], p["friction"], steps)


def _gpu(ctx, scene, steps, driver=0):
    from delta_b200.engine import Simulation, StepParams

    sim = Simulation(ctx, scene, driver)
    cps = sim.step(steps, StepParams.make(**PARAMS))
    st = sim.state()
    c = sim.contacts()
    sim.close()
    return st, cps, c


@pytest.mark.parametrize("steps", [1, 2, 40])
def test_trajectory_bit_exact(ctx, oracle, scene, steps):
    o_state, o_cps, o_c = _oracle(oracle, scene, steps)
    g_state, g_cps, g_c = _gpu(ctx, scene, steps)
    assert list(g_cps) == list(o_cps)
    assert len(g_c) == len(o_c)
    for f in FIELDS:
        assert np.array_equal(g_c[f], o_c[f]), f
    for k in STATE:
        assert np.array_equal(g_state[k], o_state[k]), k


@pytest.mark.parametrize("driver", [8, 9])
def test_culled_drivers_give_the_same_trajectory(ctx, scene, driver):
    """The certified driver (box culling + certified FP32/FP64 solver) and the culled FP64
    driver (box culling + FP64 bfSolver) give FP64 bf's trajectory and contacts bit for bit."""
    a_state, a_cps, a_c = _gpu(ctx, scene, 20, driver=0)
    b_state, b_cps, b_c = _gpu(ctx, scene, 20, driver=driver)
    assert list(a_cps) == list(b_cps)
    for k in STATE:
        assert np.array_equal(a_state[k], b_state[k]), k
    for f in FIELDS:
        assert np.array_equal(a_c[f], b_c[f]), f


def test_culled_fp64_driver_graph_equals_stepping(ctx, scene):
    from delta_b200.engine import Simulation, StepParams

    p = StepParams.make(**PARAMS)
    a_state, a_cps, _ = _gpu(ctx, scene, 25, driver=9)
    sim = Simulation(ctx, scene, 9)
    cps = sim.step(25, p, graph=True)
    st = sim.state()
    sim.close()
    assert list(cps) == list(a_cps)
    for k in STATE:
        assert np.array_equal(st[k], a_state[k]), k


@pytest.mark.parametrize("driver", [8, 9, 10])
def test_autotuned_time_step_keeps_the_trajectory(ctx, scene, driver, tmp_path):
    """delta_sim_autotune picks launch shapes of the culling and survivor kernels; the
    trajectory and contacts after tuning (stepped and replayed in a graph) equal those of an
    untuned simulation bit for bit, and a cache hit sets the same shape without timing."""
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.narrowphase import Context

    p = StepParams.make(**PARAMS)
    ref = Simulation(ctx, scene, driver)
    r_cps = list(ref.step(10, p)) + list(ref.step(10, p, graph=True))
    r_state, r_c = ref.state(), ref.contacts()
    ref.close()
    tctx = Context(0)
    try:
        sim = Simulation(tctx, scene, driver)
        cps = list(sim.step(10, p))
        cache = tmp_path / "tune.json"
        t = sim.autotune(reps=2, cache=cache)
        assert not t["cached"] and t["ms"] > 0
        assert t["cull_blocks_per_sm"] >= 1 and t["survivor_blocks_per_sm"] >= 1
        assert sim.counters()["steps"] == 10
        cps += list(sim.step(10, p, graph=True))
        st, c = sim.state(), sim.contacts()
        assert sim.autotune(cache=cache) == dict(t, cached=True)
        sim.close()
    finally:
        tctx.close()
    assert cps == r_cps
    for k in STATE:
        assert np.array_equal(st[k], r_state[k]), k
    for f in FIELDS:
        assert np.array_equal(c[f], r_c[f]), f


@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (0, 0)])
def test_every_cull_launch_shape_gives_the_same_contacts(ctx, scene, shape):
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.narrowphase import Context

    p = StepParams.make(**PARAMS)
    a_state, a_cps, a_c = _gpu(ctx, scene, 15, driver=8)
    tctx = Context(0)
    try:
        tctx.set_cull_launch(*shape)
        sim = Simulation(tctx, scene, 8)
        cps = sim.step(15, p, graph=True)
        st, c = sim.state(), sim.contacts()
        sim.close()
    finally:
        tctx.close()
    assert list(cps) == list(a_cps)
    for k in STATE:
        assert np.array_equal(st[k], a_state[k]), k
    for f in FIELDS:
        assert np.array_equal(c[f], a_c[f]), f


def test_friction_trajectory_bit_exact(ctx, oracle):
    from delta_b200.scenarios import lattice_scene

    sc = lattice_scene(seed=5, nx=4, ny=2, nz=4, friction=True)
    p = dict(PARAMS, friction=0.5)
    o_state, o_cps, _ = oracle.simulate(sc, p["dt"], p["gravity"], p["spring"], p["damper"], p["friction"], 30)
    from delta_b200.engine import Simulation, StepParams

    sim = Simulation(ctx, sc, 0)
    cps = sim.step(30, StepParams.make(**p))
    g_state = sim.state()
    assert list(cps) == list(o_cps)
    for k in STATE:
        assert np.array_equal(g_state[k], o_state[k]), k


def test_broadphase_covers_every_contact_pair(ctx, scene):
    from delta_b200.engine import DeviceScene, broadphase

    dev = DeviceScene(scene)
    pa, pb = broadphase(ctx, dev)
    keys = pa.astype(np.int64) * (1 << 32) + pb
    assert np.all(pa < pb) and np.all(np.diff(keys) > 0)
    # all pairs whose bounding spheres (grown by eps) overlap, by brute force on the host
    n = scene["n_bodies"]
    P = scene["pos"].reshape(n, 3)
    reach = scene["radius"] + scene["eps"]
    d = np.linalg.norm(P[:, None] - P[None], axis=2)
    want = set()
    for i in range(n):
        for j in range(i + 1, n):
            if scene["obstacle"][i] and scene["obstacle"][j]:
                continue
            if not scene["obstacle"][i] and not scene["obstacle"][j] and d[i, j] <= reach[i] + reach[j]:
                want.add((i, j))
    got = set(zip(pa.tolist(), pb.tolist()))
    assert want <= got


@pytest.mark.parametrize("caps", [None, (8, 8)])
def test_graph_replay_equals_stepping(ctx, oracle, scene, caps):
    """The graph-captured step gives the stepped trajectory bit for bit; with tiny
    capacities every replay overflows and the recovery path (repeat the detection with
    larger buffers, record again) must give the same result."""
    from delta_b200.engine import Simulation, StepParams

    p = StepParams.make(**PARAMS)
    o_state, o_cps, o_c = _oracle(oracle, scene, 30)
    sim = Simulation(ctx, scene, 8)
    if caps:
        sim.step(1, p)
        sim.set_graph_capacity(*caps)
        cps = np.concatenate([[-1], sim.step(29, p, graph=True)])
        cps[0] = o_cps[0]
    else:
        cps = sim.step(30, p, graph=True)
    st = sim.state()
    c = sim.contacts()
    sim.close()
    assert list(cps) == list(o_cps)
    for k in STATE:
        assert np.array_equal(st[k], o_state[k]), k
    assert len(c) == len(o_c)
    for f in FIELDS:
        assert np.array_equal(c[f], o_c[f]), f


def test_graph_counters_and_repeated_calls_match_stepping(ctx, scene):
    """Graph replays spread over several calls (1, 3, then 16 steps) give the stepped
    trajectory and the same step, body-pair and triangle-pair counters."""
    from delta_b200.engine import Simulation, StepParams

    p = StepParams.make(**PARAMS)
    ref = Simulation(ctx, scene, 8)
    ref.step(20, p)
    r_state, r_cnt = ref.state(), ref.counters()
    ref.close()
    sim = Simulation(ctx, scene, 8)
    sim.set_graph_capacity(1 << 14, 1 << 16)
    for n in (1, 3, 16):
        sim.step(n, p, graph=True)
    st, cnt = sim.state(), sim.counters()
    sim.close()
    for k in STATE:
        assert np.array_equal(st[k], r_state[k]), k
    for k in ("steps", "body_pairs", "triangle_pairs", "solved"):
        assert cnt[k] == r_cnt[k], (k, cnt[k], r_cnt[k])


def _obstacles_first(scene):
    """The same scene with the obstacles moved to the front of the body order."""
    n = scene["n_bodies"]
    obst = np.flatnonzero(scene["obstacle"])
    order = np.concatenate([obst, np.flatnonzero(scene["obstacle"] == 0)])
    off = scene["tri_offset"]
    tris = np.concatenate([np.arange(off[i], off[i + 1]) for i in order])
    verts = (3 * tris[:, None] + np.arange(3)[None]).reshape(-1)
    counts = np.diff(off)[order]
    out = dict(scene)
    out["tri_offset"] = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    out["tri_body"] = np.repeat(np.arange(n, dtype=np.int32), counts)
    for k in ("x", "y", "z", "rx", "ry", "rz"):
        out[k] = scene[k][verts].copy()
    for k, w in (("pos", 3), ("ref_pos", 3), ("vel", 3), ("ang", 3), ("ref_ang", 3), ("rot", 9), ("inertia", 9),
                 ("inverse", 9)):
        out[k] = scene[k].reshape(n, w)[order].reshape(-1).copy()
    for k in ("mass", "eps", "radius", "friction", "obstacle"):
        out[k] = scene[k][order].copy()
    return out


def test_obstacles_first_graph_equals_stepping_and_oracle(ctx, oracle, scene):
    """The floor as body 0 (partners above the obstacle in the pair order): the graph
    step's per-slave force lists and the hash grid give the stepped trajectory and the
    oracle's bit for bit."""
    from delta_b200.engine import Simulation, StepParams

    sc = _obstacles_first(scene)
    p = StepParams.make(**PARAMS)
    o_state, o_cps, _ = _oracle(oracle, sc, 20)
    ref = Simulation(ctx, sc, 8)
    ref.step(20, p)
    r_state = ref.state()
    ref.close()
    sim = Simulation(ctx, sc, 8)
    for n in (2, 18):
        sim.step(n, p, graph=True)
    g_state = sim.state()
    sim.close()
    for k in STATE:
        assert np.array_equal(r_state[k], o_state[k]), k
        assert np.array_equal(g_state[k], o_state[k]), k


def _grid(n, x0, x1, z0, z1, y, up):
    """n x n quads (2 n^2 triangles) over [x0, x1] x [z0, z1] at height y, normals +y
    (`up`) or -y."""
    xs, zs = np.linspace(x0, x1, n + 1), np.linspace(z0, z1, n + 1)
    V = np.array([(x, y, z) for x in xs for z in zs])
    F = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = i * (n + 1) + j, (i + 1) * (n + 1) + j, (i + 1) * (n + 1) + j + 1, i * (n + 1) + j + 1
            F += [[a, c, b], [a, d, c]] if up else [[a, b, c], [a, c, d]]
    return V, np.array(F)


def _tile(n, x0, z0, w, h, y0):
    """A closed w x h x w box whose bottom face (at y0) is an n x n grid of quads."""
    from delta_b200.scenarios import _outward

    Vb, Fb = _grid(n, x0, x0 + w, z0, z0 + w, y0, False)
    c = [(x0, y0, z0), (x0 + w, y0, z0), (x0 + w, y0, z0 + w), (x0, y0, z0 + w)]
    Vs = np.array(c + [(x, y0 + h, z) for x, _, z in c])
    Fs = [[4, 5, 6], [4, 6, 7]]
    for k in range(4):
        a, b = k, (k + 1) % 4
        Fs += [[a, b, b + 4], [a, b + 4, a + 4]]
    V = np.concatenate([Vb, Vs])
    return V, _outward(V, np.concatenate([Fb, np.array(Fs) + len(Vb)]))


def test_graph_many_contacts_per_pair_equals_stepping_and_oracle(ctx, oracle):
    """Two tiles resting face down on a finely meshed floor: 768 and 512 contacts per body
    pair, far more than a warp, so the graph step's per-pair ordering of the contacts ranks
    several chunks of keys.  Graph replays over several calls, stepping and the oracle give
    the same trajectory and contact list bit for bit."""
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.scenarios import build_scene

    eps = 1e-4
    sc = build_scene([_tile(8, -0.045, -0.02, 0.04, 0.01, 2 * eps - 6e-7),
                      _tile(8, 0.0051, -0.02, 0.04, 0.01, 2 * eps - 4e-7)],
                     obstacles=[_grid(12, -0.06, 0.06, -0.06, 0.06, 0.0, True)], eps=eps)
    prm = dict(PARAMS, spring=1e3)  # a softer spring: hundreds of contacts act on each tile
    o_state, o_cps, o_c = oracle.simulate(sc, prm["dt"], prm["gravity"], prm["spring"], prm["damper"],
                                          prm["friction"], 20)
    p = StepParams.make(**prm)
    ref = Simulation(ctx, sc, 8)
    r_cps = ref.step(20, p)
    r_state = ref.state()
    ref.close()
    sim = Simulation(ctx, sc, 8)
    g_cps = np.concatenate([sim.step(n, p, graph=True) for n in (1, 4, 15)])
    g_state, g_c = sim.state(), sim.contacts()
    sim.close()
    per_pair = np.unique(np.stack([g_c["master"], g_c["slave"]]), axis=1, return_counts=True)[1]
    assert per_pair.max() > 256, per_pair
    assert list(r_cps) == list(o_cps) and list(g_cps) == list(o_cps)
    for k in STATE:
        assert np.array_equal(r_state[k], o_state[k]), k
        assert np.array_equal(g_state[k], o_state[k]), k
    assert len(g_c) == len(o_c)
    for f in FIELDS:
        assert np.array_equal(g_c[f], o_c[f]), f


@pytest.fixture(scope="module")
def hopper():
    from delta_b200.scenarios import hopper_scene

    return hopper_scene(10000, seed=7)


@pytest.fixture(scope="module")
def hopper_oracle(oracle, hopper):
    p = PARAMS
    return oracle.simulate(hopper, 5e-6, p["gravity"], p["spring"], p["damper"], p["friction"], 4)


@pytest.mark.parametrize("driver,graph", [(0, False), (8, True), (9, True)])
def test_hopper_steps_bit_exact(ctx, hopper, hopper_oracle, driver, graph):
    """The uneven hopper (10,000 particles of 40-320 triangles over a 2,048-triangle cone,
    ~3,700 contacts per step): 4 steps of the plain FP64 driver (stepped) and of the culled
    drivers (graph-replayed) equal the oracle's bit for bit, trajectory and contacts."""
    from delta_b200.engine import Simulation, StepParams

    o_state, o_cps, o_c = hopper_oracle
    assert min(o_cps) > 1000
    prm = dict(PARAMS, dt=5e-6)
    sim = Simulation(ctx, hopper, driver)
    cps = sim.step(4, StepParams.make(**prm), graph=graph)
    st, c = sim.state(), sim.contacts()
    sim.close()
    assert list(cps) == list(o_cps)
    for k in STATE:
        assert np.array_equal(st[k], o_state[k]), k
    assert len(c) == len(o_c)
    for f in FIELDS:
        assert np.array_equal(c[f], o_c[f]), f


def _digests(state):
    import hashlib

    return {k: hashlib.sha256(np.ascontiguousarray(state[k], np.float64).tobytes()).hexdigest() for k in STATE}


def _fixture(name):
    import json
    from pathlib import Path

    return json.loads((Path(__file__).resolve().parent / "golden" / name).read_text())


@pytest.mark.parametrize("case,driver,graph", [("lattice", 0, False), ("lattice", 8, True), ("hopper", 0, False),
                                               ("hopper", 8, True), ("hopper", 9, True), ("hopper", 10, True)])
def test_full_length_runs_equal_the_reference(hopper, case, driver, graph):
    """Two configurations at their full length against the reference's own time step
    (tests/golden/make_timestep_golden.py: the reference's bf(), getContactsForces with
    forces.cpp's compiled constants, and dynamics.cpp's updates, run on the host): the
    256-icosphere lattice for 1000 steps and the 10,000-particle hopper for 2000.  The
    contacts of every step and every state array after the last step (SHA-256 of the
    bytes) equal the reference's, for the plain FP64 driver and for the culled drivers
    replayed as a CUDA graph.  The learned driver (FP32 hybrid) matches the contact
    counts but is not bit-exact: its trajectory stays within 1e-9 m of the reference's.
    Each run has a context of its own, as a user's first simulation does: its scratch
    buffers grow with the contact count during the run (a context whose buffers earlier
    tests had grown once hid a scratch layout larger than its allocation)."""
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.narrowphase import Context
    from delta_b200.scenarios import lattice_scene

    fx = _fixture("timestep_lattice_1000.json" if case == "lattice" else "timestep_hopper_2000.json")
    scene = lattice_scene(seed=2024) if case == "lattice" else hopper
    m = fx["material"]
    prm = StepParams.make(dt=fx["dt"], gravity=tuple(fx["gravity"]), spring=m["spring"], damper=m["damper"],
                          friction=m["friction"])
    own = Context(0)
    try:
        sim = Simulation(own, scene, driver)
        cps = sim.step(fx["steps"], prm, graph=graph)
        st = sim.state()
        sim.close()
    finally:
        own.close()
    if driver == 10:
        assert np.abs(np.asarray(st["pos"][:24]) - np.asarray(fx["pos_first_bodies"])).max() < 1e-9
        return
    assert [int(x) for x in cps] == fx["contacts_per_step"]
    assert _digests(st) == fx["sha256"]


@pytest.mark.parametrize("bodies", [40000, 70000])
def test_graph_sort_and_scan_paths_agree(ctx, bodies):
    """The graph step sorts a candidate list of at most 8,192 entries in one CTA (32-bit
    keys up to 2^16 bodies, 64-bit keys above; sized at run time to the step's pair
    count) and prefix-sums count arrays of at most 8,192 entries in one CTA; longer ones
    go to cub's device-wide sort and scan.  A box of 40,000 or 70,000 particles (its body
    and bucket arrays are longer than 8,192) replayed with the default pair capacity, with
    8,000 (the largest block sort, mostly padding) and with one above 8,192 gives the
    stepped trajectory and contacts bit for bit."""
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.scenarios import box_scene

    scene = box_scene(bodies, seed=11)
    prm = StepParams.make(dt=2e-6, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0)
    runs = []
    for graph, cap in ((False, None), (True, None), (True, 8000), (True, 9000)):
        sim = Simulation(ctx, scene, 8)
        if cap:
            sim.set_graph_capacity(cap, 1 << 16)
        cps = sim.step(6, prm, graph=graph)
        runs.append((list(cps), sim.state(), sim.contacts()))
        assert sim.counters()["body_pairs"] > 0  # candidate pairs to sort every step
        sim.close()
    (c0, s0, k0) = runs[0]
    for cps, st, c in runs[1:]:
        assert cps == c0
        for k in STATE:
            assert np.array_equal(st[k], s0[k]), k
        for f in FIELDS:
            assert np.array_equal(c[f], k0[f]), f


def _graph_and_stepped(ctx, scene, driver, steps, prm):
    """Runs `steps` with delta_sim_step and with the graph (one call); returns both
    (contacts per step, state, counters) and the graph run's skin list statistics."""
    from delta_b200.engine import Simulation

    out = []
    for graph in (False, True):
        sim = Simulation(ctx, scene, driver)
        cps = sim.step(steps, prm, graph=graph)
        out.append((list(cps), sim.state(), sim.counters()))
        skin = sim.skin_stats()
        sim.close()
    return out[0], out[1], skin


def _assert_same_run(a, b):
    (c0, s0, n0), (c1, s1, n1) = a, b
    assert c1 == c0
    for k in STATE:
        assert np.array_equal(s1[k], s0[k]), k
    for k in ("steps", "body_pairs", "triangle_pairs", "solved"):
        assert n1[k] == n0[k], (k, n1[k], n0[k])


@pytest.mark.parametrize("driver", [0, 8])
def test_graph_skin_list_rebuilds_inside_the_graph(ctx, driver):
    """The graph step takes its candidates from a skin list (pairs within reach + skin,
    filtered each step) that a conditional node rebuilds whenever a body has moved more
    than skin/2.  A lattice whose bodies move at up to 3 m/s crosses the skin many times in
    300 steps: the graph run, with its rebuilds inside the replays, equals delta_sim_step
    bit for bit, counters included."""
    from delta_b200.engine import StepParams
    from delta_b200.scenarios import lattice_scene

    scene = lattice_scene(seed=5)
    rng = np.random.default_rng(5)
    n = scene["n_bodies"]
    vel = rng.uniform(-3.0, 3.0, (n, 3))
    vel[scene["obstacle"] != 0] = 0.0
    scene["vel"] = vel.reshape(-1).copy()
    prm = StepParams.make(**PARAMS)
    stepped, graph, skin = _graph_and_stepped(ctx, scene, driver, 300, prm)
    assert skin["skin"] > 0 and skin["capacity"] > 0
    assert skin["rebuilds"] > 10, skin
    assert sum(stepped[0]) > 0  # the moving bodies touch
    _assert_same_run(stepped, graph)


def test_graph_skin_list_overflow_recovers(ctx):
    """An 8 x 8 x 8 lattice just wider than the skin list's reach, squeezed towards its
    centre: the pairs within reach + skin grow past the list's capacity (sized from the
    first, empty search), the replay freezes at the overflowing step and the host
    re-sizes the list and records the graph again; the run equals delta_sim_step's."""
    from delta_b200.engine import StepParams
    from delta_b200.scenarios import particle_cloud_scene

    sp, k = 0.027, 8
    g = (np.arange(k) - (k - 1) / 2) * sp
    cen = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    n = cen.shape[0]
    scene = particle_cloud_scene(cen, np.full(n, 0.0095), np.full(n, 80), [], seed=9)
    scene["vel"] = (-30.0 * cen).reshape(-1).copy()  # neighbours close at 0.81 m/s: spacing 0.022 m after 6 ms
    prm = StepParams.make(dt=1e-5, gravity=(0.0, 0.0, 0.0), spring=1e6, damper=0.1, friction=0.0)
    stepped, graph, skin = _graph_and_stepped(ctx, scene, 0, 600, prm)
    assert skin["capacity"] > 1024 + 1024 // 2, skin  # grown past the first list
    assert sum(stepped[0]) > 0
    _assert_same_run(stepped, graph)
