"""The C++ host layer (delta_b200/cpp/delta_b200.hpp): a C++ program built with g++
against it calls the drivers with the reference's signatures; its contacts must equal
the oracle's bit for bit."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def shim_exe(tmp_path_factory):
    lib = ROOT / "delta_b200"
    if not (lib / "libdelta_b200_cpp.so").exists():
        pytest.fail("libdelta_b200_cpp.so not built")
    exe = tmp_path_factory.mktemp("shim") / "shim_driver"
    subprocess.run(["g++", "-std=c++17", "-O1", str(ROOT / "tests/cpp/shim_driver.cpp"), f"-I{lib / 'cpp'}",
                    f"-L{lib}", "-ldelta_b200_cpp", "-ldelta_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)],
                   check=True)
    return exe


def test_cpp_drivers_match_oracle(shim_exe, oracle, tmp_path):
    from delta_b200.scenarios import sphere_mesh

    rng = np.random.default_rng(21)
    VA, FA = sphere_mesh(80, rng, 0.05, (0.9, 1.1))
    VB, FB = sphere_mesh(40, rng, 0.05, (0.9, 1.1))
    A = VA[FA].reshape(-1, 3).T.copy()
    B = (VB[FB].reshape(-1, 3) + [0.078, 0.005, 0.0]).T.copy()
    nA, nB, eps = 80, 40, 0.003
    f = tmp_path / "in.bin"
    with open(f, "wb") as fh:
        fh.write(np.array([nA, nB], np.int32).tobytes())
        fh.write(A.tobytes()); fh.write(B.tobytes())
        fh.write(np.array([eps, eps]).tobytes())
    out = subprocess.run([str(shim_exe), str(f)], check=True, capture_output=True, text=True).stdout.splitlines()
    rows = {}
    for line in out:
        name, *vals = line.split()
        rows.setdefault(name, []).append(vals)
    for name, drv in (("bf", 0), ("penalty", 1), ("hybrid_batch", 3), ("bf_cert", 0), ("penalty_stat", 2)):
        o, st = oracle.detect(drv, A, nA, eps, 1, 3, B, nB, eps, 1, 8, stats=True)
        got = rows.get(name, [])
        assert len(got) == len(o) and len(o) > 0, name
        for g, c in zip(got, o):
            vals = [float.fromhex(v) for v in g[:9]]
            want = [*c["x"], *c["normal"], c["depth"], c["P"][0], c["Q"][0]]
            assert vals == want, name
            assert [int(g[9]), int(g[10]), int(g[11])] == [c["master"], c["slave"], c["friction"]]
    hist = [int(v) for v in rows["hist"][0]]
    o, st = oracle.detect(2, A, nA, eps, 1, 3, B, nB, eps, 1, 8, stats=True)
    assert hist == list(st.newton_hist)


# ---- the per-call signatures: solvers, forces, dynamics, and the zoltan/ functions ----------
@pytest.fixture(scope="module")
def calls_exe(tmp_path_factory):
    lib = ROOT / "delta_b200"
    exe = tmp_path_factory.mktemp("calls") / "shim_calls"
    subprocess.run(["g++", "-std=c++17", "-O1", str(ROOT / "tests/cpp/shim_calls.cpp"), f"-I{lib / 'cpp'}",
                    f"-L{lib}", "-ldelta_b200_cpp", "-ldelta_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)],
                   check=True)
    return exe


def _call(exe, mode, values, tmp_path):
    f = tmp_path / f"{mode}.bin"
    np.asarray(np.concatenate([np.ravel(np.asarray(v, np.float64)) for v in values]), np.float64).tofile(f)
    out = subprocess.run([str(exe), mode, str(f)], check=True, capture_output=True, text=True).stdout.split()
    return np.array([float.fromhex(v) for v in out])


def test_cpp_pair_solvers_match_oracle(calls_exe, oracle, tmp_path):
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, _ = narrowphase_pairs(64, seed=23)
    n, me = a.shape[1], 1e-3
    vals = [[n, me]] + [np.concatenate([a[:, i], b[:, i]]) for i in range(n)]
    got = _call(calls_exe, "pairs", vals, tmp_path).reshape(n, 20)
    op, oq, _, _ = oracle.pairs(0, a, b)
    pp, pq, _, pf = oracle.pairs(1, a, b, max_error=me)
    ip, iq, _, itf = oracle.pairs(2, a, b, max_error=me)
    assert np.array_equal(got[:, 0:6], np.concatenate([op, oq]).T)
    assert np.array_equal(got[:, 6:12], np.concatenate([pp, pq]).T) and np.array_equal(got[:, 12], pf)
    assert np.array_equal(got[:, 13:19], np.concatenate([ip, iq]).T) and np.array_equal(got[:, 19], itf)


@pytest.mark.parametrize("sphere", [0, 1])
def test_cpp_get_contacts_forces_matches_oracle(calls_exe, oracle, tmp_path, sphere):
    import ctypes as C

    from oracle.oracle import CONTACT_DTYPE, Material

    rng = np.random.default_rng(24 + sphere)
    nc = 40
    c = np.zeros(nc, CONTACT_DTYPE)
    c["x"] = rng.normal(size=(nc, 3)); c["normal"] = rng.normal(size=(nc, 3))
    c["depth"] = rng.uniform(-1e-3, 1e-3, nc); c["friction"] = rng.integers(0, 2, nc)
    kin = [rng.normal(size=3) for _ in range(3)], [rng.normal(size=3) for _ in range(3)]
    mA, mB = 2.5, 0.7
    F0, T0 = rng.normal(size=3), rng.normal(size=3)
    vals = [[nc, sphere]] + [np.concatenate([c["x"][i], c["normal"][i], [c["depth"][i], c["friction"][i]]])
                             for i in range(nc)]
    vals += [*kin[0], [mA], *kin[1], [mB], F0, T0]
    got = _call(calls_exe, "forces", vals, tmp_path)
    F, T = F0.copy(), T0.copy()
    mat = Material(2e5, 0.5, 1.0) if sphere else Material(1e4, 0.5, 0.5)
    arr = [np.ascontiguousarray(x) for x in (*kin[0], *kin[1])]
    oracle.lib.dor_contacts_forces(c.ctypes.data, nc, 1.0, arr[0].ctypes.data, arr[1].ctypes.data,
                                   arr[2].ctypes.data, mA, arr[3].ctypes.data, arr[4].ctypes.data, arr[5].ctypes.data,
                                   mB, C.byref(mat), F.ctypes.data, T.ctypes.data)
    assert np.array_equal(got, np.concatenate([F, T]))


def test_cpp_dynamics_match_oracle(calls_exe, oracle, tmp_path):
    from tests import zoltan_cases

    s = zoltan_cases.system(nb=1, seed=25, omega=0.5)
    W, R = s["angular"][:3, 0].copy(), s["rotation"][:, 0].copy()
    J, Ji, tq = (np.ascontiguousarray(s[k][:, 0]) for k in ("inertia", "inverse", "torque"))
    step, r = 1e-3, np.array([0.1, -0.2, 0.3])
    pos, rpos = np.array([1.0, 2.0, 3.0]), np.array([0.05, 0.0, -0.02])
    got = _call(calls_exe, "dynamics", [W, R, J, Ji, tq, [step], r, pos, rpos], tmp_path)
    oracle.lib.dor_update_angular(W.ctypes.data, R.ctypes.data, J.ctypes.data, Ji.ctypes.data, tq.ctypes.data, step)
    ang = np.zeros(3)
    oracle.lib.dor_update_rotation(ang.ctypes.data, W.ctypes.data, R.ctypes.data, step)
    C = r - rpos
    x = pos + np.array([R[0] * C[0] + R[3] * C[1] + R[6] * C[2], R[1] * C[0] + R[4] * C[1] + R[7] * C[2],
                        R[2] * C[0] + R[5] * C[1] + R[8] * C[2]])
    assert np.array_equal(got, np.concatenate([W, ang, R, x]))


def test_cpp_zoltan_narrowphase_matches_oracle(calls_exe, oracle, tmp_path):
    from delta_b200.scenarios import narrowphase_pairs

    a, b, _, _ = narrowphase_pairs(256, seed=26)
    b[3:6, :3] = b[0:3, :3]
    n, it, nt = b.shape[1], 2, 253
    abc = a[:, 0].reshape(3, 3)
    got = _call(calls_exe, "znarrow", [[n], abc, b[0:3], b[3:6], b[6:9], [it, nt]], tmp_path).reshape(3, 6, n)
    fill = np.full((3, n), 7.0)
    for m, method in enumerate(("bf_soa", "penalty", "hybrid")):
        p, q = oracle.zoltan_soa(method, it, nt, abc, b[0:3], b[3:6], b[6:9], fill, fill)
        want = np.concatenate([p, q])
        exact = ((got[m] == want) | (np.isnan(got[m]) & np.isnan(want))).all(0)
        if method == "bf_soa":
            assert exact.all()
        else:  # the oracle for a penalty weight within 40 ulps: see tests/test_zoltan_gpu.py
            shifted = oracle.zoltan_r_shifted(method, it, nt, abc, b[0:3], b[3:6], b[6:9], fill, fill,
                                              shifts=range(-40, 41))
            match = np.zeros(n, bool)
            for x in shifted:
                match |= ((got[m] == x) | (np.isnan(got[m]) & np.isnan(x))).all(0)
            assert match.all()


def test_cpp_zoltan_system_matches_oracle(calls_exe, oracle, tmp_path):
    from tests import zoltan_cases

    nb, step, g = 20, 1e-3, np.array([0.0, 0.0, -9.81])
    s = zoltan_cases.system(nb=nb, tris_per_body=5, seed=27, omega=0.5)
    c = zoltan_cases.contacts(nb=nb, seed=27)
    nt, nc = s["t"].shape[2], len(c["slave"])
    master = np.repeat(np.arange(nb), np.diff(c["offset"]))
    con = [np.concatenate([[master[k], c["slave"][k]], c["point"][:, k], c["normal"][:, k], [c["depth"][k]]])
           for k in range(nc)]
    vals = [[nb, nt, nc, step], g, s["t"].reshape(18, nt), s["angular"], s["linear"], s["rotation"], s["position"],
            s["inertia"], s["inverse"], s["mass"], s["force"], s["torque"], s["pid"], *con]
    got = _call(calls_exe, "zsystem", vals, tmp_path)
    F, T = oracle.zoltan_force(c["offset"], c["slave"], c["point"], c["normal"], c["depth"], s["position"],
                               s["angular"], s["linear"], s["mass"], s["force"], s["torque"], g, 1e2, 1.0)
    t, ang, lin, rot, pos, F2, T2 = oracle.zoltan_update(s["t"], s["pid"], s["angular"], s["linear"], s["rotation"],
                                                         s["position"], s["inertia"], s["inverse"], s["mass"], F, T,
                                                         step)
    ang3, rot3, pos3 = oracle.zoltan_euler(ang, lin, rot, pos, step)
    vel = t[0] - t[3]
    t4, vel4 = oracle.zoltan_integrate(step, [-1, -1, -1], [1, 1, 1], t[:3], vel)
    want = np.concatenate([np.ravel(x) for x in (F, T, t, ang, lin, rot, pos, F2, T2, ang3, rot3, pos3, t4, vel4)])
    assert got.shape == want.shape and np.array_equal(got, want)
