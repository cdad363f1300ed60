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
