"""On-disk formats through the library (host code, no GPU): the legacy VTK snapshot byte for
byte against the restatement of writeGeometryToVTK, and the .mbfcp reader against the
restatement of readmbfcp (oracle/io_oracle.py)."""
import numpy as np
import pytest

from oracle import io_oracle


def _bodies(rng, counts):
    return [rng.normal(scale=0.05, size=(3, 3 * n)) + rng.normal(size=(3, 1)) for n in counts]


@pytest.mark.parametrize("counts", [(80, 20, 1), (5,), ()])
def test_write_vtk_matches_reference_format(tmp_path, counts):
    from delta_b200.io import write_vtk_host

    rng = np.random.default_rng(len(counts))
    bodies = _bodies(rng, counts)
    bodies.append(np.array([[-0.0, 1e-7, -1e-7], [2.5, -2.5, 0.0], [1e5, -1e-5, 0.123456789]]))
    fn = write_vtk_host(tmp_path, 7, bodies)
    assert fn.endswith("geometry_7.vtk")
    with open(fn) as f:
        assert f.read() == io_oracle.vtk_text(bodies)


def _mbfcp_text(spheres, with_materials=True, convex=True):
    lines = []
    if with_materials:
        lines += ["SURFACE_MATERIALS:\t1", "SURF1:\tANY", "SURF2:\tANY", "MODEL:\tSPRING_DASHPOT", "FRICTION:\t0.3",
                  "COHESION:\t0", "SPRING:\t1e+06", "DASHPOT:\t-1", "", "BULK_MATERIALS:\t1",
                  "LABEL:\tBULK_MATERIAL_0", "MODEL:\tKIRCHHOFF", "YOUNG:\t1e+09", "POISSON:\t0.25",
                  "DENSITY:\t2500.5", "", "GRAVITY:", "CONSTANT:\t0", "CONSTANT:\t-9.81", "CONSTANT:\t0", ""]
    lines.append(f"BODIES:\t{len(spheres) + (1 if convex else 0)}")
    lines.append("")
    if convex:
        lines += ["ID:\t126", "LABEL:\t(null)", "KINEMATICS:\tOBSTACLE", "BULK_MATERIAL:\tBULK_MATERIAL_0",
                  "SHAPES:\t1", "CONVEXES:\t1", "VERTEXES:\t3", "1  -0.1  0", "0  -0.1  1", "0  -0.1  0",
                  "FACES:\t1", "3  0  3  6  2", "VELOCITY:  0  0  0  0  0  0", "FORCES:\t0", ""]
    for ident, c, r in spheres:
        lines += [f"ID:\t{ident}", "LABEL:\t(null)", "KINEMATICS:\tRIGID", "BULK_MATERIAL:\tBULK_MATERIAL_0",
                  "SHAPES:\t1", "SPHERES:\t1",
                  "CENTRE: " + "  ".join(f"{v:4.2f}" for v in c), f"RADIUS: {r:4.2f}",
                  "VELOCITY:  0  0  0  0  0  0", "FORCES:\t0", ""]
    return "\n".join(lines) + "\n"


def test_read_mbfcp_matches_reference_parse(tmp_path):
    from delta_b200.io import read_mbfcp

    rng = np.random.default_rng(3)
    spheres = [(int(i), list(rng.uniform(0, 9, 3)), float(rng.uniform(0.1, 0.9))) for i in range(1, 40)]
    text = _mbfcp_text(spheres)
    p = tmp_path / "scene.mbfcp"
    p.write_text(text)
    got = read_mbfcp(p, capacity=4)  # grows past the capacity error
    ref = io_oracle.mbfcp_spheres(text)
    assert got["bodies"] == ref["bodies"] == 40
    assert got["materials"] == ref["materials"]
    assert got["materials"]["gravity"] == [0.0, np.float32(-9.81), 0.0]
    assert list(got["id"]) == [s[0] for s in ref["spheres"]]
    assert np.array_equal(got["centre"], np.array([s[1] for s in ref["spheres"]]))
    assert np.array_equal(got["radius"], np.array([s[2] for s in ref["spheres"]]))


def test_read_mbfcp_without_materials_and_errors(tmp_path):
    from delta_b200._lib import DeltaError
    from delta_b200.io import read_mbfcp

    p = tmp_path / "plain.mbfcp"
    p.write_text(_mbfcp_text([(5, [0.1, 0.2, 0.3], 0.05)], with_materials=False, convex=False))
    got = read_mbfcp(p)
    assert got["materials"] is None and list(got["id"]) == [5] and got["bodies"] == 1
    with pytest.raises(DeltaError):
        read_mbfcp(tmp_path / "missing.mbfcp")
    bad = tmp_path / "bad.mbfcp"
    bad.write_text("ID:\tx\n")
    with pytest.raises(DeltaError):
        read_mbfcp(bad)


@pytest.mark.parametrize("n", [0, 1, 257])
def test_write_vtu_holds_the_reference_arrays(tmp_path, n):
    """writeGeometryToVTKVTK's grid (write.cpp:10-70) written without VTK: Float32 centres,
    "direction" = linear velocity, "epsilon" (the active scalars; the reference's second
    SetScalars call replaces "radius"), no cells; values round-trip exactly."""
    from delta_b200.io import read_vtu, write_vtu_host

    rng = np.random.default_rng(n)
    centre = rng.normal(size=(3, n))
    vel = rng.normal(size=(3, n)) * 1e-3
    eps = rng.uniform(1e-5, 1e-3, n)
    fn = write_vtu_host(tmp_path, 12, centre, vel, eps)
    assert fn.endswith("geometry_12.vtu")
    v = read_vtu(fn)
    assert v["cells"] == 0 and v["active_scalars"] == "epsilon" and v["active_vectors"] == "direction"
    assert "radius" not in v
    assert np.array_equal(v["points"].reshape(n, 3), centre.T.astype(np.float32))
    assert np.array_equal(v["direction"].reshape(n, 3), vel.T)
    assert np.array_equal(v["epsilon"].reshape(n), eps)
