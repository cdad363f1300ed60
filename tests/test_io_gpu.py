"""VTK snapshots from device meshes and from a running simulation, against the
writeGeometryToVTK restatement (oracle/io_oracle.py) and the oracle's trajectory."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_write_vtk_from_device_meshes(ctx, tmp_path):
    from delta_b200.detection import Meshes
    from delta_b200.io import write_vtk

    from oracle import io_oracle

    rng = np.random.default_rng(0)
    bodies = [rng.normal(size=(3, 3 * n)) for n in (10, 1, 33)]
    m = Meshes.from_bodies(bodies, np.full(3, 1e-3), np.zeros(3, np.uint8))
    fn = write_vtk(ctx, tmp_path, 3, m)
    with open(fn) as f:
        assert f.read() == io_oracle.vtk_text(bodies)


def test_simulation_snapshot(ctx, tmp_path):
    """After 5 steps the simulation's snapshot is its current vertices (obstacles included)
    printed in the reference's format."""
    from delta_b200.engine import Simulation, StepParams
    from delta_b200.scenarios import lattice_scene

    from oracle import io_oracle

    scene = lattice_scene(1, nx=2, ny=2, nz=2)
    params = StepParams.make(dt=1e-5, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0)
    sim = Simulation(ctx, scene, 0)
    sim.step(5, params)
    fn = sim.write_vtk(tmp_path, 5)
    st = sim.state()
    sim.close()
    xyz = np.stack([np.asarray(st[k]) for k in ("x", "y", "z")])
    assert not np.array_equal(xyz[0], np.asarray(scene["x"]))  # the bodies moved
    off = np.asarray(scene["tri_offset"])
    bodies = [xyz[:, 3 * off[i]:3 * off[i + 1]] for i in range(len(off) - 1)]
    with open(fn) as f:
        assert f.read() == io_oracle.vtk_text(bodies)
