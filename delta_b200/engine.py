"""Time stepping on the GPU: forces, integration, broadphase and narrowphase in the
multiscale update order (Collision.cpp:1043-1127 forces from the previous detection,
MoveParticles.cpp:63-112 move, Collision.cpp:301-660 detection).

A scene is the dict built by delta_b200.scenarios.build_scene (per-body arrays in AoS,
3 or 9 entries per body); on the device the per-body vectors are SoA planes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib
from .detection import DRV_BF, Contacts
from .narrowphase import Context

VEC3 = ("pos", "ref_pos", "vel", "ang", "ref_ang")
MAT9 = ("rot", "inertia", "inverse")


class _Scene(C.Structure):
    _fields_ = [("n_bodies", C.c_int32), ("tri_offset", C.c_void_p), ("tri_body", C.c_void_p),
                ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p),
                ("pos", C.c_void_p), ("ref_pos", C.c_void_p), ("vel", C.c_void_p), ("ang", C.c_void_p),
                ("ref_ang", C.c_void_p), ("rot", C.c_void_p), ("inertia", C.c_void_p), ("inverse", C.c_void_p),
                ("mass", C.c_void_p), ("eps", C.c_void_p), ("radius", C.c_void_p), ("friction", C.c_void_p),
                ("obstacle", C.c_void_p)]


class StepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double * 3), ("spring", C.c_double), ("damper", C.c_double),
                ("friction", C.c_double)]

    @classmethod
    def make(cls, dt=1e-5, gravity=(0.0, -9.81, 0.0), spring=1e6, damper=0.1, friction=0.0):
        return cls(dt, (C.c_double * 3)(*gravity), spring, damper, friction)


class DeviceScene:
    """A scene dict uploaded to the device (SoA planes for per-body vectors)."""

    def __init__(self, scene: dict, device="cuda"):
        import torch

        n = scene["n_bodies"]
        self.n_bodies = n
        self.t = {}
        for k, v in scene.items():
            if k == "n_bodies":
                continue
            a = np.asarray(v)
            if k in VEC3:
                a = a.reshape(n, 3).T
            elif k in MAT9:
                a = a.reshape(n, 9).T
            self.t[k] = torch.as_tensor(np.ascontiguousarray(a)).to(device)

    def struct(self) -> _Scene:
        f = {k: v.data_ptr() for k, v in self.t.items()}
        return _Scene(self.n_bodies, f["tri_offset"], f["tri_body"], f["x"], f["y"], f["z"], f["rx"], f["ry"],
                      f["rz"], f["pos"], f["ref_pos"], f["vel"], f["ang"], f["ref_ang"], f["rot"], f["inertia"],
                      f["inverse"], f["mass"], f["eps"], f["radius"], f["friction"], f["obstacle"])

    def to_host(self) -> dict:
        out = {"n_bodies": self.n_bodies}
        for k, v in self.t.items():
            a = v.cpu().numpy()
            if k in VEC3 or k in MAT9:
                a = np.ascontiguousarray(a.T).reshape(-1)
            out[k] = a
        return out


class Simulation:
    """delta_sim: scene + contacts of the last detection, advanced by `step`."""

    def __init__(self, ctx: Context, scene: dict, driver: int = DRV_BF):
        self.ctx = ctx
        self.driver = int(driver)
        self.dev = DeviceScene(scene)
        self._s = self.dev.struct()
        self._h = C.c_void_p()
        check(lib().delta_sim_create(ctx.handle, C.byref(self._s), int(driver), C.byref(self._h)))

    def step(self, nsteps: int, params: StepParams | None = None, graph: bool = False) -> np.ndarray:
        """Advances nsteps; graph=True replays a captured CUDA graph of the step."""
        params = params or StepParams.make()
        cps = np.zeros(max(nsteps, 1), np.int64)
        fn = lib().delta_sim_step_graph if graph else lib().delta_sim_step
        check(fn(self._h, C.byref(params), int(nsteps), cps.ctypes.data))
        return cps[:nsteps]

    def set_graph_capacity(self, pairs: int, contacts: int):
        check(lib().delta_sim_set_graph_capacity(self._h, int(pairs), int(contacts)))

    def skin_stats(self) -> dict:
        """The graph step's skin list: skin distance, capacity, builds inside graph replays."""
        skin, cap, rb = C.c_double(0), C.c_int64(0), C.c_int64(0)
        check(lib().delta_sim_skin_stats(self._h, C.byref(skin), C.byref(cap), C.byref(rb)))
        return {"skin": skin.value, "capacity": cap.value, "rebuilds": rb.value}

    def autotune(self, reps: int = 5, cache=None) -> dict:
        """delta_sim_autotune: times the culled driver's detection of the current state under
        every launch shape of its culling and survivor kernels and keeps the fastest on the
        context.  Returns {"cull_blocks_per_sm", "survivor_blocks_per_sm", "ms", "cached"}.

        cache: a JSON file of earlier choices keyed by device, driver, bodies and triangles;
        a hit sets the stored shape (delta_set_cull_launch) without timing, a miss tunes and
        adds the result."""
        import json
        import os

        key = None
        if cache is not None:
            import torch

            dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
            ntri = int(self.dev.t["tri_offset"][-1].item())
            key = f"{dev}|driver={self.driver}|bodies={self.dev.n_bodies}|triangles={ntri}"
            table = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    table = json.load(f)
            if key in table:
                e = table[key]
                check(lib().delta_set_cull_launch(self.ctx.handle, int(e["cull_blocks_per_sm"]),
                                                  int(e["survivor_blocks_per_sm"])))
                return dict(e, cached=True)
        choice = np.zeros(2, np.int32)
        ms = C.c_float(0)
        check(lib().delta_sim_autotune(self._h, int(reps), choice.ctypes.data, C.byref(ms)))
        e = {"cull_blocks_per_sm": int(choice[0]), "survivor_blocks_per_sm": int(choice[1]), "ms": float(ms.value)}
        if key is not None:
            table[key] = e
            tmp = os.fspath(cache) + ".tmp"
            with open(tmp, "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        return dict(e, cached=False)

    def contacts(self) -> np.ndarray:
        n = C.c_int64(0)
        out = Contacts(1)
        st = lib().delta_sim_contacts(self._h, C.byref(out.struct()), C.byref(n))
        out = Contacts(max(int(n.value), 1))
        check(lib().delta_sim_contacts(self._h, C.byref(out.struct()), C.byref(n)))
        out.count = int(n.value)
        del st
        return out.to_numpy()

    def write_vtk(self, path, step: int) -> str:
        """Legacy VTK snapshot of the current vertices (writeGeometryToVTK's format)."""
        import os

        p = os.fspath(path)
        p = p if p.endswith(os.sep) else p + os.sep
        check(lib().delta_sim_write_vtk(self._h, p.encode(), int(step)))
        return os.path.join(p, f"geometry_{int(step)}.vtk")

    def counters(self) -> dict:
        """steps, candidate body pairs, triangle pairs tested (sum nA*nB), triangle pairs solved."""
        out = np.zeros(4, np.int64)
        check(lib().delta_sim_counters(self._h, out.ctypes.data))
        return dict(zip(("steps", "body_pairs", "triangle_pairs", "solved"), out.tolist()))

    def state(self) -> dict:
        self.ctx.synchronize()
        return self.dev.to_host()

    def close(self):
        if self._h:
            lib().delta_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def broadphase(ctx: Context, dev: DeviceScene, capacity: int = 1 << 16):
    """Candidate body pairs (a < b), sorted."""
    import torch

    while True:
        pa = torch.empty(capacity, dtype=torch.int32, device="cuda")
        pb = torch.empty_like(pa)
        n = C.c_int64(0)
        st = lib().delta_broadphase(ctx.handle, C.byref(dev.struct()), pa.data_ptr(), pb.data_ptr(), capacity,
                                    C.byref(n))
        if st == 3:
            capacity = int(n.value)
            continue
        check(st)
        return pa[: n.value].cpu().numpy(), pb[: n.value].cpu().numpy()
