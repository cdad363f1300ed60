"""Particle-pair contact detection: the drivers delta::contact::detection::{bf, penalty,
penaltyStat, hybridWithPerBatchFallBack, hybridWithPerTriangleFallBack, hybridBatchStat,
hybridTriangleStat, gjk} (delta/contact/detection/*.h) on the GPU.

``detect`` runs one driver over many candidate body pairs at once (the batched form the
time step uses).  The functions named after the reference drivers take the reference's
arguments (SoA-tri coordinates of two bodies, triangle counts, epsilon, friction flag,
particle id) and return the contact list as a numpy structured array with the fields
of struct contactpoint (contactpoint.h:42-103) plus the two triangle indices.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import DeltaError, ERR_CAPACITY, check, lib
from .narrowphase import F64, Context

(DRV_BF, DRV_PENALTY, DRV_PENALTY_STAT, DRV_HYBRID_BATCH, DRV_HYBRID_TRIANGLE, DRV_HYBRID_BATCH_STAT,
 DRV_HYBRID_TRI_STAT, DRV_GJK, DRV_BF_CERT, DRV_BF_CULLED, DRV_LEARNED) = range(11)

CONTACT_DTYPE = np.dtype(
    [("x", "<f8", 3), ("normal", "<f8", 3), ("depth", "<f8"), ("P", "<f8", 3), ("Q", "<f8", 3),
     ("friction", "<i4"), ("eps_total", "<f8"), ("master", "<i4"), ("slave", "<i4"), ("penetration", "<i4"),
     ("tri_a", "<i4"), ("tri_b", "<i4")], align=True)


class _Meshes(C.Structure):
    _fields_ = [("n_bodies", C.c_int32), ("tri_offset", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p),
                ("z", C.c_void_p), ("eps", C.c_void_p), ("friction", C.c_void_p), ("id", C.c_void_p)]


class _Contacts(C.Structure):
    _fields_ = [("capacity", C.c_int64), ("x", C.c_void_p), ("normal", C.c_void_p), ("P", C.c_void_p),
                ("Q", C.c_void_p), ("depth", C.c_void_p), ("eps_total", C.c_void_p), ("master", C.c_void_p),
                ("slave", C.c_void_p), ("tri_a", C.c_void_p), ("tri_b", C.c_void_p), ("penetration", C.c_void_p),
                ("friction", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("newton_hist", C.c_int64 * 17), ("penalty_fails", C.c_int64), ("batch_fails", C.c_int64),
                ("batch_size", C.c_int64), ("batch_error", C.c_double)]


class Meshes:
    """Triangulated bodies on the device in SoA-tri layout."""

    def __init__(self, tri_offset, x, y, z, eps, friction, ids=None, device="cuda"):
        import torch

        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(device)  # noqa: E731
        self.tri_offset = t(tri_offset, torch.int64)
        self.x, self.y, self.z = t(x, torch.float64), t(y, torch.float64), t(z, torch.float64)
        self.n_bodies = self.tri_offset.numel() - 1
        self.eps = t(eps, torch.float64)
        self.friction = t(friction, torch.uint8)
        self.id = t(ids if ids is not None else np.arange(self.n_bodies), torch.int32)

    @classmethod
    def from_bodies(cls, bodies, eps, friction, ids=None):
        """bodies: list of (3, 3*nT) host arrays."""
        counts = [b.shape[1] // 3 for b in bodies]
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        xyz = np.concatenate(bodies, 1) if bodies else np.zeros((3, 0))
        return cls(off, xyz[0], xyz[1], xyz[2], eps, friction, ids)

    def struct(self) -> _Meshes:
        return _Meshes(self.n_bodies, self.tri_offset.data_ptr(), self.x.data_ptr(), self.y.data_ptr(),
                       self.z.data_ptr(), self.eps.data_ptr(), self.friction.data_ptr(), self.id.data_ptr())


class Contacts:
    """Device contact buffer (SoA) of a given capacity."""

    def __init__(self, capacity: int, device="cuda"):
        import torch

        cap = max(int(capacity), 1)
        f8 = dict(dtype=torch.float64, device=device)
        i4 = dict(dtype=torch.int32, device=device)
        self.capacity = cap
        self.x, self.normal = torch.empty((3, cap), **f8), torch.empty((3, cap), **f8)
        self.P, self.Q = torch.empty((3, cap), **f8), torch.empty((3, cap), **f8)
        self.depth, self.eps_total = torch.empty(cap, **f8), torch.empty(cap, **f8)
        self.master, self.slave = torch.empty(cap, **i4), torch.empty(cap, **i4)
        self.tri_a, self.tri_b = torch.empty(cap, **i4), torch.empty(cap, **i4)
        self.penetration = torch.empty(cap, **i4)
        self.friction = torch.empty(cap, dtype=torch.uint8, device=device)
        self.count = 0

    def struct(self) -> _Contacts:
        p = lambda t: t.data_ptr()  # noqa: E731
        return _Contacts(self.capacity, p(self.x), p(self.normal), p(self.P), p(self.Q), p(self.depth),
                         p(self.eps_total), p(self.master), p(self.slave), p(self.tri_a), p(self.tri_b),
                         p(self.penetration), p(self.friction))

    def select(self, mask, n: int | None = None) -> "Contacts":
        """A new buffer with the first n contacts where mask (device, bool/uint8) is set."""
        n = self.count if n is None else n
        m = mask[:n].bool()
        k = int(m.sum().item())
        out = Contacts(k, device=self.x.device)
        for name in ("x", "normal", "P", "Q"):
            getattr(out, name)[:, :k] = getattr(self, name)[:, :n][:, m]
        for name in ("depth", "eps_total", "master", "slave", "tri_a", "tri_b", "penetration", "friction"):
            getattr(out, name)[:k] = getattr(self, name)[:n][m]
        out.count = k
        return out

    def to_numpy(self, n: int | None = None) -> np.ndarray:
        n = self.count if n is None else n
        out = np.zeros(n, CONTACT_DTYPE)
        for name in ("x", "normal", "P", "Q"):
            out[name] = getattr(self, name)[:, :n].cpu().numpy().T
        for name in ("depth", "eps_total", "master", "slave", "tri_a", "tri_b", "penetration", "friction"):
            out[name] = getattr(self, name)[:n].cpu().numpy()
        return out


def detect(ctx: Context, driver: int, meshes: Meshes, pair_a, pair_b, precision=F64, capacity=None,
           grow=True, stats=False):
    """Contacts of `driver` over the body pairs (pair_a[k], pair_b[k]), in (pair, A triangle,
    B triangle) order.  Returns (Contacts, Stats|None).  With grow=True a full buffer is
    reallocated and the call repeated."""
    import torch

    pa = torch.as_tensor(np.asarray(pair_a, np.int32) if not torch.is_tensor(pair_a) else pair_a,
                         dtype=torch.int32).cuda()
    pb = torch.as_tensor(np.asarray(pair_b, np.int32) if not torch.is_tensor(pair_b) else pair_b,
                         dtype=torch.int32).cuda()
    cap = capacity if capacity is not None else 4096
    while True:
        out = Contacts(cap)
        n = C.c_int64(0)
        st = Stats()
        status = lib().delta_detect(ctx.handle, int(driver), int(precision), C.byref(meshes.struct()),
                                    pa.data_ptr(), pb.data_ptr(), pa.numel(), C.byref(out.struct()), C.byref(n),
                                    C.byref(st))
        if status == ERR_CAPACITY and grow:
            cap = int(n.value)
            continue
        if status == ERR_CAPACITY:
            out.count = min(int(n.value), out.capacity)
            raise DeltaError(status, f"capacity {out.capacity} < {n.value} contacts")
        check(status)
        out.count = int(n.value)
        return out, (st if stats else None)


# ---- the reference drivers, one body pair per call ---------------------------------------
_ctx = None


def _default_ctx():
    global _ctx
    if _ctx is None:
        _ctx = Context(0)
    return _ctx


def _one_pair(driver, xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB, precision=F64,
              ctx=None, stats=False):
    A = np.stack([np.asarray(xA, float)[:3 * nA], np.asarray(yA, float)[:3 * nA], np.asarray(zA, float)[:3 * nA]])
    B = np.stack([np.asarray(xB, float)[:3 * nB], np.asarray(yB, float)[:3 * nB], np.asarray(zB, float)[:3 * nB]])
    m = Meshes.from_bodies([A, B], [epsA, epsB], [int(bool(fricA)), int(bool(fricB))], [idA, idB])
    out, st = detect(ctx or _default_ctx(), driver, m, [0], [1], precision=precision, stats=True)
    c = out.to_numpy()
    return (c, st) if stats else c


def bf(*args, **kw):
    """bf(xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB), bf.h:65-81."""
    return _one_pair(DRV_BF, *args, **kw)


def penalty(*args, **kw):
    """penalty(...), penalty.h:99-115."""
    return _one_pair(DRV_PENALTY, *args, **kw)


def penaltyStat(*args, **kw):  # noqa: N802 (reference name)
    """penaltyStat(...), penalty.h:59-74; stats=True also returns the iteration histogram."""
    return _one_pair(DRV_PENALTY_STAT, *args, **kw)


def hybridWithPerBatchFallBack(*args, **kw):  # noqa: N802
    """hybrid.h:113-128."""
    return _one_pair(DRV_HYBRID_BATCH, *args, **kw)


def hybridWithPerTriangleFallBack(*args, **kw):  # noqa: N802
    """hybrid.h:76-91 (the A-triangle loop runs over A's triangles)."""
    return _one_pair(DRV_HYBRID_TRIANGLE, *args, **kw)


def hybridBatchStat(*args, **kw):  # noqa: N802
    """hybrid.h:130-144."""
    return _one_pair(DRV_HYBRID_BATCH_STAT, *args, **kw)


def hybridTriangleStat(*args, **kw):  # noqa: N802
    """hybrid.h:146-160."""
    return _one_pair(DRV_HYBRID_TRI_STAT, *args, **kw)


def gjk(nA, xA, yA, zA, epsA, fricA, idA, nB, xB, yB, zB, epsB, fricB, idB, **kw):
    """gjk argument order (gjk.h:32-47); per triangle pair with bf()'s contact rule."""
    return _one_pair(DRV_GJK, xA, yA, zA, nA, epsA, fricA, idA, xB, yB, zB, nB, epsB, fricB, idB, **kw)


def filter_new_mask(ctx: Context, contacts: Contacts, n: int | None = None, eps: float = 1e-4):
    """keep flags (device uint8) of filterNewContacts (filter.cpp:80-101) per particle pair."""
    import torch

    n = contacts.count if n is None else n
    keep = torch.empty(max(n, 1), dtype=torch.uint8, device=contacts.x.device)
    check(lib().delta_filter_new_contacts(ctx.handle, C.byref(contacts.struct()), n, float(eps), keep.data_ptr()))
    return keep[:n]


def filter_old_mask(ctx: Context, stored: Contacts, fresh: Contacts, eps: float = 1e-4):
    """keep flags (device uint8) of filterOldContacts (filter.cpp:3-78) for fresh vs stored."""
    import torch

    keep = torch.empty(max(fresh.count, 1), dtype=torch.uint8, device=fresh.x.device)
    check(lib().delta_filter_old_contacts(ctx.handle, C.byref(stored.struct()), stored.count,
                                          C.byref(fresh.struct()), fresh.count, float(eps), keep.data_ptr()))
    return keep[:fresh.count]


def filterNewContacts(ctx: Context, contacts: Contacts, eps: float = 1e-4) -> Contacts:  # noqa: N802
    """delta::contact::filterNewContacts over every particle pair's contacts."""
    return contacts.select(filter_new_mask(ctx, contacts, eps=eps))


def filterOldContacts(ctx: Context, stored: Contacts, fresh: Contacts, eps: float = 1e-4) -> Contacts:  # noqa: N802
    """delta::contact::filterOldContacts: the fresh contacts not near a stored one of their pair."""
    return fresh.select(filter_old_mask(ctx, stored, fresh, eps=eps))


# ---- sphere model (sphere.cpp) ----------------------------------------------------------
class _Spheres(C.Structure):
    _fields_ = [("n", C.c_int64), ("centre", C.c_void_p), ("diameter", C.c_void_p), ("eps", C.c_void_p),
                ("friction", C.c_void_p), ("id", C.c_void_p)]


class Spheres:
    """Spherical particles on the device: centres (3, n), diameters, halo eps, friction, ids."""

    def __init__(self, centre, diameter, eps, friction, ids=None, device="cuda"):
        import torch

        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt).to(device)  # noqa: E731
        self.centre = t(centre, torch.float64)
        self.n = self.centre.shape[1]
        self.diameter = t(diameter, torch.float64)
        self.eps = t(eps, torch.float64)
        self.friction = t(friction, torch.uint8)
        self.id = t(ids if ids is not None else np.arange(self.n), torch.int32)

    def struct(self) -> _Spheres:
        return _Spheres(self.n, self.centre.data_ptr(), self.diameter.data_ptr(), self.eps.data_ptr(),
                        self.friction.data_ptr(), self.id.data_ptr())


def _pairs_dev(a):
    import torch

    return torch.as_tensor(np.asarray(a, np.int32) if not torch.is_tensor(a) else a, dtype=torch.int32).cuda()


def _grow(call, capacity):
    cap = capacity
    while True:
        out = Contacts(cap)
        n = C.c_int64(0)
        status = call(out, n)
        if status == ERR_CAPACITY:
            cap = int(n.value)
            continue
        check(status)
        out.count = int(n.value)
        return out


def sphere(ctx: Context, spheres: Spheres, pair_a, pair_b, capacity: int = 1024) -> Contacts:
    """delta::contact::detection::sphere (sphere.cpp:29-77) over sphere pairs, in pair order."""
    pa, pb = _pairs_dev(pair_a), _pairs_dev(pair_b)
    return _grow(lambda out, n: lib().delta_sphere_contacts(ctx.handle, C.byref(spheres.struct()), pa.data_ptr(),
                                                            pb.data_ptr(), pa.numel(), C.byref(out.struct()),
                                                            C.byref(n)), capacity)


def _sphere_mesh(ctx, spheres, meshes, sphere_idx, body_idx, sphere_is_b, capacity):
    ps, pm = _pairs_dev(sphere_idx), _pairs_dev(body_idx)
    return _grow(lambda out, n: lib().delta_sphere_mesh_contacts(
        ctx.handle, C.byref(spheres.struct()), C.byref(meshes.struct()), ps.data_ptr(), pm.data_ptr(), ps.numel(),
        int(sphere_is_b), C.byref(out.struct()), C.byref(n)), capacity)


def sphereWithBarrierAB(ctx: Context, spheres: Spheres, meshes: Meshes, sphere_idx, body_idx,  # noqa: N802
                        capacity: int = 4096) -> Contacts:
    """sphere.cpp:79-140: sphere A against the triangles of mesh B, in (pair, triangle) order."""
    return _sphere_mesh(ctx, spheres, meshes, sphere_idx, body_idx, 0, capacity)


def sphereWithBarrierBA(ctx: Context, spheres: Spheres, meshes: Meshes, sphere_idx, body_idx,  # noqa: N802
                        capacity: int = 4096) -> Contacts:
    """sphere.cpp:142-201: sphere B against the triangles of mesh A (mesh point first)."""
    return _sphere_mesh(ctx, spheres, meshes, sphere_idx, body_idx, 1, capacity)


def isSphereOverlayInContact(ctx: Context, centre, radius, pair_a, pair_b):  # noqa: N802
    """sphere.cpp:203-218 for each pair: |cA - cB| <= rA + rB (device uint8 flags)."""
    import torch

    c = torch.as_tensor(np.ascontiguousarray(centre) if not torch.is_tensor(centre) else centre,
                        dtype=torch.float64).cuda().contiguous()
    r = torch.as_tensor(np.ascontiguousarray(radius) if not torch.is_tensor(radius) else radius,
                        dtype=torch.float64).cuda().contiguous()
    pa, pb = _pairs_dev(pair_a), _pairs_dev(pair_b)
    out = torch.empty(max(pa.numel(), 1), dtype=torch.uint8, device="cuda")
    check(lib().delta_sphere_overlap(ctx.handle, c.data_ptr(), c.shape[1], r.data_ptr(), pa.data_ptr(),
                                     pb.data_ptr(), pa.numel(), out.data_ptr()))
    return out[:pa.numel()]
