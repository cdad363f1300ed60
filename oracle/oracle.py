"""ctypes bindings for the checker libraries (test infrastructure, not the product).

``Oracle`` wraps ``liboracle.so`` (the C restatement in ``delta_oracle.c``) and
``Reference`` wraps ``_ref/libdelta_ref*.so`` (the reference's own sources compiled by
``oracle/Makefile``).  Only tests/, the smoke check and the CPU-baseline leg of bench.py
import this module.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

BF, PENALTY, PENALTY_ITER, GJK, HYBRID_PAIR = 0, 1, 2, 3, 4
DRV_BF, DRV_PENALTY, DRV_PENALTY_STAT, DRV_HYBRID_BATCH, DRV_HYBRID_TRIANGLE = 0, 1, 2, 3, 4
DRV_HYBRID_BATCH_STAT, DRV_HYBRID_TRI_STAT, DRV_GJK = 5, 6, 7

CONTACT_DTYPE = np.dtype(
    [
        ("x", "<f8", 3),
        ("normal", "<f8", 3),
        ("depth", "<f8"),
        ("P", "<f8", 3),
        ("Q", "<f8", 3),
        ("friction", "<i4"),
        ("eps_total", "<f8"),
        ("master", "<i4"),
        ("slave", "<i4"),
        ("penetration", "<i4"),
        ("tri_a", "<i4"),
        ("tri_b", "<i4"),
    ],
    align=True,
)


class Stats(C.Structure):
    _fields_ = [
        ("newton_hist", C.c_int64 * 17),
        ("penalty_fails", C.c_int64),
        ("batch_fails", C.c_int64),
        ("batch_size", C.c_int64),
        ("batch_error", C.c_double),
    ]


class Material(C.Structure):
    _fields_ = [("spring", C.c_double), ("damper", C.c_double), ("friction", C.c_double)]


class Scene(C.Structure):
    _fields_ = [
        ("n_bodies", C.c_int32),
        ("tri_offset", C.c_void_p),
        ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
        ("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p),
        ("pos", C.c_void_p), ("ref_pos", C.c_void_p),
        ("vel", C.c_void_p), ("ang", C.c_void_p), ("ref_ang", C.c_void_p),
        ("rot", C.c_void_p), ("inertia", C.c_void_p), ("inverse", C.c_void_p),
        ("mass", C.c_void_p), ("eps", C.c_void_p), ("radius", C.c_void_p),
        ("friction", C.c_void_p), ("obstacle", C.c_void_p),
    ]


class StepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double * 3), ("mat", Material)]


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def _build_if_missing(path: Path):
    if not path.exists():
        os.system(f"make -s -C {HERE} >/dev/null 2>&1")
    return path.exists()


class _Lib:
    prefix = ""

    def _sig(self):
        L, pre = self.lib, self.prefix
        vp, i32, i64, f8 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        getattr(L, pre + "pairs").argtypes = [i32, i64, vp, vp, i64, f8, vp, vp, vp, vp, i32]
        getattr(L, pre + "pairs").restype = None
        getattr(L, pre + "detect").argtypes = [i32, vp, vp, vp, i32, f8, i32, i32, vp, vp, vp, i32, f8, i32, i32,
                                               vp, i64, vp]
        getattr(L, pre + "detect").restype = i64
        for name in ("bf_solver",):
            getattr(L, pre + name).argtypes = [vp] * 7
        getattr(L, pre + "penalty_solver").argtypes = [vp] * 6 + [f8, vp, vp]
        getattr(L, pre + "penalty_solver_iter").argtypes = [vp] * 6 + [f8, vp, vp]
        getattr(L, pre + "gjk").argtypes = [vp, i32, vp, i32, vp, vp]
        getattr(L, pre + "gjk").restype = f8
        getattr(L, pre + "expmap").argtypes = [f8, f8, f8, vp]
        getattr(L, pre + "pt").argtypes = [vp] * 5
        getattr(L, pre + "pt").restype = f8
        getattr(L, pre + "sphere").argtypes = [vp, f8, f8, i32, i32, vp, f8, f8, i32, i32, vp]
        getattr(L, pre + "sphere").restype = i64
        getattr(L, pre + "sphere_mesh").argtypes = [i32, vp, f8, f8, i32, i32, vp, vp, vp, i32, f8, i32, i32, vp, i64]
        getattr(L, pre + "sphere_mesh").restype = i64
        getattr(L, pre + "sphere_overlay").argtypes = [vp, f8, vp, f8]
        getattr(L, pre + "sphere_overlay").restype = i32

    # ---- pair list -------------------------------------------------------------
    def pairs(self, method, a, b, max_error=0.0, nthreads=0, with_flags=True):
        """a, b: float64 arrays of shape (9, n) (plane 3*vertex+coord).  Returns p, q, dist, flags."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        n = a.shape[1]
        p = np.empty((3, n)); q = np.empty((3, n)); d = np.empty(n)
        fl = np.zeros(n, np.uint8) if with_flags else None
        getattr(self.lib, self.prefix + "pairs")(method, n, _p(a), _p(b), n, max_error, _p(p), _p(q), _p(d),
                                                 _p(fl), nthreads)
        return p, q, d, fl

    # ---- particle pair -----------------------------------------------------------
    def detect(self, driver, A, nA, epsA, fricA, idA, B, nB, epsB, fricB, idB, cap=None, stats=False):
        """A, B: (3, 3*nT) float64 SoA-tri coordinates.  Returns (contacts, Stats|None)."""
        A = np.ascontiguousarray(A, dtype=np.float64)
        B = np.ascontiguousarray(B, dtype=np.float64)
        cap = cap if cap is not None else max(1, nA * nB)
        out = np.zeros(cap, CONTACT_DTYPE)
        st = Stats() if stats else None
        n = getattr(self.lib, self.prefix + "detect")(
            driver, _p(A[0]), _p(A[1]), _p(A[2]), nA, epsA, int(fricA), idA,
            _p(B[0]), _p(B[1]), _p(B[2]), nB, epsB, int(fricB), idB,
            _p(out), cap, C.byref(st) if st is not None else None)
        return out[: min(n, cap)], st

    # ---- sphere model ----------------------------------------------------------------
    def pt(self, T1, T2, T3, c):
        """point.cpp pt(): (distance, closest point)."""
        a = [np.ascontiguousarray(v, np.float64) for v in (T1, T2, T3, c)]
        tq = np.empty(3)
        d = getattr(self.lib, self.prefix + "pt")(_p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(tq))
        return d, tq

    def sphere(self, cA, dA, epsA, fA, idA, cB, dB, epsB, fB, idB):
        """sphere(): the contact (array of 0 or 1 records)."""
        out = np.zeros(1, CONTACT_DTYPE)
        cA = np.ascontiguousarray(cA, np.float64); cB = np.ascontiguousarray(cB, np.float64)
        n = getattr(self.lib, self.prefix + "sphere")(_p(cA), dA, epsA, int(fA), int(idA), _p(cB), dB, epsB,
                                                      int(fB), int(idB), _p(out))
        return out[:n]

    def sphere_mesh(self, ba, c, d, epsS, fS, idS, M, nT, epsM, fM, idM):
        """sphereWithBarrierAB (ba=0) / BA (ba=1) against the SoA-tri mesh M (3, 3*nT)."""
        M = np.ascontiguousarray(M, np.float64)
        c = np.ascontiguousarray(c, np.float64)
        out = np.zeros(max(nT, 1), CONTACT_DTYPE)
        n = getattr(self.lib, self.prefix + "sphere_mesh")(int(ba), _p(c), d, epsS, int(fS), int(idS), _p(M[0]),
                                                           _p(M[1]), _p(M[2]), nT, epsM, int(fM), int(idM), _p(out),
                                                           len(out))
        return out[:n]

    def sphere_overlay(self, cA, rA, cB, rB):
        cA = np.ascontiguousarray(cA, np.float64); cB = np.ascontiguousarray(cB, np.float64)
        return int(getattr(self.lib, self.prefix + "sphere_overlay")(_p(cA), rA, _p(cB), rB))

    def expmap(self, o):
        L = np.empty(9)
        getattr(self.lib, self.prefix + "expmap")(float(o[0]), float(o[1]), float(o[2]), _p(L))
        return L


class _Zoltan:
    """The zoltan/ narrowphase functions (SoA "one triangle against a list" shape)."""

    zprefix = ""

    def _zsig(self):
        L, pre = self.zlib, self.zprefix
        vp, i32, i64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
        getattr(L, pre + "bf").argtypes = [vp] * 7
        getattr(L, pre + "penalty").argtypes = [u32, u32, vp, vp, vp, vp, vp, vp, i64, vp, vp]
        getattr(L, pre + "hybrid").argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, i64, vp, vp]

    def zoltan_bf_pairs(self, a, b, p0=None, q0=None):
        """zoltan/bf.cpp's per-pair bf over pair-list planes a, b (9, n); p0/q0 (3, n) are
        the values left where it returns early (default NaN)."""
        a = np.ascontiguousarray(a, np.float64); b = np.ascontiguousarray(b, np.float64)
        n = a.shape[1]
        p = np.full((3, n), np.nan) if p0 is None else np.array(p0, np.float64)
        q = np.full((3, n), np.nan) if q0 is None else np.array(q0, np.float64)
        f = getattr(self.zlib, self.zprefix + "bf")
        pq = np.empty(6)
        for i in range(n):
            xa, ya, za = (np.ascontiguousarray(a[[k, 3 + k, 6 + k], i]) for k in range(3))
            xb, yb, zb = (np.ascontiguousarray(b[[k, 3 + k, 6 + k], i]) for k in range(3))
            pq[:3] = p[:, i]; pq[3:] = q[:, i]
            f(_p(xa), _p(ya), _p(za), _p(xb), _p(yb), _p(zb), _p(pq))
            p[:, i] = pq[:3]; q[:, i] = pq[3:]
        return p, q

    def zoltan_soa(self, method, it, nt, abc, d, e, f, p0=None, q0=None):
        """method "penalty" or "hybrid" (and "bf" for the oracle): triangle abc (3, 3) rows
        a, b, c against the list d, e, f (3, n); returns p, q (3, n) starting from p0, q0."""
        abc = np.ascontiguousarray(abc, np.float64)
        d, e, f = (np.ascontiguousarray(x, np.float64) for x in (d, e, f))
        n = d.shape[1]
        p = np.full((3, n), np.nan) if p0 is None else np.array(p0, np.float64)
        q = np.full((3, n), np.nan) if q0 is None else np.array(q0, np.float64)
        fn = getattr(self.zlib, self.zprefix + method)
        fn(it, nt, _p(abc[0]), _p(abc[1]), _p(abc[2]), _p(d), _p(e), _p(f), n, _p(p), _p(q))
        return p, q


class Oracle(_Lib, _Zoltan):
    """The C restatement (liboracle.so)."""

    prefix = "dor_"
    zprefix = "dzo_"

    def __init__(self, path: str | os.PathLike | None = None):
        path = Path(path) if path else HERE / "liboracle.so"
        if not _build_if_missing(path):
            raise RuntimeError(f"oracle library missing: {path}")
        self.lib = C.CDLL(str(path))
        self.zlib = self.lib
        self._sig()
        self._zsig()
        vp0, i32_, i64_, u32_, f8_ = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32, C.c_double
        self.lib.dzo_bf_soa.argtypes = [u32_, u32_, vp0, vp0, vp0, vp0, vp0, vp0, i64_, vp0, vp0]
        self.lib.dzo_penalty_shifted.argtypes = [u32_, u32_, vp0, vp0, vp0, vp0, vp0, vp0, i64_, vp0, vp0, i32_]
        self.lib.dzo_hybrid_shifted.argtypes = [i32_, i32_, vp0, vp0, vp0, vp0, vp0, vp0, i64_, vp0, vp0, i32_,
                                                i32_]
        self.lib.dzo_update.argtypes = [i32_, i32_, vp0, i64_, vp0, vp0, vp0, vp0, vp0, vp0, vp0, vp0, vp0, vp0,
                                        f8_]
        self.lib.dzo_euler.argtypes = [i32_, vp0, vp0, vp0, vp0, f8_]
        self.lib.dzo_integrate.argtypes = [f8_, vp0, vp0, i32_, vp0, i64_, vp0]
        self.lib.dzo_force.argtypes = [i32_, vp0, vp0, vp0, vp0, vp0, i64_, vp0, vp0, vp0, vp0, vp0, vp0, vp0,
                                       f8_, f8_]
        L = self.lib
        vp, i32, i64, f8 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.dor_contacts_forces.argtypes = [vp, i64, f8, vp, vp, vp, f8, vp, vp, vp, f8, vp, vp, vp]
        L.dor_update_rotation.argtypes = [vp, vp, vp, f8]
        L.dor_update_angular.argtypes = [vp, vp, vp, vp, vp, f8]
        L.dor_sim_create.restype = vp
        L.dor_sim_destroy.argtypes = [vp]
        L.dor_sim_run.argtypes = [vp, vp, vp, i32, vp]
        L.dor_sim_run.restype = i64
        L.dor_sim_contacts.argtypes = [vp, vp, i64]
        L.dor_sim_contacts.restype = i64
        L.dor_filter_new.argtypes = [i64, vp, i64, vp, vp, f8, vp]
        L.dor_filter_old.argtypes = [i64, vp, i64, vp, vp, i64, vp, i64, vp, vp, f8, vp]

    def zoltan_r_shifted(self, method, it, nt, abc, d, e, f, p0=None, q0=None, shifts=range(-12, 13)):
        """The results penalty / hybrid can give when the penalty weight r (formed with pow
        and log/log10, whose last bit depends on the math library) moves by each of `shifts`
        units in the last place: array (k, 6, n) of (p, q) planes.  For hybrid: the 7-step
        penalty points for every shift (no fallback), and the fallback points of every batch
        (bf, which does not depend on r)."""
        abc = np.ascontiguousarray(abc, np.float64)
        d, e, f = (np.ascontiguousarray(x, np.float64) for x in (d, e, f))
        n = d.shape[1]

        def run(u, mode):
            p = np.full((3, n), np.nan) if p0 is None else np.array(p0, np.float64)
            q = np.full((3, n), np.nan) if q0 is None else np.array(q0, np.float64)
            args = [it, nt, _p(abc[0]), _p(abc[1]), _p(abc[2]), _p(d), _p(e), _p(f), n, _p(p), _p(q), int(u)]
            if method == "hybrid":
                self.lib.dzo_hybrid_shifted(*args, mode)
            else:
                self.lib.dzo_penalty_shifted(*args)
            return np.concatenate([p, q])
        out = [run(u, 1) for u in shifts]
        if method == "hybrid":
            out.append(run(0, 2))
        return np.stack(out)

    # ---- zoltan dynamics and forces (zoltan_oracle.c) ------------------------------------
    def zoltan_update(self, t, pid, angular, linear, rotation, position, inertia, inverse, mass, force, torque, step):
        """dynamics::update on copies; t (6, 3, nt), per-body arrays (k, nb).  Returns the
        updated (t, angular, linear, rotation, position, force, torque)."""
        t = np.array(t, np.float64, copy=True).reshape(18, -1)
        nt = t.shape[1]
        out = [np.array(x, np.float64, copy=True) for x in (angular, linear, rotation, position, force, torque)]
        inertia = np.ascontiguousarray(inertia, np.float64); inverse = np.ascontiguousarray(inverse, np.float64)
        mass = np.ascontiguousarray(mass, np.float64); pid = np.ascontiguousarray(pid, np.int32)
        self.lib.dzo_update(nt, len(mass), _p(t), nt, _p(pid), _p(out[0]), _p(out[1]), _p(out[2]), _p(out[3]),
                            _p(inertia), _p(inverse), _p(mass), _p(out[4]), _p(out[5]), step)
        return (t.reshape(6, 3, nt), *out)

    def zoltan_euler(self, angular, linear, rotation, position, step):
        out = [np.array(x, np.float64, copy=True) for x in (angular, rotation, position)]
        linear = np.ascontiguousarray(linear, np.float64)
        self.lib.dzo_euler(linear.shape[1], _p(out[0]), _p(linear), _p(out[1]), _p(out[2]), step)
        return tuple(out)

    def zoltan_integrate(self, step, lo, hi, t, v):
        t = np.array(t, np.float64, copy=True).reshape(9, -1)
        v = np.array(v, np.float64, copy=True)
        lo = np.ascontiguousarray(lo, np.float64); hi = np.ascontiguousarray(hi, np.float64)
        nt = t.shape[1]
        self.lib.dzo_integrate(step, _p(lo), _p(hi), nt, _p(t), nt, _p(v))
        return t.reshape(3, 3, nt), v

    def zoltan_force(self, offset, slave, point, normal, depth, position, angular, linear, mass, force, torque,
                     gravity, spring=1e2, damper=1.0):
        """forces::force; returns the accumulated (force, torque) copies."""
        F = np.array(force, np.float64, copy=True); T = np.array(torque, np.float64, copy=True)
        offset = np.ascontiguousarray(offset, np.int64); slave = np.ascontiguousarray(slave, np.int32)
        point, normal, position, angular, linear = (np.ascontiguousarray(x, np.float64)
                                                    for x in (point, normal, position, angular, linear))
        depth = np.ascontiguousarray(depth, np.float64); mass = np.ascontiguousarray(mass, np.float64)
        g = np.ascontiguousarray(gravity, np.float64)
        self.lib.dzo_force(len(mass), _p(offset), _p(slave), _p(point), _p(normal), _p(depth), len(slave),
                           _p(position), _p(angular), _p(linear), _p(mass), _p(F), _p(T), _p(g), spring, damper)
        return F, T

    def filter_new(self, x, master, slave, eps=1e-4):
        """keep flags of filterNewContacts per (master, slave) segment; x is (3, n)."""
        x = np.ascontiguousarray(x, np.float64)
        m = np.ascontiguousarray(master, np.int32); s = np.ascontiguousarray(slave, np.int32)
        n = x.shape[1]
        keep = np.zeros(n, np.uint8)
        self.lib.dor_filter_new(n, _p(x), n, _p(m), _p(s), eps, _p(keep))
        return keep

    def filter_old(self, xs, ms, ss, xn, mn, sn, eps=1e-4):
        """keep flags of filterOldContacts for the new contacts xn against stored xs."""
        xs = np.ascontiguousarray(xs, np.float64); xn = np.ascontiguousarray(xn, np.float64)
        a = [np.ascontiguousarray(v, np.int32) for v in (ms, ss, mn, sn)]
        keep = np.zeros(xn.shape[1], np.uint8)
        self.lib.dor_filter_old(xs.shape[1], _p(xs), xs.shape[1], _p(a[0]), _p(a[1]), xn.shape[1], _p(xn),
                                xn.shape[1], _p(a[2]), _p(a[3]), eps, _p(keep))
        return keep

    def contacts_forces(self, contacts, sign, posA, angA, linA, mA, posB, angB, linB, mB, spring, damper, friction):
        c = np.ascontiguousarray(contacts, CONTACT_DTYPE)
        F = np.zeros(3); T = np.zeros(3)
        mat = Material(spring, damper, friction)
        arr = [np.ascontiguousarray(x, np.float64) for x in (posA, angA, linA, posB, angB, linB)]
        self.lib.dor_contacts_forces(_p(c), len(c), sign, _p(arr[0]), _p(arr[1]), _p(arr[2]), mA,
                                     _p(arr[3]), _p(arr[4]), _p(arr[5]), mB, C.byref(mat), _p(F), _p(T))
        return F, T

    def simulate(self, scene: dict, dt, gravity, spring, damper, friction, nsteps):
        """Runs nsteps on a copy of `scene` (dict of numpy arrays, see delta_b200.scenarios).
        Returns (new_scene_dict, contacts_per_step, final_contacts)."""
        s = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in scene.items()}
        sc = Scene()
        sc.n_bodies = s["n_bodies"]
        for name in ("tri_offset", "x", "y", "z", "rx", "ry", "rz", "pos", "ref_pos", "vel", "ang", "ref_ang",
                     "rot", "inertia", "inverse", "mass", "eps", "radius", "friction", "obstacle"):
            setattr(sc, name, s[name].ctypes.data)
        prm = StepParams(dt, (C.c_double * 3)(*gravity), Material(spring, damper, friction))
        cps = np.zeros(max(nsteps, 1), np.int64)
        sim = self.lib.dor_sim_create()
        try:
            n = self.lib.dor_sim_run(sim, C.byref(sc), C.byref(prm), nsteps, _p(cps))
            out = np.zeros(max(n, 1), CONTACT_DTYPE)
            self.lib.dor_sim_contacts(sim, _p(out), len(out))
        finally:
            self.lib.dor_sim_destroy(sim)
        return s, cps[:nsteps], out[:n]


class ZoltanReference(_Zoltan):
    """The reference's zoltan/{bf,penalty,hybrid}.cpp (oracle/_ref/libzoltan_ref.so)."""

    zprefix = "zref_"

    def __init__(self):
        path = HERE / "_ref" / "libzoltan_ref.so"
        if not path.exists():
            raise FileNotFoundError(path)
        self.zlib = C.CDLL(str(path))
        self._zsig()

    @staticmethod
    def available() -> bool:
        return (HERE / "_ref" / "libzoltan_ref.so").exists()


class Reference(_Lib):
    """The reference's own functions (oracle/_ref), built by oracle/Makefile."""

    prefix = "ref_"

    def __init__(self, flavour: str = "par"):
        name = "libdelta_ref.so" if flavour == "par" else "libdelta_ref_omp.so"
        path = HERE / "_ref" / name
        if not path.exists():
            raise FileNotFoundError(path)
        self.lib = C.CDLL(str(path))
        self._sig()
        L = self.lib
        vp, i64, f8 = C.c_void_p, C.c_int64, C.c_double
        L.ref_contacts_forces.argtypes = [vp, i64, vp, vp, vp, f8, vp, vp, vp, f8, vp, vp]
        L.ref_update_rotation.argtypes = [vp, vp, vp, f8]
        L.ref_update_angular.argtypes = [vp, vp, vp, vp, vp, f8]
        L.ref_filter_new.argtypes = [i64, vp, i64, vp]
        L.ref_filter_new.restype = i64
        L.ref_filter_old.argtypes = [i64, vp, i64, i64, vp, i64, vp]
        L.ref_filter_old.restype = i64

    def filter_new(self, x):
        """keep flags of the reference's filterNewContacts over one contact list x (3, n)."""
        x = np.ascontiguousarray(x, np.float64)
        keep = np.zeros(x.shape[1], np.uint8)
        self.lib.ref_filter_new(x.shape[1], _p(x), x.shape[1], _p(keep))
        return keep

    def filter_old(self, xs, xn):
        """keep flags of the reference's filterOldContacts(stored xs, new xn)."""
        xs = np.ascontiguousarray(xs, np.float64); xn = np.ascontiguousarray(xn, np.float64)
        keep = np.zeros(xn.shape[1], np.uint8)
        self.lib.ref_filter_old(xs.shape[1], _p(xs), xs.shape[1], xn.shape[1], _p(xn), xn.shape[1], _p(keep))
        return keep

    def simulate(self, scene: dict, dt, gravity, nsteps):
        """Runs nsteps of the reference-driven time step (ref_sim.cpp) on a copy of `scene`
        (force constants: those compiled into forces.cpp).  Returns (new_scene, contacts_per_step)."""
        s = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in scene.items()}
        sc = Scene()
        sc.n_bodies = s["n_bodies"]
        for name in ("tri_offset", "x", "y", "z", "rx", "ry", "rz", "pos", "ref_pos", "vel", "ang", "ref_ang",
                     "rot", "inertia", "inverse", "mass", "eps", "radius", "friction", "obstacle"):
            setattr(sc, name, s[name].ctypes.data)
        L = self.lib
        L.ref_sim_create.restype = C.c_void_p
        L.ref_sim_destroy.argtypes = [C.c_void_p]
        L.ref_sim_run.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_int32, C.c_void_p]
        L.ref_sim_run.restype = C.c_int64
        cps = np.zeros(max(nsteps, 1), np.int64)
        g = np.ascontiguousarray(gravity, np.float64)
        sim = L.ref_sim_create()
        try:
            L.ref_sim_run(sim, C.byref(sc), dt, _p(g), nsteps, _p(cps))
        finally:
            L.ref_sim_destroy(sim)
        return s, cps[:nsteps]

    @staticmethod
    def available(flavour: str = "par") -> bool:
        name = "libdelta_ref.so" if flavour == "par" else "libdelta_ref_omp.so"
        return (HERE / "_ref" / name).exists()

    def contacts_forces(self, contacts, posA, angA, linA, mA, posB, angB, linB, mB):
        c = np.ascontiguousarray(contacts, CONTACT_DTYPE)
        F = np.zeros(3); T = np.zeros(3)
        arr = [np.array(x, np.float64) for x in (posA, angA, linA, posB, angB, linB)]
        self.lib.ref_contacts_forces(_p(c), len(c), _p(arr[0]), _p(arr[1]), _p(arr[2]), mA,
                                     _p(arr[3]), _p(arr[4]), _p(arr[5]), mB, _p(F), _p(T))
        return F, T
