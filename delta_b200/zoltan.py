"""The reference's zoltan/ code path on the GPU, with its argument lists.

zoltan/ keeps the system as structure-of-arrays: the narrowphase takes one triangle
(a, b, c) against a list of triangles (d, e, f) (zoltan/bf.h, penalty.h, hybrid.h), the
integration takes per-body arrays (zoltan/dynamics.h), the forces a per-body contact list
(zoltan/forces.h).  Here every per-coordinate array is a row of a float64 CUDA tensor:
d, e, f, p, q are (3, n); t is (6, 3, nt) (vertex, coordinate, triangle; vertices 0..2
spatial, 3..5 referential); per-body arrays are (k, nb).  Each function is one call of
the C ABI (include/delta_b200.h, delta_zoltan_*), asynchronous on the context's stream.
"""
from __future__ import annotations

import ctypes as C

from ._lib import check, lib
from .narrowphase import Context


def _rows(x, k: int):
    """(C.c_void_p * k) of the row pointers of a (k, n) float64 CUDA tensor."""
    if x.dim() != 2 or x.shape[0] != k or x.stride(1) != 1:
        raise ValueError(f"expected a ({k}, n) tensor with contiguous rows")
    return (C.c_void_p * k)(*[x[r].data_ptr() for r in range(k)])


def _vec3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _narrow(fn, ctx: Context, it: int, nt: int, a, b, c, d, e, f, p, q):
    check(fn(ctx.handle, it, nt, _vec3(a), _vec3(b), _vec3(c), _rows(d, 3), _rows(e, 3), _rows(f, 3), _rows(p, 3),
             _rows(q, 3)))


def bf(ctx: Context, it: int, nt: int, a, b, c, d, e, f, p, q):
    """bf(it, nt, A, B, C, D, E, F, P, Q) (zoltan/bf.h:61-64) with zoltan/bf.cpp's per-pair
    arithmetic; entries where that returns early keep their p, q."""
    _narrow(lib().delta_zoltan_bf, ctx, it, nt, a, b, c, d, e, f, p, q)


def penalty(ctx: Context, it: int, nt: int, a, b, c, d, e, f, p, q):
    """penalty(it, nt, ...), zoltan/penalty.cpp:27-209."""
    _narrow(lib().delta_zoltan_penalty, ctx, it, nt, a, b, c, d, e, f, p, q)


def hybrid(ctx: Context, it: int, nt: int, a, b, c, d, e, f, p, q):
    """hybrid(it, nt, ...), zoltan/hybrid.cpp:37-131 (it counts batches of 4)."""
    _narrow(lib().delta_zoltan_hybrid, ctx, it, nt, a, b, c, d, e, f, p, q)


def update(ctx: Context, t, pid, angular, linear, rotation, position, inertia, inverse, mass, force, torque,
           step: float):
    """dynamics::update, zoltan/dynamics.cpp:66-250."""
    nt = t.shape[2] if t is not None else 0
    nb = mass.shape[0]
    tp = (C.c_void_p * 18)(*[t[v, k].data_ptr() for v in range(6) for k in range(3)]) if nt else None
    check(lib().delta_zoltan_update(ctx.handle, nt, nb, tp, pid.data_ptr() if nt else None, _rows(angular, 6),
                                    _rows(linear, 3), _rows(rotation, 9), _rows(position, 6), _rows(inertia, 9),
                                    _rows(inverse, 9), mass.data_ptr(), _rows(force, 3), _rows(torque, 3),
                                    float(step)))


def euler(ctx: Context, angular, linear, rotation, position, step: float):
    """dynamics::euler, zoltan/dynamics.cpp:252-297."""
    check(lib().delta_zoltan_euler(ctx.handle, angular.shape[1], _rows(angular, 6), _rows(linear, 3),
                                   _rows(rotation, 9), _rows(position, 6), float(step)))


def integrate(ctx: Context, step: float, lo, hi, t, v):
    """dynamics::integrate, zoltan/dynamics.cpp:299-335; t is (3, 3, nt), v (3, nt)."""
    nt = t.shape[2]
    tp = (C.c_void_p * 9)(*[t[w, k].data_ptr() for w in range(3) for k in range(3)])
    check(lib().delta_zoltan_integrate(ctx.handle, float(step), _vec3(lo), _vec3(hi), nt, tp, _rows(v, 3)))


def force(ctx: Context, offset, slave, point, normal, depth, position, angular, linear, mass, force_, torque,
          gravity, spring: float = 1e2, damper: float = 1.0):
    """forces::force, zoltan/forces.cpp:48-205: contacts grouped by master (body i's are
    [offset[i], offset[i+1])); force_ and torque (3, nb) accumulate."""
    nb = mass.shape[0]
    nc = slave.shape[0]
    check(lib().delta_zoltan_force(ctx.handle, nb, offset.data_ptr(), slave.data_ptr() if nc else None, nc,
                                   _rows(point, 3) if nc else None, _rows(normal, 3) if nc else None,
                                   depth.data_ptr() if nc else None, _rows(position, 6), _rows(angular, 6),
                                   _rows(linear, 3), mass.data_ptr(), _rows(force_, 3), _rows(torque, 3),
                                   _vec3(gravity), float(spring), float(damper)))
