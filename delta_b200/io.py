"""The reference's on-disk formats through the C ABI: the legacy VTK snapshot
(writeGeometryToVTK, delta/core/io/write.cpp:226-306) and the .mbfcp scene reader
(readmbfcp, delta/core/io/read.cpp:345-546)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import ERR_CAPACITY, check, lib


class _Mbfcp(C.Structure):
    _fields_ = [("id", C.c_void_p), ("centre", C.c_void_p), ("radius", C.c_void_p), ("bodies", C.c_int32),
                ("has_materials", C.c_int32), ("friction", C.c_double), ("spring", C.c_double),
                ("dashpot", C.c_double), ("density", C.c_double), ("gravity", C.c_double * 3)]


def _dir(path) -> bytes:
    p = os.fspath(path)
    return (p if p.endswith(os.sep) or p == "" else p + os.sep).encode()


def write_vtk_host(path, step: int, bodies) -> str:
    """Writes <path>/geometry_<step>.vtk for bodies given as (3, 3*nT) host arrays; returns
    the file name."""
    counts = [b.shape[1] // 3 for b in bodies]
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    xyz = np.ascontiguousarray(np.concatenate(bodies, 1) if bodies else np.zeros((3, 0)), np.float64)
    x, y, z = (np.ascontiguousarray(xyz[k]) for k in range(3))
    check(lib().delta_write_vtk_host(_dir(path), int(step), len(bodies), off.ctypes.data, x.ctypes.data,
                                     y.ctypes.data, z.ctypes.data))
    return os.path.join(os.fspath(path), f"geometry_{int(step)}.vtk")


def write_vtk(ctx, path, step: int, meshes) -> str:
    """The same from device meshes (detection.Meshes or a simulation's current vertices)."""
    check(lib().delta_write_vtk(ctx.handle, _dir(path), int(step), C.byref(meshes.struct())))
    return os.path.join(os.fspath(path), f"geometry_{int(step)}.vtk")


def write_vtu_host(path, step: int, centre, velocity, eps) -> str:
    """writeGeometryToVTKVTK (write.cpp:10-70): <path>/geometry_<step>.vtu for n particles
    (centre, velocity: (3, n); eps: (n,)); returns the file name."""
    c = np.ascontiguousarray(centre, np.float64); v = np.ascontiguousarray(velocity, np.float64)
    e = np.ascontiguousarray(eps, np.float64)
    check(lib().delta_write_vtu_host(_dir(path), int(step), e.shape[0], c.ctypes.data, v.ctypes.data,
                                     e.ctypes.data))
    return os.path.join(os.fspath(path), f"geometry_{int(step)}.vtu")


def read_vtu(filename) -> dict:
    """The arrays of a .vtu written by write_vtu_host (ASCII VTK XML): 'points' (n, 3) and
    every point-data array by name ((n, k) or (n,))."""
    import xml.etree.ElementTree as ET

    root = ET.parse(os.fspath(filename)).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    n = int(piece.get("NumberOfPoints"))

    def arr(da):
        k = int(da.get("NumberOfComponents", "1"))
        dt = np.float32 if da.get("type") == "Float32" else np.float64
        v = np.array((da.text or "").split(), dtype=dt)
        return v.reshape(n, k) if k > 1 else v
    out = {"points": arr(piece.find("Points/DataArray")), "cells": int(piece.get("NumberOfCells"))}
    for da in piece.find("PointData"):
        out[da.get("Name")] = arr(da)
    out["active_scalars"] = piece.find("PointData").get("Scalars")
    out["active_vectors"] = piece.find("PointData").get("Vectors")
    return out


def read_mbfcp(filename, capacity: int = 1024) -> dict:
    """{'bodies', 'materials' (or None), 'id', 'centre' (n, 3), 'radius'} of a .mbfcp file."""
    while True:
        ids = np.zeros(capacity, np.int32)
        centre = np.zeros((capacity, 3))
        radius = np.zeros(capacity)
        m = _Mbfcp(ids.ctypes.data, centre.ctypes.data, radius.ctypes.data)
        n = C.c_int64(0)
        st = lib().delta_read_mbfcp(os.fspath(filename).encode(), C.byref(m), capacity, C.byref(n))
        if st == ERR_CAPACITY:
            capacity = int(n.value)
            continue
        check(st)
        k = int(n.value)
        mats = None
        if m.has_materials:
            mats = {"friction": m.friction, "spring": m.spring, "dashpot": m.dashpot, "density": m.density,
                    "gravity": list(m.gravity)}
        return {"bodies": m.bodies, "materials": mats, "id": ids[:k], "centre": centre[:k], "radius": radius[:k]}
