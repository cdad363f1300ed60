"""ctypes binding of libdelta_b200.so (the C ABI declared in include/delta_b200.h).

The library is required: every compute entry point goes through it and raises when it
is missing; there is no CPU fallback.  Build it with ``make -C delta_b200``
(``__graft_entry__.build()`` does this).
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libdelta_b200.so"
HEADER = HERE.parent / "include" / "delta_b200.h"

OK, ERR_INVALID, ERR_CUDA, ERR_CAPACITY, ERR_TIMEOUT, ERR_NOMEM, ERR_UNSUPPORTED = range(7)
STATUS_NAMES = ["OK", "INVALID", "CUDA", "CAPACITY", "TIMEOUT", "NOMEM", "UNSUPPORTED"]

vp, i32, i64, f8 = C.c_void_p, C.c_int32, C.c_int64, C.c_double

# argument types of every exported function (restype int = delta_status unless listed)
SIGNATURES: dict[str, tuple[list, object]] = {
    "delta_create": ([C.POINTER(vp), C.c_int, vp], C.c_int),
    "delta_destroy": ([vp], C.c_int),
    "delta_set_stream": ([vp, vp], C.c_int),
    "delta_synchronize": ([vp], C.c_int),
    "delta_last_error": ([], C.c_char_p),
    "delta_version": ([], C.c_char_p),
    "delta_launch_count": ([vp], i64),
    "delta_pairs_run": ([vp, C.c_int, C.c_int, i64, vp, vp, i64, f8, vp, vp, vp, vp], C.c_int),
    "delta_pairs_run_host": ([vp, C.c_int, C.c_int, i64, vp, vp, i64, f8, vp, vp, vp, vp], C.c_int),
    "delta_set_pair_launch": ([vp, C.c_int, C.c_int, i32, i32], C.c_int),
    "delta_autotune_pairs": ([vp, C.c_int, C.c_int, i64, vp, vp, i64, f8, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_pairs_run_host_noalloc": ([vp, C.c_int, C.c_int, i64, vp, vp, i64, f8, vp, vp, vp, vp], C.c_int),
    "delta_detect": ([vp, C.c_int, C.c_int, vp, vp, vp, i64, vp, vp, vp], C.c_int),
    "delta_forces": ([vp, vp, vp, i64, vp, vp, vp, vp], C.c_int),
    "delta_integrate": ([vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_broadphase": ([vp, vp, vp, vp, i64, vp], C.c_int),
    "delta_sim_create": ([vp, vp, C.c_int, vp], C.c_int),
    "delta_sim_step": ([vp, vp, i32, vp], C.c_int),
    "delta_sim_step_graph": ([vp, vp, i32, vp], C.c_int),
    "delta_sim_set_graph_capacity": ([vp, i64, i64], C.c_int),
    "delta_sim_skin_stats": ([vp, vp, vp, vp], C.c_int),
    "delta_sim_contacts": ([vp, vp, vp], C.c_int),
    "delta_sim_counters": ([vp, vp], C.c_int),
    "delta_set_cull_launch": ([vp, i32, i32], C.c_int),
    "delta_sim_autotune": ([vp, i32, vp, vp], C.c_int),
    "delta_sim_destroy": ([vp], C.c_int),
    "delta_sphere_contacts": ([vp, vp, vp, vp, i64, vp, vp], C.c_int),
    "delta_sphere_mesh_contacts": ([vp, vp, vp, vp, vp, i64, C.c_int, vp, vp], C.c_int),
    "delta_sphere_overlap": ([vp, vp, i64, vp, vp, vp, i64, vp], C.c_int),
    "delta_write_vtk_host": ([C.c_char_p, i32, i32, vp, vp, vp, vp], C.c_int),
    "delta_write_vtk": ([vp, C.c_char_p, i32, vp], C.c_int),
    "delta_sim_write_vtk": ([vp, C.c_char_p, i32], C.c_int),
    "delta_write_vtu_host": ([C.c_char_p, i32, i64, vp, vp, vp], C.c_int),
    "delta_sim_write_vtu": ([vp, C.c_char_p, i32], C.c_int),
    "delta_read_mbfcp": ([C.c_char_p, vp, i64, vp], C.c_int),
    "delta_filter_new_contacts": ([vp, vp, i64, f8, vp], C.c_int),
    "delta_filter_old_contacts": ([vp, vp, i64, vp, i64, f8, vp], C.c_int),
    "delta_mlp_layout": ([vp], C.c_int),
    "delta_mlp_infer": ([vp, i64, vp, vp, i64, vp, vp, vp], C.c_int),
    "delta_mlp_infer_tcgen05": ([vp, i64, vp, vp, i64, vp, vp, vp], C.c_int),
    "delta_mlp_infer_tcgen05_wait_test": ([vp, i64, vp, vp, i64, vp, vp, vp, C.c_uint32], C.c_int),
    "delta_mlp_set_engine": ([vp, C.c_int], C.c_int),
    "delta_mlp_features": ([vp, i64, vp, vp, i64, vp, vp, vp, vp, vp], C.c_int),
    "delta_gemm_bf16": ([vp, C.c_int, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int,
                         C.c_int, C.c_int], C.c_int),
    "delta_mlp_bias_act": ([vp, i64, C.c_int, vp, vp, vp, C.c_int], C.c_int),
    "delta_mlp_mse": ([vp, i64, vp, vp, vp, C.c_float, vp, vp], C.c_int),
    "delta_mlp_act_grad": ([vp, i64, C.c_int, vp, vp, vp], C.c_int),
    "delta_mlp_colsum": ([vp, i64, C.c_int, vp, vp], C.c_int),
    "delta_adam": ([vp, i64, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, i64, vp], C.c_int),
    "delta_to_bf16": ([vp, i64, vp, vp], C.c_int),
    "delta_penalty_warm": ([vp, i64, vp, vp, i64, vp, f8, vp, vp, vp, vp], C.c_int),
    "delta_learned_refine": ([vp, i64, vp, vp, i64, vp, i32, i32, f8, vp, vp, vp, vp], C.c_int),
    "delta_pairs_run_learned": ([vp, i64, vp, vp, i64, vp, vp, i32, i32, f8, vp, vp, vp, vp, vp], C.c_int),
    "delta_pairs_run_learned_host": ([vp, i64, vp, vp, i64, vp, vp, i32, i32, f8, vp, vp, vp, vp, vp], C.c_int),
    "delta_contact_forces": ([vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_update_angular": ([vp, i32, vp, vp, vp, vp, vp, f8], C.c_int),
    "delta_update_rotation": ([vp, i32, vp, vp, vp, f8], C.c_int),
    "delta_update_vertices": ([vp, i64, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_zoltan_bf": ([vp, C.c_uint32, C.c_uint32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_zoltan_penalty": ([vp, C.c_uint32, C.c_uint32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_zoltan_hybrid": ([vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
    "delta_zoltan_update": ([vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, f8], C.c_int),
    "delta_zoltan_euler": ([vp, i32, vp, vp, vp, vp, f8], C.c_int),
    "delta_zoltan_integrate": ([vp, f8, vp, vp, i32, vp, vp], C.c_int),
    "delta_zoltan_force": ([vp, i32, vp, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, f8, f8], C.c_int),
}


class DeltaError(RuntimeError):
    def __init__(self, status: int, msg: str):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"delta_b200: {name}: {msg}")
        self.status = status


_lib = None


def header_functions() -> list[str]:
    """Names of the functions include/delta_b200.h declares."""
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(delta_\w+)\s*\(", text)))


def header_define(name: str) -> int:
    """Integer value of a ``#define`` in include/delta_b200.h."""
    m = re.search(rf"#define\s+{name}\s+(\d+)", HEADER.read_text())
    if not m:
        raise KeyError(name)
    return int(m.group(1))


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built (run `make -C {HERE}`); there is no CPU fallback")
    L = C.CDLL(str(LIB_PATH))
    for name, (args, res) in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(status: int):
    if status != OK:
        raise DeltaError(status, lib().delta_last_error().decode(errors="replace"))
