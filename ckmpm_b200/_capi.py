"""ctypes binding of the C ABI in include/ckmpm.h.

The CUDA library is required: importing a function from here loads
ckmpm_b200/_lib/libckmpm_b200.so and raises if it is missing.  There is no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libckmpm_b200.so"

CKMPM_OK = 0
CKMPM_ERR_INVALID = 1
STATUS_NAMES = {
    0: "CKMPM_OK",
    1: "CKMPM_ERR_INVALID",
    2: "CKMPM_ERR_CUDA",
    3: "CKMPM_ERR_CAPACITY",
    4: "CKMPM_ERR_NUMERIC",
    5: "CKMPM_ERR_TIMEOUT",
    6: "CKMPM_ERR_NOT_FOUND",
}

FIXED_COROTATED = 0
LINEAR = 1
DRUCKER_PRAGER = 2
FLUID = 3
VON_MISES = 4
NACC = 5
MATERIAL_PARAMS = 8

BOUNDARY_STICKY_BLOCKS = 0
BOUNDARY_SLIP_FLOOR = 1
BOUNDARY_FIELD = 2
CELL_FREE, CELL_FIXED, CELL_SLIP, CELL_VELOCITY, CELL_SEPARATE = 0, 1, 2, 3, 4

FLAG_TRACK_IDS = 1

# Every symbol include/ckmpm.h declares.
EXPORTED = (
    "ckmpm_create", "ckmpm_add_model", "ckmpm_setup", "ckmpm_step", "ckmpm_step_async",
    "ckmpm_status_check", "ckmpm_step_adaptive", "ckmpm_set_stream", "ckmpm_get_count",
    "ckmpm_get_state", "ckmpm_get_blocks", "ckmpm_get_counters", "ckmpm_get_dt",
    "ckmpm_step_profiled", "ckmpm_debug_constitutive", "ckmpm_destroy", "ckmpm_last_error",
    "ckmpm_version", "ckmpm_simulate_noalloc", "ckmpm_create_batch", "ckmpm_add_batch", "ckmpm_get_blocks_in",
    "ckmpm_set_tuning", "ckmpm_set_reorder_interval", "ckmpm_get_tuning", "ckmpm_autotune", "ckmpm_checkpoint_bytes",
    "ckmpm_checkpoint_save", "ckmpm_checkpoint_restore", "ckmpm_diff_create", "ckmpm_diff_forward", "ckmpm_diff_backward", "ckmpm_diff_timing",
    "ckmpm_diff_last_error", "ckmpm_diff_destroy", "ckmpm_set_rigid", "ckmpm_set_rigid_velocity", "ckmpm_get_time",
    "ckmpm_set_boundary_field", "ckmpm_export_positions_async", "ckmpm_export_wait",
    "ckmpm_dd_blocks", "ckmpm_dd_mark", "ckmpm_dd_pack", "ckmpm_dd_unpack",
)

MAX_BATCH_SCENES = 65536


class SceneDesc(C.Structure):
    _fields_ = [
        ("dx", C.c_float),
        ("domain_blocks", C.c_int32 * 3),
        ("gravity", C.c_float),
        ("mass_clamp", C.c_float),
        ("boundary", C.c_int32),
        ("floor_cells", C.c_float),
        ("max_particles_per_block", C.c_uint32),
        ("device", C.c_int32),
        ("flags", C.c_uint32),
    ]


class Material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("p", C.c_float * MATERIAL_PARAMS)]


class BatchScene(C.Structure):
    _fields_ = [("material", Material), ("mass", C.c_float), ("volume", C.c_float), ("n", C.c_uint32)]


class Tuning(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("graph_chunk", C.c_uint32),
                ("probe_ms", C.c_float)]

    def as_dict(self) -> dict:
        return {"threads": int(self.threads), "ctas_per_sm": int(self.ctas_per_sm),
                "graph_chunk": int(self.graph_chunk), "probe_ms": float(self.probe_ms)}


class CkmpmError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load the CUDA engine; raise loudly if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA engine first (python -m ckmpm_b200.build). "
                "There is no CPU fallback.")
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        f32p = C.POINTER(C.c_float)
        u32p = C.POINTER(C.c_uint32)
        i32p = C.POINTER(C.c_int32)
        L.ckmpm_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(P)]
        L.ckmpm_add_model.argtypes = [P, C.POINTER(Material), C.c_uint32, f32p, f32p, C.c_uint32, C.c_float,
                                      C.c_float, i32p]
        L.ckmpm_setup.argtypes = [P]
        L.ckmpm_step.argtypes = [P, C.c_uint32, C.c_float]
        L.ckmpm_step_async.argtypes = [P, C.c_uint32, C.c_float]
        L.ckmpm_status_check.argtypes = [P]
        L.ckmpm_step_adaptive.argtypes = [P, C.c_uint32, C.c_float, C.c_float, C.c_double, C.POINTER(C.c_double)]
        L.ckmpm_set_stream.argtypes = [P, P]
        L.ckmpm_set_rigid.argtypes = [P, C.c_uint32, C.POINTER(C.c_float)]
        L.ckmpm_set_rigid_velocity.argtypes = [P, C.POINTER(C.c_float)]
        L.ckmpm_get_time.argtypes = [P, C.POINTER(C.c_double)]
        L.ckmpm_set_boundary_field.argtypes = [P, C.POINTER(C.c_uint8), C.POINTER(C.c_float)]
        L.ckmpm_get_count.argtypes = [P, C.c_int32, u32p]
        L.ckmpm_get_state.argtypes = [P, C.c_int32, f32p, f32p, f32p, f32p, u32p, C.c_uint32, u32p]
        L.ckmpm_export_positions_async.argtypes = [P, C.c_int32, f32p, C.c_uint32]
        L.ckmpm_export_wait.argtypes = [P, u32p]
        L.ckmpm_get_blocks.argtypes = [P, C.c_int32, C.c_int32, i32p, u32p, C.c_uint32, u32p]
        L.ckmpm_get_counters.argtypes = [P, C.POINTER(C.c_uint64)]
        L.ckmpm_get_dt.argtypes = [P, f32p]
        L.ckmpm_step_profiled.argtypes = [P, C.c_uint32, C.c_float, C.POINTER(C.c_double)]
        L.ckmpm_debug_constitutive.argtypes = [C.POINTER(Material), C.c_uint32, f32p, C.c_float, f32p, f32p, f32p,
                                               f32p, f32p, f32p]
        L.ckmpm_simulate_noalloc.argtypes = [C.POINTER(SceneDesc), C.POINTER(Material), C.c_uint32, P, P, C.c_uint32,
                                             C.c_float, C.c_float, C.c_uint32, C.c_float, P, P, P, P, P,
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_char_p)]
        L.ckmpm_create_batch.argtypes = [C.POINTER(SceneDesc), C.c_uint32, C.POINTER(P)]
        L.ckmpm_dd_blocks.argtypes = [P, u32p]
        L.ckmpm_dd_mark.argtypes = [P, P]
        L.ckmpm_dd_pack.argtypes = [P, P, C.c_uint32, P]
        L.ckmpm_dd_unpack.argtypes = [P, P, C.c_uint32, P]
        L.ckmpm_add_batch.argtypes = [P, C.c_uint32, C.POINTER(BatchScene), f32p, f32p]
        L.ckmpm_get_blocks_in.argtypes = [P, C.c_uint32, C.c_int32, C.c_int32, i32p, u32p, C.c_uint32, u32p]
        L.ckmpm_set_tuning.argtypes = [P, C.POINTER(Tuning)]
        L.ckmpm_set_reorder_interval.argtypes = [P, C.c_uint32]
        L.ckmpm_get_tuning.argtypes = [P, C.POINTER(Tuning), u32p]
        L.ckmpm_autotune.argtypes = [P, C.c_uint32, C.c_float, C.POINTER(Tuning), C.c_uint32, u32p,
                                     C.POINTER(Tuning)]
        L.ckmpm_checkpoint_bytes.argtypes = [P, C.POINTER(C.c_uint64)]
        L.ckmpm_checkpoint_save.argtypes = [P, P]
        L.ckmpm_checkpoint_restore.argtypes = [P, P]
        L.ckmpm_destroy.argtypes = [P]
        L.ckmpm_last_error.argtypes = [P]
        L.ckmpm_last_error.restype = C.c_char_p
        L.ckmpm_version.restype = C.c_char_p
        for name in EXPORTED:
            fn = getattr(L, name)
            if name not in ("ckmpm_last_error", "ckmpm_version", "ckmpm_diff_last_error"):
                fn.restype = C.c_int
        L.ckmpm_diff_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def uptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def check(code: int, where: str, handle=None) -> None:
    if code != CKMPM_OK:
        msg = lib().ckmpm_last_error(handle)
        raise CkmpmError(code, where, msg.decode() if msg else "")
