"""ctypes binding of libpfsim.so (the C ABI declared in include/pfsim.h).

The library is loaded from this package's directory; there is no fallback:
if it is missing the import fails with instructions to build it.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libpfsim.so"

PF_OK = 0
PF_ERR_INVALID = 1
PF_ERR_CUDA = 2
PF_ERR_STATE = 3
PF_ERR_OOM = 4
PF_ERR_DEVICE = 5
PF_ERR_BUDGET = 6

PF_KEY_LINEAR = 0
PF_KEY_MORTON = 1

PF_FLUID_VISCOSITY = 1
PF_FLUID_VORTICITY = 2
PF_FLUID_SURFACE_TENSION = 4
PF_FLUID_ADHESION = 8
PF_SHAPE_MATCH_GLOBAL = 0
PF_SHAPE_MATCH_LOCAL = 1
PF_PRIM_PLANE, PF_PRIM_SPHERE, PF_PRIM_BOX, PF_PRIM_CAPSULE = 0, 1, 2, 3
PF_PRIM_INVERT, PF_PRIM_SWEEP = 1, 2

(
    PF_FIELD_POSITIONS,
    PF_FIELD_PREDICTED,
    PF_FIELD_VELOCITIES,
    PF_FIELD_INV_MASS,
    PF_FIELD_BOUNDARY_VOLUME,
    PF_FIELD_DENSITY,
    PF_FIELD_ROTATION,
    PF_FIELD_PREDICTED_ROTATION,
    PF_FIELD_ANGULAR_VELOCITY,
    PF_FIELD_LAMBDA,
    PF_FIELD_NEIGHBOR_COUNT,
    PF_FIELD_NEIGHBORS,
    PF_FIELD_CELL_PERM,
) = range(13)

MAX_NEIGHBORS = 64


class PfError(RuntimeError):
    """An error returned by libpfsim; the message carries the reference-style prefix."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class GridDesc(C.Structure):
    _fields_ = [
        ("key_kind", C.c_uint32),
        ("origin", C.c_float * 3),
        ("cell_size", C.c_float),
        ("dims", C.c_uint32 * 3),
        ("table_size", C.c_uint32),
    ]


class Range(C.Structure):
    _fields_ = [("start", C.c_uint32), ("count", C.c_uint32)]


class SceneDesc(C.Structure):
    _fields_ = [("capacity", C.c_uint32), ("particle_radius", C.c_float)]


class FluidDesc(C.Structure):
    _fields_ = [
        ("range", Range),
        ("rest_density", C.c_float),
        ("particle_spacing", C.c_float),
        ("smoothing_radius", C.c_float),
        ("compliance", C.c_float),
        ("viscosity", C.c_float),
        ("flags", C.c_uint32),
        ("n_boundaries", C.c_uint32),
        ("boundaries", C.POINTER(Range)),
        ("boundary_static", C.POINTER(C.c_uint8)),
        ("vorticity", C.c_float),
        ("surface_tension", C.c_float),
        ("adhesion", C.c_float),
    ]


class SoftbodyDef(C.Structure):
    _fields_ = [
        ("range", Range),
        ("surface_count", C.c_uint32),
        ("compliance", C.c_float),
        ("rest_positions", C.POINTER(C.c_float)),
        ("edges", C.POINTER(C.c_uint32)),
        ("n_edges", C.c_uint32),
    ]


class SoftbodyDesc(C.Structure):
    _fields_ = [
        ("n_bodies", C.c_uint32),
        ("bodies", C.POINTER(SoftbodyDef)),
        ("shape_matching", C.c_uint32),
        ("self_collision", C.c_uint32),
    ]


class ClothDesc(C.Structure):
    _fields_ = [
        ("offset", C.c_uint32),
        ("n_particles", C.c_uint32),
        ("positions", C.POINTER(C.c_float)),
        ("inv_mass", C.POINTER(C.c_float)),
        ("n_pairs", C.c_uint32),
        ("pairs", C.POINTER(C.c_uint32)),
        ("rest_lengths", C.POINTER(C.c_float)),
        ("stretch_compliance", C.c_float),
        ("n_bending", C.c_uint32),
        ("bending", C.POINTER(C.c_uint32)),
        ("bending_rest", C.POINTER(C.c_float)),
        ("bend_compliance", C.c_float),
        ("n_tethers", C.c_uint32),
        ("tether_particle", C.POINTER(C.c_uint32)),
        ("tether_anchor", C.POINTER(C.c_uint32)),
        ("tether_rest", C.POINTER(C.c_float)),
        ("tether_compliance", C.c_float),
        ("n_triangles", C.c_uint32),
        ("triangles", C.POINTER(C.c_uint32)),
        ("wind", C.c_float * 3),
        ("drag", C.c_float),
        ("lift", C.c_float),
        ("has_damping", C.c_uint32),
        ("damping", C.c_float),
    ]


class Mesh(C.Structure):
    _fields_ = [
        ("vertices", C.POINTER(C.c_float)),
        ("n_vertices", C.c_uint32),
        ("indices", C.POINTER(C.c_uint32)),
        ("n_indices", C.c_uint32),
    ]


class Voxels(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(C.c_float)),
        ("capacity", C.c_uint32),
        ("edges", C.POINTER(C.c_uint32)),
        ("edge_capacity", C.c_uint32),
        ("count", C.c_uint32),
        ("surface_count", C.c_uint32),
        ("edge_count", C.c_uint32),
    ]


class ClothParams(C.Structure):
    _fields_ = [
        ("wind", C.c_float * 3),
        ("drag", C.c_float),
        ("lift", C.c_float),
        ("damping", C.c_float),
        ("bend_compliance", C.c_float),
    ]


class TetherBuildDesc(C.Structure):
    _fields_ = [
        ("n_particles", C.c_uint32),
        ("inv_mass", C.POINTER(C.c_float)),
        ("n_pairs", C.c_uint32),
        ("pairs", C.POINTER(C.c_uint32)),
        ("rest_lengths", C.POINTER(C.c_double)),
        ("max_attachments", C.c_uint32),
        ("stretch_tolerance", C.c_double),
    ]


class Primitive(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("flags", C.c_uint32),
        ("data0", C.c_float * 4),
        ("data1", C.c_float * 4),
        ("velocity", C.c_float * 4),
        ("rotation", C.c_float * 4),
        ("spin", C.c_float * 4),
    ]


class SdfDesc(C.Structure):
    _fields_ = [
        ("res", C.c_uint32 * 3),
        ("data", C.POINTER(C.c_float)),
        ("origin", C.c_float * 3),
        ("voxel_size", C.c_float * 3),
        ("position", C.c_float * 3),
        ("rotation", C.c_float * 4),
        ("scale", C.c_float),
        ("thickness", C.c_float),
        ("mu_s", C.c_float),
        ("mu_k", C.c_float),
    ]


class LoopDesc(C.Structure):
    _fields_ = [
        ("substeps", C.c_uint32),
        ("iterations", C.c_uint32),
        ("gravity", C.c_float * 3),
        ("hash_origin", C.c_float * 3),
        ("grid_min", C.c_float * 3),
        ("grid_max", C.c_float * 3),
        ("contact", C.c_uint32),
        ("contact_mu_s", C.c_float),
        ("contact_mu_k", C.c_float),
        ("max_contacts", C.c_uint32),
    ]


class Overflow(C.Structure):
    _fields_ = [
        ("positions", C.c_uint32),
        ("velocities", C.c_uint32),
        ("grid", C.c_uint32),
        ("contacts", C.c_uint32),
        ("neighbors", C.c_uint32),
        ("device_error", C.c_uint32),
        ("grid_clamped", C.c_uint32),
    ]


class BatchOpts(C.Structure):
    _fields_ = [("use_graph", C.c_uint32), ("block_size", C.c_uint32)]


class ServerOpts(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("max_scenes", C.c_uint32),
        ("use_graph", C.c_uint32),
        ("max_cohorts", C.c_uint32),
        ("mode", C.c_uint32),
        ("async_build", C.c_uint32),
    ]


PF_SERVER_BATCHED, PF_SERVER_PLAIN = 0, 1
PF_REQ_QUEUED, PF_REQ_BUILDING, PF_REQ_LIVE, PF_REQ_DONE = 0, 1, 2, 3


class ServerStats(C.Structure):
    _fields_ = [
        ("live", C.c_uint32),
        ("queued", C.c_uint32),
        ("building", C.c_uint32),
        ("finished", C.c_uint32),
        ("cohorts", C.c_uint32),
        ("reserved0", C.c_uint32),
        ("ticks", C.c_uint64),
        ("particle_substeps", C.c_uint64),
        ("state_bytes", C.c_uint64),
        ("rebuilds", C.c_uint64),
        ("busy_ms", C.c_double),
        ("last_tick_ms", C.c_float),
        ("p50_tick_ms", C.c_float),
        ("p99_tick_ms", C.c_float),
        ("max_tick_ms", C.c_float),
        ("max_swap_ms", C.c_float),
        ("max_admit_ms", C.c_float),
        ("last_admit_ms", C.c_float),
        ("max_step_ms", C.c_float),
        ("max_free_ms", C.c_float),
    ]


_P = C.c_void_p
_u32p = C.POINTER(C.c_uint32)
_f32p = C.POINTER(C.c_float)

# name -> (restype, argtypes). Declarations follow include/pfsim.h.
SIGNATURES = {
    "pf_last_error": (C.c_char_p, []),
    "pf_abi_version": (C.c_int, []),
    "pf_trim_device_memory": (C.c_int, []),
    "pf_grid_cells": (C.c_uint64, [C.POINTER(GridDesc)]),
    "pf_sort": (C.c_int, [_P, C.c_uint32, C.POINTER(GridDesc), _P, _P, _P, _P, _P, _P]),
    "pf_sort_device_errors": (C.c_int, [_P, _u32p]),
    "pf_sort_noalloc": (C.c_int, [_P, C.c_uint32, C.POINTER(GridDesc), _P, _P, _P, _P, _P, _P]),
    "pf_sort_host": (C.c_int, [_f32p, C.c_uint32, C.POINTER(GridDesc), _u32p, _u32p, _u32p, _u32p, _u32p]),
    "pf_scene_create": (C.c_int, [C.POINTER(SceneDesc), C.POINTER(_P)]),
    "pf_scene_destroy": (None, [_P]),
    "pf_upload_particles": (C.c_int, [_P, _f32p, _f32p, _f32p, _u32p, C.c_uint32, C.c_uint32]),
    "pf_set_inv_mass": (C.c_int, [_P, Range, C.c_float]),
    "pf_add_fluid": (C.c_int, [_P, C.POINTER(FluidDesc), _u32p]),
    "pf_add_softbodies": (C.c_int, [_P, C.POINTER(SoftbodyDesc), _u32p]),
    "pf_add_cloth": (C.c_int, [_P, C.POINTER(ClothDesc), _u32p]),
    "pf_add_no_self_contacts": (C.c_int, [_P, Range]),
    "pf_voxelize_mesh": (C.c_int, [C.POINTER(Mesh), C.c_double, C.c_uint32, C.POINTER(Voxels)]),
    "pf_voxelize_sdf": (C.c_int, [_f32p, _u32p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double, C.c_double,
                                  C.c_uint32, C.POINTER(Voxels)]),
    "pf_bake_sdf": (C.c_int, [C.POINTER(Mesh), C.c_uint32, C.c_double, _f32p, C.POINTER(C.c_double),
                              C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "pf_contacts_read": (C.c_int, [_P, _u32p, C.c_uint32, _u32p, _u32p]),
    "pf_cloth_get_params": (C.c_int, [_P, C.c_uint32, C.POINTER(ClothParams)]),
    "pf_cloth_set_params": (C.c_int, [_P, C.c_uint32, C.POINTER(ClothParams)]),
    "pf_cloth_build_tethers": (C.c_int, [C.POINTER(TetherBuildDesc), _u32p, _u32p, _f32p, C.c_uint32, _u32p]),
    "pf_add_primitive": (C.c_int, [_P, C.POINTER(Primitive), _u32p]),
    "pf_set_primitive": (C.c_int, [_P, C.c_uint32, C.POINTER(Primitive)]),
    "pf_loop_build": (C.c_int, [_P, C.POINTER(LoopDesc)]),
    "pf_step": (C.c_int, [_P, C.c_double]),
    "pf_readback": (C.c_int, [_P, C.c_uint32, _P, C.c_size_t]),
    "pf_overflow_read": (C.c_int, [_P, C.POINTER(Overflow)]),
    "pf_last_step_ms": (C.c_int, [_P, _f32p]),
    "pf_batch_create": (C.c_int, [C.POINTER(_P), C.c_uint32, C.POINTER(BatchOpts), C.POINTER(_P)]),
    "pf_add_sdf_collider": (C.c_int, [_P, C.POINTER(SdfDesc), _u32p]),
    "pf_set_sdf_transform": (C.c_int, [_P, C.c_uint32, _f32p, _f32p, C.c_float]),
    "pf_batch_tuning": (C.c_int, [_P, _u32p, _u32p, _u32p, _u32p, _u32p]),
    "pf_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(_P)]),
    "pf_server_destroy": (None, [_P]),
    "pf_server_submit": (C.c_int, [_P, _P, C.POINTER(LoopDesc), C.c_uint32, C.POINTER(C.c_uint64)]),
    "pf_server_tick": (C.c_int, [_P, C.c_double]),
    "pf_server_drain_build": (C.c_int, [_P]),
    "pf_server_request_state": (C.c_int, [_P, C.c_uint64, _u32p, _u32p]),
    "pf_server_readback": (C.c_int, [_P, C.c_uint64, C.c_uint32, _P, C.c_size_t]),
    "pf_server_estimate_bytes": (C.c_int, [_P, C.POINTER(LoopDesc), C.POINTER(C.c_uint64)]),
    "pf_server_stats_read": (C.c_int, [_P, C.POINTER(ServerStats)]),
    "pf_batch_destroy": (None, [_P]),
    "pf_batch_step": (C.c_int, [_P, C.c_double]),
    "pf_batch_set_primitive": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(Primitive)]),
    "pf_batch_cloth_set_params": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.POINTER(ClothParams)]),
    "pf_batch_write": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_void_p, C.c_size_t]),
    "pf_write": (C.c_int, [_P, C.c_uint32, C.c_void_p, C.c_size_t]),
    "pf_batch_readback": (C.c_int, [_P, C.c_uint32, C.c_uint32, _P, C.c_size_t]),
    "pf_batch_overflow_read": (C.c_int, [_P, C.c_uint32, C.POINTER(Overflow)]),
    "pf_batch_last_step_ms": (C.c_int, [_P, _f32p]),
    "pf_batch_particle_substeps": (C.c_uint64, [_P]),
    "pf_batch_stream": (_P, [_P]),
    "pf_batch_launches_per_step": (C.c_uint64, [_P]),
    "pf_batch_step_upload_bytes": (C.c_uint64, [_P]),
    "pf_scene_stream": (_P, [_P]),
    "pf_batch_read_positions": (C.c_int, [_P, _f32p, C.c_size_t]),
    "pf_batch_read_positions_async": (C.c_int, [_P, _f32p, C.c_size_t]),
    "pf_batch_wait_reads": (C.c_int, [_P]),
    "pf_batch_profile_stage": (C.c_int, [_P, C.c_uint32, C.c_uint32, _f32p, C.POINTER(C.c_uint64)]),
}

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Load libpfsim.so once and bind the signatures that it exports."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"pfsim: {LIB_PATH} is missing. Build the CUDA extension first "
            "(python threejs-particle-fluids_b200/build_native.py)."
        )
    handle = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


def check(status: int) -> None:
    if status != PF_OK:
        msg = lib().pf_last_error().decode("utf-8", "replace")
        raise PfError(status, msg or f"pfsim: status {status}")


def ptr(a: np.ndarray | None, ctype=C.c_float):
    """ctypes pointer to a C-contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to libpfsim must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))
