"""Mesh -> particle setup on the GPU (src/softbody/voxelize.ts, src/sdf/bake.ts).

``voxelize_mesh`` / ``voxelize_sdf`` fill a closed mesh or a distance field
with particles on a cubic grid of spacing 2r (surface particles first, plus
the face-adjacent pairs a soft body's cluster graph uses); ``bake_sdf`` bakes
a mesh into the signed-distance grid an SDFCollider takes. The grid-point
against triangle work runs on the GPU through libpfsim.
"""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _native as N


@dataclass
class Voxels:
    """VoxelizeResult (voxelize.ts:23-36)."""

    positions: np.ndarray  # (count, 3) float32, surface particles first
    surface_count: int
    edges: np.ndarray  # (m, 2) uint32, i < j

    @property
    def count(self) -> int:
        return int(self.positions.shape[0])


def mesh_struct(vertices, indices):
    """A pf_mesh over float32 vertices and uint32 indices; returns the struct
    and the arrays it points into (keep them alive while it is used)."""
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1)
    if v.size % 3:
        raise N.PfError(N.PF_ERR_INVALID, f"TriangleMesh: vertices length {v.size} is not a multiple of 3")
    i = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    m = N.Mesh(v.ctypes.data_as(C.POINTER(C.c_float)), v.size // 3, i.ctypes.data_as(C.POINTER(C.c_uint32)), i.size)
    return m, (v, i)


def run_voxelize(call, vertices, indices) -> Voxels:
    """Two calls of a voxeliser entry point: the first sizes, the second fills."""
    keep = None
    m = None
    if vertices is not None:
        m, keep = mesh_struct(vertices, indices)
    out = N.Voxels()
    _check(call(m, out))
    pos = np.empty((max(out.count, 1), 3), np.float32)
    edges = np.empty((max(out.edge_count, 1), 2), np.uint32)
    out.positions = pos.ctypes.data_as(C.POINTER(C.c_float))
    out.capacity = out.count
    out.edges = edges.ctypes.data_as(C.POINTER(C.c_uint32))
    out.edge_capacity = out.edge_count
    _check(call(m, out))
    del keep
    return Voxels(pos[: out.count].copy(), int(out.surface_count), edges[: out.edge_count].copy())


def _check(rc) -> None:
    # oracle entry points return plain ints; library ones pf_status
    if rc:
        N.check(rc)


def voxelize_mesh(vertices, indices, particle_radius: float, largest_piece: bool = False) -> Voxels:
    """voxelize(mesh, {particleRadius, largestPiece}) (voxelize.ts:50-161)."""
    L = N.lib()
    return run_voxelize(lambda m, v: L.pf_voxelize_mesh(C.byref(m), float(particle_radius),
                                                        1 if largest_piece else 0, C.byref(v)), vertices, indices)


def voxelize_sdf(data, res, origin, voxel_size, particle_radius: float, dilation: float = 0.0,
                 largest_piece: bool = False) -> Voxels:
    """voxelize(SDFData, {particleRadius, dilation, largestPiece})."""
    L = N.lib()
    d = np.ascontiguousarray(data, np.float32).reshape(-1)
    r = np.ascontiguousarray(res, np.uint32)
    o = np.ascontiguousarray(origin, np.float64)
    vs = np.ascontiguousarray(voxel_size, np.float64)
    return run_voxelize(lambda m, v: L.pf_voxelize_sdf(d.ctypes.data_as(C.POINTER(C.c_float)),
                                                       r.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                       o.ctypes.data_as(C.POINTER(C.c_double)),
                                                       vs.ctypes.data_as(C.POINTER(C.c_double)), float(particle_radius),
                                                       float(dilation), 1 if largest_piece else 0, C.byref(v)),
                        None, None)


def bake_sdf(vertices, indices, resolution: int, padding: float | None = None):
    """bakeMeshToSdf(mesh, {resolution, padding}) (bake.ts:84-139): returns
    (data (res, res, res) float32 indexed [z, y, x], origin (3,), voxel size,
    voxels whose axis votes split)."""
    m, keep = mesh_struct(vertices, indices)
    out = np.empty(int(resolution) ** 3, np.float32)
    org = np.zeros(3, np.float64)
    vs = C.c_double(0)
    bad = C.c_uint64(0)
    N.check(N.lib().pf_bake_sdf(C.byref(m), int(resolution), -1.0 if padding is None else float(padding),
                                out.ctypes.data_as(C.POINTER(C.c_float)), org.ctypes.data_as(C.POINTER(C.c_double)),
                                C.byref(vs), C.byref(bad)))
    del keep
    return out.reshape(resolution, resolution, resolution), org, vs.value, bad.value


# ------------------------------------------------------- procedural meshes ----
def box_mesh(half=(0.5, 0.5, 0.5)):
    """A closed box of 8 corners and 12 outward triangles (half extents
    `half`), the unit cube of softbody-voxelize.test.ts:20-62 by default."""
    hx, hy, hz = half
    v = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [-hx, hy, -hz], [hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [-hx, hy, hz], [hx, hy, hz]], np.float32)
    i = np.array([0, 2, 1, 1, 2, 3, 4, 5, 6, 5, 7, 6, 0, 1, 4, 1, 5, 4, 2, 6, 3, 3, 6, 7, 0, 4, 2, 2, 4, 6,
                  1, 3, 5, 3, 7, 5], np.uint32)
    return v, i


def uv_sphere(radius: float, stacks: int, slices: int):
    """A closed UV sphere (the layout of the reference's test mesh,
    tests/_helpers/sdf-test-meshes.ts:23-87): poles
    at +-radius, stacks - 1 rings of `slices` vertices, fans at the poles and
    two triangles per quad; float32 vertices."""
    n = 2 + (stacks - 1) * slices
    pos = np.zeros((n, 3), np.float64)
    pos[0] = (0, radius, 0)
    pos[n - 1] = (0, -radius, 0)
    for s in range(1, stacks):
        phi = math.pi * s / stacks
        y, rr = math.cos(phi) * radius, math.sin(phi) * radius
        for k in range(slices):
            th = 2 * math.pi * k / slices
            pos[1 + (s - 1) * slices + k] = (math.cos(th) * rr, y, math.sin(th) * rr)
    ring = lambda s: 1 + (s - 1) * slices
    idx = []
    for k in range(slices):
        idx += [0, ring(1) + k, ring(1) + (k + 1) % slices]
    for s in range(1, stacks - 1):
        for k in range(slices):
            kn = (k + 1) % slices
            a, b, c, d = ring(s) + k, ring(s) + kn, ring(s + 1) + k, ring(s + 1) + kn
            idx += [a, c, d, a, d, b]
    last = ring(stacks - 1)
    for k in range(slices):
        idx += [last + k, n - 1, last + (k + 1) % slices]
    return pos.astype(np.float32), np.array(idx, np.uint32)


def torus(ring_radius: float, tube_radius: float, ring_segs: int, tube_segs: int):
    """A closed torus (the layout of sdf-test-meshes.ts:102-141), float32
    vertices."""
    pos = np.zeros((ring_segs * tube_segs, 3), np.float64)
    for i in range(ring_segs):
        u = 2 * math.pi * i / ring_segs
        for j in range(tube_segs):
            v = 2 * math.pi * j / tube_segs
            r = ring_radius + tube_radius * math.cos(v)
            pos[i * tube_segs + j] = (r * math.cos(u), tube_radius * math.sin(v), r * math.sin(u))
    idx = []
    for i in range(ring_segs):
        inx = (i + 1) % ring_segs
        for j in range(tube_segs):
            jn = (j + 1) % tube_segs
            a, b, c, d = i * tube_segs + j, i * tube_segs + jn, inx * tube_segs + j, inx * tube_segs + jn
            idx += [a, c, d, a, d, b]
    return pos.astype(np.float32), np.array(idx, np.uint32)
