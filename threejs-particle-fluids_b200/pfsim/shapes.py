"""Host-side scene construction: voxelised solids and cloth graphs.

``voxelize_shape`` follows the reference's voxelize (src/softbody/voxelize.ts:
50-146) for analytic shapes: lattice cells of size 2r over the shape's box,
a cell is occupied when its centre is inside, surface cells (fewer than six
occupied face neighbours) come first, and edges join neighbouring occupied
cells. The reference joins face neighbours only; ``neighborhood=26`` joins
all 26 neighbours, which makes each particle's shape-matching group a
3x3x3 cluster of 27.

``plane_geometry`` + ``create_cloth_graph`` follow three.js' PlaneGeometry
index layout and the reference's createClothGraph (src/cloth/graph.ts:130-342):
unique triangle edges in first-seen order as distance constraints (structural
edges plus one shear diagonal per quad), lumped vertex masses from a third of
each incident triangle's area, pinned vertices at zero inverse mass, and a
bending tuple with its signed rest angle for every edge two triangles share.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Voxelized:
    positions: np.ndarray  # (count, 3) float32
    count: int
    surface_count: int
    edges: np.ndarray  # (m, 2) uint32, i < j


def voxelize_shape(inside, lo, hi, particle_radius: float, neighborhood: int = 6) -> Voxelized:
    spacing = 2.0 * particle_radius
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    nx, ny, nz = [max(1, int(np.ceil((hi[a] - lo[a]) / spacing))) for a in range(3)]
    cells = np.arange(nx * ny * nz)
    cx, cy, cz = cells % nx, (cells // nx) % ny, cells // (nx * ny)
    centers = np.stack([lo[0] + particle_radius + spacing * cx, lo[1] + particle_radius + spacing * cy,
                        lo[2] + particle_radius + spacing * cz], -1)
    occ = np.asarray(inside(centers), bool).reshape(nz, ny, nx)
    pad = np.zeros((nz + 2, ny + 2, nx + 2), bool)
    pad[1:-1, 1:-1, 1:-1] = occ

    def shifted(dx, dy, dz):
        return pad[1 + dz: 1 + dz + nz, 1 + dy: 1 + dy + ny, 1 + dx: 1 + dx + nx]

    face = [(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    nface = sum(shifted(*d).astype(np.int32) for d in face)
    occ_f = occ.ravel()
    surf = np.nonzero(occ_f & (nface.ravel() < 6))[0]
    inner = np.nonzero(occ_f & (nface.ravel() >= 6))[0]
    ordered = np.concatenate([surf, inner])
    index = np.full(nx * ny * nz, -1, np.int64)
    index[ordered] = np.arange(ordered.size)
    offs = face if neighborhood == 6 else [(a, b, c) for c in (-1, 0, 1) for b in (-1, 0, 1) for a in (-1, 0, 1)
                                           if (a, b, c) != (0, 0, 0)]
    # edges in the reference's order: by particle, then by neighbour offset
    ocx, ocy, ocz = cx[ordered], cy[ordered], cz[ordered]
    ii, jj, kk = [], [], []
    for o, (dx, dy, dz) in enumerate(offs):
        x, y, z = ocx + dx, ocy + dy, ocz + dz
        ok = (x >= 0) & (x < nx) & (y >= 0) & (y < ny) & (z >= 0) & (z < nz)
        j = np.full(ordered.size, -1, np.int64)
        j[ok] = index[(x + nx * (y + ny * z))[ok]]
        i = np.arange(ordered.size)
        keep = (j > i)
        ii.append(i[keep]); jj.append(j[keep]); kk.append(np.full(keep.sum(), o))
    i = np.concatenate(ii); j = np.concatenate(jj); k = np.concatenate(kk)
    order = np.lexsort((k, i))
    edges = np.stack([i[order], j[order]], -1).astype(np.uint32)
    pos = centers[ordered].astype(np.float32)
    return Voxelized(pos, int(ordered.size), int(surf.size), edges)


def voxel_sphere(center, radius: float, particle_radius: float, neighborhood: int = 6) -> Voxelized:
    c = np.asarray(center, np.float64)
    return voxelize_shape(lambda p: ((p - c) ** 2).sum(-1) < radius * radius, c - radius, c + radius,
                          particle_radius, neighborhood)


def voxel_box(center, half, particle_radius: float, neighborhood: int = 6) -> Voxelized:
    c = np.asarray(center, np.float64)
    h = np.asarray(half, np.float64)
    return voxelize_shape(lambda p: (np.abs(p - c) <= h).all(-1), c - h, c + h, particle_radius, neighborhood)


# ------------------------------------------------------------------ cloth ----
def plane_geometry(width: float, height: float, seg_w: int, seg_h: int):
    """three.js PlaneGeometry: vertices row by row from the top (y = +h/2),
    two triangles (a, b, d), (b, c, d) per quad."""
    gx, gy = seg_w + 1, seg_h + 1
    sw, sh = width / seg_w, height / seg_h
    iy, ix = np.meshgrid(np.arange(gy), np.arange(gx), indexing="ij")
    pos = np.stack([ix * sw - width / 2, -(iy * sh - height / 2), np.zeros_like(ix, float)], -1).reshape(-1, 3)
    idx = []
    for y in range(seg_h):
        for x in range(seg_w):
            a = x + gx * y
            b = x + gx * (y + 1)
            c = (x + 1) + gx * (y + 1)
            d = (x + 1) + gx * y
            idx += [a, b, d, b, c, d]
    return pos, np.array(idx, np.int64)


@dataclass
class ClothGraph:
    positions: np.ndarray  # (n, 3) float64
    inv_mass: np.ndarray  # (n,)
    pairs: np.ndarray  # (m, 2)
    rest_lengths: np.ndarray  # (m,)
    bending: np.ndarray  # (b, 4): (p1, p2, p3, p4) per edge shared by two triangles
    bending_rest: np.ndarray  # (b,) signed rest dihedral angles
    triangles: np.ndarray  # (t, 3) non-degenerate triangles in index order


def dihedral_angles(pos: np.ndarray, tuples: np.ndarray) -> np.ndarray:
    """graph.ts:346-402: the signed dihedral angle of each (p1, p2, p3, p4)
    tuple, atan2((N1 x N2).E, (N1.N2)|E|) with E = p2 - p1,
    N1 = (p3 - p1) x (p3 - p2), N2 = (p4 - p2) x (p4 - p1); 0 for a degenerate
    edge or triangle."""
    p1, p2, p3, p4 = (pos[tuples[:, k]] for k in range(4))
    e = p2 - p1
    el = np.sqrt((e * e).sum(1))
    n1 = np.cross(p3 - p1, p3 - p2)
    n2 = np.cross(p4 - p2, p4 - p1)
    s = (np.cross(n1, n2) * e).sum(1)
    c = (n1 * n2).sum(1) * el
    ang = np.arctan2(s, c)
    bad = (el < 1e-12) | ((n1 * n1).sum(1) < 1e-24) | ((n2 * n2).sum(1) < 1e-24)
    return np.where(bad, 0.0, ang)


def create_cloth_graph(positions, index, surface_density: float = 0.2, pinned=()) -> ClothGraph:
    """graph.ts:130-342 for a mesh without coincident vertices: lumped masses,
    unique edges in first-seen order (a-b, b-c, c-a of each triangle)."""
    pos = np.asarray(positions, np.float64)
    n = pos.shape[0]
    tri = np.asarray(index, np.int64).reshape(-1, 3)
    a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
    ar = 0.5 * np.linalg.norm(np.cross(pos[b] - pos[a], pos[c] - pos[a]), axis=1)
    good = (a != b) & (b != c) & (a != c) & (ar > 0)
    a, b, c, ar = a[good], b[good], c[good], ar[good]
    area = np.zeros(n)
    for v in (a, b, c):
        np.add.at(area, v, ar / 3)
    eu = np.stack([a, b, c], 1).reshape(-1)
    ev = np.stack([b, c, a], 1).reshape(-1)
    key = np.minimum(eu, ev) * n + np.maximum(eu, ev)
    uniq, first = np.unique(key, return_index=True)
    order = np.argsort(first, kind="stable")
    keys = uniq[order]
    pairs = np.stack([keys // n, keys % n], -1).astype(np.uint32)
    inv = np.where(area > 0, 1.0 / np.where(area > 0, area * surface_density, 1.0), 0.0)
    inv[list(pinned)] = 0.0
    rest = np.linalg.norm(pos[pairs[:, 0]] - pos[pairs[:, 1]], axis=1)
    # graph.ts:300-330: every edge with exactly two incident triangles gives a
    # bending tuple (edge endpoints ascending, then the two far vertices in
    # triangle order), in the edges' first-seen order
    far = np.stack([c, a, b], 1).reshape(-1)
    order_e = np.argsort(key, kind="stable")
    sk = key[order_e]
    starts = np.flatnonzero(np.r_[True, sk[1:] != sk[:-1]])
    counts = np.diff(np.r_[starts, sk.size])
    two = counts == 2
    k2 = sk[starts[two]]
    f1 = far[order_e[starts[two]]]
    f2 = far[order_e[starts[two] + 1]]
    ordr = np.argsort(_edge_rank(keys, k2), kind="stable")
    tuples = np.stack([k2 // n, k2 % n, f1, f2], -1)[ordr].astype(np.uint32)
    bending_rest = dihedral_angles(pos, tuples.astype(np.int64))
    triangles = np.stack([a, b, c], -1).astype(np.uint32)
    return ClothGraph(pos, inv, pairs, rest, tuples, bending_rest, triangles)


def _edge_rank(edge_keys_in_order: np.ndarray, query: np.ndarray) -> np.ndarray:
    """Index of each query key in the first-seen edge order."""
    idx = np.argsort(edge_keys_in_order, kind="stable")
    pos = np.searchsorted(edge_keys_in_order[idx], query)
    return idx[pos]


def build_tethers(inv_mass, pairs, rest_lengths, max_attachments: int = 4, stretch_tolerance: float = 0.0):
    """buildTethers (src/cloth/tetherBuild.ts:84-219) in the native library
    (pf_cloth_build_tethers): for every free particle, one long-range
    attachment to the nearest pinned particle of each of its
    `max_attachments` geodesically closest pinned islands. Returns cloth-local
    (particle, anchor) uint32 arrays and float32 rest radii, particle-major."""
    import ctypes as C

    from . import _native as N

    if not (isinstance(max_attachments, int) and max_attachments > 0):
        raise N.PfError(N.PF_ERR_INVALID,
                        f"buildTethers: maxAttachmentsPerParticle must be a positive integer, got {max_attachments}")
    inv = np.ascontiguousarray(inv_mass, np.float32)
    pr = np.ascontiguousarray(pairs, np.uint32).reshape(-1)
    rl = np.ascontiguousarray(rest_lengths, np.float64)
    n = inv.size
    d = N.TetherBuildDesc()
    d.n_particles = n
    d.inv_mass = inv.ctypes.data_as(C.POINTER(C.c_float))
    d.n_pairs = pr.size // 2
    d.pairs = pr.ctypes.data_as(C.POINTER(C.c_uint32))
    d.rest_lengths = rl.ctypes.data_as(C.POINTER(C.c_double))
    d.max_attachments = max_attachments
    d.stretch_tolerance = float(stretch_tolerance)
    cap = max(1, n * max_attachments)
    part = np.empty(cap, np.uint32)
    anch = np.empty(cap, np.uint32)
    rest = np.empty(cap, np.float32)
    cnt = C.c_uint32(0)
    N.check(N.lib().pf_cloth_build_tethers(C.byref(d), part.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           anch.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           rest.ctypes.data_as(C.POINTER(C.c_float)), cap, C.byref(cnt)))
    k = cnt.value
    return part[:k].copy(), anch[:k].copy(), rest[:k].copy()
