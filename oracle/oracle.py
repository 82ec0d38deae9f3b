"""ctypes loader of the CPU oracle (libpf_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module. It restates the reference algorithm (see pf_oracle.cpp's header for
the reference files each function follows) and is never part of the product.
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpf_oracle.so"


def build() -> Path:
    """Compile the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _bind(_lib)
    return _lib


def _bind(L: C.CDLL) -> None:
    import sys

    sys.path.insert(0, str(HERE.parent / "threejs-particle-fluids_b200"))
    from pfsim import _native as N  # struct layouts only

    P = C.c_void_p
    u32p = C.POINTER(C.c_uint32)
    f32p = C.POINTER(C.c_float)
    sig = {
        "or_last_error": (C.c_char_p, []),
        "or_part1by2": (C.c_uint32, [C.c_uint32]),
        "or_morton": (C.c_uint32, [C.c_int32, C.c_int32, C.c_int32]),
        "or_set_threads": (None, [C.c_int]),
        "or_max_threads": (C.c_int, []),
        "or_hardware_threads": (C.c_int, []),
        "or_grid_cells": (C.c_uint64, [C.POINTER(N.GridDesc)]),
        "or_sort": (C.c_int, [f32p, C.c_uint32, C.POINTER(N.GridDesc), u32p, u32p, u32p, u32p, u32p]),
        "or_walk": (C.c_int, [f32p, C.POINTER(N.GridDesc), u32p, u32p, u32p, u32p, C.c_uint32, u32p]),
        "or_polar": (None, [f32p, f32p]),
        "or_polar_f64": (None, [C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "or_color_constraints": (C.c_uint32, [u32p, C.c_uint32, u32p]),
        "or_scene_create": (P, [C.POINTER(N.SceneDesc), C.c_int]),
        "or_scene_destroy": (None, [P]),
        "or_upload_particles": (C.c_int, [P, f32p, f32p, f32p, u32p, C.c_uint32, C.c_uint32]),
        "or_set_inv_mass": (C.c_int, [P, N.Range, C.c_float]),
        "or_add_fluid": (C.c_int, [P, C.POINTER(N.FluidDesc), u32p]),
        "or_add_softbodies": (C.c_int, [P, C.POINTER(N.SoftbodyDesc), u32p]),
        "or_add_cloth": (C.c_int, [P, C.POINTER(N.ClothDesc), u32p]),
        "or_add_primitive": (C.c_int, [P, C.POINTER(N.Primitive), u32p]),
        "or_add_sdf_collider": (C.c_int, [P, C.POINTER(N.SdfDesc), u32p]),
        "or_set_sdf_transform": (C.c_int, [P, C.c_uint32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float]),
        "or_sdf_sample": (C.c_int, [C.POINTER(N.SdfDesc), C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
        "or_set_primitive": (C.c_int, [P, C.c_uint32, C.POINTER(N.Primitive)]),
        "or_cloth_set_params": (C.c_int, [P, C.c_uint32, C.POINTER(N.ClothParams)]),
        "or_write": (C.c_int, [P, C.c_uint32, f32p, C.c_size_t]),
        "or_voxelize_mesh": (C.c_int, [C.POINTER(N.Mesh), C.c_double, C.c_uint32, C.POINTER(N.Voxels)]),
        "or_voxelize_sdf": (C.c_int, [f32p, u32p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                      C.c_double, C.c_uint32, C.POINTER(N.Voxels)]),
        "or_bake_sdf": (C.c_int, [C.POINTER(N.Mesh), C.c_uint32, C.c_double, f32p, C.POINTER(C.c_double),
                                  C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
        "or_add_no_self_contacts": (C.c_int, [P, N.Range]),
        "or_contacts_read": (C.c_int, [P, u32p, C.c_uint32, u32p, u32p]),
        "or_loop_build": (C.c_int, [P, C.POINTER(N.LoopDesc), C.c_uint32]),
        "or_step": (C.c_int, [P, C.c_double]),
        "or_readback": (C.c_int, [P, C.c_uint32, P, C.c_size_t, C.c_int]),
        "or_overflow_read": (C.c_int, [P, C.POINTER(N.Overflow)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


class OracleError(RuntimeError):
    pass


def check(rc: int) -> None:
    if rc != 0:
        raise OracleError(lib().or_last_error().decode())


def _p(a, t=C.c_float):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def sort(positions: np.ndarray, desc) -> dict:
    """Stable counting sort on the CPU (the oracle of pf_sort)."""
    L = lib()
    pos = np.ascontiguousarray(positions, dtype=np.float32)
    n = pos.shape[0]
    cells = int(L.or_grid_cells(C.byref(desc)))
    out = {
        "keys": np.empty(n, np.uint32),
        "perm": np.empty(n, np.uint32),
        "start": np.empty(cells, np.uint32),
        "count": np.empty(cells, np.uint32),
        "overflow": np.zeros(1, np.uint32),
    }
    check(
        L.or_sort(
            _p(pos), n, C.byref(desc), _p(out["keys"], C.c_uint32), _p(out["perm"], C.c_uint32),
            _p(out["start"], C.c_uint32), _p(out["count"], C.c_uint32), _p(out["overflow"], C.c_uint32),
        )
    )
    return out


def walk(query: np.ndarray, desc, perm, start, count, cap: int = 1 << 20) -> np.ndarray:
    """Candidates of the 27-cell walk around one point (query.ts order)."""
    L = lib()
    q = np.ascontiguousarray(query, dtype=np.float32)
    out = np.empty(cap, np.uint32)
    n = C.c_uint32(0)
    check(
        L.or_walk(_p(q), C.byref(desc), _p(perm, C.c_uint32), _p(start, C.c_uint32),
                  _p(count, C.c_uint32), _p(out, C.c_uint32), cap, C.byref(n))
    )
    return out[: min(n.value, cap)].copy()


def polar(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(9)
    r = np.empty(9, np.float32)
    lib().or_polar(_p(a), _p(r))
    return r.reshape(3, 3)


def polar_f64(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    r = np.empty(9, np.float64)
    lib().or_polar_f64(_p(a, C.c_double), _p(r, C.c_double))
    return r.reshape(3, 3)


def sdf_sample(sdf, points: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """phi and world gradient of an SDF collider (pfsim.recipe.Sdf) at points."""
    from pfsim import recipe as R

    keep = R._Keep()
    d = sdf.cstruct(keep)
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    phi = np.empty(len(pts), np.float32)
    grad = np.empty((len(pts), 3), np.float32)
    check(lib().or_sdf_sample(C.byref(d), _p(pts), len(pts), _p(phi), _p(grad)))
    return phi, grad


def color_constraints(pairs: np.ndarray) -> tuple[np.ndarray, int]:
    p = np.ascontiguousarray(pairs, dtype=np.uint32).reshape(-1)
    n = p.size // 2
    g = np.empty(n, np.uint32)
    k = lib().or_color_constraints(_p(p, C.c_uint32), n, _p(g, C.c_uint32))
    return g, int(k)


def voxelize_mesh(vertices, indices, particle_radius: float, largest_piece: bool = False):
    """voxelize(mesh) on the CPU: (positions (n, 3) float32, surface count,
    edges (m, 2) uint32)."""
    from pfsim import mesh as M

    return M.run_voxelize(lambda m, v: lib().or_voxelize_mesh(C.byref(m), float(particle_radius),
                                                              1 if largest_piece else 0, C.byref(v)),
                          vertices, indices)


def voxelize_sdf(data, res, origin, voxel_size, particle_radius: float, dilation: float = 0.0,
                 largest_piece: bool = False):
    from pfsim import mesh as M

    d = np.ascontiguousarray(data, np.float32)
    r = np.ascontiguousarray(res, np.uint32)
    o = np.ascontiguousarray(origin, np.float64)
    vs = np.ascontiguousarray(voxel_size, np.float64)
    return M.run_voxelize(lambda m, v: lib().or_voxelize_sdf(_p(d), _p(r, C.c_uint32), _p(o, C.c_double),
                                                             _p(vs, C.c_double), float(particle_radius),
                                                             float(dilation), 1 if largest_piece else 0,
                                                             C.byref(v)), None, None)


def bake_sdf(vertices, indices, resolution: int, padding: float | None = None):
    """bakeMeshToSdf on the CPU: (data (res, res, res) float32 z-major,
    origin, voxel size, inconsistent voxels)."""
    from pfsim import mesh as M

    m, keep = M.mesh_struct(vertices, indices)
    out = np.empty(resolution ** 3, np.float32)
    org = np.zeros(3, np.float64)
    vs = C.c_double(0)
    bad = C.c_uint64(0)
    check(lib().or_bake_sdf(C.byref(m), resolution, -1.0 if padding is None else float(padding), _p(out),
                            _p(org, C.c_double), C.byref(vs), C.byref(bad)))
    return out.reshape(resolution, resolution, resolution), org, vs.value, bad.value


class _RefHeap:
    """tetherBuild.ts:226-275: binary min-heap ordered on the distance alone,
    strict comparisons in both sifts (equal distances keep heap order)."""

    def __init__(self):
        self.d = []

    def push(self, item):
        d = self.d
        d.append(item)
        i = len(d) - 1
        while i > 0:
            p = (i - 1) >> 1
            if d[i][0] < d[p][0]:
                d[i], d[p] = d[p], d[i]
                i = p
            else:
                break

    def pop(self):
        d = self.d
        top = d[0]
        last = d.pop()
        if d:
            d[0] = last
            i, n = 0, len(d)
            while True:
                l, r, m = 2 * i + 1, 2 * i + 2, i
                if l < n and d[l][0] < d[m][0]:
                    m = l
                if r < n and d[r][0] < d[m][0]:
                    m = r
                if m == i:
                    break
                d[i], d[m] = d[m], d[i]
                i = m
        return top


def build_tethers(inv_mass, pairs, rest_lengths, max_attachments: int = 4, stretch_tolerance: float = 0.0):
    """buildTethers (tetherBuild.ts:84-219) in pure Python for small graphs:
    pinned islands over pinned-only edges, one multi-source Dijkstra per
    island over the rest-length-weighted edges, the nearest max_attachments
    islands of each free particle. Returns (particle, anchor, rest radius
    as float32) arrays, particle-major."""
    inv = np.asarray(inv_mass, np.float32)
    n = inv.size
    pr = np.asarray(pairs, np.int64).reshape(-1, 2)
    rl = [float(x) for x in np.asarray(rest_lengths, np.float64)]
    pinned = [bool(inv[i] == 0) for i in range(n)]
    empty = (np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float32))
    if not any(pinned):
        return empty
    adj = [[] for _ in range(n)]
    for e, (a, b) in enumerate(pr.tolist()):
        adj[a].append((b, rl[e]))
        adj[b].append((a, rl[e]))
    island = [-1] * n
    n_isl = 0
    for s0 in range(n):
        if not pinned[s0] or island[s0] != -1:
            continue
        ident = n_isl
        n_isl += 1
        stack = [s0]
        island[s0] = ident
        while stack:
            u = stack.pop()
            for t, _ in adj[u]:
                if pinned[t] and island[t] == -1:
                    island[t] = ident
                    stack.append(t)
    per = [[] for _ in range(n)]
    inf = float("inf")
    for ident in range(n_isl):
        dist = [inf] * n
        near = [-1] * n
        heap = _RefHeap()
        for i in range(n):
            if pinned[i] and island[i] == ident:
                dist[i] = 0.0
                near[i] = i
                heap.push((0.0, i))
        while heap.d:
            du, u = heap.pop()
            if du > dist[u]:
                continue
            for t, w in adj[u]:
                nd = du + w
                if nd < dist[t]:
                    dist[t] = nd
                    near[t] = near[u]
                    heap.push((nd, t))
        for v in range(n):
            if not pinned[v] and dist[v] != inf:
                per[v].append((dist[v], ident, near[v]))
    scale = 1.0 + float(stretch_tolerance)
    part, anch, rad = [], [], []
    for v in range(n):
        if pinned[v] or not per[v]:
            continue
        lst = sorted(per[v], key=lambda a: (a[0], a[1]))
        for dv, _, an in lst[:max_attachments]:
            part.append(v)
            anch.append(an)
            rad.append(dv * scale)
    return np.asarray(part, np.uint32), np.asarray(anch, np.uint32), np.asarray(rad, np.float32)


# ----------------------------------------------------------- scene backend ----
class OracleScene:
    """A recipe replayed on the CPU oracle; same methods as pfsim's Scene."""

    def __init__(self, handle, recipe, precision: int):
        self.h = handle
        self.recipe = recipe
        self.capacity = recipe.capacity
        self.precision = precision
        self.steps = 0

    def step(self, dt: float) -> None:
        L = lib()
        if self.recipe.motion is not None:
            for slot, prim in self.recipe.motion(self.steps, dt).items():
                p = prim.cstruct()
                check(L.or_set_primitive(self.h, slot, C.byref(p)))
        check(L.or_step(self.h, float(dt)))
        self.steps += 1

    def set_primitive(self, slot, prim) -> None:
        p = prim.cstruct()
        check(lib().or_set_primitive(self.h, slot, C.byref(p)))

    def set_cloth_params(self, material: int, params) -> None:
        """params: a pfsim._native.ClothParams (ClothSystem setters)."""
        check(lib().or_cloth_set_params(self.h, material, C.byref(params)))

    def contacts(self) -> tuple:
        """(pairs found in the last substep, the stored pairs (m, 2), each
        ascending, sorted)."""
        cap = max(1, 32 * self.capacity)
        out = np.empty(2 * cap, np.uint32)
        count, stored = C.c_uint32(0), C.c_uint32(0)
        check(lib().or_contacts_read(self.h, _p(out, C.c_uint32), cap, C.byref(count), C.byref(stored)))
        m = min(stored.value, cap)
        return int(count.value), out[: 2 * m].reshape(-1, 2).copy()

    def write(self, field_id: int, data: np.ndarray) -> None:
        a = np.ascontiguousarray(data, np.float32)
        check(lib().or_write(self.h, field_id, _p(a), a.nbytes))

    def readback(self, field_id: int, as_f64: bool = False) -> "np.ndarray":
        from pfsim import recipe as R

        out = R.alloc_field(field_id, self.capacity)
        if as_f64 and out.dtype == np.float32:
            out = out.astype(np.float64)
        check(lib().or_readback(self.h, field_id, out.ctypes.data_as(C.c_void_p), out.nbytes, 1 if as_f64 else 0))
        return out

    def overflow(self) -> dict:
        from pfsim import _native as N

        o = N.Overflow()
        check(lib().or_overflow_read(self.h, C.byref(o)))
        return {k: bool(getattr(o, k)) for k, _ in N.Overflow._fields_}

    def close(self) -> None:
        if self.h:
            lib().or_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleBackend:
    """Replays pfsim recipes on the oracle (FP32, or FP64 with precision=64)."""

    def __init__(self, precision: int = 32, threads: int = 1, table_size: int = 0):
        self.precision = precision
        self.threads = threads
        self.table_size = table_size
        self.name = f"oracle-f{precision}"

    def build(self, r) -> OracleScene:
        from pfsim import _native as N
        from pfsim import recipe as R

        L = lib()
        set_threads(self.threads)
        desc = N.SceneDesc(r.capacity, r.radius)
        h = L.or_scene_create(C.byref(desc), self.precision)
        if not h:
            raise OracleError(L.or_last_error().decode())
        scene = OracleScene(h, r, self.precision)
        keep = R._Keep()
        for u in r.uploads:
            p = R.pos4(u.pos)
            v = None if u.vel is None else keep.f32(R.pos4(u.vel))
            w = None if u.inv_mass is None else keep.f32(u.inv_mass)
            g = None if u.group is None else keep.u32(np.asarray(u.group, np.uint32))
            check(L.or_upload_particles(h, keep.f32(p), v, w, g, u.start, p.shape[0]))
        for kind, opts in r.materials:
            if kind == "fluid":
                check(L.or_add_fluid(h, C.byref(R.fluid_desc(opts, keep)), None))
            elif kind == "soft":
                check(L.or_add_softbodies(h, C.byref(R.softbody_desc(opts, keep)), None))
            elif kind == "cloth":
                check(L.or_add_cloth(h, C.byref(R.cloth_desc(opts, keep)), None))
        for q in r.quiet:
            check(L.or_add_no_self_contacts(h, N.Range(*q)))
        for p in r.prims:
            cs = p.cstruct()
            check(L.or_add_primitive(h, C.byref(cs), None))
        for g in r.sdfs:
            check(L.or_add_sdf_collider(h, C.byref(g.cstruct(keep)), None))
        ld = R.loop_desc(r.loop)
        check(L.or_loop_build(h, C.byref(ld), self.table_size))
        return scene
