"""The C ABI library loads and exports every symbol include/pfsim.h declares.

CPU only: no compute call is made (there is no GPU here).
"""

import ctypes as C
import re

import numpy as np
from pathlib import Path

from pfsim import _native as N

HEADER = Path(__file__).resolve().parent.parent / "include" / "pfsim.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^PF_API\s+[\w\s\*]+?\b(pf_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for must in ("pf_sort", "pf_sort_host", "pf_grid_cells", "pf_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libpfsim.so lacks {missing}"


def test_abi_version_and_error_text():
    lib = N.lib()
    assert lib.pf_abi_version() == 3
    # An invalid descriptor is rejected on the host before any device work.
    d = N.GridDesc()
    d.key_kind = N.PF_KEY_MORTON
    d.cell_size = 0.1
    d.table_size = 3
    assert lib.pf_grid_cells(C.byref(d)) == 0


def test_server_admission_estimate_is_host_only():
    """pf_server_estimate_bytes plans a scene's world on the host (no GPU):
    the estimate grows with the particle count and holds at least the
    double-buffered per-particle state."""
    from pfsim import recipe as R
    from pfsim import workloads as W

    small = R.Server.estimate_bytes(W.dam_break(4000, seed=1))
    big = R.Server.estimate_bytes(W.dam_break(16000, seed=1))
    n_small = W.dam_break(4000, seed=1).capacity
    assert small > 2 * 56 * n_small
    assert 2.5 < big / small < 5.5


def test_unbuilt_scene_is_refused_without_loop_options():
    from pfsim import recipe as R
    from pfsim import workloads as W

    scene = R.NativeBackend().build(W.dam_break(2000, seed=1), build_loop=False)
    out = C.c_uint64(0)
    rc = N.lib().pf_server_estimate_bytes(scene.h, None, C.byref(out))
    assert rc == N.PF_ERR_STATE
    assert b"SimLoop" in N.lib().pf_last_error()


def test_api_validation_is_host_side():
    """The reference's constructor checks run before any device work."""
    import pytest

    from pfsim import api as A

    with pytest.raises(N.PfError, match="Simulation: give exactly one"):
        A.Simulation(particles=100, particle_radius=0.01)
    with pytest.raises(N.PfError, match="ParticleSystem: capacity"):
        A.ParticleSystem(0, 0.01)
    with pytest.raises(N.PfError, match="SoftbodySystem: shapeMatching"):
        A.SoftbodySystem(A.ParticleSystem(4, 0.01), [], shape_matching="x")
    with pytest.raises(N.PfError, match="SDFCollider: resolution"):
        A.SDFCollider(A.ParticleSystem(4, 0.01), np.zeros((2, 4, 4)), (0, 0, 0), (1, 1, 1))


def test_sort_buffers_are_checked_before_device_work():
    """pf_sort and pf_sort_noalloc refuse missing and misaligned device
    buffers with an error (positions are read as float4, so they must be
    16-byte aligned) before they touch the device. The pointers here are
    never dereferenced."""
    import pytest

    from pfsim import hashgrid as H
    from pfsim import workloads as W

    L = N.lib()
    g = H.GridOptions(cell_size=W.SORT_CELL, kind="linear", dims=(8, 8, 8))
    n = 100
    d = g.desc(n)
    p = lambda a: C.c_void_p(a)  # noqa: E731
    for entry in (L.pf_sort, L.pf_sort_noalloc):
        with pytest.raises(N.PfError, match="16-byte aligned"):
            N.check(entry(p(0x10004), n, C.byref(d), p(0x20000), p(0x30000), p(0x40000), None, None, None))
        with pytest.raises(N.PfError, match="4-byte aligned"):
            N.check(entry(p(0x10000), n, C.byref(d), p(0x20002), p(0x30000), p(0x40000), None, None, None))
        with pytest.raises(N.PfError, match="NULL start or count"):
            N.check(entry(p(0x10000), n, C.byref(d), p(0x20000), None, p(0x40000), None, None, None))
