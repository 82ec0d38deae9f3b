"""The reference-named host API (pfsim.api) drives the same CUDA path: a
scene built through ParticleSystem / FluidSystem / PrimitiveSet / SimLoop is
bit-identical to the same scene built from a recipe, and the Simulation
façade steps a container with a fluid, a soft body and a cloth."""

import numpy as np
import pytest

from pfsim import _native as N
from pfsim import api as A
from pfsim import recipe as R
from pfsim import workloads as W

pytestmark = pytest.mark.gpu
DT = 1.0 / 60.0


def test_low_level_api_equals_recipe():
    r = W.dam_break(4000, seed=21)
    fo = r.materials[0][1]
    ps = A.ParticleSystem(r.capacity, r.radius)
    ps.upload_particles(r.uploads[0].pos)
    fluid = A.FluidSystem(ps, range=fo.range, rest_density=fo.rest_density, particle_spacing=fo.particle_spacing,
                          smoothing_radius=fo.smoothing_radius, compliance=fo.compliance, viscosity=fo.viscosity)
    prims = A.PrimitiveSet(ps)
    for p in r.prims:
        prims.prims.append(p)
    loop = A.SimLoop(ps, substeps=r.loop.substeps, iterations=r.loop.iterations, gravity=r.loop.gravity,
                     materials=[fluid], colliders=[prims], grid_min=r.loop.grid_min, grid_max=r.loop.grid_max)
    ref = R.NativeBackend().build(r)
    for _ in range(3):
        loop.step(DT)
        ref.step(DT)
    snap = ps.readback()
    np.testing.assert_array_equal(snap.positions, ref.readback(N.PF_FIELD_POSITIONS))
    np.testing.assert_array_equal(snap.velocities, ref.readback(N.PF_FIELD_VELOCITIES))
    loop.dispose()
    with pytest.raises(N.PfError, match="SimLoop: has been disposed"):
        loop.step(DT)


def test_simulation_facade_steps():
    sim = A.Simulation(container=((-0.5, 0.0, -0.3), (0.5, 0.8, 0.3)), particles=8000)
    sim.add_fluid(box=((-0.5, 0.0, -0.3), (-0.1, 0.4, 0.3)))
    sim.add_softbody("sphere", center=(0.25, 0.3, 0.0), size=0.1, softness=0.3)
    sim.add_cloth(0.4, 0.3, position=(0.2, 0.6, 0.0))
    for _ in range(10):
        sim.step(DT)
    snap = sim.readback()
    x = snap.positions[:, :3]
    assert np.isfinite(x).all()
    assert (x[:, 1] > -0.05).all() and (np.abs(x[:, 0]) < 0.55).all()
    with pytest.raises(N.PfError, match="addFluid"):
        sim.add_fluid(box=((0, 0, 0), (0.1, 0.1, 0.1)))
    sim.dispose()


def test_facade_validation():
    with pytest.raises(N.PfError, match="exactly one of"):
        A.Simulation(particles=100, particle_radius=0.01)
    with pytest.raises(N.PfError, match="substeps"):
        A.SimLoop(A.ParticleSystem(4, 0.01), substeps=0)
