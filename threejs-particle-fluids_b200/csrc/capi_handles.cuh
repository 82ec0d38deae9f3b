// capi_handles.cuh — the opaque handles of the C ABI (pfsim.h) as the
// library's translation units see them.
#pragma once

#include <memory>
#include <vector>

#include "world.cuh"

// A ParticleSystem with its materials, primitives and (once built) SimLoop.
struct pf_scene {
  pf::SceneSpec spec;
  std::unique_ptr<pf::World> world;
};

// Scenes stepped together as one world.
struct pf_batch {
  std::vector<std::unique_ptr<pf::SceneSpec>> specs;
  std::unique_ptr<pf::World> world;
};

namespace pf {
// Host copy of a scene's state fields (positions, velocities, inverse mass,
// boundary volume, rotation, angular velocity) in the layout of pf_readback.
pf_status spec_readback(const SceneSpec& spec, uint32_t field, void* dst, size_t bytes);
// Collision groups handed out when a scene's SimLoop is built (loop.ts:163-166,
// SoftbodySystem.ts:218-234).
pf_status allocate_collision_groups(SceneSpec& spec);
}  // namespace pf
