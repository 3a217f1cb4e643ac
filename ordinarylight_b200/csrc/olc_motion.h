// Motion product kernels (olc_motion.cu).
#pragma once

#include "olc_internal.h"

namespace olc {

// A run of a scene's triangle slots for the world-space snapshot.
struct MotionSegment {
  uint32_t first;        // first snapshot thread of the segment
  uint32_t slot_begin;   // global slot of its first triangle
  uint32_t instance;     // global instance record (BLAS slots)
  uint32_t prim_offset;  // packed index base; ~0 for baked world-space slots
};

// A visible mesh of the current frame: its packed triangle range and where
// the same mesh's triangles start in the previous snapshot (~0: no motion).
struct MotionMesh {
  uint32_t first, count, previous_first, pad;
};

// _project_positions' camera frame in double precision.
struct MotionCamera {
  double origin[3], forward[3], right[3], up[3];
  double scale;   // tan(vertical fov / 2)
};

// World-space vertices of every packed triangle of one scene:
// out[3 * packed + k], num_packed triangles.
void world_triangles(const SceneView& s, const MotionSegment* segs, const uint32_t* prefix, uint32_t num_segs,
                     uint32_t total, uint32_t num_packed, float4* out, cudaStream_t stream);

void motion_vectors(const uint32_t* prim, const float4* position, const float2* bary, uint32_t width,
                    uint32_t height, const MotionMesh* meshes, uint32_t num_meshes, const float4* previous,
                    const MotionCamera& now, const MotionCamera& before, float2* out, cudaStream_t stream);

}  // namespace olc
