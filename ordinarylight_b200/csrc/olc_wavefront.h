// Launch interface of the wavefront stages and the camera model shared by
// the raygen kernels.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

#include "olc_common.cuh"

namespace olc {

// Camera ray of (pixel, sample) following ReferencePathTracer._camera_rays
// (ordinarylight/renderers/reference/path_tracer.py:110-151):
//   ndc = ((x, y) + jitter) / (w, h) * 2 - 1 with y flipped;
//   perspective: d = forward + ndc_x*(aspect*tan(fov/2))*right + ndc_y*tan(fov/2)*up;
//   orthographic: o = position + ndc_x*(aspect*half)*right + ndc_y*half*up, d = forward;
//   panoramic: yaw/pitch = ndc * half angles.
// The jitter is the counter-based draw of (pixel, sample, frame) unless an
// override is given.
OLC_D void camera_ray(const JobRec& job, uint32_t pixel, uint32_t sample, const float2* jit, float3& o, float3& d) {
  uint32_t y = pixel / job.width;
  uint32_t x = pixel - y * job.width;
  float2 j = jit ? *jit : olc_camera_jitter(pixel, sample, job.frame);
  float ndc_x = ((float)x + j.x) / (float)job.width * 2.0f - 1.0f;
  float ndc_y = 1.0f - ((float)y + j.y) / (float)job.height * 2.0f;
  float3 pos = f3(job.cam_pos), fwd = f3(job.cam_forward), right = f3(job.cam_right), up = f3(job.cam_up);
  float sx = job.cam_pos.w, sy = job.cam_forward.w;
  if (job.projection == 2u) {
    float yaw = ndc_x * sx, pitch = ndc_y * sy;
    float cp = cosf(pitch), sp = sinf(pitch), cy = cosf(yaw), sy2 = sinf(yaw);
    d = fwd * (cp * cy) + right * (cp * sy2) + up * sp;
    o = pos;
  } else if (job.projection == 1u) {
    o = pos + right * (ndc_x * sx) + up * (ndc_y * sy);
    d = fwd;
  } else {
    d = fwd + right * (ndc_x * sx) + up * (ndc_y * sy);
    o = pos;
  }
  d = normalize(d);
}

struct LaunchShape {
  uint32_t block = 256;        // simple grid-stride kernels
  uint32_t trace_block = 128;  // traversal and shading kernels (64, 128 or 256)
  uint32_t grid_simple = 148 * 8;
  uint32_t grid_trace = 148 * 8;
  uint32_t grid_shade = 148 * 8;
  uint32_t stack_depth = 24;
  uint32_t scheduler = 0;      // traversal scheduling (olc_config.trace_scheduler)
  uint32_t sort_rays = 0;      // reorder extension rays before tracing them
};

// First-sample primary-hit products of the job flagged `products` (a plain
// frame), indexed by pixel.
struct ProductPtrs {
  float* depth = nullptr;
  float4* normal = nullptr;
  uint32_t* instance_id = nullptr;
  uint32_t* material_id = nullptr;
  uint32_t* primitive_id = nullptr;
  float4* position = nullptr;      // world hit point (xyz)
  float2* barycentric = nullptr;   // (u, v) of the hit in the triangle's index order
  float4* signals = nullptr;       // specular-lobe probability, opaque (1) or transmissive (0) hit
  float4* secondary = nullptr;     // hit point of the path's next vertex (xyz), recorded (w = 1)
};

void configure_trace_kernels();
// Grid of a grid-stride kernel: the blocks of `block` threads (and `smem`
// bytes of dynamic shared memory) that all SMs of the current device hold at
// once, at most `max_grid`.  A grid-stride loop over a fixed share of the
// items per block then runs in one wave; a larger grid leaves a partial
// second wave whose blocks start only as the first ones finish.
uint32_t resident_grid(const void* fn, uint32_t block, size_t smem, uint32_t max_grid);
// Where camera-ray traversal lists the chunk's primary hits of ReSTIR jobs
// (path slots, in completion order; `count` zeroed before the launch), or
// list == nullptr for no list.
struct HitListOut {
  const JobRec* jobs = nullptr;
  const uint4* meta = nullptr;   // path records (job index in .w)
  uint32_t* list = nullptr;
  uint32_t* count = nullptr;
};
// The chunk whose camera paths bounce-0 traversal starts: its header (path
// count, segments), job segments, scene records and path records.
struct CameraPaths {
  const ChunkHeader* hdr = nullptr;
  const JobRec* jobs = nullptr;
  const SceneRec* scenes = nullptr;
  PathState ps{};
};
// Closest-hit traversal of a bounce's queue; with `cam` (bounce 0) the
// kernel generates the chunk's camera rays into the queue and initialises
// the path records itself.
void launch_trace_closest(const LaunchShape& ls, const SceneView& s, const RayQueue& q, const HitBuf& h,
                          Counters* cnt, uint32_t bounce, const HitListOut& hl, const CameraPaths* cam,
                          cudaStream_t stream);
void launch_trace_shadow(const LaunchShape& ls, const SceneView& s, const ShadowQueue& sq, const PathState& ps,
                         Counters* cnt, uint32_t bounce, cudaStream_t stream);
// fresh: every path of the queue is at its camera vertex with the initial
// state that camera-ray generation wrote (bounce 0 without the reference
// volume pass), so shading does not read it back.
void launch_shade(const LaunchShape& ls, const JobRec* jobs, const SceneView& s, const RayQueue& qin,
                  const HitBuf& hits, const RayQueue& qout, const ShadowQueue& sq, const PathState& ps,
                  Counters* cnt, uint32_t bounce, uint32_t capacity, const ProductPtrs& prod, const uint4* restir,
                  bool textures, bool media, bool fresh, cudaStream_t stream);
// Reorder the bounce's ray queue `in` into `out` by origin cell and direction
// bin (keys: one word per queue slot; bins: sort_bins_bytes() of scratch).
void launch_sort_rays(const LaunchShape& ls, const SceneView& s, const RayQueue& in, const RayQueue& out,
                      Counters* cnt, uint32_t bounce, uint32_t* keys, uint32_t* bins, cudaStream_t stream);
size_t sort_bins_bytes();
void launch_ref_volumes(const LaunchShape& ls, const JobRec* jobs, const SceneView& s, const RayQueue& q,
                        const HitBuf& hits, const PathState& ps, const Counters* cnt, uint32_t bounce,
                        cudaStream_t stream);
void launch_accumulate(const LaunchShape& ls, const ChunkHeader* hdr, const JobRec* jobs, const PathState& ps,
                       unsigned long long* accum, float* sample_lum, Counters* cnt, cudaStream_t stream);
// Per-pixel luminance variance of npix pixels from spp sample planes.
void launch_sample_variance(const LaunchShape& ls, const float* sample_lum, uint32_t npix, uint32_t spp, float* out,
                            cudaStream_t stream);
void launch_resolve(const LaunchShape& ls, const ResolveEntry* entries, const uint32_t* num_entries,
                    const unsigned long long* accum, float4* out, cudaStream_t stream);
void launch_sample_textures(const LaunchShape& ls, const SceneRec* scenes, uint32_t scene, float binding, uint32_t n,
                            const float2* uv0, const float2* uv1, const float* fp0, const float* fp1, int srgb,
                            float4* out, cudaStream_t stream);
void launch_camera_rays(const LaunchShape& ls, const JobRec* job, uint32_t sample, const float* jitter,
                        float* origins, float* dirs, cudaStream_t stream);
void launch_trace_rays(const LaunchShape& ls, const SceneView& s, uint32_t root, uint32_t n, const float* origins,
                       const float* dirs, float t_min, uint32_t* inst_id, int32_t* prim, float* t, float* bary,
                       Counters* cnt, cudaStream_t stream);
void launch_occluded_rays(const LaunchShape& ls, const SceneView& s, uint32_t root, uint32_t n, const float* origins,
                          const float* dirs, float t_min, const float* t_max, uint8_t* occ, Counters* cnt,
                          cudaStream_t stream);

}  // namespace olc
