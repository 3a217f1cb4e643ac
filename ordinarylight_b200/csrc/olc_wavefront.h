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
OLC_D void camera_ray(const FrameParams& fp, uint32_t pixel, uint32_t sample, const float2* jit, float3& o,
                      float3& d) {
  uint32_t y = pixel / fp.width;
  uint32_t x = pixel - y * fp.width;
  float2 j = jit ? *jit : olc_camera_jitter(pixel, sample, fp.frame);
  float ndc_x = ((float)x + j.x) / (float)fp.width * 2.0f - 1.0f;
  float ndc_y = 1.0f - ((float)y + j.y) / (float)fp.height * 2.0f;
  float3 pos = f3(fp.cam_pos), fwd = f3(fp.cam_forward), right = f3(fp.cam_right), up = f3(fp.cam_up);
  float sx = fp.cam_pos.w, sy = fp.cam_forward.w;
  if (fp.projection == 2u) {
    float yaw = ndc_x * sx, pitch = ndc_y * sy;
    float cp = cosf(pitch), sp = sinf(pitch), cy = cosf(yaw), sy2 = sinf(yaw);
    d = fwd * (cp * cy) + right * (cp * sy2) + up * sp;
    o = pos;
  } else if (fp.projection == 1u) {
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
  uint32_t grid_simple = 148 * 8;
  uint32_t grid_trace = 148 * 8;
  uint32_t grid_shade = 148 * 8;
  uint32_t stack_depth = 24;
  uint32_t scheduler = 0;      // traversal scheduling (olc_config.trace_scheduler)
};

struct ProductPtrs {
  float* depth = nullptr;
  float4* normal = nullptr;
  uint32_t* instance_id = nullptr;
  uint32_t* material_id = nullptr;
  uint32_t* primitive_id = nullptr;
};

void configure_trace_kernels();
void launch_raygen(const LaunchShape& ls, const FrameParams* fp, uint64_t chunk_begin, uint32_t chunk_count,
                   const RayQueue& q, const PathState& ps, Counters* cnt, float t_min, cudaStream_t stream);
void launch_trace_closest(const LaunchShape& ls, const SceneView& s, const RayQueue& q, const HitBuf& h,
                          Counters* cnt, uint32_t bounce, cudaStream_t stream);
void launch_trace_shadow(const LaunchShape& ls, const SceneView& s, const ShadowQueue& sq, const PathState& ps,
                         Counters* cnt, uint32_t bounce, cudaStream_t stream);
void launch_shade(const LaunchShape& ls, uint32_t mode, const FrameParams* fp, const SceneView& s,
                  const RayQueue& qin, const HitBuf& hits, const RayQueue& qout, const ShadowQueue& sq,
                  const PathState& ps, Counters* cnt, uint32_t bounce, uint32_t capacity, const ProductPtrs& prod,
                  const uint4* restir, cudaStream_t stream);
void launch_accumulate(const LaunchShape& ls, const PathState& ps, uint32_t chunk_count, unsigned long long* accum,
                       Counters* cnt, cudaStream_t stream);
void launch_resolve(const LaunchShape& ls, const unsigned long long* accum, uint32_t npix, uint32_t spp,
                    float4* out, cudaStream_t stream);
void launch_camera_rays(const LaunchShape& ls, const FrameParams* fp, uint32_t sample, const float* jitter,
                        float* origins, float* dirs, cudaStream_t stream);
void launch_trace_rays(const LaunchShape& ls, const SceneView& s, uint32_t n, const float* origins, const float* dirs,
                       float t_min, uint32_t* inst_id, int32_t* prim, float* t, float* bary, Counters* cnt,
                       cudaStream_t stream);
void launch_occluded_rays(const LaunchShape& ls, const SceneView& s, uint32_t n, const float* origins,
                          const float* dirs, float t_min, const float* t_max, uint8_t* occ, Counters* cnt,
                          cudaStream_t stream);

}  // namespace olc
