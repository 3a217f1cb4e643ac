// Motion product of render_products: per-pixel screen-space motion of the
// first sample's primary hit between the previous products frame and this
// one (_motion_product, ordinarylight/targets/vulkan/api.py:1151-1200, with
// the projection of _project_positions, api.py:1118-1136).
//
// The reference keeps the previous frame's meshes on the host and
// re-interpolates the hit triangle there.  Here the previous frame is a
// device snapshot of every triangle's world-space vertices in packed order
// (the windowed reference keeps the same thing on the device as its
// previous vertex buffer, targets/vulkan/core.py:4783-4792), and one kernel
// maps each pixel's packed primitive to the same mesh's triangle in that
// snapshot, interpolates it with the hit's barycentrics, and projects both
// points in double precision.
#include "olc_internal.h"
#include "olc_motion.h"

namespace olc {

namespace {

// Segment of a scene's triangle slots: an instance's BLAS slots (packed
// index = prim_offset + mesh-local index) or the baked world-space slots
// (packed index stored in tri_index, prim_offset = ~0).
OLC_D uint32_t segment_of(const uint32_t* prefix, uint32_t n, uint32_t g) {
  uint32_t lo = 0, hi = n - 1u;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1u) >> 1;
    if (prefix[mid] <= g) lo = mid; else hi = mid - 1u;
  }
  return lo;
}

__global__ void k_world_triangles(SceneView s, const MotionSegment* __restrict__ segs,
                                  const uint32_t* __restrict__ prefix, uint32_t num_segs, uint32_t total,
                                  uint32_t num_packed, float4* out) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const MotionSegment sg = segs[segment_of(prefix, num_segs, g)];
    const uint32_t slot = sg.slot_begin + (g - sg.first);
    const float4* tv = s.tri_verts + 3ull * slot;
    uint32_t packed;
    float3 v[3];
    if (sg.prim_offset == 0xffffffffu) {
      packed = s.tri_index[slot];
      for (int k = 0; k < 3; ++k) v[k] = f3(tv[k]);
    } else {
      packed = sg.prim_offset + s.tri_index[slot];
      const InstanceRec& ir = s.instances[sg.instance];
      const Affine o2w{ir.o2w0, ir.o2w1, ir.o2w2};
      for (int k = 0; k < 3; ++k) v[k] = xform_point(o2w, f3(tv[k]));
    }
    if (packed >= num_packed) continue;
    for (int k = 0; k < 3; ++k) out[3ull * packed + k] = make_float4(v[k].x, v[k].y, v[k].z, 0.0f);
  }
}

struct Projected {
  double x, y;
  bool valid;
};

// _project_positions (api.py:1118-1136) for one point.
OLC_D Projected project(const MotionCamera& c, double px, double py, double pz, double width, double height) {
  const double rx = px - c.origin[0], ry = py - c.origin[1], rz = pz - c.origin[2];
  const double distance = rx * c.forward[0] + ry * c.forward[1] + rz * c.forward[2];
  const double safe = fmax(distance, 1e-12);
  const double ndc_x = (rx * c.right[0] + ry * c.right[1] + rz * c.right[2]) / (safe * c.scale * (width / height));
  const double ndc_y = -(rx * c.up[0] + ry * c.up[1] + rz * c.up[2]) / (safe * c.scale);
  return Projected{(ndc_x + 1.0) * 0.5 * width, (ndc_y + 1.0) * 0.5 * height, distance > 1e-8};
}

__global__ void k_motion(const uint32_t* __restrict__ prim, const float4* __restrict__ position,
                         const float2* __restrict__ bary, uint32_t width, uint32_t height,
                         const MotionMesh* __restrict__ meshes, uint32_t num_meshes,
                         const float4* __restrict__ previous, MotionCamera now, MotionCamera before, float2* out) {
  const uint32_t npix = width * height;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    float2 m = make_float2(0.0f, 0.0f);
    const uint32_t t = prim[p];
    if (t != 0xffffffffu && num_meshes > 0u) {
      // the visible mesh holding packed triangle t (meshes sorted by first)
      uint32_t lo = 0, hi = num_meshes - 1u;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (meshes[mid].first <= t) lo = mid; else hi = mid - 1u;
      }
      const MotionMesh mm = meshes[lo];
      if (t >= mm.first && t - mm.first < mm.count && mm.previous_first != 0xffffffffu) {
        const uint64_t old = (uint64_t)mm.previous_first + (t - mm.first);
        const float4 a = previous[3 * old + 0], b = previous[3 * old + 1], c = previous[3 * old + 2];
        const float2 uv = bary[p];
        const double w0 = (double)(1.0f - uv.x - uv.y), w1 = (double)uv.x, w2 = (double)uv.y;
        const double ox = w0 * a.x + w1 * b.x + w2 * c.x;
        const double oy = w0 * a.y + w1 * b.y + w2 * c.y;
        const double oz = w0 * a.z + w1 * b.z + w2 * c.z;
        const float4 q = position[p];
        const Projected cur = project(now, q.x, q.y, q.z, width, height);
        const Projected prev = project(before, ox, oy, oz, width, height);
        if (cur.valid && prev.valid) m = make_float2((float)(cur.x - prev.x), (float)(cur.y - prev.y));
      }
    }
    out[p] = m;
  }
}

}  // namespace

void world_triangles(const SceneView& s, const MotionSegment* segs, const uint32_t* prefix, uint32_t num_segs,
                     uint32_t total, uint32_t num_packed, float4* out, cudaStream_t stream) {
  if (total == 0 || num_segs == 0) return;
  const uint32_t blocks = std::min<uint32_t>((total + 255u) / 256u, 148u * 16u);
  k_world_triangles<<<blocks, 256, 0, stream>>>(s, segs, prefix, num_segs, total, num_packed, out);
  OLC_LAUNCH_CHECK("k_world_triangles");
}

void motion_vectors(const uint32_t* prim, const float4* position, const float2* bary, uint32_t width,
                    uint32_t height, const MotionMesh* meshes, uint32_t num_meshes, const float4* previous,
                    const MotionCamera& now, const MotionCamera& before, float2* out, cudaStream_t stream) {
  const uint32_t npix = width * height;
  if (npix == 0) return;
  const uint32_t blocks = std::min<uint32_t>((npix + 255u) / 256u, 148u * 16u);
  k_motion<<<blocks, 256, 0, stream>>>(prim, position, bary, width, height, meshes, num_meshes, previous, now,
                                       before, out);
  OLC_LAUNCH_CHECK("k_motion");
}

}  // namespace olc
