// ReSTIR DI at the primary vertex: resampled importance sampling over the
// emissive triangles, temporal reuse of the previous frame's reservoir and
// spatial reuse of neighbouring pixels' reservoirs.
//
// Reservoir algebra follows the reference's CPU oracle
// (DirectLightReservoir, ordinarylight/integrations/restir_di.py:29-162):
//   update:  M += m; w_sum += w; select if u * w_sum < w
//   merge:   w = p_hat_here(y) * w_sum_src / p_hat_src(y), represented M_src
//   W = w_sum / (M * p_hat(y))
// and the flow of the reference's fused primary kernel
// (wavefront_primary_impl.glsl:1547-1687): initial candidates, temporal
// merge, spatial merge, final visibility (here: the bounce-0 shadow ray).
// Target p_hat = luminance(f * Le * G) without visibility.
//
// Storage: two uint4 words per reservoir,
//   w0 = (light index, barycentrics as half2, w_sum, M)
//   w1 = (p_hat of the selected sample, primary depth, octahedral normal, valid)
// indexed by sample stream * npix + pixel, so a stream's history survives
// chunking and batching.
#include <cuda_fp16.h>

#include "olc_restir.h"
#include "olc_shading.cuh"

namespace olc {

namespace {

constexpr uint32_t kRestirStream = 0x52455354u;  // stream key offset of the reuse passes

OLC_D uint32_t oct_encode(float3 n) {
  float s = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
  float x = n.x / s, y = n.y / s;
  if (n.z < 0.0f) {
    float ox = (1.0f - fabsf(y)) * (x >= 0.0f ? 1.0f : -1.0f);
    float oy = (1.0f - fabsf(x)) * (y >= 0.0f ? 1.0f : -1.0f);
    x = ox;
    y = oy;
  }
  uint32_t ux = (uint32_t)__float2int_rn(clampf(x, -1.0f, 1.0f) * 32767.0f) & 0xffffu;
  uint32_t uy = (uint32_t)__float2int_rn(clampf(y, -1.0f, 1.0f) * 32767.0f) & 0xffffu;
  return ux | (uy << 16);
}
OLC_D float3 oct_decode(uint32_t v) {
  float x = (float)(int16_t)(v & 0xffffu) / 32767.0f;
  float y = (float)(int16_t)(v >> 16) / 32767.0f;
  float z = 1.0f - fabsf(x) - fabsf(y);
  if (z < 0.0f) {
    float ox = (1.0f - fabsf(y)) * (x >= 0.0f ? 1.0f : -1.0f);
    float oy = (1.0f - fabsf(x)) * (y >= 0.0f ? 1.0f : -1.0f);
    x = ox;
    y = oy;
  }
  return normalize(f3(x, y, z));
}

struct Surface {
  float3 p, n, view;
  SurfaceMat m;
  float depth;
  bool valid;
};

struct Res {
  uint32_t light;
  uint32_t bary;
  float w_sum;
  uint32_t M;
  float target;
};

OLC_D float2 unpack_bary(uint32_t b) {
  return __half22float2(*reinterpret_cast<const __half2*>(&b));
}
OLC_D uint32_t pack_bary(float b1, float b2) {
  __half2 h = __floats2half2_rn(b1, b2);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Unshadowed target of light sample (light, bary) at surface s.
OLC_D float target_of(const SceneView& sc, const Surface& s, uint32_t light, uint32_t bary) {
  const EmitterRec e = sc.emitters[light];
  float2 b = unpack_bary(bary);
  float3 lp = f3(e.a) * fmaxf(1.0f - b.x - b.y, 0.0f) + f3(e.b) * b.x + f3(e.c) * b.y;
  float3 off = lp - s.p;
  float d2 = dot(off, off);
  if (!(d2 > 1e-12f)) return 0.0f;
  float dist = sqrtf(d2);
  float3 l = off / dist;
  float cs = dot(s.n, l);
  if (cs <= 0.0f) return 0.0f;
  float cl = emitter_cosine(e, l);
  if (cl <= 1e-6f) return 0.0f;
  float3 f = pbr_eval(s.m, s.n, s.view, l);
  float t = luminance(f * f3(e.emission_area)) * cs * cl / d2;
  return (t == t && t < 3.0e38f) ? fmaxf(t, 0.0f) : 0.0f;
}

OLC_D bool res_update(Res& r, uint32_t light, uint32_t bary, float target, float w, uint32_t m, float u) {
  r.M += m;
  r.w_sum += w;
  bool sel = w > 0.0f && (r.light == 0xffffffffu || u * r.w_sum < w);
  if (sel) {
    r.light = light;
    r.bary = bary;
    r.target = target;
  }
  return sel;
}

OLC_D Surface primary_surface(const SceneView& s, const RayQueue& q, const HitBuf& h, uint32_t i) {
  Surface su;
  su.valid = false;
  float4 hit = h.tuv_slot[i];
  if (hit.x < 0.0f) return su;
  float4 dt = q.dir_tmax[i];
  float4 ot = q.origin_tmin[i];
  const float3 d = f3(dt);
  const uint32_t slot = __float_as_uint(hit.w);
  const InstanceRec& ir = s.instances[h.instance[i]];
  Affine o2w{ir.o2w0, ir.o2w1, ir.o2w2};
  Affine w2o{ir.w2o0, ir.w2o1, ir.w2o2};
  const float4* tv = s.tri_verts + 3u * slot;
  float3 v0 = xform_point(o2w, f3(tv[0])), v1 = xform_point(o2w, f3(tv[1])), v2 = xform_point(o2w, f3(tv[2]));
  float3 ng = normalize(cross(v1 - v0, v2 - v0));
  const float4* tn = s.tri_normals + 3u * slot;
  float w0 = 1.0f - hit.y - hit.z;
  float3 nobj = f3(tn[0]) * w0 + f3(tn[1]) * hit.y + f3(tn[2]) * hit.z;
  float3 ns = normalize(xform_normal_by_inverse(w2o, nobj));
  if (!(dot(ns, ns) > 0.5f)) ns = ng;
  if (dot(ns, ng) < 0.0f) ns = -ns;
  const bool entering = dot(d, ng) < 0.0f;
  su.n = entering ? ns : -ns;
  su.p = f3(ot) + d * hit.x;
  su.view = -d;
  su.m = load_material(s, ir.material);
  su.depth = hit.x;
  su.valid = true;
  return su;
}

OLC_D bool similar(const Surface& s, uint32_t w1_normal, float depth) {
  float3 n = oct_decode(w1_normal);
  if (dot(n, s.n) < 0.9f) return false;
  return fabsf(depth - s.depth) <= 0.1f * s.depth;
}

OLC_D void store_res(uint4* w0, uint4* w1, uint64_t g, const Res& r, const Surface& s) {
  w0[g] = make_uint4(r.light, r.bary, __float_as_uint(r.w_sum), r.M);
  w1[g] = make_uint4(__float_as_uint(r.target), __float_as_uint(s.valid ? s.depth : -1.0f),
                     s.valid ? oct_encode(s.n) : 0u, s.valid ? 1u : 0u);
}

OLC_D Res load_res(const uint4* w0, const uint4* w1, uint64_t g, float& depth, uint32_t& nrm, bool& valid) {
  uint4 a = w0[g], b = w1[g];
  Res r;
  r.light = a.x;
  r.bary = a.y;
  r.w_sum = __uint_as_float(a.z);
  r.M = a.w;
  r.target = __uint_as_float(b.x);
  depth = __uint_as_float(b.y);
  nrm = b.z;
  valid = b.w != 0u;
  return r;
}

struct RestirArgs {
  const FrameParams* fp;
  SceneView s;
  RayQueue q;
  HitBuf h;
  PathState ps;
  uint64_t chunk_begin;
  uint32_t chunk_count;
  uint32_t npix;
  uint32_t candidates;
  uint32_t use_history;
  uint32_t history_cap;     // M cap of the temporal history
  uint32_t neighbours;
  float radius;
  const uint4* hist0;
  const uint4* hist1;
  const uint4* in0;
  const uint4* in1;
  uint4* out0;
  uint4* out1;
  uint32_t pass;
  uint4* selected;
  uint32_t finalize;
};

__global__ void __launch_bounds__(128) k_restir_initial(RestirArgs a) {
  const FrameParams& fp = *a.fp;
  const SceneView& s = a.s;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.chunk_count; i += gridDim.x * blockDim.x) {
    uint4 meta = a.ps.meta[i];
    const uint64_t g = a.chunk_begin + i;
    Surface su = primary_surface(s, a.q, a.h, i);
    Res r{0xffffffffu, 0u, 0.0f, 0u, 0.0f};
    if (su.valid) {
      uint32_t rng = olc_bounce_state(olc_path_seed(meta.x, meta.y, fp.frame), kRestirStream);
      for (uint32_t c = 0; c < a.candidates; ++c) {
        float sel = olc_rand(rng);
        uint32_t li = select_emitter(s, sel);
        float ru = sqrtf(olc_rand(rng));
        float rv = olc_rand(rng);
        uint32_t bary = pack_bary(ru * (1.0f - rv), ru * rv);
        float t = target_of(s, su, li, bary);
        const EmitterRec& e = s.emitters[li];
        float p_src = e.dist.y / fmaxf(e.emission_area.w, 1e-12f);
        float w = p_src > 0.0f ? t / p_src : 0.0f;
        res_update(r, li, bary, t, w, 1u, olc_rand(rng));
      }
      // temporal reuse
      if (a.use_history) {
        float pd;
        uint32_t pn;
        bool pv;
        Res prev = load_res(a.hist0, a.hist1, g, pd, pn, pv);
        if (pv && prev.light != 0xffffffffu && prev.M > 0u && prev.target > 0.0f && similar(su, pn, pd)) {
          uint32_t m = min(prev.M, a.history_cap);
          float wsum = prev.w_sum * ((float)m / (float)prev.M);
          float t = target_of(s, su, prev.light, prev.bary);
          float w = t * wsum / prev.target;
          res_update(r, prev.light, prev.bary, t, w, m, olc_rand(rng));
        }
      }
    }
    store_res(a.out0, a.out1, g, r, su);
  }
}

__global__ void __launch_bounds__(128) k_restir_spatial(RestirArgs a) {
  const FrameParams& fp = *a.fp;
  const SceneView& s = a.s;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.chunk_count; i += gridDim.x * blockDim.x) {
    uint4 meta = a.ps.meta[i];
    const uint64_t g = a.chunk_begin + i;
    const uint64_t stream_base = g - meta.x;  // stream * npix
    Surface su = primary_surface(s, a.q, a.h, i);
    float d0;
    uint32_t n0;
    bool v0;
    Res r = load_res(a.in0, a.in1, g, d0, n0, v0);
    if (su.valid && a.neighbours > 0u) {
      uint32_t rng = olc_bounce_state(olc_path_seed(meta.x, meta.y, fp.frame), kRestirStream + 1u + a.pass);
      const int px = (int)(meta.x % fp.width), py = (int)(meta.x / fp.width);
      for (uint32_t k = 0; k < a.neighbours; ++k) {
        float rr = a.radius * sqrtf(olc_rand(rng));
        float th = 2.0f * OLC_PI * olc_rand(rng);
        float u = olc_rand(rng);
        int qx = px + __float2int_rn(rr * cosf(th));
        int qy = py + __float2int_rn(rr * sinf(th));
        if (qx < 0 || qy < 0 || qx >= (int)fp.width || qy >= (int)fp.height || (qx == px && qy == py)) continue;
        uint64_t gq = stream_base + (uint64_t)qy * fp.width + (uint64_t)qx;
        float dq;
        uint32_t nq;
        bool vq;
        Res nb = load_res(a.in0, a.in1, gq, dq, nq, vq);
        if (!vq || nb.light == 0xffffffffu || nb.M == 0u || !(nb.target > 0.0f) || !similar(su, nq, dq)) continue;
        float t = target_of(s, su, nb.light, nb.bary);
        float w = t * nb.w_sum / nb.target;
        res_update(r, nb.light, nb.bary, t, w, nb.M, u);
      }
    }
    store_res(a.out0, a.out1, g, r, su);
    if (a.finalize) {
      float W = (r.light != 0xffffffffu && r.M > 0u && r.target > 0.0f) ? r.w_sum / ((float)r.M * r.target) : 0.0f;
      if (!(W == W) || W > 3.0e38f) W = 0.0f;
      a.selected[i] = make_uint4(W > 0.0f ? r.light : 0xffffffffu, r.bary, __float_as_uint(W), 0u);
    }
  }
}

}  // namespace

void restir_prepare(RestirState& st, const olc_config& cfg, uint32_t w, uint32_t h, uint32_t spp,
                    uint32_t frame_index, uint32_t slots, const FrameParams& cam) {
  uint64_t n = (uint64_t)w * h * spp;
  if (n > st.reservoirs) {
    st.res_a0.allocate(n * 16);
    st.res_a1.allocate(n * 16);
    st.res_b0.allocate(n * 16);
    st.res_b1.allocate(n * 16);
    st.hist0.allocate(n * 16);
    st.hist1.allocate(n * 16);
    st.reservoirs = n;
    st.history_valid = false;
  }
  if (slots > st.slots) {
    st.selected.allocate((size_t)slots * 16);
    st.slots = slots;
  }
  auto same = [](const float4& x, const float4& y) {
    return x.x == y.x && x.y == y.y && x.z == y.z && x.w == y.w;
  };
  bool camera_same = same(cam.cam_pos, st.hist_camera.cam_pos) && same(cam.cam_forward, st.hist_camera.cam_forward) &&
                     same(cam.cam_right, st.hist_camera.cam_right) && same(cam.cam_up, st.hist_camera.cam_up) &&
                     cam.projection == st.hist_camera.projection;
  st.history_used = cfg.restir_temporal && st.history_valid && st.hist_w == w && st.hist_h == h &&
                    st.hist_spp == spp && st.hist_frame + 1u == frame_index && camera_same;
  st.cur_w = w;
  st.cur_h = h;
  st.cur_spp = spp;
  st.cur_frame = frame_index;
  st.hist_camera = cam;
}

const uint4* restir_run(RestirState& st, const olc_config& cfg, const LaunchShape& ls, const SceneView& s,
                        const FrameParams* fp, const RayQueue& q, const HitBuf& hits, const PathState& ps,
                        Counters* /*cnt*/, uint64_t chunk_begin, uint32_t chunk_count, uint32_t npix,
                        cudaStream_t stream) {
  RestirArgs a{};
  a.fp = fp;
  a.s = s;
  a.q = q;
  a.h = hits;
  a.ps = ps;
  a.chunk_begin = chunk_begin;
  a.chunk_count = chunk_count;
  a.npix = npix;
  a.candidates = cfg.restir_candidates;
  a.use_history = st.history_used ? 1u : 0u;
  a.history_cap = std::max<uint32_t>(1u, cfg.restir_max_history ? cfg.restir_max_history : 20u) * cfg.restir_candidates;
  a.neighbours = cfg.restir_neighbours;
  a.radius = cfg.restir_radius > 0.0f ? cfg.restir_radius : 30.0f;
  a.hist0 = st.hist0.as<uint4>();
  a.hist1 = st.hist1.as<uint4>();
  a.selected = st.selected.as<uint4>();
  a.out0 = st.res_a0.as<uint4>();
  a.out1 = st.res_a1.as<uint4>();
  uint32_t grid = ls.grid_shade;
  k_restir_initial<<<grid, 128, 0, stream>>>(a);
  OLC_LAUNCH_CHECK("k_restir_initial");
  // spatial passes ping-pong A -> B -> A ...; the last pass finalises.
  uint32_t passes = std::max<uint32_t>(cfg.restir_spatial, 1u);
  bool in_a = true;
  for (uint32_t p = 0; p < passes; ++p) {
    RestirArgs b = a;
    b.pass = p;
    b.neighbours = cfg.restir_spatial ? cfg.restir_neighbours : 0u;
    b.in0 = in_a ? st.res_a0.as<uint4>() : st.res_b0.as<uint4>();
    b.in1 = in_a ? st.res_a1.as<uint4>() : st.res_b1.as<uint4>();
    b.out0 = in_a ? st.res_b0.as<uint4>() : st.res_a0.as<uint4>();
    b.out1 = in_a ? st.res_b1.as<uint4>() : st.res_a1.as<uint4>();
    b.finalize = (p + 1 == passes) ? 1u : 0u;
    k_restir_spatial<<<grid, 128, 0, stream>>>(b);
    OLC_LAUNCH_CHECK("k_restir_spatial");
    in_a = !in_a;
  }
  st.final_in_b = !in_a;  // the final reservoirs are where the last pass wrote
  return st.selected.as<uint4>();
}

void restir_finish(RestirState& st) {
  // the final reservoirs become the next frame's temporal history
  if (st.final_in_b) {
    std::swap(st.hist0, st.res_b0);
    std::swap(st.hist1, st.res_b1);
  } else {
    std::swap(st.hist0, st.res_a0);
    std::swap(st.hist1, st.res_a1);
  }
  st.history_valid = true;
  st.hist_w = st.cur_w;
  st.hist_h = st.cur_h;
  st.hist_spp = st.cur_spp;
  st.hist_frame = st.cur_frame;
}

void restir_reset(RestirState& st) {
  st.history_valid = false;
  st.history_used = false;
}

void restir_release(RestirState& st) {
  st.res_a0.release();
  st.res_a1.release();
  st.res_b0.release();
  st.res_b1.release();
  st.hist0.release();
  st.hist1.release();
  st.selected.release();
  st.reservoirs = 0;
  st.slots = 0;
  st.history_valid = false;
}

}  // namespace olc
