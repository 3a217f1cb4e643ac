// Wavefront path-tracing stages: camera raygen, closest-hit and any-hit
// traversal, shading with NEE and warp-aggregated queue compaction, and the
// fixed-point HDR accumulation.
//
// Stage map against the reference wavefront (ordinarylight/shaders/):
//   start_camera_path wavefront_generate.comp:86-167 (+ path init), run by
//                    bounce-0 k_trace_closest for each ray it takes
//   k_trace_closest  wavefront_intersect.comp:317-356 (software traversal)
//   k_shade          wavefront_shade.comp:262-596
//   k_trace_shadow   nativeOccluded in transport_v1/lighting.glsl
//   k_accumulate     wavefront_resolve.comp:45-54 plus the host float64
//                    accumulation of api.py:1404-1422, moved on device
//   k_resolve        colour = sum / spp, alpha 0 (path_tracer.py:89-95)
// Every kernel serves a wavefront of one or many jobs (JobRec): a path's job
// is in its state, a queued ray carries its scene's TLAS root.  Queue counts
// never leave the device: persistent kernels read them, so the bounce loop
// can be captured once as a CUDA graph.
#include <algorithm>
#include <mutex>
#include <vector>

#include "olc_internal.h"
#include "olc_shading.cuh"
#include "olc_refvolume.cuh"
#include "olc_textures.cuh"
#include "olc_trace.cuh"
#include "olc_volume.cuh"
#include "olc_wavefront.h"

namespace olc {

namespace {

OLC_D uint32_t lane_id() { return threadIdx.x & 31u; }

// Entry k of a path's medium stack (entry 0 is the outside, IOR 1).
OLC_D float medium_ior(const float4* stack, uint32_t path, uint32_t k) {
  if (k == 0u) return 1.0f;
  const float4 v = stack[4ull * path + ((k - 1u) >> 2)];
  const uint32_t c = (k - 1u) & 3u;
  return c == 0u ? v.x : c == 1u ? v.y : c == 2u ? v.z : v.w;
}
OLC_D void set_medium_ior(float4* stack, uint32_t path, uint32_t k, float ior) {
  float* v = reinterpret_cast<float*>(stack + 4ull * path + ((k - 1u) >> 2));
  v[(k - 1u) & 3u] = ior;
}

// GLSL refract(i, n, eta): the transmitted direction for unit i and n, or
// zero on total internal reflection.
OLC_D float3 refract_dir(float3 i, float3 n, float eta) {
  const float ni = dot(n, i);
  const float k = 1.0f - eta * eta * (1.0f - ni * ni);
  if (k < 0.0f) return f3(0.0f, 0.0f, 0.0f);
  return i * eta - n * (eta * ni + sqrtf(k));
}

// Warp-aggregated slot reservation: one atomic per warp for all lanes that
// want a slot (reserveOutputIndex, wavefront_shade.comp:199-213).  Must be
// called by all 32 lanes.
OLC_D uint32_t warp_reserve(uint32_t* counter, bool want) {
  uint32_t ballot = __ballot_sync(0xffffffffu, want);
  if (ballot == 0u) return 0xffffffffu;
  uint32_t leader = __ffs(ballot) - 1u;
  uint32_t base = 0;
  if (lane_id() == leader) base = atomicAdd(counter, __popc(ballot));
  base = __shfl_sync(0xffffffffu, base, leader);
  return want ? base + __popc(ballot & ((1u << lane_id()) - 1u)) : 0xffffffffu;
}

// Segment owning chunk-local path index g (segments are ordered by seg_begin).
OLC_D uint32_t segment_of_path(const JobRec* jobs, uint32_t num_segments, uint64_t g) {
  uint32_t lo = 0, hi = num_segments - 1u;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1u) >> 1;
    if (jobs[mid].seg_begin <= g) lo = mid; else hi = mid - 1u;
  }
  return lo;
}

OLC_D float job_t_min(const JobRec& j) { return j.mode == 1u ? 1e-4f : 0.001f; }

// Pixel of index k (0 <= k < w * h) of a sample stream: 8x4-pixel tiles in
// bands of 4 rows (the band's last w % 8 columns and a last short band in
// row order), so the 32 consecutive camera rays of a warp cover one tile.
// A bijection per stream: each pixel still gets exactly one path per sample.
OLC_D uint32_t stream_pixel(uint32_t k, uint32_t w, uint32_t h) {
  const uint32_t band_pixels = 4u * w;
  const uint32_t band = k / band_pixels;
  const uint32_t y0 = band * 4u;
  uint32_t r = k - band * band_pixels;
  if (h - y0 < 4u) return y0 * w + r;
  const uint32_t full = (w >> 3) * 32u;
  if (r < full) {
    const uint32_t tile = r >> 5, within = r & 31u;
    return (y0 + (within >> 3)) * w + tile * 8u + (within & 7u);
  }
  r -= full;
  const uint32_t rem = w & 7u;
  return (y0 + r / rem) * w + (w - rem) + r % rem;
}

// Camera ray and initial state of chunk path i (the ray generation of
// wavefront_generate.comp:86-167 and the path init): writes the bounce-0
// queue entry and the path record, and returns the ray.  Bounce-0
// closest-hit traversal calls it for each ray it takes, so no separate pass
// writes the queue for the traversal to read back.
OLC_D void start_camera_path(const JobRec* __restrict__ jobs, uint32_t num_segments,
                             const SceneRec* __restrict__ scenes, const RayQueue& q, const PathState& ps, uint32_t i,
                             float3& o, float3& d, float& tmin, uint32_t& root) {
  const uint32_t j = segment_of_path(jobs, num_segments, i);
  const JobRec& job = jobs[j];
  const uint64_t local = job.seg_first + (i - job.seg_begin);
  const uint32_t local_sample = (uint32_t)(local / job.npix);
  const uint32_t pixel = stream_pixel((uint32_t)(local - (uint64_t)local_sample * job.npix), job.width, job.height);
  const uint32_t sample = job.sample_base + local_sample;   // the RNG key's sample index
  camera_ray(job, pixel, sample, nullptr, o, d);
  tmin = job_t_min(job);
  root = scenes[job.scene].tlas_root;
  q.origin_tmin[i] = make_float4(o.x, o.y, o.z, tmin);
  q.dir_root[i] = make_float4(d.x, d.y, d.z, __uint_as_float(root));
  q.path[i] = i;
  ps.throughput[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
  ps.radiance[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ps.shadow[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  ps.meta[i] = make_uint4(pixel, sample, 0u, j);
}

// Persistent traversal (Aila and Laine, "Understanding the Efficiency of Ray
// Traversal on GPUs", HPG 2009: persistent threads with dynamic fetch).
// Scheduler 0 (refill): each lane runs its ray for up to 16 loop iterations;
// lanes whose ray finished are refilled from the queue with one
// warp-aggregated atomic once at least 8 of them are idle, so SIMD lanes stay
// busy instead of waiting for the warp's longest ray.  Scheduler 1 (batch): a
// warp takes 32 rays and runs all of them to completion before fetching more.
template <int SCHED>
struct TraceSchedule;
template <>
struct TraceSchedule<0> {
  static constexpr int kSteps = 16;
  static constexpr uint32_t kRefillLanes = 8;
};
template <>
struct TraceSchedule<1> {
  static constexpr int kSteps = 1 << 30;
  static constexpr uint32_t kRefillLanes = 32;
};

template <int STACK, bool ANY_HIT, int SCHED, class Load, class Store>
OLC_D void persistent_trace(const SceneView& s, uint32_t n, uint32_t* cursor, int* smem, Load load, Store store,
                            uint32_t& err) {
  constexpr int kTraceSteps = TraceSchedule<SCHED>::kSteps;
  constexpr uint32_t kRefillLanes = TraceSchedule<SCHED>::kRefillLanes;
  Traversal<STACK, ANY_HIT> tr;
  int spill[OLC_SPILL];
  uint32_t my = 0xffffffffu;
  bool exhausted = false;
  const uint32_t lt = (1u << lane_id()) - 1u;
  // A queue shorter than the grid's warp count is spread one ray per warp,
  // so its rays run in separate warps instead of diverging in a few: the
  // launch then takes about one ray's latency.
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  const uint32_t cap = n < warps ? 1u : 32u;
  while (true) {
    const bool idle = my == 0xffffffffu;
    if (!exhausted) {
      const uint32_t idle_mask = __ballot_sync(0xffffffffu, idle);
      const uint32_t want = __popc(idle_mask);
      const uint32_t busy = 32u - want;
      const uint32_t take = busy >= cap ? 0u : min(want, cap - busy);
      if (take > 0u && (want >= kRefillLanes || idle_mask == 0xffffffffu || cap < 32u)) {
        const uint32_t leader = __ffs(idle_mask) - 1u;
        uint32_t base = 0;
        if (lane_id() == leader) base = atomicAdd(cursor, take);
        base = __shfl_sync(0xffffffffu, base, leader);
        const uint32_t rank = __popc(idle_mask & lt);
        if (idle && rank < take) {
          const uint32_t cand = base + rank;
          if (cand < n) {
            my = cand;
            float3 o, d;
            float tmin, tmax;
            uint32_t root;
            load(my, o, d, tmin, tmax, root);
            tr.begin(s, o, d, tmin, tmax, root, smem, spill);
          }
        }
        if (base + take >= n) exhausted = true;
      }
    }
    if (__ballot_sync(0xffffffffu, my != 0xffffffffu) == 0u) break;
    if (my != 0xffffffffu && tr.advance(s, kTraceSteps, err)) {
      store(my, tr);
      my = 0xffffffffu;
    }
  }
}

// Register cap of the traversal kernels: 64 registers hold the traversal
// state without spilling (the world ray and the hit's barycentrics live in
// shared memory), so eight blocks of 128 threads stay resident per SM.
constexpr int kTraceRegisters = 64;

// kCamera: bounce 0, whose rays the kernel generates itself (the chunk's
// paths in order, `cam` their jobs and path records) and whose primary hits
// of ReSTIR jobs it lists for the resampling passes.
template <int STACK, int SCHED, bool kCamera>
__global__ void __maxnreg__(kTraceRegisters) k_trace_closest(SceneView s, RayQueue q, HitBuf h, Counters* cnt,
                                                              uint32_t bounce, HitListOut hl, CameraPaths cam) {
  extern __shared__ int smem_stack[];
  uint32_t n, num_segments = 0;
  if (kCamera) {
    n = cam.hdr->count;
    num_segments = cam.hdr->num_segments;
    if (blockIdx.x == 0 && threadIdx.x == 0) cnt->queue_count[0] = n;
  } else {
    n = cnt->queue_count[bounce];
  }
  uint32_t err = 0;
  persistent_trace<STACK, false, SCHED>(
      s, n, &cnt->closest_cursor[bounce], smem_stack,
      [&](uint32_t i, float3& o, float3& d, float& tmin, float& tmax, uint32_t& root) {
        tmax = CUDART_INF_F;
        if (kCamera) {
          start_camera_path(cam.jobs, num_segments, cam.scenes, q, cam.ps, i, o, d, tmin, root);
        } else {
          float4 ot = q.origin_tmin[i];
          float4 dr = q.dir_root[i];
          o = f3(ot);
          d = f3(dr);
          tmin = ot.w;
          root = __float_as_uint(dr.w);
        }
      },
      [&](uint32_t i, const Traversal<STACK, false>& tr) {
        h.tuv_slot[i] = tr.found() ? make_float4(tr.hit_t, tr.hit_u(), tr.hit_v(), __uint_as_float(tr.hit_slot))
                                   : make_float4(-1.0f, 0.0f, 0.0f, 0.0f);
        h.instance[i] = tr.found() ? tr.hit_inst : 0xffffffffu;
        if (kCamera && hl.list != nullptr) {
          // (path slot i is queue slot i): list the primary hits of ReSTIR
          // jobs, one atomic per group of lanes finishing together; the list
          // order affects no result
          const bool take = tr.found() && hl.jobs[hl.meta[i].w].restir != 0u;
          const uint32_t group = __activemask();
          const uint32_t ballot = __ballot_sync(group, take);
          if (ballot != 0u) {
            const uint32_t leader = __ffs(ballot) - 1u;
            uint32_t base = 0;
            if (lane_id() == leader) base = atomicAdd(hl.count, __popc(ballot));
            base = __shfl_sync(group, base, leader);
            if (take) hl.list[base + __popc(ballot & ((1u << lane_id()) - 1u))] = i;
          }
        }
      },
      err);
  if (err) atomicAdd(&cnt->traversal_errors, 1u);
}

template <int STACK, int SCHED>
__global__ void __maxnreg__(kTraceRegisters) k_trace_shadow(SceneView s, ShadowQueue sq, PathState ps,
                                                             Counters* cnt, uint32_t bounce) {
  extern __shared__ int smem_stack[];
  const uint32_t n = cnt->shadow_count[bounce];
  uint32_t err = 0;
  persistent_trace<STACK, true, SCHED>(
      s, n, &cnt->shadow_cursor[bounce], smem_stack,
      [&](uint32_t i, float3& o, float3& d, float& tmin, float& tmax, uint32_t& root) {
        float4 ot = sq.origin_tmax[i];
        float4 dp = sq.dir_path[i];
        o = f3(ot);
        d = f3(dp);
        tmin = 0.001f;
        tmax = ot.w;
        root = __float_as_uint(sq.contrib_root[i].w);
      },
      [&](uint32_t i, const Traversal<STACK, true>& tr) {
        if (!tr.found()) {
          uint32_t path = __float_as_uint(sq.dir_path[i].w);
          float4 c = sq.contrib_root[i];
          float4 r = ps.shadow[path];
          ps.shadow[path] = make_float4(r.x + c.x, r.y + c.y, r.z + c.z, r.w);
        }
      },
      err);
  if (err) atomicAdd(&cnt->traversal_errors, 1u);
}

struct ShadeArgs {
  const JobRec* jobs;
  SceneView s;
  RayQueue qin;
  HitBuf hits;
  RayQueue qout;
  ShadowQueue sq;
  PathState ps;
  Counters* cnt;
  uint32_t bounce;
  uint32_t capacity;
  ProductPtrs prod;
  const uint4* restir;   // per-path selected light sample (bounce 0), or null
  uint32_t fresh;        // every path is at its camera vertex with its initial state (throughput 1,
                         // previous pdf 0, radiance 0), which then is not read back
};

// One next-event sample from p: an area emitter (alias-table choice, uniform
// point; sampleAreaLightTechnique, lighting.glsl:341-403) or an analytic light
// (samplePointLights, lighting.glsl:260-312), chosen with probability
// p_area = 0.5 when the scene has both.  At a surface vertex the BSDF and the
// cosine weight the light (MIS against the BSDF pdf); at a medium vertex
// (`medium`) the isotropic phase function does (MIS against 1 / (4 pi)).
// With `lights_only` only the analytic lights are sampled (a ReSTIR vertex,
// whose emitter light comes from its reservoir).  Returns false when the
// sample contributes nothing.
OLC_D bool next_event(const SceneView& s, const SceneRec& sc, const SurfaceMat& m, float3 p, float3 nrm, float3 view,
                      float3 tp, bool medium, uint32_t& rng, float3& sh_o, float3& sh_d, float& sh_tmax,
                      float3& sh_c, bool lights_only = false) {
  constexpr float kPhase = 0.25f / OLC_PI;
  const float p_area =
      (sc.num_emitters > 0u && !lights_only) ? (sc.num_lights > 0u ? 0.5f : 1.0f) : 0.0f;
  const float choose = olc_rand(rng);
  float3 c = f3(0.0f, 0.0f, 0.0f);
  float3 ldir;
  float dist = 1e4f;
  bool directional = false;
  if (choose < p_area) {
    const float sel = olc_rand(rng);
    const uint32_t li = select_emitter(s, sc, sel);
    const EmitterRec e = load_emitter(s, li);
    const float ru = sqrtf(olc_rand(rng));
    const float rv = olc_rand(rng);
    const float3 lp = emitter_point(e, ru * (1.0f - rv), ru * rv);
    const float3 off = lp - p;
    const float dist2 = dot(off, off);
    dist = sqrtf(dist2);
    ldir = off / fmaxf(dist, 1e-6f);
    const float scos = medium ? 1.0f : fmaxf(dot(nrm, ldir), 0.0f);
    const float lc = emitter_cosine(e, ldir);
    if (!(scos > 0.0f && lc > 1e-6f)) return false;
    const float eff_pdf = e.a_pdf.w * dist2 / fmaxf(lc * e.e1_area.w, 1e-6f) * p_area;
    const float scatter_pdf = medium ? kPhase : pbr_pdf(m, nrm, view, ldir);
    const float mis = power_heuristic(eff_pdf, scatter_pdf);
    const float3 f = medium ? f3(kPhase, kPhase, kPhase) : pbr_eval(m, nrm, view, ldir);
    c = tp * f * f3(e.emission) * (scos * mis / fmaxf(eff_pdf, 1e-6f));
  } else if (sc.num_lights > 0u) {
    const float pick = olc_rand(rng);
    const uint32_t li = min((uint32_t)(pick * (float)sc.num_lights), sc.num_lights - 1u);
    const float p_sel = (1.0f - p_area) / (float)sc.num_lights;
    const LightRec L = s.lights[sc.light_base + li];
    const int type = (int)(L.position_type.w + 0.5f);
    float dist2 = 1.0f;
    if (type == 1) {
      ldir = -normalize(f3(L.direction_range));
      directional = true;
    } else {
      const float3 off = f3(L.position_type) - p;
      dist2 = fmaxf(dot(off, off), 1e-6f);
      dist = sqrtf(dist2);
      ldir = off / dist;
    }
    const bool in_range = !(type != 1 && L.direction_range.w > 0.0f && dist > L.direction_range.w);
    float atten = type == 1 ? 1.0f : 1.0f / dist2;
    if (type == 2) {
      const float cone = dot(normalize(f3(L.direction_range)), -ldir);
      const float x = clampf((cone - L.spot.y) / (L.spot.x - L.spot.y), 0.0f, 1.0f);
      atten *= x * x * (3.0f - 2.0f * x);
    }
    const float scos = medium ? 1.0f : fmaxf(dot(nrm, ldir), 0.0f);
    if (!(in_range && atten > 0.0f && scos > 0.0f)) return false;
    const float3 f = medium ? f3(kPhase, kPhase, kPhase) : pbr_eval(m, nrm, view, ldir);
    c = tp * f * f3(L.color_intensity) * (L.color_intensity.w * atten * scos / p_sel);
  } else {
    return false;
  }
  if (!(c.x > 0.0f || c.y > 0.0f || c.z > 0.0f)) return false;
  sh_o = medium ? p : p + nrm * 0.002f;
  sh_d = ldir;
  sh_tmax = directional ? 1e4f : fmaxf(dist - 0.004f, 0.001f);
  sh_c = c;
  return true;
}

// The shading kernel is latency bound, and the occupancy gained by a
// register cap outweighs its spills: 80 registers (six blocks of 128
// threads per SM) with media, 72 (seven) without.  kTextures: a variant for
// runs with a textured scene; the untextured one carries none of the texture
// code's registers.  kMedia: the same for participating media (delta
// tracking at the vertex, ratio tracking of the shadow ray), whose code
// raises the uncapped kernel from 90 to 110 registers (312 bytes of spills
// at 80 registers with it, 96 at 72 without it).
template <bool kMedia>
struct ShadeRegisters {
  static constexpr int kCap = kMedia ? 80 : 72;
};
template <bool kTextures, bool kMedia>
__global__ void __maxnreg__(ShadeRegisters<kMedia>::kCap) k_shade(ShadeArgs a) {
  const SceneView& s = a.s;
  const uint32_t bounce = a.bounce;
  const uint32_t n = a.cnt->queue_count[bounce];
  // Warps take the queue 32 paths at a time (one atomic per grab), so a
  // block whose paths cost more (media crossings, refractions) does not
  // hold the launch open while others idle.
  uint32_t grab = 0, grab_end = 0;
  while (true) {
    if (grab == grab_end) {
      uint32_t g = 0;
      if (lane_id() == 0u) g = atomicAdd(&a.cnt->shade_cursor[bounce], 32u);
      grab = __shfl_sync(0xffffffffu, g, 0);
      grab_end = grab + 32u;
    }
    const uint32_t base = grab;
    grab += 32u;
    if (base >= n) break;
    const uint32_t i = base + lane_id();
    const bool valid = i < n;
    bool want_next = false, want_shadow = false, is_miss = false;
    float3 next_o = f3(0, 0, 0), next_d = f3(0, 0, 0);
    float3 sh_o = f3(0, 0, 0), sh_d = f3(0, 0, 0), sh_c = f3(0, 0, 0);
    float sh_tmax = 0.0f, next_tmin = 0.0f;
    uint32_t path = 0, root = 0;
    if (valid) {
      path = a.qin.path[i];
      const float4 ot = a.qin.origin_tmin[i];
      const float4 dr = a.qin.dir_root[i];
      const float4 hit = a.hits.tuv_slot[i];
      const float4 tp4 = a.fresh ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : a.ps.throughput[path];
      const float4 rad4 = a.fresh ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : a.ps.radiance[path];
      const uint4 meta = a.ps.meta[path];
      const JobRec& job = a.jobs[meta.w];
      const SceneRec& sc = s.scenes[job.scene];
      const bool cpu_mode = job.mode == 1u;
      root = __float_as_uint(dr.w);
      next_tmin = job_t_min(job);
      float3 tp = f3(tp4), rad = f3(rad4);
      const float3 o = f3(ot), d = f3(dr);
      const uint32_t flags = meta.z >> 8;
      const uint32_t out_pixel = meta.x;  // products belong to one plain frame's job
      const bool write_products = job.products && bounce == 0u && meta.y == job.sample_base && a.prod.depth;
      const bool write_secondary = job.products && bounce == 1u && meta.y == job.sample_base && a.prod.depth;
      uint32_t rng = olc_bounce_state(olc_path_seed(meta.x, meta.y, job.frame), bounce);
      uint32_t new_flags = flags & OLC_PATH_DEPTH_MASK;   // the medium stack depth carries over
      float new_pdf = 0.0f;
      const uint32_t next_bounce = bounce + 1u;
      // ---- participating medium (production transport): a real collision
      // before the surface (or before leaving the scene) makes this vertex a
      // scattering event in the medium
      Medium med;
      const bool has_medium = kMedia && !cpu_mode && load_medium(sc, med);
      float t_med = 0.0f;
      const bool scattered =
          has_medium && medium_collision(med, o, d, ot.w, hit.x < 0.0f ? CUDART_INF_F : hit.x, rng, t_med);
      if (scattered) {
        const float3 p = o + d * t_med;
        tp *= med.albedo;
        if (kTextures && sc.tex_words != nullptr) {
          const float2 c = bounce > 0u ? a.ps.cone[path] : make_float2(0.0f, 0.0f);
          a.ps.cone[path] = make_float2(c.x + t_med * c.y, c.y);
        }
        if (write_products) {
          a.prod.depth[out_pixel] = t_med;
          a.prod.normal[out_pixel] = make_float4(0, 0, 0, 0);
          a.prod.instance_id[out_pixel] = 0xffffffffu;
          a.prod.material_id[out_pixel] = 0xffffffffu;
          a.prod.primitive_id[out_pixel] = 0xffffffffu;
          a.prod.position[out_pixel] = make_float4(p.x, p.y, p.z, 0.0f);
          a.prod.barycentric[out_pixel] = make_float2(0.0f, 0.0f);
          a.prod.signals[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          a.prod.secondary[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (next_bounce < job.max_bounces) {
          if (job.nee && (sc.num_emitters > 0u || sc.num_lights > 0u)) {
            SurfaceMat none{};
            want_shadow = next_event(s, sc, none, p, f3(0, 0, 1), -d, tp, true, rng, sh_o, sh_d, sh_tmax, sh_c);
            if (sc.num_emitters > 0u) new_flags |= OLC_PATH_FLAG_PREV_NEE;
          }
          const float u1 = olc_rand(rng), u2 = olc_rand(rng);
          next_d = uniform_sphere(u1, u2);
          new_pdf = 0.25f / OLC_PI;
          bool alive = max3(tp) > 0.0f;
          if (alive && job.rr_start > 0u && next_bounce >= job.rr_start) {
            const float survival = clampf(max3(tp), job.rr_min_survival, 0.95f);
            if (olc_rand(rng) >= survival) alive = false;
            else tp = tp * (1.0f / survival);
          }
          if (alive) {
            next_o = p;
            want_next = true;
          }
        }
      } else if (hit.x < 0.0f) {
        is_miss = true;
        // miss: environment (no environment NEE, so BSDF sampling carries it
        // with MIS weight 1)
        rad += tp * environment_radiance(sc, d, cpu_mode);
        if (write_products) {
          a.prod.depth[out_pixel] = CUDART_INF_F;
          a.prod.normal[out_pixel] = make_float4(0, 0, 0, 0);
          a.prod.instance_id[out_pixel] = 0xffffffffu;
          a.prod.material_id[out_pixel] = 0xffffffffu;
          a.prod.primitive_id[out_pixel] = 0xffffffffu;
          a.prod.position[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          a.prod.barycentric[out_pixel] = make_float2(0.0f, 0.0f);
          a.prod.signals[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          a.prod.secondary[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
      } else {
        const float t = hit.x, bu = hit.y, bv = hit.z;
        const uint32_t slot = __float_as_uint(hit.w);
        const uint32_t inst = a.hits.instance[i];
        const InstanceRec& ir = s.instances[inst];
        Affine o2w{ir.o2w0, ir.o2w1, ir.o2w2};
        Affine w2o{ir.w2o0, ir.w2o1, ir.w2o2};
        const float4* tv = s.tri_verts + 3u * slot;
        float3 v0 = xform_point(o2w, f3(tv[0])), v1 = xform_point(o2w, f3(tv[1])), v2 = xform_point(o2w, f3(tv[2]));
        float3 e1 = v1 - v0, e2 = v2 - v0;
        float3 gcross = cross(e1, e2);
        float3 ng = normalize(gcross);
        float3 p = o + d * t;
        const InstanceRec& orec = s.instances[owner_instance(s.instances, s.tri_owner, inst, slot)];
        SurfaceMat m = load_material(s, orec.material);
        if (write_products) {
          a.prod.depth[out_pixel] = t;
          float3 fn = dot(ng, d) > 0.0f ? -ng : ng;
          a.prod.normal[out_pixel] = make_float4(fn.x, fn.y, fn.z, 0.0f);
          a.prod.instance_id[out_pixel] = orec.instance_id;
          a.prod.material_id[out_pixel] = s.material_aux[orec.material].material_id;
          a.prod.primitive_id[out_pixel] = ir.prim_offset + s.tri_index[slot];
          a.prod.position[out_pixel] = make_float4(p.x, p.y, p.z, 0.0f);
          a.prod.barycentric[out_pixel] = make_float2(bu, bv);
          a.prod.signals[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          a.prod.secondary[out_pixel] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        if (cpu_mode) {
          // CPU reference transport (path_tracer.py:74-87)
          float3 nrm = dot(ng, d) > 0.0f ? -ng : ng;
          rad += tp * m.emission;
          tp *= m.base;
          if (next_bounce < job.max_bounces) {
            float u1 = olc_rand(rng), u2 = olc_rand(rng);
            next_o = p + nrm * 1e-4f;
            next_d = reference_bounce_direction(nrm, u1, u2);
            want_next = true;
          }
        } else {
          // shading normal: interpolated vertex normals in world space
          const float4* tn = s.tri_normals + 3u * slot;
          float w0 = 1.0f - bu - bv;
          float3 nobj = f3(tn[0]) * w0 + f3(tn[1]) * bu + f3(tn[2]) * bv;
          float3 ns = normalize(xform_normal_by_inverse(w2o, nobj));
          if (!(dot(ns, ns) > 0.5f)) ns = ng;
          if (dot(ns, ng) < 0.0f) ns = -ns;
          const bool entering = dot(d, ng) < 0.0f;
          // textures (wavefront_shade.comp:368-391), looked up with the ray
          // cone's footprint; camera rays start with width and spread 0
          const bool textured = kTextures && sc.tex_words != nullptr;
          float cone_w = 0.0f, cone_s = 0.0f, occlusion = 1.0f;
          if (textured) {
            if (bounce > 0u) {
              const float2 c = a.ps.cone[path];
              cone_s = c.y;
              cone_w = c.x + t * c.y;
            }
            const TexturedHit th = apply_textures(sc, orec.material - sc.material_base, slot, v0, v1, v2, o2w, w2o,
                                                  tn, bu, bv, cone_w, ng, ns, m);
            m = th.m;
            ns = th.ns;
            occlusion = th.occlusion;
          }
          const float3 nrm = entering ? ns : -ns;
          // denoiser path signals (the secondary path state of
          // wavefront_shade.comp:406-410, :561-568): the specular-lobe
          // probability of the (textured) primary material and whether it is
          // opaque, then the position of the path's next surface vertex
          if (write_products)
            a.prod.signals[out_pixel] = make_float4(spec_probability(m), m.transmission <= 0.001f ? 1.0f : 0.0f, 0.0f, 0.0f);
          if (write_secondary) a.prod.secondary[out_pixel] = make_float4(p.x, p.y, p.z, 1.0f);
          // emission with power-heuristic MIS against the previous BSDF pdf
          // (wavefront_shade.comp:412-433)
          if ((entering || m.two_sided) && (m.emission.x > 0.0f || m.emission.y > 0.0f || m.emission.z > 0.0f)) {
            float mis = 1.0f;
            if (flags & OLC_PATH_FLAG_PREV_RESTIR) {
              mis = 0.0f;  // the primary vertex's area lighting came from ReSTIR
            } else if ((flags & OLC_PATH_FLAG_PREV_NEE) && sc.num_emitters > 0u) {
              float area = 0.5f * length(gcross);
              float lc_raw = dot(ng, -d);
              float lc = m.two_sided ? fabsf(lc_raw) : fmaxf(lc_raw, 0.0f);
              float sel = area * luminance(m.emission) / fmaxf(sc.emissive_weight, 1e-6f);
              float p_area = sc.num_lights > 0u ? 0.5f : 1.0f;
              float light_pdf = sel * t * t / fmaxf(lc * area, 1e-6f) * p_area;
              mis = power_heuristic(tp4.w, light_pdf);
            }
            rad += tp * m.emission * mis;
          }
          if (next_bounce < job.max_bounces && m.transmission > 0.001f) {
            // ---- dielectric interface (wavefront_shade.comp:480-505): refract
            // into or out of the medium stack, reflect on total internal
            // reflection; no light sampling, no roulette, previous pdf kept
            uint32_t depth = ((flags & OLC_PATH_DEPTH_MASK) >> OLC_PATH_DEPTH_SHIFT) + 1u;
            const float current = medium_ior(a.ps.ior_stack, path, depth - 1u);
            const float target = entering ? fmaxf(m.ior, 1.0001f) : (depth > 1u ? medium_ior(a.ps.ior_stack, path, depth - 2u) : 1.0f);
            float3 wdir = refract_dir(d, nrm, current / target);
            if (dot(wdir, wdir) < 0.01f) {
              wdir = d - nrm * (2.0f * dot(nrm, d));
            } else if (entering && depth < OLC_MAX_MEDIUM_DEPTH) {
              set_medium_ior(a.ps.ior_stack, path, depth, target);
              ++depth;
            } else if (!entering && depth > 1u) {
              --depth;
            }
            tp *= (f3(0.8f, 0.8f, 0.8f) + m.base * 0.2f) * m.transmission;
            new_flags = (depth - 1u) << OLC_PATH_DEPTH_SHIFT;
            new_pdf = tp4.w;
            if (textured) a.ps.cone[path] = make_float2(cone_w, cone_s);
            wdir = normalize(wdir);
            if (max3(tp) > 0.0f) {
              next_o = p + wdir * 0.002f;
              next_d = wdir;
              want_next = true;
            }
          } else if (next_bounce < job.max_bounces) {
            const float3 view = -d;
            bool did_restir = false;
            // ---- next-event estimation: one shadow ray per path per bounce
            if (bounce == 0u && job.restir && a.restir != nullptr && sc.num_emitters > 0u) {
              uint4 rs = a.restir[path];
              did_restir = true;
              // A scene that also has analytic lights: one of the two
              // estimators runs, the reservoir's emitter sample or one
              // analytic light, each with probability 1/2 and its
              // contribution divided by that probability.
              const bool with_lights = job.nee && sc.num_lights > 0u;
              const bool use_reservoir = !with_lights || olc_rand(rng) < 0.5f;
              const float pick = with_lights ? 2.0f : 1.0f;
              float Wr = __uint_as_float(rs.z) * pick;
              if (!use_reservoir) {
                want_shadow = next_event(s, sc, m, p, nrm, view, tp, false, rng, sh_o, sh_d, sh_tmax, sh_c, true);
                sh_c *= pick;
              } else if (rs.x != 0xffffffffu && Wr > 0.0f) {
                const EmitterRec e = load_emitter(s, rs.x);
                float2 bary = __half22float2(*reinterpret_cast<const __half2*>(&rs.y));
                float3 lp = emitter_point(e, bary.x, bary.y);
                float3 off = lp - p;
                float dist2 = dot(off, off);
                float dist = sqrtf(dist2);
                float3 ldir = off / fmaxf(dist, 1e-6f);
                float scos = fmaxf(dot(nrm, ldir), 0.0f);
                float lc = emitter_cosine(e, ldir);
                if (scos > 0.0f && lc > 1e-6f) {
                  float3 f = pbr_eval(m, nrm, view, ldir);
                  float G = lc / fmaxf(dist2, 1e-12f);
                  float3 c = tp * f * f3(e.emission) * (scos * G * Wr);
                  if (c.x > 0.0f || c.y > 0.0f || c.z > 0.0f) {
                    sh_o = p + nrm * 0.002f;
                    sh_d = ldir;
                    sh_tmax = fmaxf(dist - 0.004f, 0.001f);
                    sh_c = c;
                    want_shadow = true;
                  }
                }
              }
            } else if (job.nee && (sc.num_emitters > 0u || sc.num_lights > 0u)) {
              want_shadow = next_event(s, sc, m, p, nrm, view, tp, false, rng, sh_o, sh_d, sh_tmax, sh_c);
            }
            // ---- BSDF sample
            float3 wdir, weight;
            float pdf;
            const bool sampled = pbr_sample(m, nrm, d, rng, wdir, weight, pdf);
            if (textured) {
              // occlusion map on the sampled weight (ordinarylight_pbr_weight,
              // ordinaryshade_primary.glsl:605-609); the cone spreads with
              // roughness (wavefront_shade.comp:546)
              weight = weight * (occlusion * (1.0f - m.metallic) + m.metallic);
              a.ps.cone[path] = make_float2(cone_w, cone_s + m.roughness * 0.25f);
            }
            tp *= weight;
            new_pdf = pdf;
            if (did_restir) new_flags |= OLC_PATH_FLAG_PREV_RESTIR;
            else if (job.nee && sc.num_emitters > 0u) new_flags |= OLC_PATH_FLAG_PREV_NEE;
            // (the reference also ends paths whose throughput falls below 1e-4,
            // wavefront_shade.comp:322-327; that cut-off is biased, so only
            // exactly-zero throughput ends a path here and Russian roulette
            // handles the rest)
            bool alive = sampled && max3(tp) > 0.0f;
            // Russian roulette (wavefront_shade.comp:569-580)
            if (alive && job.rr_start > 0u && next_bounce >= job.rr_start) {
              float survival = clampf(max3(tp), job.rr_min_survival, 0.95f);
              if (olc_rand(rng) >= survival) alive = false;
              else tp = tp * (1.0f / survival);
            }
            if (alive) {
              next_o = p + wdir * 0.002f;
              next_d = wdir;
              want_next = true;
            }
          }
        }
      }
      // shadow rays crossing the medium carry its ratio-tracked transmittance
      if (want_shadow && has_medium) {
        sh_c *= medium_transmittance(med, sh_o, sh_d, sh_tmax, rng);
        want_shadow = sh_c.x > 0.0f || sh_c.y > 0.0f || sh_c.z > 0.0f;
      }
      a.ps.throughput[path] = make_float4(tp.x, tp.y, tp.z, new_pdf);
      a.ps.radiance[path] = make_float4(rad.x, rad.y, rad.z, 0.0f);
      a.ps.meta[path] = make_uint4(meta.x, meta.y, (bounce + 1u) | (new_flags << 8), meta.w);
    }
    // miss statistics (per-bounce hit/miss split of the shade roofline)
    {
      uint32_t ballot = __ballot_sync(0xffffffffu, is_miss);
      if (ballot && lane_id() == (uint32_t)(__ffs(ballot) - 1)) atomicAdd(&a.cnt->miss_count[bounce], __popc(ballot));
    }
    // compaction of the next queue and the shadow queue
    uint32_t slot = warp_reserve(&a.cnt->queue_count[bounce + 1u], want_next);
    if (want_next) {
      if (slot < a.capacity) {
        a.qout.origin_tmin[slot] = make_float4(next_o.x, next_o.y, next_o.z, next_tmin);
        a.qout.dir_root[slot] = make_float4(next_d.x, next_d.y, next_d.z, __uint_as_float(root));
        a.qout.path[slot] = path;
      } else {
        atomicAdd(&a.cnt->overflow, 1u);
      }
    }
    uint32_t sslot = warp_reserve(&a.cnt->shadow_count[bounce], want_shadow);
    if (want_shadow) {
      if (sslot < a.capacity) {
        a.sq.origin_tmax[sslot] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_tmax);
        a.sq.dir_path[sslot] = make_float4(sh_d.x, sh_d.y, sh_d.z, __uint_as_float(path));
        a.sq.contrib_root[sslot] = make_float4(sh_c.x, sh_c.y, sh_c.z, __uint_as_float(root));
      } else {
        atomicAdd(&a.cnt->overflow, 1u);
      }
    }
  }
}

// ---- ray reordering -------------------------------------------------------
// Secondary rays leave the shading stage in path order, so a warp holds rays
// that start anywhere in the scene and point anywhere, and its lanes
// traverse unrelated parts of the hierarchy.  Before an extension bounce is
// traced, the queue is reordered by a 15-bit key: an 8x8 octahedral
// direction bin above the 9-bit Morton code of the origin within its scene's
// root box (after the ray-sorting idea of Garanzha and Loop, "Fast Ray
// Sorting and Breadth-First Packet Traversal for GPU Ray Tracing", EG 2010).
// A counting sort over the 32,768 keys with warp-aggregated atomics; the
// order inside a key is arbitrary, which changes no result because every ray
// is traced independently and accumulation is order independent.
constexpr uint32_t kSortBits = 15;
constexpr uint32_t kSortBins = 1u << kSortBits;

OLC_D uint32_t ray_sort_key(const SceneView& s, float3 o, float3 d, uint32_t root) {
  const float4* p = reinterpret_cast<const float4*>(s.nodes + root);
  const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  const float3 lo = f3(fminf(a.x, b.x), fminf(a.z, b.z), fminf(c.x, c.z));
  const float3 hi = f3(fmaxf(a.y, b.y), fmaxf(a.w, b.w), fmaxf(c.y, c.w));
  const float3 ext = hi - lo;
  auto cell = [](float v, float l, float e) -> uint32_t {
    const float u = e > 0.0f ? (v - l) / e : 0.0f;
    return (uint32_t)clampf(u * 8.0f, 0.0f, 7.0f);
  };
  const uint32_t cx = cell(o.x, lo.x, ext.x), cy = cell(o.y, lo.y, ext.y), cz = cell(o.z, lo.z, ext.z);
  uint32_t morton = 0u;
#pragma unroll
  for (int bit = 0; bit < 3; ++bit)
    morton |= (((cx >> bit) & 1u) << (3 * bit)) | (((cy >> bit) & 1u) << (3 * bit + 1)) |
              (((cz >> bit) & 1u) << (3 * bit + 2));
  const float l1 = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
  float ox = l1 > 0.0f ? d.x / l1 : 0.0f, oy = l1 > 0.0f ? d.y / l1 : 0.0f;
  if (d.z < 0.0f) {
    const float tx = (1.0f - fabsf(oy)) * (ox >= 0.0f ? 1.0f : -1.0f);
    const float ty = (1.0f - fabsf(ox)) * (oy >= 0.0f ? 1.0f : -1.0f);
    ox = tx;
    oy = ty;
  }
  const uint32_t ux = (uint32_t)clampf((ox * 0.5f + 0.5f) * 8.0f, 0.0f, 7.0f);
  const uint32_t uy = (uint32_t)clampf((oy * 0.5f + 0.5f) * 8.0f, 0.0f, 7.0f);
  return ((ux | (uy << 3)) << 9) | morton;
}

// Adds `amount` per lane to counter[key], one atomic per distinct key of the
// warp; returns each lane's previous count plus its rank among equal keys.
OLC_D uint32_t warp_bin_add(uint32_t* counter, uint32_t key, bool active) {
  const uint32_t mask = __ballot_sync(0xffffffffu, active);
  if (!active) return 0u;
  const uint32_t peers = __match_any_sync(mask, key);
  const uint32_t leader = __ffs(peers) - 1u;
  uint32_t base = 0u;
  if (lane_id() == leader) base = atomicAdd(counter + key, (uint32_t)__popc(peers));
  base = __shfl_sync(peers, base, leader);
  return base + __popc(peers & ((1u << lane_id()) - 1u));
}

__global__ void k_sort_keys(SceneView s, RayQueue q, const uint32_t* __restrict__ count, uint32_t* keys,
                            uint32_t* hist) {
  const uint32_t n = *count;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool active = i < n;
    uint32_t key = 0u;
    if (active) {
      const float4 ot = q.origin_tmin[i];
      const float4 dr = q.dir_root[i];
      key = ray_sort_key(s, f3(ot), f3(dr), __float_as_uint(dr.w));
      keys[i] = key;
    }
    warp_bin_add(hist, key, active);
  }
}

// Exclusive prefix sum of the kSortBins counts, in place (one block of 1024).
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* hist) {
  constexpr uint32_t kPer = kSortBins / 1024u;
  __shared__ uint32_t warp_sums[32];
  const uint32_t t = threadIdx.x;
  uint32_t local[kPer];
  uint32_t sum = 0u;
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    local[k] = hist[t * kPer + k];
    sum += local[k];
  }
  uint32_t incl = sum;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane_id() >= (uint32_t)off) incl += v;
  }
  if (lane_id() == 31u) warp_sums[t >> 5] = incl;
  __syncthreads();
  if (t < 32u) {
    uint32_t w = warp_sums[t];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, w, off);
      if (t >= (uint32_t)off) w += v;
    }
    warp_sums[t] = w;
  }
  __syncthreads();
  uint32_t run = incl - sum + ((t >> 5) ? warp_sums[(t >> 5) - 1u] : 0u);
#pragma unroll
  for (uint32_t k = 0; k < kPer; ++k) {
    hist[t * kPer + k] = run;
    run += local[k];
  }
}

__global__ void k_sort_scatter(RayQueue in, const uint32_t* __restrict__ count, const uint32_t* __restrict__ keys,
                               uint32_t* cursor, RayQueue out) {
  const uint32_t n = *count;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool active = i < n;
    const uint32_t key = active ? keys[i] : 0u;
    const uint32_t pos = warp_bin_add(cursor, key, active);
    if (active) {
      out.origin_tmin[pos] = in.origin_tmin[i];
      out.dir_root[pos] = in.dir_root[i];
      out.path[pos] = in.path[i];
    }
  }
}

// ---- the reference volume model (reference-compatible mode) ---------------
// Each queued ray of a reference-compatible path whose scene has visible
// volumes crosses them over [0, hit distance] (unbounded for a miss) before
// shading: path radiance += throughput * volume radiance, throughput *=
// volume transmittance (ReferencePathTracer.render_hdr,
// renderers/reference/path_tracer.py:55-65; the march is in
// olc_refvolume.cuh).  A grid-stride pass over the bounce's queue; rays of
// other paths are skipped.
__global__ void __launch_bounds__(128) k_ref_volumes(const JobRec* __restrict__ jobs, SceneView s, RayQueue q,
                                                     HitBuf h, PathState ps, const Counters* __restrict__ cnt,
                                                     uint32_t bounce) {
  const uint32_t n = cnt->queue_count[bounce];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t path = q.path[i];
    const uint4 meta = ps.meta[path];
    const JobRec& job = jobs[meta.w];
    if (job.mode != 1u) continue;
    const SceneRec& sc = s.scenes[job.scene];
    if (sc.num_ref_vols == 0u) continue;
    const float4 hit = h.tuv_slot[i];
    const float t_max = hit.x < 0.0f ? CUDART_INF_F : hit.x;
    float3 rad;
    float T;
    rv_integrate(ref_volumes_of(sc), s.lights + sc.light_base, sc.num_lights, f3(q.origin_tmin[i]),
                 f3(q.dir_root[i]), t_max, rad, T);
    if (T == 1.0f && rad.x == 0.0f && rad.y == 0.0f && rad.z == 0.0f) continue;
    const float4 tp = ps.throughput[path];
    const float4 r = ps.radiance[path];
    ps.radiance[path] = make_float4(r.x + tp.x * rad.x, r.y + tp.y * rad.y, r.z + tp.z * rad.z, r.w);
    ps.throughput[path] = make_float4(tp.x * T, tp.y * T, tp.z * T, tp.w);
  }
}

OLC_D unsigned long long to_fixed(float v, uint32_t* nan_counter) {
  if (!(v == v)) {  // NaN
    atomicAdd(nan_counter, 1u);
    return 0ull;
  }
  v = fminf(fmaxf(v, 0.0f), OLC_SAMPLE_CLAMP);
  return __float2ull_rn(v * OLC_ACCUM_SCALE);
}

// A sample's colour channel as a one-sample image shows it: the fixed-point
// value divided back (the division k_resolve does for spp = 1).
OLC_D float from_fixed(unsigned long long v) { return (float)((double)v * (1.0 / (double)OLC_ACCUM_SCALE)); }

// Path samples into their pixels' fixed-point sums.  A segment made of whole
// sample streams (its first path and its length multiples of the image's
// pixel count, as ReSTIR jobs and single-chunk frames are) holds every one of
// its samples of a pixel at the same position of each stream, so the thread
// of the first stream's path adds them all with one atomic per channel
// instead of one per sample; other segments add path by path.  Integer sums
// make the result independent of the grouping and the order.
__global__ void k_accumulate(const ChunkHeader* __restrict__ hdr, const JobRec* __restrict__ jobs, PathState ps,
                             unsigned long long* accum, float* sample_lum, Counters* cnt) {
  const uint32_t count = hdr->count;
  const uint32_t num_segments = hdr->num_segments;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    // the segment from the chunk's job table (L1-resident), so the paths of
    // later sample streams, added by their pixel's first-stream path, read
    // nothing of their own
    const uint32_t j = segment_of_path(jobs, num_segments, i);
    const JobRec& job = jobs[j];
    const uint32_t seg_begin = (uint32_t)job.seg_begin;
    const uint32_t seg_end = j + 1u < num_segments ? (uint32_t)jobs[j + 1u].seg_begin : count;
    const uint32_t seg_count = seg_end - seg_begin;
    uint32_t samples = 1u;
    if (job.seg_first % job.npix == 0ull && seg_count % job.npix == 0u) {
      if (i - seg_begin >= job.npix) continue;   // added with its pixel's first-stream path
      samples = seg_count / job.npix;
    }
    const uint4 meta = ps.meta[i];
    unsigned long long fr = 0ull, fg = 0ull, fb = 0ull;
    for (uint32_t k = 0; k < samples; ++k) {
      // the path's own emission terms, then its shadow rays' sum
      const float4 r = ps.radiance[i + k * job.npix];
      const float4 sh = ps.shadow[i + k * job.npix];
      const unsigned long long sr = to_fixed(r.x + sh.x, &cnt->nan_samples);
      const unsigned long long sg = to_fixed(r.y + sh.y, &cnt->nan_samples);
      const unsigned long long sb = to_fixed(r.z + sh.z, &cnt->nan_samples);
      fr += sr;
      fg += sg;
      fb += sb;
      if (job.lum_base != ~0ull) {
        // luminance in float32 in the reference's operation order
        // (api.py:1404-1410: r * 0.2126 + g * 0.7152 + b * 0.0722), unfused
        const float l = __fadd_rn(__fadd_rn(__fmul_rn(from_fixed(sr), 0.2126f), __fmul_rn(from_fixed(sg), 0.7152f)),
                                  __fmul_rn(from_fixed(sb), 0.0722f));
        sample_lum[job.lum_base + (uint64_t)(meta.y - job.sample_base + k) * job.npix + meta.x] = l;
      }
    }
    unsigned long long* dst = accum + 3ull * (job.pixel_base + meta.x);
    atomicAdd(dst + 0, fr);
    atomicAdd(dst + 1, fg);
    atomicAdd(dst + 2, fb);
  }
}

// Unbiased luminance variance over the samples of each pixel, summed in
// double precision in sample order (api.py:1411-1431).
__global__ void k_sample_variance(const float* __restrict__ sample_lum, uint32_t npix, uint32_t spp, float* out) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
    if (spp <= 1u) {
      out[p] = 0.0f;
      continue;
    }
    double sum = 0.0, sq = 0.0;
    for (uint32_t s = 0; s < spp; ++s) {
      const double l = (double)sample_lum[(uint64_t)s * npix + p];
      sum = __dadd_rn(sum, l);
      sq = __dadd_rn(sq, __dmul_rn(l, l));
    }
    const double v = __ddiv_rn(__dsub_rn(sq, __ddiv_rn(__dmul_rn(sum, sum), (double)spp)), (double)(spp - 1u));
    out[p] = (float)fmax(v, 0.0);
  }
}

// Mean of the accumulated samples of each finished job (the host
// accumulate-and-divide of render_wavefront_outputs,
// ordinarylight/targets/vulkan/api.py:1404-1422, done on the device).
__global__ void k_resolve(const ResolveEntry* __restrict__ entries, const uint32_t* __restrict__ num_entries,
                          const unsigned long long* __restrict__ accum, float4* out) {
  const uint32_t n = *num_entries;
  for (uint32_t e = 0; e < n; ++e) {
    const ResolveEntry en = entries[e];
    const double scale = 1.0 / ((double)OLC_ACCUM_SCALE * (double)en.spp);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < en.npix; p += gridDim.x * blockDim.x) {
      const unsigned long long* a = accum + 3ull * (en.pixel_base + p);
      out[en.pixel_base + p] = make_float4((float)((double)a[0] * scale), (float)((double)a[1] * scale),
                                           (float)((double)a[2] * scale), 0.0f);
    }
  }
}

// Material texture lookups of a scene for given coordinates and footprints
// (the sampler alone, for its parity tests).
__global__ void k_sample_textures(const SceneRec* __restrict__ scenes, uint32_t scene, float binding, uint32_t n,
                                  const float2* __restrict__ uv0, const float2* __restrict__ uv1,
                                  const float* __restrict__ fp0, const float* __restrict__ fp1, int srgb, float4* out) {
  const SceneRec& sc = scenes[scene];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = sample_material_texture(sc, binding, uv0[i], uv1[i], srgb != 0, fp0[i], fp1[i]);
}

__global__ void k_camera_rays(const JobRec* __restrict__ job_ptr, uint32_t sample, float2 jitter_override,
                              int use_override, float* origins, float* dirs) {
  const JobRec job = *job_ptr;
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < job.npix; p += gridDim.x * blockDim.x) {
    float3 o, d;
    camera_ray(job, p, sample, use_override ? &jitter_override : nullptr, o, d);
    origins[3ull * p + 0] = o.x;
    origins[3ull * p + 1] = o.y;
    origins[3ull * p + 2] = o.z;
    dirs[3ull * p + 0] = d.x;
    dirs[3ull * p + 1] = d.y;
    dirs[3ull * p + 2] = d.z;
  }
}

template <int STACK>
__global__ void __launch_bounds__(256) k_trace_rays(SceneView s, uint32_t root, uint32_t n,
                                                    const float* __restrict__ origins, const float* __restrict__ dirs,
                                                    float t_min, uint32_t* inst_id, int32_t* prim, float* tout,
                                                    float* bary, Counters* cnt) {
  extern __shared__ int smem_stack[];
  uint32_t err = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 o = f3(origins[3ull * i], origins[3ull * i + 1], origins[3ull * i + 2]);
    float3 d = f3(dirs[3ull * i], dirs[3ull * i + 1], dirs[3ull * i + 2]);
    HitResult hr;
    bool hit = olc_traverse<STACK, false>(s, root, o, d, t_min, CUDART_INF_F, hr, smem_stack, err);
    if (inst_id)
      inst_id[i] = hit ? s.instances[owner_instance(s.instances, s.tri_owner, hr.instance, hr.slot)].instance_id
                       : 0xffffffffu;
    if (prim) prim[i] = hit ? (int32_t)hr.packed : -1;
    if (tout) tout[i] = hit ? hr.t : CUDART_INF_F;
    if (bary) {
      bary[2ull * i] = hit ? hr.u : 0.0f;
      bary[2ull * i + 1] = hit ? hr.v : 0.0f;
    }
  }
  if (err) atomicAdd(&cnt->traversal_errors, 1u);
}

template <int STACK>
__global__ void __launch_bounds__(256) k_occluded_rays(SceneView s, uint32_t root, uint32_t n,
                                                       const float* __restrict__ origins,
                                                       const float* __restrict__ dirs, float t_min,
                                                       const float* __restrict__ t_max, uint8_t* occ, Counters* cnt) {
  extern __shared__ int smem_stack[];
  uint32_t err = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float3 o = f3(origins[3ull * i], origins[3ull * i + 1], origins[3ull * i + 2]);
    float3 d = f3(dirs[3ull * i], dirs[3ull * i + 1], dirs[3ull * i + 2]);
    HitResult hr;
    occ[i] = olc_traverse<STACK, true>(s, root, o, d, t_min, t_max[i], hr, smem_stack, err) ? 1 : 0;
  }
  if (err) atomicAdd(&cnt->traversal_errors, 1u);
}

constexpr int kTraceThreads = 128;

template <class F>
void dispatch_stack(uint32_t depth, F&& f) {
  if (depth <= 16) f(std::integral_constant<int, 16>{});
  else if (depth <= 24) f(std::integral_constant<int, 24>{});
  else f(std::integral_constant<int, 32>{});
}

inline size_t stack_bytes(uint32_t depth, uint32_t threads) {
  uint32_t d = depth <= 16 ? 16 : (depth <= 24 ? 24 : 32);
  return (size_t)(d + OLC_RAY_SAVE) * threads * sizeof(int);
}

}  // namespace

void launch_trace_closest(const LaunchShape& ls, const SceneView& s, const RayQueue& q, const HitBuf& h,
                          Counters* cnt, uint32_t bounce, const HitListOut& hl, const CameraPaths* cam,
                          cudaStream_t stream) {
  dispatch_stack(ls.stack_depth, [&](auto depth) {
    constexpr int D = decltype(depth)::value;
    const size_t smem = stack_bytes(D, ls.trace_block);
    // camera rays come in 8x4-pixel tiles: a warp keeps its 32 coherent rays
    // to the end instead of refilling lanes with rays of other tiles
    if (cam != nullptr)
      k_trace_closest<D, 1, true><<<ls.grid_trace, ls.trace_block, smem, stream>>>(s, q, h, cnt, 0u, hl, *cam);
    else if (ls.scheduler == 1)
      k_trace_closest<D, 1, false><<<ls.grid_trace, ls.trace_block, smem, stream>>>(s, q, h, cnt, bounce,
                                                                                    HitListOut{}, CameraPaths{});
    else
      k_trace_closest<D, 0, false><<<ls.grid_trace, ls.trace_block, smem, stream>>>(s, q, h, cnt, bounce,
                                                                                    HitListOut{}, CameraPaths{});
  });
  OLC_LAUNCH_CHECK("k_trace_closest");
}

void launch_trace_shadow(const LaunchShape& ls, const SceneView& s, const ShadowQueue& sq, const PathState& ps,
                         Counters* cnt, uint32_t bounce, cudaStream_t stream) {
  dispatch_stack(ls.stack_depth, [&](auto depth) {
    constexpr int D = decltype(depth)::value;
    if (ls.scheduler == 1)
      k_trace_shadow<D, 1><<<ls.grid_trace, ls.trace_block, stack_bytes(D, ls.trace_block), stream>>>(s, sq, ps, cnt,
                                                                                                       bounce);
    else
      k_trace_shadow<D, 0><<<ls.grid_trace, ls.trace_block, stack_bytes(D, ls.trace_block), stream>>>(s, sq, ps, cnt,
                                                                                                       bounce);
  });
  OLC_LAUNCH_CHECK("k_trace_shadow");
}

uint32_t resident_grid(const void* fn, uint32_t block, size_t smem, uint32_t max_grid) {
  struct Entry {
    const void* fn;
    uint32_t block;
    size_t smem;
    int device;
    uint32_t grid;
  };
  static std::mutex mu;
  static std::vector<Entry> cache;
  int device = 0;
  OLC_CUDA(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mu);
  for (const Entry& e : cache)
    if (e.fn == fn && e.block == block && e.smem == smem && e.device == device) return std::min(e.grid, max_grid);
  int per_sm = 0, sms = 0;
  OLC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, (int)block, smem));
  OLC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const uint32_t grid = (uint32_t)std::max(1, per_sm) * (uint32_t)std::max(1, sms);
  cache.push_back(Entry{fn, block, smem, device, grid});
  return std::min(grid, max_grid);
}

void launch_shade(const LaunchShape& ls, const JobRec* jobs, const SceneView& s, const RayQueue& qin,
                  const HitBuf& hits, const RayQueue& qout, const ShadowQueue& sq, const PathState& ps,
                  Counters* cnt, uint32_t bounce, uint32_t capacity, const ProductPtrs& prod, const uint4* restir,
                  bool textures, bool media, bool fresh, cudaStream_t stream) {
  ShadeArgs a;
  a.jobs = jobs;
  a.s = s;
  a.qin = qin;
  a.hits = hits;
  a.qout = qout;
  a.sq = sq;
  a.ps = ps;
  a.cnt = cnt;
  a.bounce = bounce;
  a.capacity = capacity;
  a.prod = prod;
  a.restir = restir;
  a.fresh = fresh ? 1u : 0u;
  auto launch = [&](auto kernel) {
    kernel<<<resident_grid((const void*)kernel, ls.trace_block, 0, ls.grid_shade), ls.trace_block, 0, stream>>>(a);
  };
  if (textures && media) launch(k_shade<true, true>);
  else if (textures) launch(k_shade<true, false>);
  else if (media) launch(k_shade<false, true>);
  else launch(k_shade<false, false>);
  OLC_LAUNCH_CHECK("k_shade");
}

void launch_sort_rays(const LaunchShape& ls, const SceneView& s, const RayQueue& in, const RayQueue& out,
                      Counters* cnt, uint32_t bounce, uint32_t* keys, uint32_t* bins, cudaStream_t stream) {
  OLC_CUDA(cudaMemsetAsync(bins, 0, kSortBins * sizeof(uint32_t), stream));
  const uint32_t* count = &cnt->queue_count[bounce];
  k_sort_keys<<<ls.grid_simple, 256, 0, stream>>>(s, in, count, keys, bins);
  OLC_LAUNCH_CHECK("k_sort_keys");
  k_sort_scan<<<1, 1024, 0, stream>>>(bins);
  OLC_LAUNCH_CHECK("k_sort_scan");
  k_sort_scatter<<<ls.grid_simple, 256, 0, stream>>>(in, count, keys, bins, out);
  OLC_LAUNCH_CHECK("k_sort_scatter");
}

size_t sort_bins_bytes() { return kSortBins * sizeof(uint32_t); }

void launch_ref_volumes(const LaunchShape& ls, const JobRec* jobs, const SceneView& s, const RayQueue& q,
                        const HitBuf& hits, const PathState& ps, const Counters* cnt, uint32_t bounce,
                        cudaStream_t stream) {
  k_ref_volumes<<<resident_grid((const void*)k_ref_volumes, 128, 0, ls.grid_shade), 128, 0, stream>>>(
      jobs, s, q, hits, ps, cnt, bounce);
  OLC_LAUNCH_CHECK("k_ref_volumes");
}

void launch_accumulate(const LaunchShape& ls, const ChunkHeader* hdr, const JobRec* jobs, const PathState& ps,
                       unsigned long long* accum, float* sample_lum, Counters* cnt, cudaStream_t stream) {
  k_accumulate<<<resident_grid((const void*)k_accumulate, ls.block, 0, ls.grid_simple), ls.block, 0, stream>>>(
      hdr, jobs, ps, accum, sample_lum, cnt);
  OLC_LAUNCH_CHECK("k_accumulate");
}

void launch_sample_variance(const LaunchShape& ls, const float* sample_lum, uint32_t npix, uint32_t spp, float* out,
                            cudaStream_t stream) {
  k_sample_variance<<<ls.grid_simple, ls.block, 0, stream>>>(sample_lum, npix, spp, out);
  OLC_LAUNCH_CHECK("k_sample_variance");
}

void launch_resolve(const LaunchShape& ls, const ResolveEntry* entries, const uint32_t* num_entries,
                    const unsigned long long* accum, float4* out, cudaStream_t stream) {
  k_resolve<<<resident_grid((const void*)k_resolve, ls.block, 0, ls.grid_simple), ls.block, 0, stream>>>(
      entries, num_entries, accum, out);
  OLC_LAUNCH_CHECK("k_resolve");
}

void launch_sample_textures(const LaunchShape& ls, const SceneRec* scenes, uint32_t scene, float binding, uint32_t n,
                            const float2* uv0, const float2* uv1, const float* fp0, const float* fp1, int srgb,
                            float4* out, cudaStream_t stream) {
  if (n == 0) return;
  k_sample_textures<<<ls.grid_simple, ls.block, 0, stream>>>(scenes, scene, binding, n, uv0, uv1, fp0, fp1, srgb, out);
  OLC_LAUNCH_CHECK("k_sample_textures");
}

void launch_camera_rays(const LaunchShape& ls, const JobRec* job, uint32_t sample, const float* jitter,
                        float* origins, float* dirs, cudaStream_t stream) {
  float2 j = make_float2(0.5f, 0.5f);
  if (jitter) j = make_float2(jitter[0], jitter[1]);
  k_camera_rays<<<ls.grid_simple, ls.block, 0, stream>>>(job, sample, j, jitter ? 1 : 0, origins, dirs);
  OLC_LAUNCH_CHECK("k_camera_rays");
}

void launch_trace_rays(const LaunchShape& ls, const SceneView& s, uint32_t root, uint32_t n, const float* origins,
                       const float* dirs, float t_min, uint32_t* inst_id, int32_t* prim, float* t, float* bary,
                       Counters* cnt, cudaStream_t stream) {
  dispatch_stack(ls.stack_depth, [&](auto depth) {
    constexpr int D = decltype(depth)::value;
    uint32_t grid = std::max<uint32_t>(1u, std::min<uint32_t>((n + kTraceThreads - 1) / kTraceThreads, ls.grid_trace));
    k_trace_rays<D><<<grid, kTraceThreads, stack_bytes(D, kTraceThreads), stream>>>(s, root, n, origins, dirs, t_min,
                                                                                     inst_id, prim, t, bary, cnt);
  });
  OLC_LAUNCH_CHECK("k_trace_rays");
}

void launch_occluded_rays(const LaunchShape& ls, const SceneView& s, uint32_t root, uint32_t n, const float* origins,
                          const float* dirs, float t_min, const float* t_max, uint8_t* occ, Counters* cnt,
                          cudaStream_t stream) {
  dispatch_stack(ls.stack_depth, [&](auto depth) {
    constexpr int D = decltype(depth)::value;
    uint32_t grid = std::max<uint32_t>(1u, std::min<uint32_t>((n + kTraceThreads - 1) / kTraceThreads, ls.grid_trace));
    k_occluded_rays<D><<<grid, kTraceThreads, stack_bytes(D, kTraceThreads), stream>>>(s, root, n, origins, dirs,
                                                                                        t_min, t_max, occ, cnt);
  });
  OLC_LAUNCH_CHECK("k_occluded_rays");
}

void configure_trace_kernels() {
  // Prefer the largest shared-memory carve-out for the traversal kernels so
  // more blocks (each holding its short stacks) share one SM, and allow the
  // largest launch's stacks (32 entries, 256 threads: above the 48 KB that
  // needs no opt-in).
  const int most = (int)stack_bytes(32, 256);
  auto prefer = [most](const void* fn) {
    cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, most);
  };
  prefer((const void*)k_trace_closest<16, 0, false>);
  prefer((const void*)k_trace_closest<24, 0, false>);
  prefer((const void*)k_trace_closest<32, 0, false>);
  prefer((const void*)k_trace_closest<16, 1, true>);
  prefer((const void*)k_trace_closest<24, 1, true>);
  prefer((const void*)k_trace_closest<32, 1, true>);
  prefer((const void*)k_trace_shadow<16, 0>);
  prefer((const void*)k_trace_shadow<24, 0>);
  prefer((const void*)k_trace_shadow<32, 0>);
  prefer((const void*)k_trace_closest<16, 1, false>);
  prefer((const void*)k_trace_closest<24, 1, false>);
  prefer((const void*)k_trace_closest<32, 1, false>);
  prefer((const void*)k_trace_shadow<16, 1>);
  prefer((const void*)k_trace_shadow<24, 1>);
  prefer((const void*)k_trace_shadow<32, 1>);
  prefer((const void*)k_trace_rays<16>);
  prefer((const void*)k_trace_rays<24>);
  prefer((const void*)k_trace_rays<32>);
  prefer((const void*)k_occluded_rays<16>);
  prefer((const void*)k_occluded_rays<24>);
  prefer((const void*)k_occluded_rays<32>);
}

}  // namespace olc
