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
// Storage: three uint4 words per reservoir,
//   w0 = (light index, barycentrics as half2, w_sum, M)
//   w1 = (p_hat of the selected sample, primary depth, octahedral normal, stamp)
//   w2 = (primary surface position, 0): where the support test of the
//        unbiased combination evaluates a reused reservoir's target
// indexed by the job's reservoir base + sample stream * npix + pixel, so a
// stream's reservoirs survive chunking and batching.  A reservoir is valid
// only when its stamp equals the stamp of the wavefront that should have
// written it, so pixels whose primary ray missed never need clearing.
//
// Only primary rays that hit take part: the bounce-0 traversal lists them
// (k_trace_closest's hit list), so the candidate loop runs with full warps
// even when much of the image is sky.
#include <cuda_fp16.h>

#include "olc_restir.h"
#include "olc_shading.cuh"
#include "olc_textures.cuh"
#include "olc_volume.cuh"

namespace olc {

namespace {

constexpr uint32_t kRestirStream = 0x52455354u;  // stream key offset of the reuse passes
constexpr uint32_t kMaxNeighbours = 16;          // restir_neighbours' upper bound
constexpr uint32_t kPoolStream = 0x504f4f4cu;    // stream key of the light pool and its block starts
constexpr uint32_t kPoolSize = 1u << 15;         // light-pool entries per ReSTIR job and frame

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

// BSDF of one surface with the light-independent terms hoisted
// (preparePrimaryPbr, transport_v1/lighting.glsl:116-133): every candidate
// then costs only the half-vector terms.
struct PreparedBsdf {
  float3 n, view, f0, diffuse;
  float nv, a2;
  float spec_scale;   // a2 G1(v) / (2 pi n.v): the GGX lobe's light-independent factor
};

OLC_D PreparedBsdf prepare_bsdf(const SurfaceMat& m, float3 n, float3 view) {
  PreparedBsdf b;
  b.n = n;
  b.view = view;
  b.nv = fmaxf(dot(n, view), 0.0f);
  b.f0 = lerp3(f3(0.04f, 0.04f, 0.04f), m.base, m.metallic);
  b.diffuse = m.base * ((1.0f - m.metallic) / OLC_PI);
  b.a2 = ggx_alpha2(m.roughness);
  b.spec_scale = b.nv > 0.0f ? b.a2 * ggx_g1(b.nv, b.a2) / (2.0f * OLC_PI * b.nv) : 0.0f;
  return b;
}

// The BSDF times the cosine-free factors for candidate direction l, with
// hardware reciprocal square roots, one approximate division and the GGX
// bracket's sin^2(n, h) as 1 - (n.h)^2.  The specular lobe
// F D G1(v) G1(l) / (4 n.v n.l), with D = a2 / (pi den^2) and
// G1(l) = 2 n.l / (n.l + sqrt(a2 + (1 - a2) (n.l)^2)), is evaluated as
// F spec_scale / (den^2 (n.l + sqrt(...))) (n.l cancels), and
// (1 - F) diffuse + F spec as diffuse + F (spec - diffuse).  The resampling
// target only has to be one fixed function of the sample, positive where
// both cosines are (the estimator stays unbiased for any such target).
OLC_D float3 prepared_eval(const PreparedBsdf& b, float3 l, float nl) {
  const float3 hv = b.view + l;
  const float3 h = hv * rsqrtf(fmaxf(dot(hv, hv), 1e-30f));
  const float nh = fmaxf(dot(b.n, h), 0.0f);
  const float vh = fmaxf(dot(b.view, h), 0.0f);
  const float w = 1.0f - fminf(vh, 1.0f);
  const float w2 = w * w;
  const float w5 = w2 * w2 * w;
  const float iw5 = 1.0f - w5;
  const float den = fmaf(nh * nh, b.a2, fmaxf(fmaf(-nh, nh, 1.0f), 0.0f));   // the GGX bracket of ggx_d
  const float x = fmaf(1.0f - b.a2, nl * nl, b.a2);
  const float spec = __fdividef(b.spec_scale, fmaxf(den * den * (nl + x * rsqrtf(x)), 1e-30f));
  const float3 F = f3(fmaf(b.f0.x, iw5, w5), fmaf(b.f0.y, iw5, w5), fmaf(b.f0.z, iw5, w5));
  return f3(fmaf(F.x, spec - b.diffuse.x, b.diffuse.x), fmaf(F.y, spec - b.diffuse.y, b.diffuse.y),
            fmaf(F.z, spec - b.diffuse.z, b.diffuse.z));
}

struct Surface {
  float3 p;
  PreparedBsdf bsdf;
  float depth;
};

struct Res {
  uint32_t light;
  uint32_t bary;
  float w_sum;
  uint32_t M;
  float target;
};

OLC_D float2 unpack_bary(uint32_t b) { return __half22float2(*reinterpret_cast<const __half2*>(&b)); }
OLC_D uint32_t pack_bary(float b1, float b2) {
  __half2 h = __floats2half2_rn(b1, b2);
  return *reinterpret_cast<uint32_t*>(&h);
}

// The emitter radiance weighted by the luminance coefficients, so that
// luminance(f Le) = dot(f, luminance_weighted(Le)).
OLC_D float3 luminance_weighted(float3 Le) { return f3(Le.x * 0.2126f, Le.y * 0.7152f, Le.z * 0.0722f); }

// Unshadowed target of a light sample at surface s, given the sample's point,
// the emitter's normal, sidedness and luminance-weighted radiance Lw:
// dot(f, Lw) cos_s cos_l / d^2 = luminance(f Le) cos_s cos_l / d^2.
OLC_D float target_at(const Surface& s, float3 lp, float3 lnormal, bool two_sided, float3 Lw) {
  float3 off = lp - s.p;
  float d2 = dot(off, off);
  if (!(d2 > 1e-12f)) return 0.0f;
  float inv = rsqrtf(d2);
  float3 l = off * inv;
  float cs = dot(s.bsdf.n, l);
  if (cs <= 0.0f || s.bsdf.nv <= 0.0f) return 0.0f;
  const float c = -dot(lnormal, l);
  float cl = two_sided ? fabsf(c) : fmaxf(c, 0.0f);   // emitter_cosine
  if (cl <= 1e-6f) return 0.0f;
  float3 f = prepared_eval(s.bsdf, l, cs);
  float t = dot(f, Lw) * cs * cl * (inv * inv);
  return (t == t && t < 3.0e38f) ? fmaxf(t, 0.0f) : 0.0f;
}

// Unshadowed target of light sample (light, bary) at surface s, from the
// emitter record (the reuse passes; the light pool stores the same terms).
OLC_D float target_of(const SceneView& sc, const Surface& s, uint32_t light, uint32_t bary) {
  const EmitterRec e = load_emitter(sc, light);
  const float2 b = unpack_bary(bary);
  return target_at(s, emitter_point(e, b.x, b.y), f3(e.normal), e.e2_sided.w > 0.5f,
                   luminance_weighted(f3(e.emission)));
}

// Returns whether the offered sample was selected.
OLC_D bool res_update(Res& r, uint32_t light, uint32_t bary, float target, float w, uint32_t m, float u) {
  r.M += m;
  r.w_sum += w;
  if (w > 0.0f && (r.light == 0xffffffffu || u * r.w_sum < w)) {
    r.light = light;
    r.bary = bary;
    r.target = target;
    return true;
  }
  return false;
}

// Whether the light sample at point lp of emitter e lies in the support of
// the target at a surface (position p, viewer-side shading normal n): both
// cosines positive.  Only reservoirs with a positive target of their own
// sample are ever reused, so their surfaces face the viewer (n.v > 0); the
// BSDF of an opaque surface is positive wherever both cosines are, and
// emitters have positive luminance, so this is where target_of is not zero.
OLC_D bool in_support(const EmitterRec& e, float3 lp, float3 p, float3 n) {
  const float3 off = lp - p;
  const float d2 = dot(off, off);
  if (!(d2 > 1e-12f)) return false;
  const float3 l = off * rsqrtf(d2);
  return dot(n, l) > 0.0f && emitter_cosine(e, l) > 1e-6f;
}

// Unbiased normalisation of a combined reservoir (Bitterli et al. 2020,
// "Spatiotemporal reservoir resampling", Algorithm 6): W = w_sum / (Z p_hat)
// with Z the sample counts of only those combined reservoirs whose own target
// is positive at the selected sample, instead of all of them (1 / M weights
// darken wherever a reused reservoir could not have produced the sample).
// Stored as w_sum M / Z, so W = w_sum / (M p_hat) and the reuse weight
// p_hat w_sum / p_hat_src of later passes stay as they are.
OLC_D void normalise_support(Res& r, uint32_t Z) {
  if (Z > 0u && Z < r.M) r.w_sum *= (float)r.M / (float)Z;
}

// The primary vertex of path slot i (its ray hit: only listed hits get
// here) as the shading stage sees it at bounce 0: position, viewer-side
// shading normal (normal-mapped when textured), material (textured; the
// camera ray's cone has width 0), view direction, depth.
struct PrimaryVertex {
  float3 p, n, view;
  SurfaceMat m;
  float depth;
};

template <bool kTextures>
OLC_D PrimaryVertex primary_vertex(const SceneView& s, const RayQueue& q, const HitBuf& h, uint32_t i,
                                   uint32_t scene) {
  PrimaryVertex pv;
  const float4 hit = h.tuv_slot[i];
  const float4 dr = q.dir_root[i];
  const float4 ot = q.origin_tmin[i];
  const float3 d = f3(dr);
  const uint32_t slot = __float_as_uint(hit.w);
  const uint32_t inst = h.instance[i];
  const InstanceRec& ir = s.instances[inst];
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
  pv.p = f3(ot) + d * hit.x;
  const uint32_t owner = owner_instance(s.instances, s.tri_owner, inst, slot);
  const uint32_t mi = s.instances[owner].material;
  pv.m = load_material(s, mi);
  const SceneRec& sc = s.scenes[scene];
  if (kTextures && sc.tex_words != nullptr) {
    const TexturedHit th = apply_textures(sc, mi - sc.material_base, slot, v0, v1, v2, o2w, w2o, tn, hit.y, hit.z,
                                          0.0f, ng, ns, pv.m);
    pv.m = th.m;
    ns = th.ns;
  }
  pv.n = entering ? ns : -ns;
  pv.view = -d;
  pv.depth = hit.x;
  return pv;
}

template <bool kTextures>
OLC_D Surface primary_surface(const SceneView& s, const RayQueue& q, const HitBuf& h, uint32_t i, uint32_t scene) {
  const PrimaryVertex pv = primary_vertex<kTextures>(s, q, h, i, scene);
  Surface su;
  su.p = pv.p;
  su.bsdf = prepare_bsdf(pv.m, pv.n, pv.view);
  su.depth = pv.depth;
  return su;
}

OLC_D bool similar(const Surface& s, uint32_t w1_normal, float depth) {
  if (dot(oct_decode(w1_normal), s.bsdf.n) < 0.9f) return false;
  return fabsf(depth - s.depth) <= 0.1f * s.depth;
}

OLC_D void store_res(uint4* w0, uint4* w1, uint4* w2, uint64_t g, const Res& r, const Surface& s, uint32_t stamp) {
  w0[g] = make_uint4(r.light, r.bary, __float_as_uint(r.w_sum), r.M);
  w1[g] = make_uint4(__float_as_uint(r.target), __float_as_uint(s.depth), oct_encode(s.bsdf.n), stamp);
  w2[g] = make_uint4(__float_as_uint(s.p.x), __float_as_uint(s.p.y), __float_as_uint(s.p.z), 0u);
}

OLC_D float3 stored_position(const uint4* w2, uint64_t g) {
  const uint4 v = w2[g];
  return f3(__uint_as_float(v.x), __uint_as_float(v.y), __uint_as_float(v.z));
}

OLC_D Res load_res(const uint4* w0, const uint4* w1, uint64_t g, float& depth, uint32_t& nrm, uint32_t& stamp) {
  uint4 a = w0[g], b = w1[g];
  Res r;
  r.light = a.x;
  r.bary = a.y;
  r.w_sum = __uint_as_float(a.z);
  r.M = a.w;
  r.target = __uint_as_float(b.x);
  depth = __uint_as_float(b.y);
  nrm = b.z;
  stamp = b.w;
  return r;
}

// Reservoir index of (job, sample stream, pixel).
OLC_D uint64_t reservoir_index(const JobRec& job, uint32_t sample, uint32_t pixel) {
  return job.reservoir_base + (uint64_t)(sample - job.sample_base) * job.npix + pixel;
}

struct RestirArgs {
  const ChunkHeader* hdr;
  const JobRec* jobs;
  SceneView s;
  RayQueue q;
  HitBuf h;
  PathState ps;
  const uint32_t* hit_list;
  const uint32_t* hit_count;
  uint32_t* cursor;           // work cursor of this launch (zeroed with hit_count)
  uint32_t candidates;
  uint32_t history_cap;     // M cap of the temporal history
  uint32_t neighbours;
  float radius;
  const uint4* hist0;
  const uint4* hist1;
  const uint4* hist2;
  const uint4* in0;
  const uint4* in1;
  const uint4* in2;
  uint4* out0;
  uint4* out1;
  uint4* out2;
  uint32_t pass;
  uint4* selected;
  uint32_t finalize;
  const float4* pool0;      // light pool: kPoolSize entries per chunk segment
  const float4* pool1;
  const float4* pool2;
};

// Light pool of every ReSTIR job of the chunk (after the presampled light
// tiles of Wyman and Panteleev, HPG 2021): kPoolSize emitter samples drawn
// from the scene's source distribution (alias-table emitter, uniform point
// with the reference's square-root mapping, ordinaryshade_primary.glsl:668-671),
// each stored with the terms the resampling target reads: the point and the
// reciprocal source pdf per unit area (negative for a two-sided emitter), the
// emitter's normal and the sample's half-precision barycentrics, its
// luminance-weighted radiance and index.  Entries are keyed by (entry, job.frame) only, so every chunking
// and batch mix draws the same pool.
__global__ void k_restir_pool(const ChunkHeader* __restrict__ hdr, const JobRec* __restrict__ jobs, SceneView s,
                              float4* __restrict__ p0, float4* __restrict__ p1, float4* __restrict__ p2) {
  const uint64_t n = (uint64_t)hdr->num_segments * kPoolSize;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const JobRec& job = jobs[k / kPoolSize];
    if (!job.restir) continue;
    const SceneRec& sc = s.scenes[job.scene];
    if (sc.num_emitters == 0u) continue;
    const uint32_t entry = (uint32_t)(k % kPoolSize);
    uint32_t rng = olc_bounce_state(olc_path_seed(entry, kPoolStream, job.frame), kPoolStream);
    const uint32_t li = select_emitter(s, sc, olc_rand(rng));
    // The barycentrics are stored in half precision, so 16 bits of each of
    // their two uniforms suffice: both come from one word (each half placed
    // in a float's mantissa, [1, 2) minus 1).
    const uint32_t bits = olc_rand_word(rng);
    const float u0 = __uint_as_float(0x3f800000u | ((bits >> 16) << 7)) - 1.0f;
    const float rv = __uint_as_float(0x3f800000u | ((bits & 0xffffu) << 7)) - 1.0f;
    const float ru = u0 > 0.0f ? u0 * rsqrtf(u0) : 0.0f;
    const uint32_t bary = pack_bary(ru * (1.0f - rv), ru * rv);
    const EmitterRec e = load_emitter(s, li);
    const float2 b = unpack_bary(bary);
    const float3 lp = emitter_point(e, b.x, b.y);
    p0[k] = make_float4(lp.x, lp.y, lp.z, e.e2_sided.w > 0.5f ? -e.emission.w : e.emission.w);
    p1[k] = make_float4(e.normal.x, e.normal.y, e.normal.z, __uint_as_float(bary));
    const float3 lw = luminance_weighted(f3(e.emission));
    p2[k] = make_float4(lw.x, lw.y, lw.z, __uint_as_float(li));
  }
}

// Eight blocks of 128 threads per SM for the untextured kernel (64
// registers, 20 bytes of spills outside the candidate loop): the candidate
// loop is issue-bound and gains from the extra warps (1.657 -> 1.625 ms of
// ReSTIR per 1080p frame).  The textured kernel keeps its 128 registers.
template <bool kTextures>
__global__ void __launch_bounds__(128, kTextures ? 4 : 8) k_restir_initial(RestirArgs a) {
  const SceneView& s = a.s;
  const uint32_t n = *a.hit_count;
  // warps take the hit list 32 entries at a time (one atomic per grab),
  // so blocks whose hits cost more do not hold the launch open
  for (uint32_t grab = 0, grab_end = 0;;) {
    if (grab == grab_end) {
      uint32_t g = 0;
      if ((threadIdx.x & 31u) == 0u) g = atomicAdd(a.cursor, 32u);
      grab = __shfl_sync(0xffffffffu, g, 0);
      grab_end = grab + 32u;
    }
    const uint32_t k = grab + (threadIdx.x & 31u);
    grab += 32u;
    if (grab - 32u >= n) break;
    if (k >= n) continue;
    const uint32_t i = a.hit_list[k];
    const uint4 meta = a.ps.meta[i];
    const JobRec& job = a.jobs[meta.w];
    const SceneRec& sc = s.scenes[job.scene];
    const uint64_t g = reservoir_index(job, meta.y, meta.x);
    const Surface su = primary_surface<kTextures>(s, a.q, a.h, i, job.scene);
    const uint32_t stamp = a.hdr->stamp;
    Res r{0xffffffffu, 0u, 0.0f, 0u, 0.0f};
    uint32_t rng = olc_bounce_state(olc_path_seed(meta.x, meta.y, job.frame), kRestirStream);
    if (sc.num_emitters > 0u) {
      // Candidates come from the job's light pool: the 32 pixels of an 8x4
      // block of one sample stream read 32 consecutive entries per candidate
      // from a block-specific start, so each pixel's candidates are distinct
      // pool entries, i.e. independent draws of the source distribution.
      const uint32_t px = meta.x % job.width, py = meta.x / job.width;
      const uint32_t block = (py >> 2) * ((job.width + 7u) >> 3) + (px >> 3);
      uint32_t e = olc_hash(olc_path_seed(block, meta.y, job.frame) ^ kPoolStream) + ((px & 7u) | ((py & 3u) << 3));
      const size_t base = (size_t)meta.w * kPoolSize;
      const float4* q0 = a.pool0 + base;
      const float4* q1 = a.pool1 + base;
      const float4* q2 = a.pool2 + base;
      for (uint32_t c = 0; c < a.candidates; ++c, e += 32u) {
        const uint32_t k = e & (kPoolSize - 1u);
        const float4 w0 = __ldg(q0 + k), w1 = __ldg(q1 + k), w2 = __ldg(q2 + k);
        const float t = target_at(su, f3(w0), f3(w1), w0.w < 0.0f, f3(w2));
        res_update(r, __float_as_uint(w2.w), __float_as_uint(w1.w), t, t * fabsf(w0.w), 1u, olc_rand(rng));
      }
    }
    // temporal reuse
    if (job.history) {
      float pd;
      uint32_t pn, pstamp;
      const uint64_t gh = job.history_base + (uint64_t)(meta.y - job.sample_base) * job.npix + meta.x;
      Res prev = load_res(a.hist0, a.hist1, gh, pd, pn, pstamp);
      if (pstamp != 0u && pstamp >= a.hdr->history_first && pstamp <= a.hdr->history_last && prev.light != 0xffffffffu && prev.M > 0u && prev.target > 0.0f &&
          similar(su, pn, pd)) {
        uint32_t m = min(prev.M, a.history_cap);
        float wsum = prev.w_sum * ((float)m / (float)prev.M);
        float t = target_of(s, su, prev.light, prev.bary);
        res_update(r, prev.light, prev.bary, t, t * wsum / prev.target, m, olc_rand(rng));
        // the candidates always count; the history only where the selected
        // sample is in the support of the previous frame's target
        if (r.light != 0xffffffffu) {
          const EmitterRec e = load_emitter(s, r.light);
          const float2 b = unpack_bary(r.bary);
          const bool supported =
              in_support(e, emitter_point(e, b.x, b.y), stored_position(a.hist2, gh), oct_decode(pn));
          normalise_support(r, r.M - (supported ? 0u : m));
        }
      }
    }
    store_res(a.out0, a.out1, a.out2, g, r, su, stamp);
  }
}

// Eight blocks of 128 threads per SM for the untextured kernel too (64
// registers instead of 69, 20 bytes of spills): with its grid one resident
// wave, the eighth block per SM took its ReSTIR time from 1.495 to 1.468 ms
// per 1080p instanced frame.
template <bool kTextures>
__global__ void __launch_bounds__(128, kTextures ? 4 : 8) k_restir_spatial(RestirArgs a) {
  const SceneView& s = a.s;
  const uint32_t n = *a.hit_count;
  // warps take the hit list 32 entries at a time (one atomic per grab),
  // so blocks whose hits cost more do not hold the launch open
  for (uint32_t grab = 0, grab_end = 0;;) {
    if (grab == grab_end) {
      uint32_t g = 0;
      if ((threadIdx.x & 31u) == 0u) g = atomicAdd(a.cursor, 32u);
      grab = __shfl_sync(0xffffffffu, g, 0);
      grab_end = grab + 32u;
    }
    const uint32_t k = grab + (threadIdx.x & 31u);
    grab += 32u;
    if (grab - 32u >= n) break;
    if (k >= n) continue;
    const uint32_t i = a.hit_list[k];
    const uint4 meta = a.ps.meta[i];
    const JobRec& job = a.jobs[meta.w];
    const uint64_t g = reservoir_index(job, meta.y, meta.x);
    const uint64_t stream_base = g - meta.x;
    const Surface su = primary_surface<kTextures>(s, a.q, a.h, i, job.scene);
    const uint32_t stamp = a.hdr->stamp;
    float d0;
    uint32_t n0, st0;
    Res r = load_res(a.in0, a.in1, g, d0, n0, st0);
    if (a.neighbours > 0u) {
      const uint32_t rng0 = olc_bounce_state(olc_path_seed(meta.x, meta.y, job.frame), kRestirStream + 1u + a.pass);
      const int px = (int)(meta.x % job.width), py = (int)(meta.x / job.width);
      // The j-th neighbour of this pixel from the pass's stream; false when
      // it is off the image, this pixel, invalid or not similar.
      auto neighbour = [&](uint32_t& rng, uint32_t& q, Res& nb, float& dq, uint32_t& nq, float& u) {
        float rr = a.radius * sqrtf(olc_rand(rng));
        float th = 2.0f * OLC_PI * olc_rand(rng);
        u = olc_rand(rng);
        float sn, cs;
        __sincosf(th, &sn, &cs);
        int qx = px + __float2int_rn(rr * cs);
        int qy = py + __float2int_rn(rr * sn);
        if (qx < 0 || qy < 0 || qx >= (int)job.width || qy >= (int)job.height || (qx == px && qy == py)) return false;
        q = (uint32_t)qy * job.width + (uint32_t)qx;
        uint32_t sq;
        nb = load_res(a.in0, a.in1, stream_base + q, dq, nq, sq);
        return sq == stamp && nb.light != 0xffffffffu && nb.M != 0u && nb.target > 0.0f && similar(su, nq, dq);
      };
      uint32_t rng = rng0;
      uint32_t reused_q[kMaxNeighbours];
      uint32_t reused = 0;
      uint32_t winner = kMaxNeighbours;   // the reused neighbour whose sample was selected last
      for (uint32_t j = 0; j < a.neighbours; ++j) {
        uint32_t q, nq;
        Res nb;
        float dq, u;
        if (!neighbour(rng, q, nb, dq, nq, u)) continue;
        float t = target_of(s, su, nb.light, nb.bary);
        if (res_update(r, nb.light, nb.bary, t, t * nb.w_sum / nb.target, nb.M, u)) winner = reused;
        reused_q[reused++] = q;
      }
      if (reused && r.light != 0xffffffffu) {
        // this pixel's reservoir always counts (the selected sample has a
        // positive target here), and so does the neighbour whose own sample
        // won (reused only with a positive target of it); each other reused
        // neighbour where the sample is in the support of its own target
        const EmitterRec e = load_emitter(s, r.light);
        const float2 b = unpack_bary(r.bary);
        const float3 lp = emitter_point(e, b.x, b.y);
        uint32_t Z = r.M;
        for (uint32_t k = 0; k < reused; ++k) {
          if (k == winner) continue;
          const uint64_t gq = stream_base + reused_q[k];
          const uint4 w0 = a.in0[gq];
          const uint4 w1 = a.in1[gq];
          if (!in_support(e, lp, stored_position(a.in2, gq), oct_decode(w1.z))) Z -= w0.w;
        }
        normalise_support(r, Z);
      }
    }
    store_res(a.out0, a.out1, a.out2, g, r, su, stamp);
    if (a.finalize) {
      float W = (r.light != 0xffffffffu && r.M > 0u && r.target > 0.0f) ? r.w_sum / ((float)r.M * r.target) : 0.0f;
      if (!(W == W) || W > 3.0e38f) W = 0.0f;
      a.selected[i] = make_uint4(W > 0.0f ? r.light : 0xffffffffu, r.bary, __float_as_uint(W), 0u);
    }
  }
}

}  // namespace

void restir_prepare(RestirState& st, uint64_t reservoirs, uint32_t slots, uint32_t chunks, uint32_t segments) {
  if (reservoirs > st.reservoirs) {
    // the history survives only if its buffers are kept
    for (DeviceBuffer* b : {&st.res_a0, &st.res_a1, &st.res_a2, &st.res_b0, &st.res_b1, &st.res_b2, &st.hist0,
                            &st.hist1, &st.hist2})
      b->allocate(reservoirs * 16);
    // stamps start at 1: zero-filled reservoirs are never valid
    for (DeviceBuffer* b : {&st.res_a1, &st.res_b1, &st.hist1}) OLC_CUDA(cudaMemset(b->get(), 0, reservoirs * 16));
    st.reservoirs = reservoirs;
    st.history_valid = false;
  }
  if (segments > st.pool_segments) {
    for (DeviceBuffer* b : {&st.pool0, &st.pool1, &st.pool2}) b->allocate((size_t)segments * kPoolSize * 16);
    st.pool_segments = segments;
  }
  if (slots > st.slots) {
    st.selected.allocate((size_t)slots * 16);
    st.hit_list.allocate((size_t)slots * 4);
    st.slots = slots;
  }
  if (!st.hit_count.get()) st.hit_count.allocate(32);
  if ((uint64_t)st.next_stamp + chunks >= 0xffffffffull) {
    // stamps would wrap: clear every stored stamp and start again at 1
    for (DeviceBuffer* b : {&st.res_a1, &st.res_b1, &st.hist1}) OLC_CUDA(cudaMemset(b->get(), 0, st.reservoirs * 16));
    st.next_stamp = 1;
    st.history_valid = false;
    st.hist_first = st.hist_last = 0;
  }
  st.run_first = st.next_stamp;
  st.run_last = st.next_stamp + chunks - 1u;
  st.next_stamp += chunks;
}

const uint4* restir_run(RestirState& st, const olc_config& cfg, const LaunchShape& ls, const SceneView& s,
                        const ChunkHeader* hdr, const JobRec* jobs, const RayQueue& q, const HitBuf& hits,
                        const PathState& ps, bool textures, cudaStream_t stream) {
  RestirArgs a{};
  a.hdr = hdr;
  a.jobs = jobs;
  a.s = s;
  a.q = q;
  a.h = hits;
  a.ps = ps;
  a.hit_list = st.hit_list.as<uint32_t>();
  a.hit_count = st.hit_count.as<uint32_t>();
  a.candidates = cfg.restir_candidates;
  a.history_cap = std::max<uint32_t>(1u, cfg.restir_max_history ? cfg.restir_max_history : 20u) * cfg.restir_candidates;
  a.neighbours = cfg.restir_neighbours;
  a.radius = cfg.restir_radius > 0.0f ? cfg.restir_radius : 30.0f;
  a.hist0 = st.hist0.as<uint4>();
  a.hist1 = st.hist1.as<uint4>();
  a.hist2 = st.hist2.as<uint4>();
  a.selected = st.selected.as<uint4>();
  a.out0 = st.res_a0.as<uint4>();
  a.out1 = st.res_a1.as<uint4>();
  a.out2 = st.res_a2.as<uint4>();
  a.pool0 = st.pool0.as<float4>();
  a.pool1 = st.pool1.as<float4>();
  a.pool2 = st.pool2.as<float4>();
  k_restir_pool<<<resident_grid((const void*)k_restir_pool, 256, 0, ls.grid_simple), 256, 0, stream>>>(
      hdr, jobs, s, st.pool0.as<float4>(), st.pool1.as<float4>(), st.pool2.as<float4>());
  OLC_LAUNCH_CHECK("k_restir_pool");
  const uint32_t grid = ls.grid_shade;
  a.cursor = st.hit_count.as<uint32_t>() + 1;
  if (textures)
    k_restir_initial<true><<<resident_grid((const void*)k_restir_initial<true>, 128, 0, grid), 128, 0, stream>>>(a);
  else
    k_restir_initial<false><<<resident_grid((const void*)k_restir_initial<false>, 128, 0, grid), 128, 0, stream>>>(a);
  OLC_LAUNCH_CHECK("k_restir_initial");
  // spatial passes ping-pong A -> B -> A ...; the last pass finalises.
  uint32_t passes = std::max<uint32_t>(cfg.restir_spatial, 1u);
  bool in_a = true;
  for (uint32_t p = 0; p < passes; ++p) {
    RestirArgs b = a;
    b.pass = p;
    b.cursor = st.hit_count.as<uint32_t>() + 2 + p;
    b.neighbours = cfg.restir_spatial ? cfg.restir_neighbours : 0u;
    b.in0 = in_a ? st.res_a0.as<uint4>() : st.res_b0.as<uint4>();
    b.in1 = in_a ? st.res_a1.as<uint4>() : st.res_b1.as<uint4>();
    b.in2 = in_a ? st.res_a2.as<uint4>() : st.res_b2.as<uint4>();
    b.out0 = in_a ? st.res_b0.as<uint4>() : st.res_a0.as<uint4>();
    b.out1 = in_a ? st.res_b1.as<uint4>() : st.res_a1.as<uint4>();
    b.out2 = in_a ? st.res_b2.as<uint4>() : st.res_a2.as<uint4>();
    b.finalize = (p + 1 == passes) ? 1u : 0u;
    if (textures)
      k_restir_spatial<true><<<resident_grid((const void*)k_restir_spatial<true>, 128, 0, grid), 128, 0, stream>>>(b);
    else
      k_restir_spatial<false><<<resident_grid((const void*)k_restir_spatial<false>, 128, 0, grid), 128, 0, stream>>>(
          b);
    OLC_LAUNCH_CHECK("k_restir_spatial");
    in_a = !in_a;
  }
  st.final_in_b = !in_a;  // the final reservoirs are where the last pass wrote
  return st.selected.as<uint4>();
}

void restir_finish(RestirState& st) {
  // the final reservoirs become the next frame's temporal history
  st.hist_first = st.run_first;
  st.hist_last = st.run_last;
  if (st.final_in_b) {
    std::swap(st.hist0, st.res_b0);
    std::swap(st.hist1, st.res_b1);
    std::swap(st.hist2, st.res_b2);
  } else {
    std::swap(st.hist0, st.res_a0);
    std::swap(st.hist1, st.res_a1);
    std::swap(st.hist2, st.res_a2);
  }
}

void restir_reset(RestirState& st) {
  st.history_valid = false;
  st.history_used = false;
}

void restir_release(RestirState& st) {
  for (DeviceBuffer* b : {&st.res_a0, &st.res_a1, &st.res_a2, &st.res_b0, &st.res_b1, &st.res_b2, &st.hist0,
                          &st.hist1, &st.hist2})
    b->release();
  st.selected.release();
  for (DeviceBuffer* b : {&st.pool0, &st.pool1, &st.pool2}) b->release();
  st.pool_segments = 0;
  st.hit_list.release();
  st.hit_count.release();
  st.reservoirs = 0;
  st.slots = 0;
  st.history_valid = false;
}

}  // namespace olc
