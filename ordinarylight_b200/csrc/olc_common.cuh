// Shared device definitions: vector math, the counter-based sampling
// sequence, and the HBM layouts of the resident scene and wavefront queues.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>

#define OLC_HD __host__ __device__ __forceinline__
#define OLC_D __device__ __forceinline__

// ---------------------------------------------------------------------------
// float3 helpers
// ---------------------------------------------------------------------------
OLC_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
OLC_HD float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
OLC_HD float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
OLC_HD float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
OLC_HD float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
OLC_HD float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
OLC_HD float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
OLC_HD float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
OLC_HD float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
OLC_HD float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
OLC_HD float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
OLC_HD float3& operator*=(float3& a, float s) { a = a * s; return a; }
OLC_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
OLC_HD float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
OLC_HD float length(float3 a) { return sqrtf(dot(a, a)); }
OLC_HD float3 normalize(float3 a) {
  float l = sqrtf(dot(a, a));
  return l > 0.0f ? a * (1.0f / l) : a;
}
OLC_HD float3 fminf3(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
OLC_HD float3 fmaxf3(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
OLC_HD float max3(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
OLC_HD float get(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
OLC_HD float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
OLC_HD float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
OLC_HD float3 lerp3(float3 a, float3 b, float t) { return a + (b - a) * t; }

// Affine 3x4 row-major transform.
struct Affine {
  float4 r0, r1, r2;
};
OLC_HD float3 xform_point(const Affine& m, float3 p) {
  return f3(m.r0.x * p.x + m.r0.y * p.y + m.r0.z * p.z + m.r0.w,
            m.r1.x * p.x + m.r1.y * p.y + m.r1.z * p.z + m.r1.w,
            m.r2.x * p.x + m.r2.y * p.y + m.r2.z * p.z + m.r2.w);
}
OLC_HD float3 xform_vector(const Affine& m, float3 v) {
  return f3(m.r0.x * v.x + m.r0.y * v.y + m.r0.z * v.z,
            m.r1.x * v.x + m.r1.y * v.y + m.r1.z * v.z,
            m.r2.x * v.x + m.r2.y * v.y + m.r2.z * v.z);
}
// Normal transform by the inverse transpose: given W = world->object,
// n_world = W^T n_object.
OLC_HD float3 xform_normal_by_inverse(const Affine& w2o, float3 n) {
  return f3(w2o.r0.x * n.x + w2o.r1.x * n.y + w2o.r2.x * n.z,
            w2o.r0.y * n.x + w2o.r1.y * n.y + w2o.r2.y * n.z,
            w2o.r0.z * n.x + w2o.r1.z * n.y + w2o.r2.z * n.z);
}

// ---------------------------------------------------------------------------
// Counter-based sampling sequence.
//
// The mixing function is the 32-bit integer hash the reference wavefront uses
// for its per-path seed (waveHash, ordinarylight/shaders/wavefront_generate.comp:71-79:
// xor-shift 16, multiply 0x7feb352d, xor-shift 15, multiply 0x846ca68b,
// xor-shift 16 — C. Wellons' published "lowbias32"), and the per-draw
// generator is the PCG-RXS-M-XS 32-bit step of randomFloat
// (ordinarylight/shaders/transport_v1/sampling.glsl:16-22; M. O'Neill, PCG).
// Unlike the reference, the stream is re-keyed for every bounce from
// (pixel, sample, bounce, frame), so a path's random numbers never depend on
// how many numbers an earlier bounce consumed or on which queue slot or
// launch processed it.
// ---------------------------------------------------------------------------
OLC_HD uint32_t olc_hash(uint32_t v) {
  v ^= v >> 16;
  v *= 0x7feb352du;
  v ^= v >> 15;
  v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}

// Seed of (pixel, sample, frame).  The reference combines
// H(H(pixel ^ H(frame) ^ H(sample + 1))) (wavefront_generate.comp:113-116),
// whose xor makes (frame f, sample s) and (frame s + 1, sample f - 1) share a
// stream (for example every pixel of frame 1 sample 0 equals frame 2
// sample 1... and pixel 0 of frame 1 sample 0 gets jitter 0).  Nesting the
// pixel/frame hash before mixing in the sample removes that symmetry:
// H(H(pixel ^ H(frame)) ^ H(sample + 1)).
OLC_HD uint32_t olc_path_seed(uint32_t pixel, uint32_t sample, uint32_t frame) {
  return olc_hash(olc_hash(pixel ^ olc_hash(frame)) ^ olc_hash(sample + 1u));
}

// Stream state of one bounce of one path.
OLC_HD uint32_t olc_bounce_state(uint32_t path_seed, uint32_t bounce) {
  return olc_hash(path_seed ^ olc_hash(bounce * 0x9e3779b9u + 0x632be5abu));
}

// One PCG-RXS-M-XS step: a uniform 32-bit word, or a float in [0, 1).
OLC_HD uint32_t olc_rand_word(uint32_t& state) {
  state = state * 747796405u + 2891336453u;
  const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
  return (word >> 22u) ^ word;
}
OLC_HD float olc_rand(uint32_t& state) { return (float)olc_rand_word(state) * (1.0f / 4294967296.0f); }

// Camera jitter of (pixel, sample, frame): two hash steps of the path seed,
// the reference raygen's jitter draws (wavefront_generate.comp:117-121).
OLC_HD float2 olc_camera_jitter(uint32_t pixel, uint32_t sample, uint32_t frame) {
  uint32_t s = olc_path_seed(pixel, sample, frame);
  s = olc_hash(s);
  float jx = (float)s * (1.0f / 4294967296.0f);
  s = olc_hash(s);
  float jy = (float)s * (1.0f / 4294967296.0f);
  return make_float2(jx, jy);
}

// ---------------------------------------------------------------------------
// Resident scene layout in HBM.
// ---------------------------------------------------------------------------
// BVH2 node, 64 bytes, four 16-byte loads: both child boxes are stored in the
// parent so one node fetch tests two children.
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, -, -)   child >= 0: node index; child < 0: leaf
struct __align__(16) BvhNode {
  float4 a, b, c;
  int4 d;
};
// Leaf reference: ~((first << 3) | (count - 1)), count in 1..8.
#define OLC_LEAF_MAX 8
OLC_HD int olc_make_leaf(uint32_t first, uint32_t count) { return ~(int)((first << 3) | (count - 1u)); }
OLC_HD uint32_t olc_leaf_first(int ref) { return ((uint32_t)(~ref)) >> 3; }
OLC_HD uint32_t olc_leaf_count(int ref) { return (((uint32_t)(~ref)) & 7u) + 1u; }
#define OLC_EMPTY_CHILD ((int)0x80000000)

// BVH4 node, 128 bytes (one L2 line, seven 16-byte loads): up to four
// descendants of BVH2 node i (its children, each internal one opened in turn
// while the largest box still fits four slots; a leaf stands for itself),
// stored at index i of a second array parallel to the BVH2 nodes.  Traversal
// descends about two BVH2 levels per dependent fetch.  Child references keep
// the BVH2 encoding, and an internal child's index is its BVH2 index, so
// roots, instance records and leaves are shared by both forms.  Box slot k of
// the six float4 is child k; unused slots hold OLC_EMPTY_CHILD and an
// inverted box (lo +inf, hi -inf) that no ray enters.
struct __align__(16) BvhNode4 {
  float4 lox, hix, loy, hiy, loz, hiz;
  int4 child;
  int4 reserved;
};

// Instance record, 128 bytes: world->object 3x4 and identity/offsets (the
// 64 bytes traversal reads), then object->world 3x4 for shading, then flags.
//
// Instances of very small meshes (the 1,024 one-triangle emitters of the
// instanced benchmark scene, the walls of the box room) are baked at upload
// into world-space triangles that the TLAS references directly, so a ray
// reaching such an object needs no transform and no second hierarchy.  Hits
// on them report one identity record flagged OLC_INSTANCE_FLATTENED; for
// their slots tri_index holds the packed triangle index itself and tri_owner
// the record of the original instance (material, Mesh.id).
#define OLC_INSTANCE_FLATTENED 1u
struct __align__(16) InstanceRec {
  float4 w2o0, w2o1, w2o2;
  uint32_t blas_root;      // node index of the instance's BLAS root
  uint32_t material;       // material table index
  uint32_t prim_offset;    // packed triangle base (Scene.triangles order)
  uint32_t instance_id;    // Mesh.id
  float4 o2w0, o2w1, o2w2;
  uint32_t flags;          // OLC_INSTANCE_FLATTENED
  uint32_t pad[3];
};

// Material record, 32 bytes.
struct __align__(16) MaterialRec {
  float4 base_rough;       // base_color.rgb, roughness
  float4 emit_metal;       // emission.rgb, metallic
};
struct __align__(16) MaterialAux {
  uint32_t two_sided;
  uint32_t material_id;
  float transmission;      // > 0.001: a dielectric interface (wavefront_shade.comp:480-505)
  float ior;
};

// Emitter record (area light), 80 bytes: the reference's emissive-triangle
// records (Scene.emissive_triangle_data, scene/_core.py:2637-2691:
// vertices, emission, area, power pdf, two-sided flag) re-expressed at upload
// for sampling — vertex a, both edges and the unit normal precomputed, so a
// candidate costs no cross product or normalisation.
struct __align__(16) EmitterRec {
  float4 a_pdf;            // a.xyz, selection probability
  float4 e1_area;          // b - a, area
  float4 e2_sided;         // c - a, two-sided flag (0/1)
  float4 normal;           // unit normal of cross(e1, e2), area-measure source pdf (probability / area)
  float4 emission;         // rgb, reciprocal of the source pdf (area / probability; 0 if never selected)
};

// Walker/Vose alias table entry over the emitter power distribution: O(1)
// selection with the same probabilities as the reference's CDF binary
// search (transport_v1/lighting.glsl:356-377).
struct __align__(8) AliasEntry {
  float threshold;
  uint32_t alias;
};

struct __align__(16) LightRec {
  float4 position_type;
  float4 direction_range;
  float4 color_intensity;
  float4 spot;
};

// The instance that owns a hit's material and identity: the hit instance
// itself, or for a baked world-space triangle the original instance.
OLC_D uint32_t owner_instance(const InstanceRec* instances, const uint32_t* tri_owner, uint32_t inst, uint32_t slot) {
  return (instances[inst].flags & OLC_INSTANCE_FLATTENED) ? tri_owner[slot] : inst;
}

// Pool record 0 is an identity transform flagged OLC_INSTANCE_FLATTENED:
// hits on baked world-space triangles report it as their instance.
#define OLC_IDENTITY_INSTANCE 0u

// TLAS leaf kinds (the leaf's count field): an instance (first = global
// instance record) or a baked world-space triangle (first = global slot).
#define OLC_TLAS_LEAF_INSTANCE 1u
#define OLC_TLAS_LEAF_TRIANGLE 2u

// One visible volume in the reference's volume model (the reference-
// compatible mode's ray march; 288 bytes, the olc_scene_desc record of 72
// floats with its integer fields as bit patterns).
struct __align__(16) RefVolume {
  float4 w2b0, w2b1, w2b2;          // world -> local unit cube (rows of the inverse transform)
  uint32_t nx, ny, nz, lut_len;     // grid size (x fastest in memory: z, y, x), transfer entries
  uint32_t grid_off, lut_off;       // offsets of the normalized grid and of the transfer table
  uint32_t address, linear;         // transfer addressing: 0 clamp, 1 repeat, 2 mirror; linear filter
  uint32_t missing, num_clip, phase_hg, orders;
  float density_scale, emission_scale, step_size, scattering_scale;
  float4 scat_color_aniso;          // scattering colour, Henyey-Greenstein anisotropy
  float4 scat_albedo;               // scattering albedo (multiple orders)
  float4 clip[8];                   // (a, b, c, d): keep (a, b, c) . p >= d
  float4 reserved;
};
static_assert(sizeof(RefVolume) == 288, "RefVolume must match the 72-float scene-description record");

// One resident scene of the pool: its TLAS root and its lighting.  Emitter
// indices of the alias table are scene-local (add emitter_base).
struct __align__(16) SceneRec {
  uint32_t tlas_root;
  uint32_t emitter_base;
  uint32_t num_emitters;
  float emissive_weight;       // Scene.emissive_light_weight
  uint32_t light_base;
  uint32_t num_lights;
  uint32_t env_kind;           // olc_environment_kind
  float env_rotation;
  float4 env_color;            // colour * intensity
  const float* env_image;      // equirect RGB
  uint32_t env_w, env_h;
  const float* volume;         // density grid (z, y, x)
  uint32_t volume_present;
  uint32_t vol_nx, vol_ny, vol_nz;
  float4 vol_w2b0, vol_w2b1, vol_w2b2;   // world -> unit box
  float vol_sigma_t_scale;
  float vol_albedo;
  float vol_max_density;
  uint32_t pad;
  // textures (tex_words == nullptr: an untextured scene)
  const uint32_t* tex_words;     // Scene.texture_data layout
  const float4* tex_bindings;    // 2 per binding: (texture, cos, sin, texcoord set), (offset, scale)
  const float4* tex_attr;        // 6 per triangle slot of the scene: per vertex (uv0, uv1), (tangent, handedness)
  const float4* mat_tex;         // 3 per material of the scene: binding indices and map parameters
  const float* srgb_lut;         // 256 sRGB-to-linear values
  uint32_t slot_base;            // first triangle slot of the scene
  uint32_t material_base;        // first material record of the scene
  // volumes in the reference's model (reference-compatible mode; none: 0)
  const RefVolume* ref_vols;
  const float* ref_grid;         // normalized values of every volume
  const float4* ref_lut;         // transfer-function entries of every volume
  uint32_t num_ref_vols;
  uint32_t pad2[3];
};

// Device view of the scene pool shared by every resident scene: all BLAS and
// TLAS nodes, triangle slots, instances, materials, emitters and lights of
// all scenes live in one set of arrays, so a wavefront may mix rays of
// different scenes and each ray needs only its scene's TLAS root.
struct SceneView {
  const BvhNode* nodes;          // BLAS and TLAS nodes
  const BvhNode4* wide;          // their BVH4 form, same indices (traversal reads only these)
  const float4* tri_verts;       // 3 float4 per triangle slot (object space)
  const float4* tri_normals;     // 3 float4 per triangle slot (object space)
  const uint32_t* tri_index;     // slot -> mesh-local triangle index (packed index for baked triangles)
  const uint32_t* tri_owner;     // slot -> original instance (baked triangles only)
  const InstanceRec* instances;
  const MaterialRec* materials;
  const MaterialAux* material_aux;
  const EmitterRec* emitters;
  const AliasEntry* emitter_alias;
  const LightRec* lights;
  const SceneRec* scenes;
};

// ---------------------------------------------------------------------------
// Wavefront queues (structure of arrays, 16-byte elements).
// ---------------------------------------------------------------------------
struct RayQueue {
  float4* origin_tmin;     // origin.xyz, t_min
  float4* dir_root;        // direction.xyz, TLAS root of the ray's scene (bits); t_max is infinite
  uint32_t* path;          // path slot
};

struct HitBuf {
  float4* tuv_slot;        // t, u, v, triangle slot bits (t < 0: miss)
  uint32_t* instance;      // instance index
};

struct ShadowQueue {
  float4* origin_tmax;     // origin.xyz, t_max
  float4* dir_path;        // direction.xyz, path slot bits
  float4* contrib_root;    // unoccluded contribution rgb, TLAS root (bits)
};

struct PathState {
  float4* throughput;      // rgb, previous BSDF pdf
  float4* radiance;        // rgb, unused
  uint4* meta;             // pixel, sample, bounce | flags << 8, job
  float4* ior_stack;       // 4 per path: indices of refraction of the media entered, entries 1..15
  float2* cone;            // ray cone (width, spread) of the path's next ray; textured scenes only
  float4* shadow;          // rgb the path's unoccluded shadow rays carried, unused; written only by the
                           // any-hit kernel, so the shadow rays of a bounce run beside later bounces
};

#define OLC_PATH_FLAG_PREV_NEE 1u     // the previous vertex sampled area lights
#define OLC_PATH_FLAG_PREV_RESTIR 2u  // area lights of the previous vertex came from ReSTIR
// Depth of the path's medium stack minus one (the reference's medium depth,
// metadata.w >> 8, wavefront_shade.comp:447); entry 0 is the outside, IOR 1.
#define OLC_PATH_DEPTH_SHIFT 4u
#define OLC_PATH_DEPTH_MASK (15u << OLC_PATH_DEPTH_SHIFT)
#define OLC_MAX_MEDIUM_DEPTH 16u      // entry 0 plus the 15 stored ones (the reference's depth)

// Fixed-point scale of the per-pixel radiance accumulator.  Sums of
// non-negative samples in unsigned 64-bit fixed point are independent of the
// order of the atomic additions, so every launch shape, chunking and batch
// mix produces the same bits.
//
// Each sample's channel is clamped to [0, 2^19 - 1] before scaling, so one
// sample adds below 2^47 and a pixel's sum over the largest frame accepted
// (65,536 = 2^16 samples, also when its sample range is split into shards)
// stays below 2^63: it fits an unsigned 64-bit word and also the signed
// 64-bit tensors the multi-GPU all-reduce adds, without wrapping.
#define OLC_PI_F 3.14159265358979f
#define OLC_ACCUM_SHIFT 28
#define OLC_ACCUM_SCALE 268435456.0f
#define OLC_SAMPLE_CLAMP 524287.0f
#define OLC_MAX_FRAME_SAMPLES 65536u

// One segment of a render job inside a chunk: the job's camera, image,
// samples, transport knobs and scene, plus where this segment's paths sit in
// the chunk and where the job's pixels and reservoirs live.  Every wavefront
// kernel reads its paths' records from device memory, so a plain frame is a
// chunk sequence over one job, batches and served requests mix many, and a
// captured graph replays for new cameras and mixes after one table copy.
struct __align__(16) JobRec {
  float4 cam_pos;          // xyz, x scale (aspect*half_height | half horizontal angle)
  float4 cam_forward;      // xyz, y scale (half_height | half vertical angle)
  float4 cam_right;        // xyz, 0
  float4 cam_up;           // xyz, 0
  uint32_t projection;
  uint32_t width, height;
  uint32_t spp;
  uint32_t frame;          // seed + frame_index
  uint32_t npix;
  uint32_t max_bounces;
  uint32_t mode;           // olc_mode
  uint32_t rr_start;
  float rr_min_survival;
  uint32_t restir;         // ReSTIR DI at the primary vertex
  uint32_t nee;            // next-event estimation (production mode)
  uint32_t scene;          // SceneRec index
  uint32_t history;        // ReSTIR temporal history valid for this job
  uint32_t products;       // write first-sample primary-hit products
  uint32_t sample_base;    // global index of the job's first sample (a shard of a frame's samples)
  unsigned long long seg_begin;       // chunk-local index of the segment's first path
  unsigned long long seg_first;       // job-local index (sample * npix + pixel) of that path
  unsigned long long pixel_base;      // first pixel of the job in the accumulator and outputs
  unsigned long long reservoir_base;  // reservoir of (sample, pixel) = base + sample * npix + pixel (mod 2^64)
  unsigned long long history_base;    // first reservoir of its temporal history
  unsigned long long lum_base;        // per-sample luminance of (sample, pixel) at base + sample * npix + pixel;
                                      // ~0: not kept
};

// Header of one chunk's table in device memory, followed by num_segments
// JobRec entries ordered by seg_begin.  The kernels read the path count from
// here rather than from launch parameters, so one captured graph serves every
// chunk with the same bounce count.
//
// ReSTIR reservoirs carry the stamp of the chunk that wrote them; stamps grow
// by one per chunk, so a reservoir is this chunk's only if its stamp equals
// `stamp`, and the previous plain frame's (its chunks' stamps form a range)
// only if its stamp lies in [history_first, history_last].
struct __align__(16) ChunkHeader {
  uint32_t count;          // paths in the chunk
  uint32_t num_segments;
  uint32_t stamp;          // ReSTIR validity stamp of this chunk
  uint32_t history_first;  // stamps of the temporal history's reservoirs
  uint32_t history_last;
  uint32_t pad[3];
};

// Jobs whose last paths finished in a run: resolved from the accumulator.
struct __align__(16) ResolveEntry {
  unsigned long long pixel_base;
  uint32_t npix;
  uint32_t spp;
};

// Work counters kept in device memory, zeroed once per chunk.
#define OLC_MAX_BOUNCES 64
struct Counters {
  uint32_t queue_count[OLC_MAX_BOUNCES + 2];    // rays in the queue of each bounce
  uint32_t shadow_count[OLC_MAX_BOUNCES + 2];   // shadow rays emitted at each bounce
  uint32_t closest_cursor[OLC_MAX_BOUNCES + 2]; // persistent closest-hit work cursor
  uint32_t shadow_cursor[OLC_MAX_BOUNCES + 2];  // persistent any-hit work cursor
  uint32_t miss_count[OLC_MAX_BOUNCES + 2];     // rays of each bounce that left the scene
  uint32_t shade_cursor[OLC_MAX_BOUNCES + 2];   // shading work cursor (32-path grabs)
  uint32_t overflow;
  uint32_t traversal_errors;
  uint32_t nan_samples;
  uint32_t pad;
};
