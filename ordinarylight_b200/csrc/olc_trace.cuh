// Software two-level BVH traversal: closest hit and any hit.
//
// Replaces the hardware ray queries of the reference wavefront
// (nativeTraceSurface, ordinarylight/shaders/wavefront_intersect.comp:96-235;
// nativeOccluded in ordinarylight/shaders/transport_v1/lighting.glsl).
// * TLAS and BLAS nodes share one node pool; a TLAS leaf is one instance.
//   Traversal reads the BVH4 form of the pool (BvhNode4: up to four
//   descendants of a BVH2 node in one 128-byte line, collapsed greedily by
//   surface area), so each dependent fetch descends about two levels of the
//   binary hierarchy.  A ray picks each axis's near and far box planes once
//   from its direction's signs, so the slab test needs no per-axis min/max.
//   Entering an instance transforms the ray to object space (t is preserved
//   because the direction is not renormalised) and pushes a marker that
//   restores the world ray when the instance's subtree is exhausted; the
//   world ray and its derived terms are kept meanwhile in OLC_RAY_SAVE shared
//   words per thread instead of being recomputed.
// * The traversal stack lives in shared memory (STACK entries per thread,
//   entry k of thread t at k * blockDim.x + t, so a warp's pushes hit 32
//   distinct banks), followed by the per-thread shared words in the same
//   column layout; a launch gives (STACK + OLC_RAY_SAVE) * blockDim.x words.
//   What a ray needs only at instance transitions or at its end (the world
//   ray, the closest hit's barycentrics) lives there rather than in
//   registers, which keeps eight blocks of 128 threads resident per SM.
//   Deeper entries spill to a bounded local array.  A push beyond both is
//   counted as a traversal error instead of writing out of bounds.
// * Triangles use the watertight test of Woop, Benthin and Wald (JCGT 2013):
//   the edge functions are evaluated without FMA contraction so that an edge
//   shared by two triangles gets exactly negated values, with a double
//   precision re-evaluation when an edge function is exactly zero.
// * Closest-hit ties (equal t) resolve to the lowest packed triangle index,
//   the rule of ReferencePathTracer._intersect (strict "<" over triangles in
//   packed order, ordinarylight/renderers/reference/path_tracer.py:159-175),
//   which also makes the result independent of traversal order.
#pragma once

#include "olc_common.cuh"

#define OLC_SPILL 96
// Shared words per thread beyond the stack: the world ray's derived terms
// (0-9), restored on leaving an instance; the world ray's origin (10-12) and
// direction (13-15); the closest hit's barycentrics (16-17).
#define OLC_RAY_SAVE 18
#define OLC_SAVE_ORIGIN 10
#define OLC_SAVE_DIR 13
#define OLC_SAVE_UV 16
#define OLC_NO_INSTANCE 0xffffffffu
#define OLC_MARKER 0x7fffffff
#define OLC_TRAVERSAL_BUDGET (1u << 22)

struct TraceRay {
  float3 o;
  float3 inv, oinv;
  int kp;              // shear permutation kx | ky << 2 | kz << 4
  float sx, sy, sz;
  int nx, ny, nz;      // float4 index of each axis's near plane in a BvhNode4 (its far plane is index ^ 1)
};

OLC_D void setup_ray(TraceRay& r, float3 o, float3 d) {
  r.o = o;
  float dx = fabsf(d.x) < 1e-20f ? copysignf(1e-20f, d.x) : d.x;
  float dy = fabsf(d.y) < 1e-20f ? copysignf(1e-20f, d.y) : d.y;
  float dz = fabsf(d.z) < 1e-20f ? copysignf(1e-20f, d.z) : d.z;
  r.inv = f3(1.0f / dx, 1.0f / dy, 1.0f / dz);
  r.oinv = f3(o.x * r.inv.x, o.y * r.inv.y, o.z * r.inv.z);
  r.nx = r.inv.x < 0.0f ? 1 : 0;
  r.ny = r.inv.y < 0.0f ? 3 : 2;
  r.nz = r.inv.z < 0.0f ? 5 : 4;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
  int kx = kz + 1 == 3 ? 0 : kz + 1;
  int ky = kx + 1 == 3 ? 0 : kx + 1;
  float dkz = get(d, kz);
  if (dkz < 0.0f) { int t = kx; kx = ky; ky = t; }
  r.kp = kx | (ky << 2) | (kz << 4);
  r.sx = get(d, kx) / dkz;
  r.sy = get(d, ky) / dkz;
  r.sz = 1.0f / dkz;
}

// Watertight ray/triangle test.  Returns true with t, b1 (weight of v1),
// b2 (weight of v2) when the ray hits with t_min < t <= t_max.
OLC_D bool intersect_triangle(const TraceRay& r, float3 v0, float3 v1, float3 v2,
                              float t_min, float t_max, float& t_out, float& b1, float& b2) {
  const int kx = r.kp & 3, ky = (r.kp >> 2) & 3, kz = r.kp >> 4;
  float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
  float Akz = get(A, kz), Bkz = get(B, kz), Ckz = get(C, kz);
  float Ax = __fmaf_rn(-r.sx, Akz, get(A, kx));
  float Ay = __fmaf_rn(-r.sy, Akz, get(A, ky));
  float Bx = __fmaf_rn(-r.sx, Bkz, get(B, kx));
  float By = __fmaf_rn(-r.sy, Bkz, get(B, ky));
  float Cx = __fmaf_rn(-r.sx, Ckz, get(C, kx));
  float Cy = __fmaf_rn(-r.sy, Ckz, get(C, ky));
  float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
  float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
  float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
  if (U == 0.0f || V == 0.0f || W == 0.0f) {
    double CxBy = (double)Cx * (double)By, CyBx = (double)Cy * (double)Bx;
    U = (float)(CxBy - CyBx);
    double AxCy = (double)Ax * (double)Cy, AyCx = (double)Ay * (double)Cx;
    V = (float)(AxCy - AyCx);
    double BxAy = (double)Bx * (double)Ay, ByAx = (double)By * (double)Ax;
    W = (float)(BxAy - ByAx);
  }
  if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
  float det = U + V + W;
  if (det == 0.0f) return false;
  float Az = r.sz * Akz, Bz = r.sz * Bkz, Cz = r.sz * Ckz;
  float T = U * Az + V * Bz + W * Cz;
  float t = __fdiv_rn(T, det);
  if (!(t > t_min) || !(t <= t_max)) return false;
  float rcp = 1.0f / det;
  t_out = t;
  b1 = V * rcp;
  b2 = W * rcp;
  return true;
}

// Save / restore the terms setup_ray derives from the world ray (o, d): the
// slab reciprocals, the shear permutation and constants; restoring also reads
// back the world origin.  `w` is this thread's column (stride threads).
OLC_D void save_ray(float* w, int stride, const TraceRay& r) {
  w[0 * stride] = r.inv.x; w[1 * stride] = r.inv.y; w[2 * stride] = r.inv.z;
  w[3 * stride] = r.oinv.x; w[4 * stride] = r.oinv.y; w[5 * stride] = r.oinv.z;
  w[6 * stride] = r.sx; w[7 * stride] = r.sy; w[8 * stride] = r.sz;
  w[9 * stride] = __int_as_float(r.kp | (r.nx << 6) | (r.ny << 9) | (r.nz << 12));
}
OLC_D void restore_ray(const float* w, int stride, TraceRay& r) {
  r.o = f3(w[(OLC_SAVE_ORIGIN + 0) * stride], w[(OLC_SAVE_ORIGIN + 1) * stride], w[(OLC_SAVE_ORIGIN + 2) * stride]);
  r.inv = f3(w[0 * stride], w[1 * stride], w[2 * stride]);
  r.oinv = f3(w[3 * stride], w[4 * stride], w[5 * stride]);
  r.sx = w[6 * stride]; r.sy = w[7 * stride]; r.sz = w[8 * stride];
  const int k = __float_as_int(w[9 * stride]);
  r.kp = k & 63;
  r.nx = (k >> 6) & 7; r.ny = (k >> 9) & 7; r.nz = (k >> 12) & 7;
}

struct HitResult {
  float t, u, v;
  uint32_t slot;       // triangle slot (BVH order)
  uint32_t instance;   // instance index (0xffffffff: miss)
  uint32_t packed;     // packed triangle index (tie-break key)
};

template <int STACK>
struct TraversalStack {
  int* smem;           // this thread's column in the shared stack
  int stride;
  int sp;
  int* spill;          // this thread's local overflow array (OLC_SPILL entries)

  OLC_D void init(int* base, int tid, int threads, int* spill_area) {
    smem = base + tid;
    stride = threads;
    sp = 0;
    spill = spill_area;
  }
  OLC_D bool push(int v, uint32_t& err) {
    if (sp < STACK) { smem[sp * stride] = v; ++sp; return true; }
    if (sp < STACK + OLC_SPILL) { spill[sp - STACK] = v; ++sp; return true; }
    err = 1u;
    return false;
  }
  OLC_D int pop() {
    --sp;
    return sp < STACK ? smem[sp * stride] : spill[sp - STACK];
  }
};

OLC_D void load_instance_w2o(const InstanceRec* inst, uint32_t i, Affine& w2o, uint32_t& root) {
  const float4* p = reinterpret_cast<const float4*>(inst + i);
  w2o.r0 = __ldg(p + 0);
  w2o.r1 = __ldg(p + 1);
  w2o.r2 = __ldg(p + 2);
  root = __ldg(&inst[i].blas_root);
}

// Packed triangle index (Scene.triangles order) of triangle slot `slot` hit
// through instance `inst`: the closest-hit tie-break key.  Record 0, the
// identity instance of baked world-space triangles, has offset 0.
OLC_D uint32_t packed_index(const SceneView& s, uint32_t inst, uint32_t slot) {
  return __ldg(&s.instances[inst].prim_offset) + __ldg(s.tri_index + slot);
}

// Three-input float max / min (one instruction on sm_100).
OLC_D float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
OLC_D float fmin3(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Slab test of one child box (Kay and Kajiya) on its near and far planes
// (chosen per ray by the direction's signs, so no min/max per axis), with the
// conservative far bound of robust traversal (Ize 2013): a few ulps of slack
// so rounding in the slab test never culls a box the ray touches.  Unused
// slots hold an inverted box (lo +inf, hi -inf), whose near distance is +inf
// and far distance -inf for every ray.
OLC_D bool child_box(float nxp, float fxp, float nyp, float fyp, float nzp, float fzp, const TraceRay& r,
                     float t_min, float t_max, float& near_t) {
  const float n = fmax3(__fmaf_rn(nxp, r.inv.x, -r.oinv.x), __fmaf_rn(nyp, r.inv.y, -r.oinv.y),
                        fmaxf(__fmaf_rn(nzp, r.inv.z, -r.oinv.z), t_min));
  const float f = fmin3(__fmaf_rn(fxp, r.inv.x, -r.oinv.x), __fmaf_rn(fyp, r.inv.y, -r.oinv.y),
                        fminf(__fmaf_rn(fzp, r.inv.z, -r.oinv.z), t_max));
  near_t = n;
  return n <= f * 1.0000004f;
}

// One compare-exchange of a sorting network over (key, child) pairs.
OLC_D void order_pair(float& ka, int& ca, float& kb, int& cb) {
  const bool swap = kb < ka;
  const float k = swap ? kb : ka;
  const int c = swap ? cb : ca;
  kb = swap ? ka : kb;
  cb = swap ? ca : cb;
  ka = k;
  ca = c;
}

// Resumable traversal of the two-level structure.  ANY_HIT stops at the
// first hit in (t_min, t_max).  advance() runs at most `iterations` loop
// iterations (node visits, leaf tests, instance transitions) and returns true
// once the ray is finished, so a persistent kernel can refill lanes whose rays
// finished while the other lanes of the warp are still traversing.
//
// Register state is kept to what every iteration reads: the current ray, the
// closest t with its slot and instance, the node, the instance being walked
// (OLC_NO_INSTANCE in the TLAS) and the stack pointer.  The world ray and the
// closest hit's barycentrics live in the thread's shared words, and the
// packed tie-break index is looked up only when two hits have equal t.
template <int STACK, bool ANY_HIT>
struct Traversal {
  TraceRay ray;
  float t_min;
  float hit_t;
  uint32_t hit_slot;   // triangle slot (BVH order) of the closest hit so far
  uint32_t hit_inst;   // its instance; OLC_NO_INSTANCE while nothing was hit
  int node;
  uint32_t cur_inst;   // instance whose BLAS is being walked, or OLC_NO_INSTANCE
  uint32_t budget;
  float* save;         // this thread's column of OLC_RAY_SAVE shared words
  TraversalStack<STACK> st;

  OLC_D bool found() const { return hit_inst != OLC_NO_INSTANCE; }
  OLC_D float hit_u() const { return save[OLC_SAVE_UV * st.stride]; }
  OLC_D float hit_v() const { return save[(OLC_SAVE_UV + 1) * st.stride]; }
  OLC_D HitResult result(const SceneView& s) const {
    HitResult h;
    h.t = hit_t;
    h.slot = hit_slot;
    h.instance = hit_inst;
    h.u = found() ? hit_u() : 0.0f;
    h.v = found() ? hit_v() : 0.0f;
    h.packed = found() ? packed_index(s, hit_inst, hit_slot) : 0xffffffffu;
    return h;
  }

  OLC_D void begin(const SceneView& s, float3 o, float3 d, float tmin, float tmax, uint32_t tlas_root,
                   int* smem_base, int* spill_area) {
    st.init(smem_base, threadIdx.x, blockDim.x, spill_area);
    save = reinterpret_cast<float*>(smem_base + STACK * blockDim.x) + threadIdx.x;
    const int w = st.stride;
    save[(OLC_SAVE_ORIGIN + 0) * w] = o.x;
    save[(OLC_SAVE_ORIGIN + 1) * w] = o.y;
    save[(OLC_SAVE_ORIGIN + 2) * w] = o.z;
    save[(OLC_SAVE_DIR + 0) * w] = d.x;
    save[(OLC_SAVE_DIR + 1) * w] = d.y;
    save[(OLC_SAVE_DIR + 2) * w] = d.z;
    t_min = tmin;
    setup_ray(ray, o, d);
    save_ray(save, w, ray);   // the world ray's terms, restored on leaving an instance
    hit_t = tmax;
    hit_inst = OLC_NO_INSTANCE;
    hit_slot = 0;
    cur_inst = OLC_NO_INSTANCE;
    node = (int)tlas_root;
    // A well-formed tree is acyclic and finite; the budget only guarantees
    // the loop ends (and reports an error) should the structure be corrupt.
    budget = OLC_TRAVERSAL_BUDGET;
  }

  // A triangle hit at t (<= hit_t) through instance `inst`: keep it if it is
  // nearer, or equally near with a lower packed index.  Returns true when the
  // ray is finished (any hit).
  OLC_D bool offer(const SceneView& s, uint32_t inst, uint32_t slot, float t, float b1, float b2) {
    if (ANY_HIT) {
      hit_t = t;
      hit_inst = inst;
      hit_slot = slot;
      return true;
    }
    if (hit_inst == OLC_NO_INSTANCE || t < hit_t ||
        packed_index(s, inst, slot) < packed_index(s, hit_inst, hit_slot)) {
      hit_t = t;
      hit_inst = inst;
      hit_slot = slot;
      save[OLC_SAVE_UV * st.stride] = b1;
      save[(OLC_SAVE_UV + 1) * st.stride] = b2;
    }
    return false;
  }

  OLC_D bool advance(const SceneView& s, int iterations, uint32_t& err) {
    // The budget is charged per call, not per iteration (a call may charge
    // more than it uses; the bound only has to end a corrupt walk).
    const uint32_t steps = min((uint32_t)iterations, budget);
    budget -= steps;
    for (uint32_t it = 0; it < steps; ++it) {
      // `node` is never the instance marker here: a marker is only popped,
      // and the pop below steps past it.
      if (node >= 0) {
        // BVH4 node: test the four child boxes, descend into the nearest
        // hit child and push the others, farthest first (closest hit) or in
        // slot order (any hit, where the order changes nothing but time).
        const float4* p = reinterpret_cast<const float4*>(s.wide + node);
        const float4 nx = __ldg(p + ray.nx), fx = __ldg(p + (ray.nx ^ 1));
        const float4 ny = __ldg(p + ray.ny), fy = __ldg(p + (ray.ny ^ 1));
        const float4 nz = __ldg(p + ray.nz), fz = __ldg(p + (ray.nz ^ 1));
        const int4 ch = __ldg(reinterpret_cast<const int4*>(p + 6));
        float n0, n1, n2, n3;
        const bool h0 = child_box(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, ray, t_min, hit_t, n0);
        const bool h1 = child_box(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, ray, t_min, hit_t, n1);
        const bool h2 = child_box(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, ray, t_min, hit_t, n2);
        const bool h3 = child_box(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, ray, t_min, hit_t, n3);
        if (ANY_HIT) {
          if (h0 || h1 || h2 || h3) {
            int next = OLC_EMPTY_CHILD;
            if (h3) next = ch.w;
            if (h2) { if (next != OLC_EMPTY_CHILD) st.push(next, err); next = ch.z; }
            if (h1) { if (next != OLC_EMPTY_CHILD) st.push(next, err); next = ch.y; }
            if (h0) { if (next != OLC_EMPTY_CHILD) st.push(next, err); next = ch.x; }
            node = next;
            continue;
          }
          // nothing to enter: fall through to the pop
        } else if (const int hits = (int)h0 + (int)h1 + (int)h2 + (int)h3) {
          // misses sort last (+inf); a hit's key is finite
          float k0 = h0 ? fminf(n0, 3.0e38f) : CUDART_INF_F, k1 = h1 ? fminf(n1, 3.0e38f) : CUDART_INF_F;
          float k2 = h2 ? fminf(n2, 3.0e38f) : CUDART_INF_F, k3 = h3 ? fminf(n3, 3.0e38f) : CUDART_INF_F;
          int c0 = ch.x, c1 = ch.y, c2 = ch.z, c3 = ch.w;
          order_pair(k0, c0, k1, c1);
          order_pair(k2, c2, k3, c3);
          order_pair(k0, c0, k2, c2);
          order_pair(k1, c1, k3, c3);
          order_pair(k1, c1, k2, c2);
          if (hits > 3) st.push(c3, err);
          if (hits > 2) st.push(c2, err);
          if (hits > 1) st.push(c1, err);
          node = c0;
          continue;
        }
      } else {
        const uint32_t first = olc_leaf_first(node);
        const uint32_t count = olc_leaf_count(node);
        if (cur_inst == OLC_NO_INSTANCE && count == OLC_TLAS_LEAF_TRIANGLE) {
          // baked world-space triangle referenced directly by the TLAS
          const uint32_t slot = first;
          const float4* tv = s.tri_verts + 3u * slot;
          float3 v0 = f3(__ldg(tv + 0)), v1 = f3(__ldg(tv + 1)), v2 = f3(__ldg(tv + 2));
          float t, b1, b2;
          if (intersect_triangle(ray, v0, v1, v2, t_min, hit_t, t, b1, b2) &&
              offer(s, OLC_IDENTITY_INSTANCE, slot, t, b1, b2))
            return true;
        } else if (cur_inst == OLC_NO_INSTANCE) {
          // instance leaf (TLAS leaves hold one instance)
          Affine w2o;
          uint32_t root;
          load_instance_w2o(s.instances, first, w2o, root);
          if (st.push(OLC_MARKER, err)) {
            const int w = st.stride;
            const float3 wd = f3(save[(OLC_SAVE_DIR + 0) * w], save[(OLC_SAVE_DIR + 1) * w],
                                 save[(OLC_SAVE_DIR + 2) * w]);
            setup_ray(ray, xform_point(w2o, ray.o), xform_vector(w2o, wd));
            cur_inst = first;
            node = (int)root;
            continue;
          }
        } else {
          for (uint32_t k = 0; k < count; ++k) {
            const uint32_t slot = first + k;
            const float4* tv = s.tri_verts + 3u * slot;
            float3 v0 = f3(__ldg(tv + 0)), v1 = f3(__ldg(tv + 1)), v2 = f3(__ldg(tv + 2));
            float t, b1, b2;
            if (intersect_triangle(ray, v0, v1, v2, t_min, hit_t, t, b1, b2) &&
                offer(s, cur_inst, slot, t, b1, b2))
              return true;
          }
        }
      }
      // pop
      if (st.sp == 0) return true;
      node = st.pop();
      if (node == OLC_MARKER) {
        cur_inst = OLC_NO_INSTANCE;
        restore_ray(save, st.stride, ray);
        if (st.sp == 0) return true;
        node = st.pop();
      }
    }
    if (budget == 0u) {
      err = 1u;
      return true;
    }
    return false;
  }
};

// Blocking traversal: the whole ray in one call.  Returns true on a hit.
template <int STACK, bool ANY_HIT>
OLC_D bool olc_traverse(const SceneView& s, uint32_t tlas_root, float3 wo, float3 wd, float t_min, float t_max,
                        HitResult& hit, int* smem_base, uint32_t& err) {
  Traversal<STACK, ANY_HIT> tr;
  int spill[OLC_SPILL];
  tr.begin(s, wo, wd, t_min, t_max, tlas_root, smem_base, spill);
  while (!tr.advance(s, 1 << 30, err)) {
  }
  hit = tr.result(s);
  return tr.found();
}
