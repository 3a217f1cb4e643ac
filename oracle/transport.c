/* ORACLE - test infrastructure only, never part of the product path.
 *
 * CPU restatement (C, double precision) of the reference GPU wavefront's
 * production transport, the estimator the CUDA renderer's production mode
 * must agree with in expectation.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU legs may load it, as the checker.
 *
 * What it restates (OrdinaryLight, ordinarylight/shaders/...):
 *
 *  BSDF (ordinaryshade_primary.glsl:506-609, the ordinarylight_pbr_* helpers
 *  that samplePbr calls, transport_v1/lighting.glsl:218-246):
 *    f0 = mix(0.04, base, metallic); F = f0 + (1 - f0)(1 - v.h)^5;
 *    alpha = max(roughness^2, 0.0009), a2 = alpha^2;
 *    D = a2 / (pi ((n.h)^2 (a2 - 1) + 1)^2) (uncapped; see ggx_d);
 *    G1(x) = 2x / max(x + sqrt(a2 + (1 - a2) x^2), 1e-6);
 *    f = (1 - F)(1 - metallic) base / pi + F D G1(n.v) G1(n.l) / max(4 n.v n.l, 1e-6);
 *    p_spec = clamp(max(f0), 0.1, 0.9);
 *    pdf = mix(n.l / pi, D n.h / (4 max(v.h, 1e-6)), p_spec), floored at 1e-6.
 *  Sampling: lobe with p_spec; diffuse = cosine hemisphere in the frame
 *  tangent = normalize(cross(n, z or y)); specular = GGX half vector
 *  cos = sqrt((1 - u) / (1 + (a2 - 1) u)), reflected.  A reflection
 *  below the surface: the reference draws a fresh cosine direction but keeps
 *  the mixture pdf (lighting.glsl:238-241), which overstates the weight of
 *  such directions; OLO_INVALID_RESAMPLE reproduces that, the default ends
 *  the path there (the unbiased estimator of the same BSDF).
 *
 *  Next-event estimation at a non-transmissive surface vertex below the
 *  bounce limit (wavefront_shade.comp:507-541):
 *    - every analytic light (samplePointLights, lighting.glsl:260-312):
 *      directional / point / spot attenuation with smoothstep cone, range
 *      cut-off, shadow ray from hit + 0.002 n, t in [0.001, d - 0.004]
 *      (10000 for directional); no MIS (delta lights);
 *    - one area-light sample (sampleAreaLightTechnique, :336-404): emitter by
 *      binary search of the power CDF (selection <= cdf), point
 *      (1 - sqrt u) a + sqrt u (1 - v) b + sqrt u v c, light pdf
 *      sel d^2 / max(cos_l A, 1e-6), power-heuristic weight against the
 *      BSDF pdf, contribution f Le cos w / pdf;
 *    - with the environment sampled (OLO_ENV_NEE): one cosine-hemisphere
 *      direction (sampleEnvironmentTechnique, :618-647) with the reference's
 *      constant weight pair: 1/2 on this sample and 1/2 on environment
 *      radiance reached by BSDF sampling from a surface vertex
 *      (ordinarylight_environment_mis, ordinaryshade_primary.glsl:727-734;
 *      wavefront_shade.comp:331-348), so the two weights sum to one.
 *  Emission of a hit (wavefront_shade.comp:412-433): visible when entering or
 *  two-sided; after a surface vertex that sampled area lights, weighted by
 *  power(prev_pdf, sel d^2 / (cos_l A)) with sel = A lum / total power.
 *  Russian roulette (:569-580): from bounce rr_start, survival
 *  clamp(max(throughput), rr_min, 0.95).  Path length: emission is added at
 *  every vertex; NEE and continuation only while bounce + 1 < max_bounces
 *  (:433-440).  The reference's throughput cut-off at 1e-4 (:322-327) is a
 *  biased early exit and is not restated.
 *
 * Independent of the CUDA renderer by construction: its own bounding volume
 * hierarchy (median split), Moller-Trumbore in double precision, its own
 * random numbers (SplitMix64 streams keyed by seed, pixel and sample), and
 * the reference's estimator structure (all analytic lights, CDF emitter
 * choice, environment NEE) where the CUDA renderer draws one light per vertex
 * from an alias table and leaves the environment to BSDF sampling.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OLO_PI 3.14159265358979323846

enum {
  OLO_NEE = 1,               /* next-event estimation (lights + one area sample) */
  OLO_ENV_NEE = 2,           /* also sample the environment at surface vertices */
  OLO_INVALID_RESAMPLE = 4,  /* the reference's resampling of invalid reflections */
};

typedef struct {
  int32_t num_triangles;
  const float* positions;   /* (T, 3, 3) world space */
  const float* normals;     /* (T, 3, 3) world vertex normals */
  const int32_t* material;  /* (T) index into materials */
  int32_t num_materials;
  const float* materials;   /* (M, 10): base rgb, roughness, metallic, emission rgb, two_sided, unused */
  int32_t num_emitters;
  const int32_t* emitter_triangle;  /* (E) triangle of each emitter record */
  const double* emitter_cdf;        /* (E) cumulative power, last = 1 */
  const double* emitter_pdf;        /* (E) selection probability */
  double total_power;               /* sum of area * luminance over emitters */
  int32_t num_lights;
  const float* lights;      /* (L, 16): type, position xyz, direction xyz, radiance rgb, range, cos inner, cos outer */
  int32_t env_kind;         /* 0 analytic sky of the GPU shaders, 1 constant */
  float env_color[3];
} olo_scene;

typedef struct {
  int32_t projection;       /* 0 perspective, 1 orthographic, 2 panoramic */
  float position[3], forward[3], right[3], up[3];
  float scale_x, scale_y;   /* aspect * tan(fov / 2) and tan(fov / 2); half sizes; half angles */
} olo_camera;

typedef struct {
  int32_t width, height;
  int32_t x0, y0, win_w, win_h;   /* the pixel window to render */
  int32_t samples, first_sample;
  int32_t max_bounces;
  int32_t rr_start;
  float rr_min_survival;
  uint32_t flags;
  uint64_t seed;
} olo_params;

/* ---- vectors ---------------------------------------------------------- */
typedef struct { double x, y, z; } v3;
static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 scl(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double len(v3 a) { return sqrt(dot(a, a)); }
static inline v3 nrm(v3 a) { double l = len(a); return l > 0.0 ? scl(a, 1.0 / l) : a; }
static inline double maxc(v3 a) { return fmax(a.x, fmax(a.y, a.z)); }
static inline double clampd(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }
static inline v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

/* ---- random numbers: SplitMix64 ---------------------------------------- */
static inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
typedef struct { uint64_t s; } rng_t;
static inline double rnd(rng_t* r) {
  r->s += 0x9e3779b97f4a7c15ull;
  return (double)(mix64(r->s) >> 11) * (1.0 / 9007199254740992.0);
}

/* ---- bounding volume hierarchy ------------------------------------------ */
typedef struct {
  double lo[3], hi[3];
  int32_t left, count;      /* inner: left child index (right = left + 1), count = 0; leaf: first, count */
} node_t;

typedef struct {
  node_t* nodes;
  int32_t* order;
  int32_t num_nodes;
  const olo_scene* s;
  v3* centroid;
} bvh_t;

static void tri_box(const olo_scene* s, int32_t t, double* lo, double* hi) {
  for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
  for (int k = 0; k < 3; ++k)
    for (int a = 0; a < 3; ++a) {
      double v = s->positions[9 * t + 3 * k + a];
      lo[a] = fmin(lo[a], v);
      hi[a] = fmax(hi[a], v);
    }
}

static int32_t g_sort_axis;
static const v3* g_sort_centroid;
static int cmp_centroid(const void* a, const void* b) {
  const v3* c = g_sort_centroid;
  int32_t i = *(const int32_t*)a, j = *(const int32_t*)b;
  double x = g_sort_axis == 0 ? c[i].x : (g_sort_axis == 1 ? c[i].y : c[i].z);
  double y = g_sort_axis == 0 ? c[j].x : (g_sort_axis == 1 ? c[j].y : c[j].z);
  return x < y ? -1 : (x > y ? 1 : (i < j ? -1 : (i > j)));
}

static void build_node(bvh_t* b, int32_t index, int32_t first, int32_t count) {
  node_t* n = &b->nodes[index];
  for (int a = 0; a < 3; ++a) { n->lo[a] = INFINITY; n->hi[a] = -INFINITY; }
  double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int32_t k = first; k < first + count; ++k) {
    double lo[3], hi[3];
    tri_box(b->s, b->order[k], lo, hi);
    const v3 c = b->centroid[b->order[k]];
    const double cc[3] = {c.x, c.y, c.z};
    for (int a = 0; a < 3; ++a) {
      n->lo[a] = fmin(n->lo[a], lo[a]);
      n->hi[a] = fmax(n->hi[a], hi[a]);
      clo[a] = fmin(clo[a], cc[a]);
      chi[a] = fmax(chi[a], cc[a]);
    }
  }
  if (count <= 4) {
    n->left = first;
    n->count = count;
    return;
  }
  int axis = 0;
  for (int a = 1; a < 3; ++a)
    if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
  g_sort_axis = axis;
  g_sort_centroid = b->centroid;
  qsort(b->order + first, (size_t)count, sizeof(int32_t), cmp_centroid);
  const int32_t half = count / 2;
  const int32_t left = b->num_nodes;
  b->num_nodes += 2;
  n->left = left;
  n->count = 0;
  build_node(b, left, first, half);
  build_node(b, left + 1, first + half, count - half);
}

static int bvh_build(bvh_t* b, const olo_scene* s) {
  const int32_t t = s->num_triangles;
  b->s = s;
  b->num_nodes = 0;
  b->nodes = (node_t*)calloc((size_t)(2 * (t > 0 ? t : 1)), sizeof(node_t));
  b->order = (int32_t*)malloc(sizeof(int32_t) * (size_t)(t > 0 ? t : 1));
  b->centroid = (v3*)malloc(sizeof(v3) * (size_t)(t > 0 ? t : 1));
  if (!b->nodes || !b->order || !b->centroid) return -1;
  for (int32_t i = 0; i < t; ++i) {
    b->order[i] = i;
    const float* p = s->positions + 9 * i;
    b->centroid[i] = scl(add(add(ld3(p), ld3(p + 3)), ld3(p + 6)), 1.0 / 3.0);
  }
  b->num_nodes = 1;
  if (t > 0) build_node(b, 0, 0, t);
  return 0;
}

static void bvh_free(bvh_t* b) {
  free(b->nodes);
  free(b->order);
  free(b->centroid);
}

static inline int box_hit(const node_t* n, v3 o, v3 inv, double tmax) {
  double t0 = 0.0, t1 = tmax;
  const double oo[3] = {o.x, o.y, o.z}, ii[3] = {inv.x, inv.y, inv.z};
  for (int a = 0; a < 3; ++a) {
    double u = (n->lo[a] - oo[a]) * ii[a], v = (n->hi[a] - oo[a]) * ii[a];
    if (u > v) { double w = u; u = v; v = w; }
    v *= 1.0 + 1e-12;
    t0 = u > t0 ? u : t0;
    t1 = v < t1 ? v : t1;
    if (t0 > t1) return 0;
  }
  return 1;
}

/* Moller-Trumbore; returns t in (tmin, tmax) or -1. */
static inline double tri_hit(const olo_scene* s, int32_t t, v3 o, v3 d, double tmin, double tmax, double* bu,
                             double* bv) {
  const float* p = s->positions + 9 * t;
  v3 a = ld3(p), e1 = sub(ld3(p + 3), a), e2 = sub(ld3(p + 6), a);
  v3 pv = cross(d, e2);
  double det = dot(e1, pv);
  if (fabs(det) < 1e-300) return -1.0;
  double inv = 1.0 / det;
  v3 tv = sub(o, a);
  double u = dot(tv, pv) * inv;
  if (u < 0.0 || u > 1.0) return -1.0;
  v3 q = cross(tv, e1);
  double v = dot(d, q) * inv;
  if (v < 0.0 || u + v > 1.0) return -1.0;
  double th = dot(e2, q) * inv;
  if (!(th > tmin && th < tmax)) return -1.0;
  *bu = u;
  *bv = v;
  return th;
}

/* closest hit: triangle index or -1 */
static int32_t trace(const bvh_t* b, v3 o, v3 d, double tmin, double tmax, double* t_out, double* bu, double* bv,
                     int any) {
  if (b->s->num_triangles == 0) return -1;
  v3 inv = mk(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
  int32_t stack[128];
  int sp = 0;
  stack[sp++] = 0;
  int32_t best = -1;
  double best_t = tmax;
  while (sp) {
    const node_t* n = &b->nodes[stack[--sp]];
    if (!box_hit(n, o, inv, best_t)) continue;
    if (n->count) {
      for (int32_t k = n->left; k < n->left + n->count; ++k) {
        double u, v;
        double th = tri_hit(b->s, b->order[k], o, d, tmin, best_t, &u, &v);
        if (th > 0.0) {
          best = b->order[k];
          best_t = th;
          *bu = u;
          *bv = v;
          if (any) {
            *t_out = th;
            return best;
          }
        }
      }
    } else if (sp < 126) {
      stack[sp++] = n->left;
      stack[sp++] = n->left + 1;
    }
  }
  *t_out = best_t;
  return best;
}

/* ---- the reference's shading formulas ------------------------------------ */
typedef struct {
  v3 base, emission;
  double roughness, metallic;
  int two_sided;
} mat_t;

static mat_t load_mat(const olo_scene* s, int32_t t) {
  const float* m = s->materials + 10 * s->material[t];
  mat_t r;
  r.base = ld3(m);
  r.roughness = m[3];
  r.metallic = m[4];
  r.emission = ld3(m + 5);
  r.two_sided = m[8] > 0.5f;
  return r;
}

static inline void frame_of(v3 n, v3* t, v3* b) {
  *t = nrm(fabs(n.z) < 0.999 ? cross(n, mk(0, 0, 1)) : cross(n, mk(0, 1, 0)));
  *b = cross(n, *t);
}

static inline v3 cosine_dir(v3 n, double u, double v) {
  v3 t, b;
  frame_of(n, &t, &b);
  double r = sqrt(u), phi = 2.0 * OLO_PI * v;
  return nrm(add(add(scl(t, r * cos(phi)), scl(b, r * sin(phi))), scl(n, sqrt(fmax(0.0, 1.0 - u)))));
}

static inline double alpha2_of(double roughness) {
  double a = fmax(roughness * roughness, 0.0009);
  return a * a;
}
/* GGX D with the bracket (n.h)^2 (a2 - 1) + 1 written as |n x h|^2 + (n.h)^2 a2
 * and not capped: the reference floors pi den^2 at 1e-6, which for roughness
 * below about 0.155 caps D near its peak while the sampler draws the uncapped
 * distribution, so f cos / pdf no longer integrates f and the estimators of
 * one scene disagree (by a fifth at roughness 0.05).  Above roughness 0.155
 * both are the same function. */
static inline double ggx_d(double nh, double s2, double a2) {
  double den = s2 + nh * nh * a2;
  return a2 / fmax(OLO_PI * den * den, 1e-300);
}
static inline double sin2_between(v3 n, v3 h, double nh) {
  if (!(nh > 0.0)) return 1.0;
  v3 c = cross(n, h);
  return dot(c, c);
}
static inline double ggx_g1(double x, double a2) { return 2.0 * x / fmax(x + sqrt(a2 + (1.0 - a2) * x * x), 1e-6); }
static inline v3 f0_of(const mat_t* m) { return add(scl(mk(0.04, 0.04, 0.04), 1.0 - m->metallic), scl(m->base, m->metallic)); }
static inline double spec_prob(const mat_t* m) { return clampd(maxc(f0_of(m)), 0.1, 0.9); }

static v3 bsdf_eval(const mat_t* m, v3 n, v3 view, v3 out) {
  double nv = fmax(dot(n, view), 0.0), nl = fmax(dot(n, out), 0.0);
  if (nv <= 0.0 || nl <= 0.0) return mk(0, 0, 0);
  v3 h = nrm(add(view, out));
  double nh = fmax(dot(n, h), 0.0), vh = fmax(dot(view, h), 0.0);
  v3 f0 = f0_of(m);
  double w = pow(1.0 - clampd(vh, 0.0, 1.0), 5.0);
  v3 F = add(f0, scl(sub(mk(1, 1, 1), f0), w));
  double a2 = alpha2_of(m->roughness);
  double spec = ggx_d(nh, sin2_between(n, h, nh), a2) * ggx_g1(nv, a2) * ggx_g1(nl, a2) / fmax(4.0 * nv * nl, 1e-6);
  v3 diff = scl(mul(sub(mk(1, 1, 1), F), m->base), (1.0 - m->metallic) / OLO_PI);
  return add(diff, scl(F, spec));
}

static double bsdf_pdf(const mat_t* m, v3 n, v3 view, v3 out) {
  double nl = fmax(dot(n, out), 0.0);
  if (nl <= 0.0) return 0.0;
  v3 h = nrm(add(view, out));
  double nh = fmax(dot(n, h), 0.0), vh = fmax(dot(view, h), 1e-6);
  double sp = ggx_d(nh, sin2_between(n, h, nh), alpha2_of(m->roughness)) * nh / (4.0 * vh);
  double dp = nl / OLO_PI;
  double p = spec_prob(m);
  return dp + (sp - dp) * p;
}

static inline double power_h(double a, double b) {
  double a2 = a * a, b2 = b * b;
  return a2 / fmax(a2 + b2, 1e-6);
}

static v3 environment(const olo_scene* s, v3 d) {
  if (s->env_kind == 1) return ld3(s->env_color);
  double sky = fmax(d.y, 0.0);  /* ordinarylight_environment_analytic, ordinaryshade_primary.glsl:703-707 */
  return add(scl(mk(0.018, 0.022, 0.032), 1.0 - sky), scl(mk(0.32, 0.46, 0.72), sky));
}

static inline double luminance(v3 c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; }

static int32_t select_emitter(const olo_scene* s, double u) {
  int32_t lo = 0, hi = s->num_emitters - 1;
  while (lo < hi) {
    int32_t mid = lo + (hi - lo) / 2;
    if (u <= s->emitter_cdf[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

static inline double tri_area(const olo_scene* s, int32_t t, v3* ng) {
  const float* p = s->positions + 9 * t;
  v3 c = cross(sub(ld3(p + 3), ld3(p)), sub(ld3(p + 6), ld3(p)));
  double l = len(c);
  if (ng) *ng = l > 0.0 ? scl(c, 1.0 / l) : mk(0, 0, 0);
  return 0.5 * l;
}

static inline int occluded(const bvh_t* b, v3 o, v3 d, double tmax) {
  double t, u, v;
  return trace(b, o, d, 0.001, tmax, &t, &u, &v, 1) >= 0;
}

/* Direct light at a surface vertex (radiance towards -d before throughput). */
static v3 next_event(const bvh_t* b, const olo_scene* s, const mat_t* m, v3 p, v3 n, v3 view, uint32_t flags,
                     rng_t* r) {
  v3 direct = mk(0, 0, 0);
  const v3 origin = add(p, scl(n, 0.002));
  for (int32_t i = 0; i < s->num_lights; ++i) {
    const float* L = s->lights + 16 * i;
    const int type = (int)(L[0] + 0.5f);
    v3 dir;
    double dist2 = 1.0, dist = 10000.0;
    if (type == 1) {
      dir = scl(nrm(ld3(L + 4)), -1.0);
    } else {
      v3 off = sub(ld3(L + 1), p);
      dist2 = fmax(dot(off, off), 1e-6);
      dist = sqrt(dist2);
      dir = scl(off, 1.0 / dist);
      if (L[10] > 0.0f && dist > L[10]) continue;
    }
    double atten = type == 1 ? 1.0 : 1.0 / dist2;
    if (type == 2) {
      double cone = dot(nrm(ld3(L + 4)), scl(dir, -1.0));
      double x = clampd((cone - L[12]) / (L[11] - L[12]), 0.0, 1.0);
      atten *= x * x * (3.0 - 2.0 * x);
    }
    if (atten <= 0.0) continue;
    double c = fmax(dot(n, dir), 0.0);
    if (c <= 0.0) continue;
    double tmax = type == 1 ? 10000.0 : fmax(dist - 0.004, 0.001);
    if (occluded(b, origin, dir, tmax)) continue;
    direct = add(direct, scl(mul(bsdf_eval(m, n, view, dir), ld3(L + 7)), atten * c));
  }
  if (s->num_emitters > 0) {
    const double sel_u = rnd(r);
    const int32_t e = select_emitter(s, sel_u);
    const int32_t t = s->emitter_triangle[e];
    const double ru = sqrt(rnd(r)), rv = rnd(r);
    const float* q = s->positions + 9 * t;
    v3 lp = add(add(scl(ld3(q), 1.0 - ru), scl(ld3(q + 3), ru * (1.0 - rv))), scl(ld3(q + 6), ru * rv));
    v3 off = sub(lp, p);
    double dist2 = dot(off, off), dist = sqrt(dist2);
    v3 dir = scl(off, 1.0 / fmax(dist, 1e-6));
    v3 ng;
    double area = tri_area(s, t, &ng);
    mat_t lm = load_mat(s, t);
    double raw = dot(ng, scl(dir, -1.0));
    double lc = lm.two_sided ? fabs(raw) : fmax(raw, 0.0);
    double sc = fmax(dot(n, dir), 0.0);
    if (sc > 0.0 && lc > 1e-6 && !occluded(b, origin, dir, fmax(dist - 0.004, 0.001))) {
      double light_pdf = s->emitter_pdf[e] * dist2 / fmax(lc * area, 1e-6);
      double w = power_h(light_pdf, bsdf_pdf(m, n, view, dir));
      direct = add(direct, scl(mul(bsdf_eval(m, n, view, dir), lm.emission), sc * w / fmax(light_pdf, 1e-6)));
    }
  }
  if (flags & OLO_ENV_NEE) {
    double u = rnd(r), v = rnd(r);
    v3 dir = cosine_dir(n, u, v);
    double c = fmax(dot(n, dir), 0.0);
    if (c > 0.0 && !occluded(b, origin, dir, 1e30)) {
      double pdf = c / OLO_PI;
      direct = add(direct, scl(mul(bsdf_eval(m, n, view, dir), environment(s, dir)), c * 0.5 / pdf));
    }
  }
  return direct;
}

/* samplePbr (lighting.glsl:226-246) with the lobe choice u[0] and the
 * direction draws u[1], u[2]; returns 0 for a reflection below the surface
 * unless OLO_INVALID_RESAMPLE, which draws a fresh cosine direction from r. */
static int sample_bsdf(const mat_t* m, v3 n, v3 d, const double* u, uint32_t flags, rng_t* r, v3* out_dir,
                       v3* weight, double* pdf_out) {
  const v3 view = scl(d, -1.0);
  v3 out;
  if (u[0] < spec_prob(m)) {
    const double a2 = alpha2_of(m->roughness);
    const double den = fmax((1.0 - u[1]) + a2 * u[1], 1e-300);   /* 1 + (a2 - 1) u */
    const double c = sqrt((1.0 - u[1]) / den);
    const double sn = sqrt(a2 * u[1] / den), phi = 2.0 * OLO_PI * u[2];
    v3 ta, bi;
    frame_of(n, &ta, &bi);
    v3 h = nrm(add(add(scl(ta, sn * cos(phi)), scl(bi, sn * sin(phi))), scl(n, c)));
    out = sub(d, scl(h, 2.0 * dot(h, d)));
  } else {
    out = cosine_dir(n, u[1], u[2]);
  }
  if (!(dot(n, out) > 0.0)) {
    if (!(flags & OLO_INVALID_RESAMPLE)) return 0;
    out = cosine_dir(n, rnd(r), rnd(r));
  }
  out = nrm(out);
  const double pdf = fmax(bsdf_pdf(m, n, view, out), 1e-6);
  *weight = scl(bsdf_eval(m, n, view, out), fmax(dot(n, out), 0.0) / pdf);
  *out_dir = out;
  *pdf_out = pdf;
  return 1;
}

static v3 radiance(const bvh_t* b, const olo_scene* s, const olo_params* prm, v3 o, v3 d, rng_t* r) {
  v3 rad = mk(0, 0, 0), tp = mk(1, 1, 1);
  double tmin = 0.001;
  int prev_surface = 0;     /* the previous vertex sampled its BSDF (and lights, with NEE) */
  double prev_pdf = 0.0;
  const int nee = (prm->flags & OLO_NEE) != 0;
  for (int bounce = 0;; ++bounce) {
    double t, bu, bv;
    int32_t tri = trace(b, o, d, tmin, 1e30, &t, &bu, &bv, 0);
    if (tri < 0) {
      double w = (prev_surface && nee && (prm->flags & OLO_ENV_NEE)) ? 0.5 : 1.0;
      return add(rad, scl(mul(tp, environment(s, d)), w));
    }
    v3 ng;
    double area = tri_area(s, tri, &ng);
    const float* nv = s->normals + 9 * tri;
    v3 ns = nrm(add(add(scl(ld3(nv), 1.0 - bu - bv), scl(ld3(nv + 3), bu)), scl(ld3(nv + 6), bv)));
    if (!(dot(ns, ns) > 0.5)) ns = ng;
    if (dot(ns, ng) < 0.0) ns = scl(ns, -1.0);
    const int entering = dot(d, ng) < 0.0;
    const v3 n = entering ? ns : scl(ns, -1.0);
    const v3 p = add(o, scl(d, t));
    const mat_t m = load_mat(s, tri);
    if ((entering || m.two_sided) && maxc(m.emission) > 0.0) {
      double w = 1.0;
      if (prev_surface && nee && s->num_emitters > 0) {
        double raw = dot(ng, scl(d, -1.0));
        double lc = m.two_sided ? fabs(raw) : fmax(raw, 0.0);
        double sel = area * luminance(m.emission) / fmax(s->total_power, 1e-6);
        double light_pdf = sel * t * t / fmax(lc * area, 1e-6);
        w = power_h(prev_pdf, light_pdf);
      }
      rad = add(rad, scl(mul(tp, m.emission), w));
    }
    if (bounce + 1 >= prm->max_bounces) return rad;
    const v3 view = scl(d, -1.0);
    if (nee) rad = add(rad, mul(tp, next_event(b, s, &m, p, n, view, prm->flags, r)));
    /* BSDF sample (samplePbr) */
    double u3[3] = {rnd(r), rnd(r), rnd(r)};
    v3 out, weight;
    double pdf;
    if (!sample_bsdf(&m, n, d, u3, prm->flags, r, &out, &weight, &pdf)) return rad;
    tp = mul(tp, weight);
    prev_surface = 1;
    prev_pdf = pdf;
    if (prm->rr_start > 0 && bounce + 1 >= prm->rr_start) {
      const double survival = clampd(maxc(tp), prm->rr_min_survival, 0.95);
      if (rnd(r) >= survival) return rad;
      tp = scl(tp, 1.0 / survival);
    }
    if (!(maxc(tp) > 0.0)) return rad;
    o = add(p, scl(out, 0.002));
    d = out;
    tmin = 0.001;
  }
}

static void camera_ray(const olo_camera* c, const olo_params* p, int32_t x, int32_t y, double jx, double jy, v3* o,
                       v3* d) {
  const double ndc_x = ((double)x + jx) / (double)p->width * 2.0 - 1.0;
  const double ndc_y = 1.0 - ((double)y + jy) / (double)p->height * 2.0;
  const v3 pos = ld3(c->position), fwd = ld3(c->forward), right = ld3(c->right), up = ld3(c->up);
  if (c->projection == 2) {
    const double yaw = ndc_x * c->scale_x, pitch = ndc_y * c->scale_y;
    *d = add(add(scl(fwd, cos(pitch) * cos(yaw)), scl(right, cos(pitch) * sin(yaw))), scl(up, sin(pitch)));
    *o = pos;
  } else if (c->projection == 1) {
    *o = add(add(pos, scl(right, ndc_x * c->scale_x)), scl(up, ndc_y * c->scale_y));
    *d = fwd;
  } else {
    *d = add(add(fwd, scl(right, ndc_x * c->scale_x)), scl(up, ndc_y * c->scale_y));
    *o = pos;
  }
  *d = nrm(*d);
}

/* Renders the window of p: sum and sum of squares per pixel and channel of the
 * samples [first_sample, first_sample + samples), each a double
 * (win_h, win_w, 3).  Returns 0, or -1 when memory runs out. */
int olo_render(const olo_scene* s, const olo_camera* c, const olo_params* p, double* sum, double* sumsq) {
  bvh_t b;
  if (bvh_build(&b, s) != 0) {
    bvh_free(&b);
    return -1;
  }
  const int64_t npix = (int64_t)p->win_w * p->win_h;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t k = 0; k < npix; ++k) {
    const int32_t x = p->x0 + (int32_t)(k % p->win_w), y = p->y0 + (int32_t)(k / p->win_w);
    const uint64_t pixel = (uint64_t)y * (uint64_t)p->width + (uint64_t)x;
    double acc[3] = {0, 0, 0}, acc2[3] = {0, 0, 0};
    for (int32_t i = 0; i < p->samples; ++i) {
      const uint64_t sample = (uint64_t)(p->first_sample + i);
      rng_t r;
      r.s = mix64(p->seed ^ mix64(pixel * 0x100000001b3ull + mix64(sample + 0x51ed27ull)));
      const double jx = rnd(&r), jy = rnd(&r);
      v3 o, d;
      camera_ray(c, p, x, y, jx, jy, &o, &d);
      const v3 L = radiance(&b, s, p, o, d, &r);
      const double l[3] = {L.x, L.y, L.z};
      for (int ch = 0; ch < 3; ++ch) {
        const double v = isfinite(l[ch]) ? l[ch] : 0.0;
        acc[ch] += v;
        acc2[ch] += v * v;
      }
    }
    for (int ch = 0; ch < 3; ++ch) {
      sum[3 * k + ch] = acc[ch];
      sumsq[3 * k + ch] = acc2[ch];
    }
  }
  bvh_free(&b);
  return 0;
}

/* Closest hits of given rays (for the oracle's own geometry checks):
 * triangle index or -1, and t. */
int olo_trace(const olo_scene* s, int32_t n, const float* origins, const float* dirs, double tmin, int32_t* tri,
              double* t) {
  bvh_t b;
  if (bvh_build(&b, s) != 0) {
    bvh_free(&b);
    return -1;
  }
#pragma omp parallel for schedule(static)
  for (int32_t i = 0; i < n; ++i) {
    double u, v;
    tri[i] = trace(&b, ld3(origins + 3 * i), nrm(ld3(dirs + 3 * i)), tmin, 1e30, &t[i], &u, &v, 0);
  }
  bvh_free(&b);
  return 0;
}

/* Known-answer hooks for the CPU tests: the BSDF value, pdf and one sample. */
void olo_bsdf(const float* material10, const double* n, const double* view, const double* out, double* f,
              double* pdf) {
  olo_scene s;
  memset(&s, 0, sizeof(s));
  int32_t zero = 0;
  s.materials = material10;
  s.material = &zero;
  mat_t m = load_mat(&s, 0);
  v3 nn = mk(n[0], n[1], n[2]), vv = mk(view[0], view[1], view[2]), oo = mk(out[0], out[1], out[2]);
  v3 e = bsdf_eval(&m, nn, vv, oo);
  f[0] = e.x;
  f[1] = e.y;
  f[2] = e.z;
  *pdf = bsdf_pdf(&m, nn, vv, oo);
}

/* Known-answer hook: n samples of the BSDF at normal nrm for the incoming
 * direction d (towards the surface), with the lobe/direction draws u (n, 3)
 * and, for OLO_INVALID_RESAMPLE, a generator seeded by seed; writes the
 * weights f cos / pdf (n, 3), zero for invalid samples. */
void olo_sample_bsdf(const float* material10, const double* nrm_in, const double* d_in, int32_t n,
                     const double* u, uint32_t flags, uint64_t seed, double* weights) {
  olo_scene s;
  memset(&s, 0, sizeof(s));
  int32_t zero = 0;
  s.materials = material10;
  s.material = &zero;
  mat_t m = load_mat(&s, 0);
  rng_t r;
  r.s = mix64(seed);
  const v3 nn = nrm(mk(nrm_in[0], nrm_in[1], nrm_in[2])), dd = nrm(mk(d_in[0], d_in[1], d_in[2]));
  for (int32_t i = 0; i < n; ++i) {
    v3 out, w;
    double pdf;
    if (!sample_bsdf(&m, nn, dd, u + 3 * i, flags, &r, &out, &w, &pdf)) w = mk(0, 0, 0);
    weights[3 * i + 0] = w.x;
    weights[3 * i + 1] = w.y;
    weights[3 * i + 2] = w.z;
  }
}
