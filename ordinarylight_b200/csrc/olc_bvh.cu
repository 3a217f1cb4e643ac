// Device LBVH construction: 30-bit Morton codes, a stable LSD radix sort,
// Karras' parallel hierarchy emission, bottom-up boxes, leaf collapse and a
// node layout of two child boxes per 64-byte node; refit; the BVH4 form
// traversal reads (up to four descendants per 128-byte node, collapsed
// greedily by surface area); validation.
//
// Replaces the driver-built hardware BLAS/TLAS of the reference
// (VulkanSceneUploader._build_scene, ordinarylight/targets/vulkan/scene.py:1484-1560):
// one BLAS per mesh resource, one TLAS over instances.
//
// Bit-exactness: the Morton quantisation uses only correctly rounded float
// operations without contraction (__fadd_rn/__fsub_rn/__fmul_rn/__fdiv_rn),
// so the codes equal a float32 host computation of the same formula, and the
// radix sort is stable, so the permutation equals
// numpy.argsort(codes, kind="stable").
#include <algorithm>
#include <cmath>

#include "olc_internal.h"
#include "olc_sah.h"

namespace olc {

namespace {

constexpr int kThreads = 256;

OLC_D uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
OLC_D float ord2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

OLC_HD uint32_t expand_bits10(uint32_t v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_triangle_boxes(const float* __restrict__ vertices, const uint32_t* __restrict__ indices,
                                 uint32_t nt, float4* lo, float4* hi, float4* centers) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  uint32_t i0 = indices[3 * i + 0], i1 = indices[3 * i + 1], i2 = indices[3 * i + 2];
  float3 a = f3(vertices[3 * i0 + 0], vertices[3 * i0 + 1], vertices[3 * i0 + 2]);
  float3 b = f3(vertices[3 * i1 + 0], vertices[3 * i1 + 1], vertices[3 * i1 + 2]);
  float3 c = f3(vertices[3 * i2 + 0], vertices[3 * i2 + 1], vertices[3 * i2 + 2]);
  float3 l = fminf3(fminf3(a, b), c), h = fmaxf3(fmaxf3(a, b), c);
  lo[i] = make_float4(l.x, l.y, l.z, 0.0f);
  hi[i] = make_float4(h.x, h.y, h.z, 0.0f);
  centers[i] = make_float4(__fmul_rn(__fadd_rn(l.x, h.x), 0.5f), __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
                           __fmul_rn(__fadd_rn(l.z, h.z), 0.5f), 0.0f);
}

__global__ void k_triangle_boxes_flat(const float* __restrict__ tri, uint32_t nt, float4* lo, float4* hi,
                                      float4* centers) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nt) return;
  const float* p = tri + 9ull * i;
  float3 a = f3(p[0], p[1], p[2]), b = f3(p[3], p[4], p[5]), c = f3(p[6], p[7], p[8]);
  float3 l = fminf3(fminf3(a, b), c), h = fmaxf3(fmaxf3(a, b), c);
  lo[i] = make_float4(l.x, l.y, l.z, 0.0f);
  hi[i] = make_float4(h.x, h.y, h.z, 0.0f);
  centers[i] = make_float4(__fmul_rn(__fadd_rn(l.x, h.x), 0.5f), __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
                           __fmul_rn(__fadd_rn(l.z, h.z), 0.5f), 0.0f);
}

__global__ void k_init_bounds(uint32_t* b) {
  if (threadIdx.x < 3) b[threadIdx.x] = 0xffffffffu;   // min
  else if (threadIdx.x < 6) b[threadIdx.x] = 0u;       // max
}

__global__ void k_center_bounds(const float4* __restrict__ centers, uint32_t n, uint32_t* bounds) {
  __shared__ uint32_t s[6];
  if (threadIdx.x < 3) s[threadIdx.x] = 0xffffffffu;
  else if (threadIdx.x < 6) s[threadIdx.x] = 0u;
  __syncthreads();
  uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 c = centers[i];
    uint32_t o[3] = {f2ord(c.x), f2ord(c.y), f2ord(c.z)};
    for (int k = 0; k < 3; ++k) { mn[k] = min(mn[k], o[k]); mx[k] = max(mx[k], o[k]); }
  }
  for (int k = 0; k < 3; ++k) { atomicMin(&s[k], mn[k]); atomicMax(&s[3 + k], mx[k]); }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(&bounds[threadIdx.x], s[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(&bounds[threadIdx.x], s[threadIdx.x]);
}

__global__ void k_morton(const float4* __restrict__ centers, uint32_t n, const uint32_t* __restrict__ bounds,
                         uint32_t* codes, uint32_t* vals) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lo[3], inv[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = ord2f(bounds[k]);
    float ext = __fsub_rn(ord2f(bounds[3 + k]), lo[k]);
    inv[k] = ext > 0.0f ? __fdiv_rn(1.0f, ext) : 0.0f;
  }
  float4 c = centers[i];
  float cc[3] = {c.x, c.y, c.z};
  uint32_t q[3];
  for (int k = 0; k < 3; ++k) {
    float v = __fmul_rn(__fmul_rn(__fsub_rn(cc[k], lo[k]), inv[k]), 1024.0f);
    v = fminf(fmaxf(v, 0.0f), 1023.0f);
    q[k] = (uint32_t)v;
  }
  codes[i] = (expand_bits10(q[0]) << 2) | (expand_bits10(q[1]) << 1) | expand_bits10(q[2]);
  if (vals) vals[i] = i;
}

// ---- radix sort ----------------------------------------------------------
constexpr int kRsWarps = 8;
constexpr int kRsRounds = 8;
constexpr int kRsTile = kRsWarps * kRsRounds * 32;  // 2048 items per block

__global__ void k_rs_hist(const uint32_t* __restrict__ keys, uint32_t n, uint32_t shift, uint32_t* hist,
                          uint32_t nblocks) {
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  uint32_t base = blockIdx.x * kRsTile;
  for (uint32_t i = threadIdx.x; i < (uint32_t)kRsTile; i += blockDim.x) {
    uint32_t idx = base + i;
    if (idx < n) atomicAdd(&cnt[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// Exclusive scan of hist[0..len) by one block of 1024 threads.
__global__ void k_exclusive_scan_1block(uint32_t* data, uint32_t len) {
  __shared__ uint32_t sums[1024];
  uint32_t per = (len + blockDim.x - 1) / blockDim.x;
  uint32_t begin = threadIdx.x * per;
  uint32_t end = min(begin + per, len);
  uint32_t local = 0;
  for (uint32_t i = begin; i < end; ++i) local += data[i];
  sums[threadIdx.x] = local;
  __syncthreads();
  for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
    uint32_t v = threadIdx.x >= off ? sums[threadIdx.x - off] : 0u;
    __syncthreads();
    sums[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = sums[threadIdx.x] - local;
  for (uint32_t i = begin; i < end; ++i) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(256) k_rs_scatter(const uint32_t* __restrict__ keys_in,
                                                    const uint32_t* __restrict__ vals_in, uint32_t* keys_out,
                                                    uint32_t* vals_out, uint32_t n, uint32_t shift,
                                                    const uint32_t* __restrict__ hist, uint32_t nblocks) {
  __shared__ uint32_t whist[kRsWarps][256];
  __shared__ uint32_t boff[256];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  for (uint32_t i = threadIdx.x; i < (uint32_t)(kRsWarps * 256); i += blockDim.x) (&whist[0][0])[i] = 0u;
  __syncthreads();
  const uint32_t lanemask_lt = (1u << lane) - 1u;
  uint32_t k[kRsRounds], v[kRsRounds], dig[kRsRounds], rank[kRsRounds];
  const uint32_t base = blockIdx.x * kRsTile + warp * (kRsRounds * 32);
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    uint32_t idx = base + r * 32 + lane;
    bool valid = idx < n;
    k[r] = valid ? keys_in[idx] : 0u;
    v[r] = valid ? vals_in[idx] : 0u;
    uint32_t d = valid ? ((k[r] >> shift) & 255u) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t leader = __ffs(peers) - 1u;
    uint32_t prior = valid ? whist[warp][d] : 0u;
    __syncwarp();
    if (valid && lane == leader) whist[warp][d] = prior + __popc(peers);
    __syncwarp();
    dig[r] = d;
    rank[r] = prior + __popc(peers & lanemask_lt);
  }
  __syncthreads();
  {
    uint32_t d = threadIdx.x;  // blockDim == 256: one digit per thread
    uint32_t run = 0;
    for (int w = 0; w < kRsWarps; ++w) {
      uint32_t t = whist[w][d];
      whist[w][d] = run;
      run += t;
    }
    boff[d] = hist[d * nblocks + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    if (dig[r] < 256u) {
      uint32_t dst = boff[dig[r]] + whist[warp][dig[r]] + rank[r];
      keys_out[dst] = k[r];
      vals_out[dst] = v[r];
    }
  }
}

// ---- Karras hierarchy ----------------------------------------------------
OLC_D int lbvh_delta(const uint32_t* codes, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = codes[i], b = codes[j];
  if (a == b) return 32 + __clz((uint32_t)(i ^ j));
  return __clz(a ^ b);
}

__global__ void k_karras(const uint32_t* __restrict__ codes, int n, int* left, int* right, int* first, int* last,
                         int* parent, int* leaf_parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (lbvh_delta(codes, n, i, i + 1) - lbvh_delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = lbvh_delta(codes, n, i, i - d);
  int lmax = 2;
  while (lbvh_delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (lbvh_delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = lbvh_delta(codes, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (lbvh_delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int gamma = i + s * d + min(d, 0);
  int lo = min(i, j), hi = max(i, j);
  // child encoding: >= 0 internal, < 0 leaf (~index)
  int lc = (lo == gamma) ? ~gamma : gamma;
  int rc = (hi == gamma + 1) ? ~(gamma + 1) : (gamma + 1);
  left[i] = lc;
  right[i] = rc;
  first[i] = lo;
  last[i] = hi;
  if (lc < 0) leaf_parent[~lc] = i; else parent[lc] = i;
  if (rc < 0) leaf_parent[~rc] = i; else parent[rc] = i;
  if (i == 0) parent[0] = -1;
}

__global__ void k_gather_sorted_boxes(const uint32_t* __restrict__ order, uint32_t n, const float4* lo,
                                      const float4* hi, float4* slo, float4* shi) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t o = order[i];
  slo[i] = lo[o];
  shi[i] = hi[o];
}

OLC_D float4 ld_cg(const float4* p) { return __ldcg(p); }

__global__ void k_bottom_up(int n, const int* __restrict__ left, const int* __restrict__ right,
                            const int* __restrict__ parent, const int* __restrict__ leaf_parent,
                            const float4* __restrict__ leaf_lo, const float4* __restrict__ leaf_hi, float4* node_lo,
                            float4* node_hi, uint32_t* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = leaf_parent[i];
  for (int guard = 0; p >= 0 && guard < n; ++guard) {
    __threadfence();
    uint32_t old = atomicAdd(&flags[p], 1u);
    if (old == 0u) return;
    __threadfence();
    int lc = left[p], rc = right[p];
    float4 llo = lc < 0 ? leaf_lo[~lc] : ld_cg(node_lo + lc);
    float4 lhi = lc < 0 ? leaf_hi[~lc] : ld_cg(node_hi + lc);
    float4 rlo = rc < 0 ? leaf_lo[~rc] : ld_cg(node_lo + rc);
    float4 rhi = rc < 0 ? leaf_hi[~rc] : ld_cg(node_hi + rc);
    node_lo[p] = make_float4(fminf(llo.x, rlo.x), fminf(llo.y, rlo.y), fminf(llo.z, rlo.z), 0.0f);
    node_hi[p] = make_float4(fmaxf(lhi.x, rhi.x), fmaxf(lhi.y, rhi.y), fmaxf(lhi.z, rhi.z), 0.0f);
    p = parent[p];
  }
}

// TLAS leaf of build primitive p: primitives [0, n_inst) are instances
// (global instance index inst_base + p), the rest baked world-space triangles
// (global slot flat_base + p - n_inst).
struct TlasRefs {
  uint32_t n_inst = 0, inst_base = 0, flat_base = 0;
  const uint32_t* remap = nullptr;   // build index -> primitive (a subset build), or identity
};
OLC_HD int tlas_prim_leaf(const TlasRefs& r, uint32_t p) {
  return p < r.n_inst ? olc_make_leaf(r.inst_base + p, OLC_TLAS_LEAF_INSTANCE)
                      : olc_make_leaf(r.flat_base + (p - r.n_inst), OLC_TLAS_LEAF_TRIANGLE);
}
OLC_D int tlas_leaf(const TlasRefs& r, uint32_t i) { return tlas_prim_leaf(r, r.remap ? r.remap[i] : i); }

// Emit final nodes.  blas: leaves reference slot ranges (collapse subtrees of
// at most leaf_max leaves); tlas: one instance or baked triangle per leaf.
__global__ void k_emit_nodes(int n, const int* __restrict__ left, const int* __restrict__ right,
                             const int* __restrict__ first, const int* __restrict__ last,
                             const float4* __restrict__ leaf_lo, const float4* __restrict__ leaf_hi,
                             const float4* __restrict__ node_lo, const float4* __restrict__ node_hi,
                             const uint32_t* __restrict__ sorted_vals, int is_tlas, TlasRefs tr,
                             uint32_t leaf_max, BvhNode* nodes, uint32_t node_base, uint32_t slot_base) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int ch[2] = {left[i], right[i]};
  float4 lo[2], hi[2];
  int ref[2];
  for (int s = 0; s < 2; ++s) {
    int c = ch[s];
    if (c < 0) {
      int leaf = ~c;
      lo[s] = leaf_lo[leaf];
      hi[s] = leaf_hi[leaf];
      ref[s] = is_tlas ? tlas_leaf(tr, sorted_vals[leaf]) : olc_make_leaf(slot_base + (uint32_t)leaf, 1u);
    } else {
      lo[s] = node_lo[c];
      hi[s] = node_hi[c];
      uint32_t size = (uint32_t)(last[c] - first[c] + 1);
      if (!is_tlas && size <= leaf_max) ref[s] = olc_make_leaf(slot_base + (uint32_t)first[c], size);
      else ref[s] = (int)(node_base + (uint32_t)c);
    }
  }
  BvhNode nd;
  nd.a = make_float4(lo[0].x, hi[0].x, lo[0].y, hi[0].y);
  nd.b = make_float4(lo[1].x, hi[1].x, lo[1].y, hi[1].y);
  nd.c = make_float4(lo[0].z, hi[0].z, lo[1].z, hi[1].z);
  nd.d = make_int4(ref[0], ref[1], 0, 0);
  nodes[node_base + i] = nd;
}

// A structure with a single primitive: one node, child 1 empty.
__global__ void k_single_leaf_node(const float4* lo, const float4* hi, int is_tlas, TlasRefs tr,
                                   const uint32_t* sorted_vals, BvhNode* nodes, uint32_t node_base,
                                   uint32_t slot_base, uint32_t n) {
  BvhNode nd;
  if (n == 0) {
    const float inf = CUDART_INF_F;
    nd.a = make_float4(inf, -inf, inf, -inf);
    nd.b = nd.a;
    nd.c = make_float4(inf, -inf, inf, -inf);
    nd.d = make_int4(OLC_EMPTY_CHILD, OLC_EMPTY_CHILD, 0, 0);
  } else {
    const float inf = CUDART_INF_F;
    nd.a = make_float4(lo[0].x, hi[0].x, lo[0].y, hi[0].y);
    nd.b = make_float4(inf, -inf, inf, -inf);
    nd.c = make_float4(lo[0].z, hi[0].z, inf, -inf);
    nd.d = make_int4(is_tlas ? tlas_leaf(tr, sorted_vals[0]) : olc_make_leaf(slot_base, 1u),
                     OLC_EMPTY_CHILD, 0, 0);
  }
  nodes[node_base] = nd;
}

__global__ void k_reorder_triangles(const uint32_t* __restrict__ order, uint32_t nt,
                                    const float* __restrict__ vertices, const float* __restrict__ normals,
                                    const uint32_t* __restrict__ indices, float4* tri_verts,
                                    float4* tri_normals, uint32_t* tri_index, uint32_t slot_base) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nt) return;
  uint32_t t = order[s];
  uint32_t dst = slot_base + s;
  for (int k = 0; k < 3; ++k) {
    uint32_t vi = indices[3 * t + k];
    tri_verts[3ull * dst + k] = make_float4(vertices[3 * vi + 0], vertices[3 * vi + 1], vertices[3 * vi + 2], 0.0f);
    tri_normals[3ull * dst + k] = make_float4(normals[3 * vi + 0], normals[3 * vi + 1], normals[3 * vi + 2], 0.0f);
  }
  tri_index[dst] = t;
}

// Boxes of world-space triangles that the TLAS references directly.
__global__ void k_flat_triangle_boxes(const float4* __restrict__ verts, uint32_t n, float4* lo, float4* hi,
                                      float4* centers) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float3 a = f3(verts[3ull * i]), b = f3(verts[3ull * i + 1]), c = f3(verts[3ull * i + 2]);
  float3 l = fminf3(fminf3(a, b), c), h = fmaxf3(fmaxf3(a, b), c);
  lo[i] = make_float4(l.x, l.y, l.z, 0.0f);
  hi[i] = make_float4(h.x, h.y, h.z, 0.0f);
  centers[i] = make_float4(__fmul_rn(__fadd_rn(l.x, h.x), 0.5f), __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
                           __fmul_rn(__fadd_rn(l.z, h.z), 0.5f), 0.0f);
}

// Tight world box of each instance: the bounds of its BLAS's vertices after
// the object-to-world transform (a rotated object-space box can be up to
// sqrt(3) wider per axis than the object it holds).  Blocks (instance, part)
// each bound a stride of the instance's vertices and merge into per-instance
// order-preserving integer bounds with atomics, so a single instance of
// millions of triangles is spread over the whole GPU; min/max make the
// result independent of the merge order.
__global__ void __launch_bounds__(256) k_instance_box_parts(const float* __restrict__ o2w, uint32_t n,
                                                            const uint2* __restrict__ slot_ranges,
                                                            const float4* __restrict__ tri_verts, uint32_t* acc_mn,
                                                            uint32_t* acc_mx) {
  __shared__ uint32_t s[6];
  const uint32_t i = blockIdx.x;   // instance; blockIdx.y is the part
  if (i >= n) return;
  if (threadIdx.x < 3) s[threadIdx.x] = 0xffffffffu;
  else if (threadIdx.x < 6) s[threadIdx.x] = 0u;
  __syncthreads();
  Affine m;
  const float* p = o2w + 12ull * i;
  m.r0 = make_float4(p[0], p[1], p[2], p[3]);
  m.r1 = make_float4(p[4], p[5], p[6], p[7]);
  m.r2 = make_float4(p[8], p[9], p[10], p[11]);
  const uint2 range = slot_ranges[i];
  uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
  const uint64_t stride = (uint64_t)gridDim.y * blockDim.x;
  for (uint64_t v = 3ull * range.x + (uint64_t)blockIdx.y * blockDim.x + threadIdx.x; v < 3ull * range.y; v += stride) {
    const float3 w = xform_point(m, f3(tri_verts[v]));
    const uint32_t o[3] = {f2ord(w.x), f2ord(w.y), f2ord(w.z)};
    for (int k = 0; k < 3; ++k) { mn[k] = min(mn[k], o[k]); mx[k] = max(mx[k], o[k]); }
  }
  for (int k = 0; k < 3; ++k) {
    for (int off = 16; off > 0; off >>= 1) {
      mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
      mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
    }
  }
  if ((threadIdx.x & 31u) == 0u)
    for (int k = 0; k < 3; ++k) { atomicMin(&s[k], mn[k]); atomicMax(&s[3 + k], mx[k]); }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(&acc_mn[3ull * i + threadIdx.x], s[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(&acc_mx[3ull * i + threadIdx.x - 3], s[threadIdx.x]);
}

__global__ void k_instance_box_init(uint32_t n, uint32_t* acc_mn, uint32_t* acc_mx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3u * n) return;
  acc_mn[i] = 0xffffffffu;
  acc_mx[i] = 0u;
}

__global__ void k_instance_box_finish(uint32_t n, const uint32_t* __restrict__ acc_mn,
                                      const uint32_t* __restrict__ acc_mx, float4* lo, float4* hi, float4* centers) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t* a = acc_mn + 3ull * i;
  const uint32_t* b = acc_mx + 3ull * i;
  float3 wl, wh;
  if (a[0] > b[0]) {  // no vertices
    wl = f3(CUDART_INF_F, CUDART_INF_F, CUDART_INF_F);
    wh = -wl;
  } else {
    wl = f3(ord2f(a[0]), ord2f(a[1]), ord2f(a[2]));
    wh = f3(ord2f(b[0]), ord2f(b[1]), ord2f(b[2]));
  }
  // Pad by a relative epsilon: the traversal transforms the ray, not the
  // vertices, so its hit points are not bit-identical to these.
  float mag = fmaxf(fmaxf(max3(fmaxf3(wh, -wl)), max3(wh - wl)), 1e-3f);
  float3 pad = f3(mag, mag, mag) * 1e-5f;
  wl = wl - pad;
  wh = wh + pad;
  lo[i] = make_float4(wl.x, wl.y, wl.z, 0.0f);
  hi[i] = make_float4(wh.x, wh.y, wh.z, 0.0f);
  centers[i] = make_float4(__fmul_rn(__fadd_rn(wl.x, wh.x), 0.5f), __fmul_rn(__fadd_rn(wl.y, wh.y), 0.5f),
                           __fmul_rn(__fadd_rn(wl.z, wh.z), 0.5f), 0.0f);
}

inline uint32_t blocks_for(uint64_t n, int threads = kThreads) { return (uint32_t)((n + threads - 1) / threads); }

// ---- binned SAH build on the host (hierarchies of up to kSahMaxPrims) -----
// olc_sah.h builds the tree; on the instanced scene's sphere and top level
// its summed inner-node area is 10-13 % below that of the Morton-order tree,
// i.e. that many fewer box tests per ray.  The nodes and the leaf order are
// written exactly as the device build writes them (same BVH2 layout, leaf
// encoding and slot order semantics), so everything downstream (the BVH4
// form, refits, validation) is shared.
constexpr uint32_t kSahMaxPrims = 1u << 17;

uint32_t build_hierarchy_sah(uint32_t n, BuildScratch& sc, int is_tlas, const TlasRefs& tr, BvhNode* nodes,
                             uint32_t node_base, uint32_t slot_base, cudaStream_t stream) {
  std::vector<float4> lo(n), hi(n), ce(n);
  OLC_CUDA(cudaMemcpyAsync(lo.data(), sc.boxes_lo.get(), n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaMemcpyAsync(hi.data(), sc.boxes_hi.get(), n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaMemcpyAsync(ce.data(), sc.centers.get(), n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaStreamSynchronize(stream));
  std::vector<sah::Node> tree;
  std::vector<uint32_t> order;
  sah::build(n, &lo[0].x, &hi[0].x, &ce[0].x, 4, tree, order);
  std::vector<BvhNode> out(tree.size());
  for (size_t i = 0; i < tree.size(); ++i) {
    const sah::Node& t = tree[i];
    int ref[2];
    for (int s = 0; s < 2; ++s) {
      const int32_t c = t.child[s];
      if (c >= 0) ref[s] = (int)(node_base + (uint32_t)c);
      else ref[s] = is_tlas ? tlas_prim_leaf(tr, order[(uint32_t)~c]) : olc_make_leaf(slot_base + (uint32_t)~c, 1u);
    }
    const sah::Box& b0 = t.box[0];
    const sah::Box& b1 = t.box[1];
    out[i].a = make_float4(b0.lo[0], b0.hi[0], b0.lo[1], b0.hi[1]);
    out[i].b = make_float4(b1.lo[0], b1.hi[0], b1.lo[1], b1.hi[1]);
    out[i].c = make_float4(b0.lo[2], b0.hi[2], b1.lo[2], b1.hi[2]);
    out[i].d = make_int4(ref[0], ref[1], 0, 0);
  }
  OLC_CUDA(cudaMemcpyAsync(nodes + node_base, out.data(), out.size() * sizeof(BvhNode), cudaMemcpyHostToDevice,
                           stream));
  OLC_CUDA(cudaMemcpyAsync(sc.vals.get(), order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
  OLC_CUDA(cudaStreamSynchronize(stream));   // the host arrays go out of scope
  return node_base;
}

// Common tail of a BLAS/TLAS build after boxes and centres exist.
uint32_t build_hierarchy(uint32_t n, BuildScratch& sc, int is_tlas, const TlasRefs& tr, uint32_t leaf_max,
                         BvhNode* nodes, uint32_t node_base, uint32_t slot_base, cudaStream_t stream) {
  if (n >= 2 && n <= kSahMaxPrims && leaf_max == 1u && tr.remap == nullptr)
    return build_hierarchy_sah(n, sc, is_tlas, tr, nodes, node_base, slot_base, stream);
  if (n <= 1) {
    if (n == 1) {
      // sorted order is the identity
      uint32_t zero = 0;
      OLC_CUDA(cudaMemcpyAsync(sc.vals.as<uint32_t>(), &zero, sizeof(zero), cudaMemcpyHostToDevice, stream));
    }
    k_single_leaf_node<<<1, 1, 0, stream>>>(sc.boxes_lo.as<float4>(), sc.boxes_hi.as<float4>(), is_tlas, tr,
                                            sc.vals.as<uint32_t>(), nodes, node_base, slot_base, n);
    OLC_LAUNCH_CHECK("k_single_leaf_node");
    OLC_CUDA(cudaStreamSynchronize(stream));
    return node_base;
  }
  uint32_t* bounds = sc.bounds.as<uint32_t>();
  morton_codes(sc.centers.as<float4>(), n, bounds, nullptr, stream);
  k_morton<<<blocks_for(n), kThreads, 0, stream>>>(sc.centers.as<float4>(), n, bounds, sc.keys.as<uint32_t>(),
                                                     sc.vals.as<uint32_t>());
  OLC_LAUNCH_CHECK("k_morton");
  radix_sort_pairs(sc.keys.as<uint32_t>(), sc.vals.as<uint32_t>(), sc.keys_alt.as<uint32_t>(),
                   sc.vals_alt.as<uint32_t>(), sc.hist.as<uint32_t>(), n, 30, stream);
  k_karras<<<blocks_for(n - 1), kThreads, 0, stream>>>(sc.keys.as<uint32_t>(), (int)n, sc.left.as<int>(),
                                                         sc.right.as<int>(), sc.first.as<int>(), sc.last.as<int>(),
                                                         sc.parent.as<int>(), sc.leaf_parent.as<int>());
  OLC_LAUNCH_CHECK("k_karras");
  k_gather_sorted_boxes<<<blocks_for(n), kThreads, 0, stream>>>(sc.vals.as<uint32_t>(), n, sc.boxes_lo.as<float4>(),
                                                                  sc.boxes_hi.as<float4>(), sc.sorted_lo.as<float4>(),
                                                                  sc.sorted_hi.as<float4>());
  OLC_LAUNCH_CHECK("k_gather_sorted_boxes");
  OLC_CUDA(cudaMemsetAsync(sc.flags.get(), 0, sizeof(uint32_t) * (n - 1), stream));
  k_bottom_up<<<blocks_for(n), kThreads, 0, stream>>>((int)n, sc.left.as<int>(), sc.right.as<int>(),
                                                        sc.parent.as<int>(), sc.leaf_parent.as<int>(),
                                                        sc.sorted_lo.as<float4>(), sc.sorted_hi.as<float4>(),
                                                        sc.node_lo.as<float4>(), sc.node_hi.as<float4>(),
                                                        sc.flags.as<uint32_t>());
  OLC_LAUNCH_CHECK("k_bottom_up");
  k_emit_nodes<<<blocks_for(n - 1), kThreads, 0, stream>>>(
      (int)n, sc.left.as<int>(), sc.right.as<int>(), sc.first.as<int>(), sc.last.as<int>(),
      sc.sorted_lo.as<float4>(), sc.sorted_hi.as<float4>(), sc.node_lo.as<float4>(), sc.node_hi.as<float4>(),
      sc.vals.as<uint32_t>(), is_tlas, tr, leaf_max, nodes, node_base, slot_base);
  OLC_LAUNCH_CHECK("k_emit_nodes");
  return node_base;  // Karras root is internal node 0
}

}  // namespace

void BuildScratch::ensure(size_t n) {
  if (n <= capacity) return;
  size_t c = std::max<size_t>(n, 1024);
  boxes_lo.allocate(c * 16);
  boxes_hi.allocate(c * 16);
  centers.allocate(c * 16);
  bounds.allocate(64);
  keys.allocate(c * 4);
  vals.allocate(c * 4);
  keys_alt.allocate(c * 4);
  vals_alt.allocate(c * 4);
  hist.allocate(radix_sort_hist_words((uint32_t)c) * 4);
  sorted_lo.allocate(c * 16);
  sorted_hi.allocate(c * 16);
  left.allocate(c * 4);
  right.allocate(c * 4);
  first.allocate(c * 4);
  last.allocate(c * 4);
  parent.allocate(c * 4);
  leaf_parent.allocate(c * 4);
  flags.allocate(c * 4);
  node_lo.allocate(c * 16);
  node_hi.allocate(c * 16);
  capacity = c;
}

size_t radix_sort_hist_words(uint32_t n) {
  uint32_t nblocks = (n + kRsTile - 1) / kRsTile;
  return (size_t)256 * std::max<uint32_t>(nblocks, 1u);
}

void morton_codes(const float4* centers, uint32_t n, uint32_t* bounds, uint32_t* codes, cudaStream_t stream) {
  k_init_bounds<<<1, 32, 0, stream>>>(bounds);
  OLC_LAUNCH_CHECK("k_init_bounds");
  uint32_t grid = std::min<uint32_t>(blocks_for(n), 148u * 8u);
  k_center_bounds<<<std::max<uint32_t>(grid, 1u), kThreads, 0, stream>>>(centers, n, bounds);
  OLC_LAUNCH_CHECK("k_center_bounds");
  if (codes) {
    k_morton<<<blocks_for(n), kThreads, 0, stream>>>(centers, n, bounds, codes, nullptr);
    OLC_LAUNCH_CHECK("k_morton");
  }
}

void triangle_centers_flat(const float* tri, uint32_t n, float4* lo, float4* hi, float4* centers,
                           cudaStream_t stream) {
  k_triangle_boxes_flat<<<blocks_for(n), kThreads, 0, stream>>>(tri, n, lo, hi, centers);
  OLC_LAUNCH_CHECK("k_triangle_boxes_flat");
}

void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint32_t* hist,
                      uint32_t n, uint32_t key_bits, cudaStream_t stream) {
  if (n <= 1) return;
  uint32_t nblocks = (n + kRsTile - 1) / kRsTile;
  uint32_t passes = (key_bits + 7) / 8;
  uint32_t* kin = keys;
  uint32_t* vin = vals;
  uint32_t* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t shift = 8 * p;
    k_rs_hist<<<nblocks, 256, 0, stream>>>(kin, n, shift, hist, nblocks);
    OLC_LAUNCH_CHECK("k_rs_hist");
    k_exclusive_scan_1block<<<1, 1024, 0, stream>>>(hist, 256 * nblocks);
    OLC_LAUNCH_CHECK("k_exclusive_scan_1block");
    k_rs_scatter<<<nblocks, 256, 0, stream>>>(kin, vin, kout, vout, n, shift, hist, nblocks);
    OLC_LAUNCH_CHECK("k_rs_scatter");
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {
    OLC_CUDA(cudaMemcpyAsync(keys, kin, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream));
    OLC_CUDA(cudaMemcpyAsync(vals, vin, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream));
  }
}

uint32_t build_blas(const BlasDesc& d, BuildScratch& sc, BvhNode* nodes, uint32_t node_base, float4* tri_verts,
                    float4* tri_normals, uint32_t* tri_index, uint32_t slot_base, uint32_t leaf_max,
                    cudaStream_t stream) {
  uint32_t n = d.num_triangles;
  sc.ensure(std::max<uint32_t>(n, 1u));
  if (n > 0) {
    k_triangle_boxes<<<blocks_for(n), kThreads, 0, stream>>>(d.vertices, d.indices, n, sc.boxes_lo.as<float4>(),
                                                               sc.boxes_hi.as<float4>(), sc.centers.as<float4>());
    OLC_LAUNCH_CHECK("k_triangle_boxes");
  }
  uint32_t root = build_hierarchy(n, sc, 0, TlasRefs{}, leaf_max, nodes, node_base, slot_base, stream);
  if (n > 0) {
    k_reorder_triangles<<<blocks_for(n), kThreads, 0, stream>>>(sc.vals.as<uint32_t>(), n, d.vertices, d.normals,
                                                                  d.indices, tri_verts, tri_normals, tri_index,
                                                                  slot_base);
    OLC_LAUNCH_CHECK("k_reorder_triangles");
  }
  return root;
}

// ---- texture attributes of triangle slots --------------------------------

// Per-slot vertex attributes of one mesh's BLAS slots, in slot order:
// (uv0, uv1) and (object tangent, handedness) of each corner.
__global__ void k_slot_attributes(const float4* __restrict__ texcoords, const float4* __restrict__ tangents,
                                  const uint32_t* __restrict__ indices, uint32_t nt, uint32_t vertex_base,
                                  const uint32_t* __restrict__ tri_index, uint32_t first_slot, uint32_t scene_slot0,
                                  float4* attr) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nt) return;
  const uint32_t slot = first_slot + s;
  const uint32_t t = tri_index[slot];
  float4* out = attr + 6ull * (slot - scene_slot0);
  for (int k = 0; k < 3; ++k) {
    const uint32_t vi = vertex_base + indices[3ull * t + k];
    out[2 * k] = texcoords[vi];
    out[2 * k + 1] = tangents[vi];
  }
}

void slot_attributes(const float4* texcoords, const float4* tangents, const uint32_t* mesh_indices, uint32_t nt,
                     uint32_t vertex_base, const uint32_t* tri_index, uint32_t first_slot, uint32_t scene_slot0,
                     float4* attr, cudaStream_t stream) {
  if (nt == 0) return;
  k_slot_attributes<<<blocks_for(nt), kThreads, 0, stream>>>(texcoords, tangents, mesh_indices, nt, vertex_base,
                                                               tri_index, first_slot, scene_slot0, attr);
  OLC_LAUNCH_CHECK("k_slot_attributes");
}

// sRGB-to-linear decode of the 256 byte values, c / 12.92 below 0.04045 and
// ((c + 0.055) / 1.055)^2.4 above (IEC 61966-2-1), in double precision.
__global__ void k_srgb_table(float* out) {
  const uint32_t i = threadIdx.x;
  if (i >= 256u) return;
  const double c = (double)i / 255.0;
  out[i] = (float)(c <= 0.04045 ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4));
}

void srgb_table(float* out, cudaStream_t stream) {
  k_srgb_table<<<1, 256, 0, stream>>>(out);
  OLC_LAUNCH_CHECK("k_srgb_table");
}

// ---- refit: new triangle positions under an unchanged hierarchy ----------

// Rewrite the triangle slots of one BLAS from new mesh arrays.  Slot order
// (and so every leaf) stays; tri_index maps a slot to its mesh triangle.
__global__ void k_refresh_slots(const float* __restrict__ vertices, const float* __restrict__ normals,
                                const uint32_t* __restrict__ indices, uint32_t nt, float4* tri_verts,
                                float4* tri_normals, const uint32_t* __restrict__ tri_index, uint32_t slot_base) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nt) return;
  const uint32_t dst = slot_base + s;
  const uint32_t t = tri_index[dst];
  for (int k = 0; k < 3; ++k) {
    uint32_t vi = indices[3 * t + k];
    tri_verts[3ull * dst + k] = make_float4(vertices[3 * vi + 0], vertices[3 * vi + 1], vertices[3 * vi + 2], 0.0f);
    tri_normals[3ull * dst + k] = make_float4(normals[3 * vi + 0], normals[3 * vi + 1], normals[3 * vi + 2], 0.0f);
  }
}

__global__ void k_refit_init(uint32_t count, int* parent, uint32_t* done) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  parent[i] = -1;
  done[i] = 0u;
}

// Parent of every internal node and how many internal children each node
// waits for.  Nodes inside subtrees that the build collapsed into leaves are
// unreachable; they get refit too, harmlessly.
__global__ void k_refit_links(const BvhNode* __restrict__ nodes, uint32_t node_base, uint32_t count, int* parent,
                              uint32_t* pending) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int4 d = nodes[node_base + i].d;
  uint32_t internal = 0;
  for (int c : {d.x, d.y})
    if (c >= 0 && (uint32_t)c - node_base < count) {
      parent[(uint32_t)c - node_base] = (int)i;
      ++internal;
    }
  pending[i] = internal;
}

OLC_D void slot_range_box(const float4* tri_verts, int ref, float3& lo, float3& hi) {
  lo = make_float3(CUDART_INF_F, CUDART_INF_F, CUDART_INF_F);
  hi = make_float3(-CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F);
  if (ref == OLC_EMPTY_CHILD) return;
  const uint32_t first = olc_leaf_first(ref), n = olc_leaf_count(ref);
  for (uint32_t k = 0; k < n; ++k)
    for (int v = 0; v < 3; ++v) {
      const float3 p = f3(tri_verts[3ull * (first + k) + v]);
      lo = fminf3(lo, p);
      hi = fmaxf3(hi, p);
    }
}

// Union of a node's two child boxes (its own box).
OLC_D void node_box(const BvhNode& n, float3& lo, float3& hi) {
  lo = make_float3(fminf(n.a.x, n.b.x), fminf(n.a.z, n.b.z), fminf(n.c.x, n.c.z));
  hi = make_float3(fmaxf(n.a.y, n.b.y), fmaxf(n.a.w, n.b.w), fmaxf(n.c.y, n.c.w));
}

// Bottom-up box pass: a thread starts at each node without internal
// children and climbs while it is the last child to finish (Karras 2012's
// atomic-counter traversal).  Boxes are min/max over the same vertices as at
// build time, so refitting unchanged geometry reproduces the built nodes.
__global__ void k_refit_up(BvhNode* nodes, uint32_t node_base, uint32_t count, const float4* __restrict__ tri_verts,
                           const int* __restrict__ parent, const uint32_t* __restrict__ pending, uint32_t* done) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count || pending[i] != 0u) return;
  uint32_t n = i;
  for (uint32_t guard = 0; guard < count; ++guard) {
    BvhNode* nd = nodes + node_base + n;
    const int4 d = nd->d;
    float3 lo[2], hi[2];
    const int ref[2] = {d.x, d.y};
    for (int c = 0; c < 2; ++c) {
      if (ref[c] >= 0 && (uint32_t)ref[c] - node_base < count) {
        const float4* cp = reinterpret_cast<const float4*>(nodes + ref[c]);
        BvhNode child;
        child.a = __ldcg(cp + 0);
        child.b = __ldcg(cp + 1);
        child.c = __ldcg(cp + 2);
        node_box(child, lo[c], hi[c]);
      } else {
        slot_range_box(tri_verts, ref[c], lo[c], hi[c]);
      }
    }
    nd->a = make_float4(lo[0].x, hi[0].x, lo[0].y, hi[0].y);
    nd->b = make_float4(lo[1].x, hi[1].x, lo[1].y, hi[1].y);
    nd->c = make_float4(lo[0].z, hi[0].z, lo[1].z, hi[1].z);
    const int p = parent[n];
    if (p < 0) return;
    __threadfence();
    const uint32_t before = atomicAdd(&done[p], 1u);
    if (before + 1u < pending[p]) return;
    __threadfence();
    n = (uint32_t)p;
  }
}

void refit_blas(const BlasDesc& d, BuildScratch& sc, BvhNode* nodes, uint32_t node_base, uint32_t node_count,
                float4* tri_verts, float4* tri_normals, const uint32_t* tri_index, uint32_t slot_base,
                cudaStream_t stream) {
  const uint32_t n = d.num_triangles;
  if (n > 0) {
    k_refresh_slots<<<blocks_for(n), kThreads, 0, stream>>>(d.vertices, d.normals, d.indices, n, tri_verts,
                                                              tri_normals, tri_index, slot_base);
    OLC_LAUNCH_CHECK("k_refresh_slots");
  }
  sc.ensure(std::max<uint32_t>(node_count, 1u));
  int* parent = sc.parent.as<int>();
  uint32_t* pending = sc.first.as<uint32_t>();
  uint32_t* done = sc.flags.as<uint32_t>();
  k_refit_init<<<blocks_for(node_count), kThreads, 0, stream>>>(node_count, parent, done);
  OLC_LAUNCH_CHECK("k_refit_init");
  k_refit_links<<<blocks_for(node_count), kThreads, 0, stream>>>(nodes, node_base, node_count, parent, pending);
  OLC_LAUNCH_CHECK("k_refit_links");
  k_refit_up<<<blocks_for(node_count), kThreads, 0, stream>>>(nodes, node_base, node_count, tri_verts, parent,
                                                                pending, done);
  OLC_LAUNCH_CHECK("k_refit_up");
}

// Large primitives (an instance or baked triangle whose box spans more than
// a quarter of the scene along some axis, such as a ground plane) make every
// ancestor in a Morton-ordered hierarchy as large as themselves, so most rays
// would descend those ancestors.  They are split off: the TLAS root joins an
// LBVH over the large primitives and an LBVH over the rest, and a ray pays
// for the large ones once near the root.
constexpr float kLargeFraction = 0.25f;
constexpr uint32_t kHoistMaxPrims = 1u << 20;   // above this, one LBVH (no host pass)

uint32_t build_tlas(const float* o2w, const uint2* slot_ranges, uint32_t n, uint32_t max_instance_triangles,
                    uint32_t instance_base, const float4* tri_verts, const float4* flat_verts, uint32_t n_flat,
                    uint32_t flat_slot_base, BuildScratch& sc, BvhNode* nodes, uint32_t node_base,
                    cudaStream_t stream) {
  const uint32_t total = n + n_flat;
  sc.ensure(std::max<uint32_t>(total, 1u));
  if (n > 0) {
    // enough parts per instance for about 16 vertices per thread in the
    // largest instance
    const uint32_t parts =
        std::max<uint32_t>(1u, std::min<uint32_t>(2048u, (uint32_t)((3ull * max_instance_triangles + 4095) / 4096)));
    // 3 words per instance in each of two 16-byte-per-primitive scratch arrays
    uint32_t* acc_mn = reinterpret_cast<uint32_t*>(sc.node_lo.get());
    uint32_t* acc_mx = reinterpret_cast<uint32_t*>(sc.node_hi.get());
    k_instance_box_init<<<blocks_for(3ull * n), kThreads, 0, stream>>>(n, acc_mn, acc_mx);
    OLC_LAUNCH_CHECK("k_instance_box_init");
    k_instance_box_parts<<<dim3(n, parts), 256, 0, stream>>>(o2w, n, slot_ranges, tri_verts, acc_mn, acc_mx);
    OLC_LAUNCH_CHECK("k_instance_box_parts");
    k_instance_box_finish<<<blocks_for(n), kThreads, 0, stream>>>(n, acc_mn, acc_mx, sc.boxes_lo.as<float4>(),
                                                                    sc.boxes_hi.as<float4>(), sc.centers.as<float4>());
    OLC_LAUNCH_CHECK("k_instance_box_finish");
  }
  if (n_flat > 0) {
    k_flat_triangle_boxes<<<blocks_for(n_flat), kThreads, 0, stream>>>(
        flat_verts, n_flat, sc.boxes_lo.as<float4>() + n, sc.boxes_hi.as<float4>() + n, sc.centers.as<float4>() + n);
    OLC_LAUNCH_CHECK("k_flat_triangle_boxes");
  }
  TlasRefs tr;
  tr.n_inst = n;
  tr.inst_base = instance_base;
  tr.flat_base = flat_slot_base;
  // up to kSahMaxPrims the SAH build places large primitives near the root by
  // itself; the Morton build above that needs them hoisted first
  if (total < 3 || total > kHoistMaxPrims || total <= kSahMaxPrims)
    return build_hierarchy(total, sc, 1, tr, 1, nodes, node_base, 0, stream);

  // classify on the host
  std::vector<float4> lo(total), hi(total), ce(total);
  OLC_CUDA(cudaMemcpyAsync(lo.data(), sc.boxes_lo.get(), total * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaMemcpyAsync(hi.data(), sc.boxes_hi.get(), total * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaMemcpyAsync(ce.data(), sc.centers.get(), total * sizeof(float4), cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaStreamSynchronize(stream));
  float slo[3] = {INFINITY, INFINITY, INFINITY}, shi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t p = 0; p < total; ++p) {
    const float l[3] = {lo[p].x, lo[p].y, lo[p].z}, h[3] = {hi[p].x, hi[p].y, hi[p].z};
    for (int a = 0; a < 3; ++a) {
      slo[a] = std::min(slo[a], l[a]);
      shi[a] = std::max(shi[a], h[a]);
    }
  }
  std::vector<uint32_t> large, small;
  for (uint32_t p = 0; p < total; ++p) {
    const float e[3] = {hi[p].x - lo[p].x, hi[p].y - lo[p].y, hi[p].z - lo[p].z};
    bool big = false;
    for (int a = 0; a < 3; ++a)
      if (shi[a] > slo[a] && e[a] > kLargeFraction * (shi[a] - slo[a])) big = true;
    (big ? large : small).push_back(p);
  }
  if (large.empty() || small.empty()) return build_hierarchy(total, sc, 1, tr, 1, nodes, node_base, 0, stream);

  // two subset builds below a root node at node_base
  DeviceBuffer remap(total * sizeof(uint32_t));
  std::vector<float4> sub_lo, sub_hi, sub_ce;
  int child_ref[2];
  float4 child_lo[2], child_hi[2];
  uint32_t next = node_base + 1;
  const std::vector<uint32_t>* subsets[2] = {&large, &small};
  uint32_t remap_off = 0;
  for (int k = 0; k < 2; ++k) {
    const std::vector<uint32_t>& ids = *subsets[k];
    const uint32_t m = (uint32_t)ids.size();
    float4 ul = make_float4(INFINITY, INFINITY, INFINITY, 0.0f), uh = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
    for (uint32_t p : ids) {
      ul = make_float4(std::min(ul.x, lo[p].x), std::min(ul.y, lo[p].y), std::min(ul.z, lo[p].z), 0.0f);
      uh = make_float4(std::max(uh.x, hi[p].x), std::max(uh.y, hi[p].y), std::max(uh.z, hi[p].z), 0.0f);
    }
    child_lo[k] = ul;
    child_hi[k] = uh;
    if (m == 1) {
      child_ref[k] = tlas_prim_leaf(tr, ids[0]);
      continue;
    }
    sub_lo.resize(m);
    sub_hi.resize(m);
    sub_ce.resize(m);
    for (uint32_t i = 0; i < m; ++i) {
      sub_lo[i] = lo[ids[i]];
      sub_hi[i] = hi[ids[i]];
      sub_ce[i] = ce[ids[i]];
    }
    OLC_CUDA(cudaMemcpyAsync(sc.boxes_lo.get(), sub_lo.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream));
    OLC_CUDA(cudaMemcpyAsync(sc.boxes_hi.get(), sub_hi.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream));
    OLC_CUDA(cudaMemcpyAsync(sc.centers.get(), sub_ce.data(), m * sizeof(float4), cudaMemcpyHostToDevice, stream));
    uint32_t* rm = remap.as<uint32_t>() + remap_off;
    OLC_CUDA(cudaMemcpyAsync(rm, ids.data(), m * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    TlasRefs sub = tr;
    sub.remap = rm;
    child_ref[k] = (int)build_hierarchy(m, sc, 1, sub, 1, nodes, next, 0, stream);
    next += m - 1;
    remap_off += m;
    OLC_CUDA(cudaStreamSynchronize(stream));   // the host staging vectors are reused
  }
  BvhNode root;
  root.a = make_float4(child_lo[0].x, child_hi[0].x, child_lo[0].y, child_hi[0].y);
  root.b = make_float4(child_lo[1].x, child_hi[1].x, child_lo[1].y, child_hi[1].y);
  root.c = make_float4(child_lo[0].z, child_hi[0].z, child_lo[1].z, child_hi[1].z);
  root.d = make_int4(child_ref[0], child_ref[1], 0, 0);
  OLC_CUDA(cudaMemcpyAsync(nodes + node_base, &root, sizeof(root), cudaMemcpyHostToDevice, stream));
  OLC_CUDA(cudaStreamSynchronize(stream));
  return node_base;
}

// ---- BVH4 form --------------------------------------------------------------
namespace {
OLC_D void set_lane(float4& v, int k, float x) {
  if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}
OLC_D void set_lane(int4& v, int k, int x) {
  if (k == 0) v.x = x; else if (k == 1) v.y = x; else if (k == 2) v.z = x; else v.w = x;
}
// Append child `which` of BVH2 node `parent` (box from the parent) as slot k.
OLC_D void put_child(BvhNode4& w, int& k, const BvhNode& parent, int which, int ref) {
  const float lx = which ? parent.b.x : parent.a.x, hx = which ? parent.b.y : parent.a.y;
  const float ly = which ? parent.b.z : parent.a.z, hy = which ? parent.b.w : parent.a.w;
  const float lz = which ? parent.c.z : parent.c.x, hz = which ? parent.c.w : parent.c.y;
  set_lane(w.lox, k, lx); set_lane(w.hix, k, hx);
  set_lane(w.loy, k, ly); set_lane(w.hiy, k, hy);
  set_lane(w.loz, k, lz); set_lane(w.hiz, k, hz);
  set_lane(w.child, k, ref);
  ++k;
}

// Half surface area of child `which` of BVH2 node `nd`.
OLC_D float child_half_area(const BvhNode& nd, int which) {
  const float dx = which ? nd.b.y - nd.b.x : nd.a.y - nd.a.x;
  const float dy = which ? nd.b.w - nd.b.z : nd.a.w - nd.a.z;
  const float dz = which ? nd.c.w - nd.c.z : nd.c.y - nd.c.x;
  return dx * dy + dy * dz + dz * dx;
}

// One slot candidate of a BVH4 node: child `which` of BVH2 node `parent`.
struct WideEntry {
  uint32_t parent;
  int which;
  int ref;
  float area;
};

// BVH4 node of BVH2 node i, collapsed greedily by surface area: start from
// i's two children and repeatedly open the internal entry with the largest
// box (replacing it, in place, by its own children) while the result still
// fits four slots.  Where one child is a leaf this fills the slots the
// fixed two-level collapse would leave empty, so fewer nodes are fetched
// per ray.  Internal nodes outside [begin, end) (the nodes of an unbuilt
// mesh in a scene's node range) are left out, so no fetch leaves the range;
// the number of openings is bounded, so a corrupt structure cannot keep the
// loop running.
OLC_D BvhNode4 bvh4_of(const BvhNode* __restrict__ nodes, uint32_t i, uint32_t begin, uint32_t end) {
  BvhNode4 w;
  const float inf = __int_as_float(0x7f800000);
  w.lox = w.loy = w.loz = make_float4(inf, inf, inf, inf);
  w.hix = w.hiy = w.hiz = make_float4(-inf, -inf, -inf, -inf);
  w.child = make_int4(OLC_EMPTY_CHILD, OLC_EMPTY_CHILD, OLC_EMPTY_CHILD, OLC_EMPTY_CHILD);
  w.reserved = make_int4(0, 0, 0, 0);
  auto admit = [&](const BvhNode& nd, int which) {
    const int ref = which ? nd.d.y : nd.d.x;
    return ref != OLC_EMPTY_CHILD && (ref < 0 || ((uint32_t)ref >= begin && (uint32_t)ref < end));
  };
  WideEntry e[4];
  int n = 0;
  {
    const BvhNode nd = nodes[i];
    for (int c = 0; c < 2; ++c)
      if (admit(nd, c)) e[n++] = WideEntry{i, c, c ? nd.d.y : nd.d.x, child_half_area(nd, c)};
  }
  for (int opening = 0; opening < 16; ++opening) {
    int best = -1;
    float best_area = -1.0f;
    for (int k = 0; k < n; ++k)
      if (e[k].ref >= 0 && e[k].area > best_area) {
        best = k;
        best_area = e[k].area;
      }
    if (best < 0) break;
    const uint32_t at = (uint32_t)e[best].ref;
    const BvhNode cn = nodes[at];
    WideEntry kids[2];
    int m = 0;
    for (int g = 0; g < 2; ++g)
      if (admit(cn, g)) kids[m++] = WideEntry{at, g, g ? cn.d.y : cn.d.x, child_half_area(cn, g)};
    if (n - 1 + m > 4) break;
    // replace entry `best` by its m children, keeping the slot order
    if (m == 0) {
      for (int k = best; k + 1 < n; ++k) e[k] = e[k + 1];
    } else if (m == 2) {
      for (int k = n - 1; k > best; --k) e[k + 1] = e[k];
      e[best + 1] = kids[1];
    }
    if (m > 0) e[best] = kids[0];
    n += m - 1;
  }
  int k = 0;
  for (int j = 0; j < n; ++j) put_child(w, k, nodes[e[j].parent], e[j].which, e[j].ref);
  return w;
}

__global__ void k_bvh4(const BvhNode* __restrict__ nodes, BvhNode4* __restrict__ wide, uint32_t begin,
                       uint32_t count) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  wide[begin + t] = bvh4_of(nodes, begin + t, begin, begin + count);
}
}  // namespace

void build_bvh4(const BvhNode* nodes, BvhNode4* wide, uint32_t begin, uint32_t count, cudaStream_t stream) {
  if (count == 0) return;
  k_bvh4<<<blocks_for(count), kThreads, 0, stream>>>(nodes, wide, begin, count);
  OLC_LAUNCH_CHECK("k_bvh4");
}

// ---- validation ----------------------------------------------------------
namespace {
// Walk each built BLAS from its root; count how often each slot is reached,
// leaves outside the BLAS's own slot range, child boxes that do not lie
// inside the box stored for them in the parent, and BVH4 nodes that differ
// from the collapse of their BVH2 node.
__global__ void k_validate(SceneView s, const BlasRange* ranges, uint32_t count, uint32_t* slot_hits,
                           unsigned long long* bad) {
  uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= count) return;
  const BlasRange r = ranges[b];
  int stack[128];
  int sp = 0;
  stack[sp++] = (int)r.root;
  for (uint32_t guard = 0; sp > 0; ++guard) {
    if (guard > (1u << 26)) {
      atomicAdd(bad, 1ull);
      break;
    }
    int node = stack[--sp];
    if (node < 0) continue;
    {
      // the BVH4 form must be current: equal to the collapse of this node
      const BvhNode4 want = bvh4_of(s.nodes, (uint32_t)node, 0u, 0x7fffffffu);
      const BvhNode4 have = s.wide[node];
      const int* a = reinterpret_cast<const int*>(&want);
      const int* h = reinterpret_cast<const int*>(&have);
      bool same = true;
      for (int k = 0; k < 28; ++k) same = same && a[k] == h[k];   // six box float4 and the child refs
      if (!same) atomicAdd(bad, 1ull);
    }
    BvhNode nd = s.nodes[node];
    int ch[2] = {nd.d.x, nd.d.y};
    for (int c = 0; c < 2; ++c) {
      if (ch[c] == OLC_EMPTY_CHILD) continue;
      if (ch[c] >= 0) {
        BvhNode cn = s.nodes[ch[c]];
        float lx = c == 0 ? nd.a.x : nd.b.x, hx = c == 0 ? nd.a.y : nd.b.y;
        float ly = c == 0 ? nd.a.z : nd.b.z, hy = c == 0 ? nd.a.w : nd.b.w;
        float lz = c == 0 ? nd.c.x : nd.c.z, hz = c == 0 ? nd.c.y : nd.c.w;
        for (int g = 0; g < 2; ++g) {
          int gc = g == 0 ? cn.d.x : cn.d.y;
          if (gc == OLC_EMPTY_CHILD) continue;
          float glx = g == 0 ? cn.a.x : cn.b.x, ghx = g == 0 ? cn.a.y : cn.b.y;
          float gly = g == 0 ? cn.a.z : cn.b.z, ghy = g == 0 ? cn.a.w : cn.b.w;
          float glz = g == 0 ? cn.c.x : cn.c.z, ghz = g == 0 ? cn.c.y : cn.c.w;
          if (glx < lx || gly < ly || glz < lz || ghx > hx || ghy > hy || ghz > hz) atomicAdd(bad, 1ull);
        }
        if (sp < 128) stack[sp++] = ch[c]; else atomicAdd(bad, 1ull);
      } else {
        uint32_t f = olc_leaf_first(ch[c]), cnt = olc_leaf_count(ch[c]);
        for (uint32_t k = 0; k < cnt; ++k) {
          if (f + k < r.slot_begin || f + k >= r.slot_end) atomicAdd(bad, 1ull);
          else atomicAdd(&slot_hits[f + k], 1u);
        }
      }
    }
  }
}
}  // namespace

uint64_t validate_bvh(const SceneView& s, const std::vector<BlasRange>& blas, cudaStream_t stream) {
  uint32_t slots = 0;
  for (const BlasRange& r : blas) slots = std::max(slots, r.slot_end);
  DeviceBuffer hits(std::max<size_t>(slots, 1) * 4), bad(8), ranges(std::max<size_t>(blas.size(), 1) * sizeof(BlasRange));
  OLC_CUDA(cudaMemsetAsync(hits.get(), 0, std::max<size_t>(slots, 1) * 4, stream));
  OLC_CUDA(cudaMemsetAsync(bad.get(), 0, 8, stream));
  if (!blas.empty()) {
    OLC_CUDA(cudaMemcpyAsync(ranges.get(), blas.data(), blas.size() * sizeof(BlasRange), cudaMemcpyHostToDevice,
                             stream));
    k_validate<<<blocks_for(blas.size(), 64), 64, 0, stream>>>(s, ranges.as<BlasRange>(), (uint32_t)blas.size(),
                                                               hits.as<uint32_t>(), bad.as<unsigned long long>());
    OLC_LAUNCH_CHECK("k_validate");
  }
  std::vector<uint32_t> h(std::max<size_t>(slots, 1));
  unsigned long long nbad = 0;
  OLC_CUDA(cudaMemcpyAsync(h.data(), hits.get(), h.size() * 4, cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaMemcpyAsync(&nbad, bad.get(), 8, cudaMemcpyDeviceToHost, stream));
  OLC_CUDA(cudaStreamSynchronize(stream));
  for (const BlasRange& r : blas)
    for (uint32_t i = r.slot_begin; i < r.slot_end; ++i)
      if (h[i] != 1u) ++nbad;
  return nbad;
}

}  // namespace olc
