// C ABI of libolcuda: context, scene residency, the wavefront frame driver.
//
// A frame is processed as chunks of at most `capacity` paths.  Path linear
// index = sample * npix + pixel (sample-major), so a chunk that spans whole
// sample streams keeps every pixel of a stream resident together (ReSTIR's
// spatial pass needs that).  Per chunk: raygen, then per bounce
// trace_closest -> [ReSTIR at bounce 0] -> shade -> trace_shadow, then
// accumulate.  With use_graphs the whole frame is captured once per
// (width, height, spp) and replayed; per-frame parameters live in device
// memory and are refreshed by one host->device copy before each replay.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "olcuda.h"
#include "olc_internal.h"
#include "olc_restir.h"
#include "olc_wavefront.h"

using namespace olc;

namespace {

thread_local std::string g_thread_error;

// Instances of meshes with at most this many triangles are baked into one
// world-space mesh at upload, up to kFlattenMaxTotal baked triangles.
constexpr uint32_t kFlattenMaxTriangles = 64;
constexpr uint64_t kFlattenMaxTotal = 1ull << 24;

struct ScenePack {
  DeviceBuffer nodes, tri_verts, tri_normals, tri_index, instances, o2w, materials, material_aux, emitters,
      emitter_alias, lights,
      env_image, volume;
  SceneView view{};
  uint32_t total_triangles = 0;
  uint32_t blas_nodes = 0, tlas_nodes = 0, blas_count = 0;
  uint64_t bytes = 0;
  double build_ms = 0.0;
  bool valid = false;
  DeviceBuffer tri_owner;
  std::vector<BlasRange> blas_ranges;
  uint32_t flattened_instances = 0, tlas_instances = 0;
};

struct TimelineEntry {
  uint32_t stage, bounce, chunk;
};

struct GraphKey {
  uint32_t w, h, spp;
  bool operator<(const GraphKey& o) const { return std::tie(w, h, spp) < std::tie(o.w, o.h, o.spp); }
};

}  // namespace

struct olc_context {
  olc_config cfg{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
  std::string error;
  ScenePack scene;
  BuildScratch scratch;
  LaunchShape ls;
  // wavefront buffers
  uint32_t capacity = 0;
  DeviceBuffer q0_o, q0_d, q0_p, q1_o, q1_d, q1_p, hit_tuv, hit_inst, sh_o, sh_d, sh_c, ps_tp, ps_rad, ps_meta;
  DeviceBuffer counters, fp_dev, accum, out_dev;
  DeviceBuffer prod_depth, prod_normal, prod_inst, prod_mat, prod_prim;
  uint32_t npix_capacity = 0;
  FrameParams* fp_host = nullptr;     // pinned
  Counters* counters_host = nullptr;  // pinned, one per chunk
  uint32_t counters_host_chunks = 0;
  RestirState restir;
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::map<GraphKey, std::vector<TimelineEntry>> graph_timelines;
  // device timeline: events[k] .. events[k+1] brackets launch k
  std::vector<cudaEvent_t> tl_events;
  std::vector<TimelineEntry> tl_entries;
  bool capturing = false;
  std::vector<olc_launch_record> last_profile;
  uint32_t last_w = 0, last_h = 0;
  bool closed = false;
};

namespace {

int fail(olc_context* ctx, int code, const std::string& msg) {
  if (ctx) ctx->error = msg;
  g_thread_error = msg;
  return code;
}

template <class F>
int guarded(olc_context* ctx, F&& f) {
  try {
    if (ctx && ctx->closed) return fail(ctx, OLC_ERR_CLOSED, "renderer context is closed");
    if (ctx) OLC_CUDA(cudaSetDevice(ctx->device));
    f();
    return OLC_OK;
  } catch (const Error& e) {
    return fail(ctx, e.code, e.what());
  } catch (const std::bad_alloc&) {
    return fail(ctx, OLC_ERR_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(ctx, OLC_ERR_RUNTIME, e.what());
  }
}

void validate_config(const olc_config& c) {
  if (c.max_bounces < 1 || c.max_bounces > OLC_MAX_BOUNCES)
    throw Error(OLC_ERR_VALUE, "max_bounces must be between 1 and 64");
  if (c.mode > 1) throw Error(OLC_ERR_VALUE, "mode must be 0 (production) or 1 (reference_compatible)");
  if (c.trace_scheduler > 1) throw Error(OLC_ERR_VALUE, "trace_scheduler must be 0 (refill) or 1 (batch)");
  if (c.restir && (c.restir_candidates < 1 || c.restir_candidates > 64))
    throw Error(OLC_ERR_VALUE, "restir_candidates must be between 1 and 64");
  if (c.restir_spatial > 4) throw Error(OLC_ERR_VALUE, "restir_spatial must be between 0 and 4");
  if (c.restir_neighbours > 16) throw Error(OLC_ERR_VALUE, "restir_neighbours must be between 0 and 16");
  if (c.stack_depth != 0 && c.stack_depth != 16 && c.stack_depth != 24 && c.stack_depth != 32)
    throw Error(OLC_ERR_VALUE, "stack_depth must be 16, 24 or 32");
  if (c.block_size != 0 && (c.block_size < 64 || c.block_size > 1024 || (c.block_size & 31u)))
    throw Error(OLC_ERR_VALUE, "block_size must be a multiple of 32 in [64, 1024]");
  if (c.russian_roulette_min_survival < 0.0f || c.russian_roulette_min_survival > 1.0f)
    throw Error(OLC_ERR_VALUE, "russian_roulette_min_survival must be in [0, 1]");
}

void apply_launch_shape(olc_context* ctx) {
  ctx->ls.block = ctx->cfg.block_size ? ctx->cfg.block_size : 256;
  ctx->ls.stack_depth = ctx->cfg.stack_depth ? ctx->cfg.stack_depth : 24;
  ctx->ls.scheduler = ctx->cfg.trace_scheduler;
  ctx->ls.grid_simple = ctx->sm_count * 8;
  ctx->ls.grid_shade = ctx->sm_count * 12;
  ctx->ls.grid_trace = ctx->sm_count * 12;
}

void drop_graphs(olc_context* ctx) {
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_timelines.clear();
}

void tl_record(olc_context* ctx, size_t index) {
  while (ctx->tl_events.size() <= index) {
    cudaEvent_t e;
    OLC_CUDA(cudaEventCreate(&e));
    ctx->tl_events.push_back(e);
  }
  if (ctx->capturing)
    OLC_CUDA(cudaEventRecordWithFlags(ctx->tl_events[index], ctx->stream, cudaEventRecordExternal));
  else
    OLC_CUDA(cudaEventRecord(ctx->tl_events[index], ctx->stream));
}

void tl_begin(olc_context* ctx) {
  ctx->tl_entries.clear();
  tl_record(ctx, 0);
}

void tl_mark(olc_context* ctx, uint32_t stage, uint32_t bounce, uint32_t chunk) {
  ctx->tl_entries.push_back(TimelineEntry{stage, bounce, chunk});
  tl_record(ctx, ctx->tl_entries.size());
}

// Inverse of a row-major 3x4 affine (double precision on the host).
void invert_affine(const float* m, float* out) {
  double a[3][4];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 4; ++c) a[r][c] = m[4 * r + c];
  double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
               a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
  if (!(std::fabs(det) > 1e-30)) throw Error(OLC_ERR_VALUE, "instance transform is not invertible");
  double inv[3][3];
  inv[0][0] = (a[1][1] * a[2][2] - a[1][2] * a[2][1]) / det;
  inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
  inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
  inv[1][0] = (a[1][2] * a[2][0] - a[1][0] * a[2][2]) / det;
  inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
  inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
  inv[2][0] = (a[1][0] * a[2][1] - a[1][1] * a[2][0]) / det;
  inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
  inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
  for (int r = 0; r < 3; ++r) {
    double t = -(inv[r][0] * a[0][3] + inv[r][1] * a[1][3] + inv[r][2] * a[2][3]);
    for (int c = 0; c < 3; ++c) out[4 * r + c] = (float)inv[r][c];
    out[4 * r + 3] = (float)t;
  }
}

template <class T>
void upload(DeviceBuffer& buf, const T* host, size_t count, cudaStream_t stream, uint64_t& bytes) {
  size_t b = std::max<size_t>(count, 1) * sizeof(T);
  buf.allocate(b);
  if (count && host) OLC_CUDA(cudaMemcpyAsync(buf.get(), host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
  else OLC_CUDA(cudaMemsetAsync(buf.get(), 0, b, stream));
  bytes += b;
}

// Emitter records for sampling from the reference layout (a, b, c, emission +
// area, cdf/pdf/two-sided; Scene.emissive_triangle_data), plus a Vose alias
// table over the pdfs (M. D. Vose, "A linear algorithm for generating random
// numbers with a given distribution", IEEE TSE 1991).
void build_emitters(const olc_scene_desc* d, std::vector<EmitterRec>& em, std::vector<AliasEntry>& alias) {
  const uint32_t n = d->num_emitters;
  em.resize(n);
  alias.resize(n);
  if (n == 0) return;
  if (!d->emitters) throw Error(OLC_ERR_VALUE, "emitter records are required");
  std::vector<double> p(n);
  double total = 0.0;
  for (uint32_t i = 0; i < n; ++i) {
    const float* r = d->emitters + 20ull * i;
    float3 a = make_float3(r[0], r[1], r[2]), b = make_float3(r[4], r[5], r[6]), c = make_float3(r[8], r[9], r[10]);
    float3 e1 = b - a, e2 = c - a;
    float3 nrm = normalize(cross(e1, e2));
    float pdf = r[17];
    if (!(pdf >= 0.0f) || !std::isfinite(pdf)) throw Error(OLC_ERR_VALUE, "emitter pdf must be finite and >= 0");
    em[i].a_pdf = make_float4(a.x, a.y, a.z, pdf);
    em[i].e1_area = make_float4(e1.x, e1.y, e1.z, r[15]);
    em[i].e2_sided = make_float4(e2.x, e2.y, e2.z, r[18] > 0.5f ? 1.0f : 0.0f);
    em[i].normal = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
    em[i].emission = make_float4(r[12], r[13], r[14], 0.0f);
    p[i] = pdf;
    total += pdf;
  }
  if (!(total > 0.0)) throw Error(OLC_ERR_VALUE, "emitter pdfs sum to zero");
  std::vector<double> scaled(n);
  std::vector<uint32_t> small, large;
  for (uint32_t i = 0; i < n; ++i) {
    scaled[i] = p[i] / total * n;
    (scaled[i] < 1.0 ? small : large).push_back(i);
  }
  while (!small.empty() && !large.empty()) {
    uint32_t s = small.back(), l = large.back();
    small.pop_back();
    alias[s].threshold = (float)scaled[s];
    alias[s].alias = l;
    scaled[l] = (scaled[l] + scaled[s]) - 1.0;
    if (scaled[l] < 1.0) {
      large.pop_back();
      small.push_back(l);
    }
  }
  for (uint32_t i : large) alias[i] = AliasEntry{1.0f, i};
  for (uint32_t i : small) alias[i] = AliasEntry{1.0f, i};
}

void build_scene(olc_context* ctx, const olc_scene_desc* d, ScenePack& sp) {
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = ctx->stream;
  if (!d) throw Error(OLC_ERR_VALUE, "scene description is null");
  const uint32_t nm = d->num_meshes, ni = d->num_instances;
  if (nm && (!d->mesh_vertex_offset || !d->mesh_triangle_offset))
    throw Error(OLC_ERR_VALUE, "mesh offsets are required");
  uint32_t total_v = nm ? d->mesh_vertex_offset[nm] : 0, total_t = nm ? d->mesh_triangle_offset[nm] : 0;
  if (total_t >= (1u << 28)) throw Error(OLC_ERR_VALUE, "scene exceeds 2^28 triangles");
  for (uint32_t m = 0; m < nm; ++m) {
    if (d->mesh_vertex_offset[m + 1] < d->mesh_vertex_offset[m] ||
        d->mesh_triangle_offset[m + 1] < d->mesh_triangle_offset[m])
      throw Error(OLC_ERR_VALUE, "mesh offsets must be non-decreasing");
    uint32_t nv = d->mesh_vertex_offset[m + 1] - d->mesh_vertex_offset[m];
    for (uint64_t k = 3ull * d->mesh_triangle_offset[m]; k < 3ull * d->mesh_triangle_offset[m + 1]; ++k)
      if (d->indices[k] >= nv) throw Error(OLC_ERR_VALUE, "an index refers to a vertex that does not exist");
  }
  for (uint32_t i = 0; i < ni; ++i) {
    if (d->instance_mesh[i] >= nm) throw Error(OLC_ERR_VALUE, "instance refers to a missing mesh");
    if (d->instance_material[i] >= d->num_materials) throw Error(OLC_ERR_VALUE, "instance refers to a missing material");
  }
  uint64_t bytes = 0;
  // geometry staging (device copies of the host arrays)
  DeviceBuffer dv, dn, di;
  upload(dv, d->vertices, 3ull * total_v, st, bytes);
  upload(dn, d->normals, 3ull * total_v, st, bytes);
  upload(di, d->indices, 3ull * total_t, st, bytes);
  bytes = 0;
  // ---- instance flattening: instances of meshes with at most
  // kFlattenMaxTriangles triangles are baked into one world-space mesh.
  auto mesh_tris = [&](uint32_t m) { return d->mesh_triangle_offset[m + 1] - d->mesh_triangle_offset[m]; };
  std::vector<uint8_t> flat(ni, 0);
  uint64_t flat_tris = 0;
  uint32_t flat_count = 0;
  for (uint32_t i = 0; i < ni; ++i) {
    uint32_t nt = mesh_tris(d->instance_mesh[i]);
    if (nt > 0 && nt <= kFlattenMaxTriangles) {
      flat[i] = 1;
      flat_tris += nt;
      ++flat_count;
    }
  }
  if (!ctx->cfg.flatten_instances || flat_count < 2 || flat_tris > kFlattenMaxTotal) {
    std::fill(flat.begin(), flat.end(), 0);
    flat_tris = 0;
    flat_count = 0;
  }
  const bool flattening = flat_count > 0;
  // internal instance order: TLAS members (instances kept as instances, then
  // the flattened mesh's identity instance), then the flattened originals.
  std::vector<uint32_t> order;
  for (uint32_t i = 0; i < ni; ++i)
    if (!flat[i]) order.push_back(i);
  const uint32_t pseudo = (uint32_t)order.size();
  const uint32_t tlas_members = pseudo + (flattening ? 1u : 0u);
  std::vector<uint32_t> internal_of(ni);
  for (uint32_t k = 0; k < pseudo; ++k) internal_of[order[k]] = k;
  {
    uint32_t k = tlas_members;
    for (uint32_t i = 0; i < ni; ++i)
      if (flat[i]) internal_of[i] = k++;
  }
  const uint32_t n_records = tlas_members + flat_count;
  // meshes that still need their own BLAS
  std::vector<uint8_t> mesh_used(nm, 0);
  for (uint32_t k = 0; k < pseudo; ++k) mesh_used[d->instance_mesh[order[k]]] = 1;
  // node pool: BLAS nodes, the flattened mesh, then TLAS nodes
  std::vector<uint32_t> node_base(nm), blas_root(nm, 0);
  uint32_t nodes_total = 0;
  for (uint32_t m = 0; m < nm; ++m) {
    node_base[m] = nodes_total;
    if (mesh_used[m]) nodes_total += blas_node_count(mesh_tris(m));
  }
  uint32_t tlas_base = nodes_total;
  const uint64_t tlas_prims = (uint64_t)pseudo + flat_tris;  // instances + direct triangles
  uint32_t tlas_nodes = tlas_prims > 1 ? (uint32_t)(tlas_prims - 1) : 1;
  nodes_total += tlas_nodes;
  const uint64_t total_slots = (uint64_t)total_t + flat_tris;
  if (total_slots >= (1ull << 28)) throw Error(OLC_ERR_VALUE, "scene exceeds 2^28 triangles");
  sp.nodes.allocate((size_t)nodes_total * sizeof(BvhNode));
  sp.tri_verts.allocate(std::max<size_t>(total_slots, 1) * 3 * sizeof(float4));
  sp.tri_normals.allocate(std::max<size_t>(total_slots, 1) * 3 * sizeof(float4));
  sp.tri_index.allocate(std::max<size_t>(total_slots, 1) * sizeof(uint32_t));
  sp.tri_owner.allocate(std::max<size_t>(total_slots, 1) * sizeof(uint32_t));
  OLC_CUDA(cudaMemsetAsync(sp.tri_owner.get(), 0, sp.tri_owner.bytes(), st));
  bytes += sp.nodes.bytes() + sp.tri_verts.bytes() + sp.tri_normals.bytes() + sp.tri_index.bytes() +
           sp.tri_owner.bytes();
  sp.blas_ranges.clear();
  for (uint32_t m = 0; m < nm; ++m) {
    if (!mesh_used[m]) continue;
    BlasDesc bd;
    uint32_t v0 = d->mesh_vertex_offset[m], t0i = d->mesh_triangle_offset[m];
    bd.vertices = dv.as<float>() + 3ull * v0;
    bd.normals = dn.as<float>() + 3ull * v0;
    bd.indices = di.as<uint32_t>() + 3ull * t0i;
    bd.num_vertices = d->mesh_vertex_offset[m + 1] - v0;
    bd.num_triangles = mesh_tris(m);
    blas_root[m] = build_blas(bd, ctx->scratch, sp.nodes.as<BvhNode>(), node_base[m], sp.tri_verts.as<float4>(),
                              sp.tri_normals.as<float4>(), sp.tri_index.as<uint32_t>(), t0i, 4, st);
    sp.blas_ranges.push_back({blas_root[m], t0i, t0i + bd.num_triangles});
  }
  // instance records (internal order)
  std::vector<InstanceRec> inst(n_records);
  std::vector<float> o2w(12ull * std::max<uint32_t>(tlas_members, 1), 0.0f);
  auto fill_record = [&](InstanceRec& r, const float* m) {
    float w2o[12];
    invert_affine(m, w2o);
    r.w2o0 = make_float4(w2o[0], w2o[1], w2o[2], w2o[3]);
    r.w2o1 = make_float4(w2o[4], w2o[5], w2o[6], w2o[7]);
    r.w2o2 = make_float4(w2o[8], w2o[9], w2o[10], w2o[11]);
    r.o2w0 = make_float4(m[0], m[1], m[2], m[3]);
    r.o2w1 = make_float4(m[4], m[5], m[6], m[7]);
    r.o2w2 = make_float4(m[8], m[9], m[10], m[11]);
    r.flags = 0;
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
  };
  for (uint32_t i = 0; i < ni; ++i) {
    const float* m = d->instance_object_to_world + 12ull * i;
    for (int k = 0; k < 12; ++k)
      if (!std::isfinite(m[k])) throw Error(OLC_ERR_VALUE, "instance transform must be finite");
    const uint32_t k = internal_of[i];
    InstanceRec& r = inst[k];
    fill_record(r, m);
    r.blas_root = blas_root[d->instance_mesh[i]];
    r.material = d->instance_material[i];
    r.prim_offset = d->instance_primitive_offset[i];
    r.instance_id = d->instance_id[i];
    if (k < tlas_members)
      for (int c = 0; c < 12; ++c) o2w[12ull * k + c] = m[c];
  }
  if (flattening) {
    // world-space triangles of the flattened instances, in packed order,
    // written straight into their slots; the TLAS references them directly
    std::vector<float4> fv(3ull * flat_tris), fn(3ull * flat_tris);
    std::vector<uint32_t> fpacked(flat_tris), fowner(flat_tris);
    uint64_t t = 0;
    for (uint32_t i = 0; i < ni; ++i) {
      if (!flat[i]) continue;
      const InstanceRec& r = inst[internal_of[i]];
      Affine mo{r.o2w0, r.o2w1, r.o2w2}, mw{r.w2o0, r.w2o1, r.w2o2};
      const uint32_t m = d->instance_mesh[i];
      const uint32_t v0 = d->mesh_vertex_offset[m];
      for (uint32_t lt = 0; lt < mesh_tris(m); ++lt, ++t) {
        for (int c = 0; c < 3; ++c) {
          uint32_t vi = v0 + d->indices[3ull * (d->mesh_triangle_offset[m] + lt) + c];
          float3 p = xform_point(mo, make_float3(d->vertices[3ull * vi], d->vertices[3ull * vi + 1],
                                                 d->vertices[3ull * vi + 2]));
          float3 nn = normalize(xform_normal_by_inverse(
              mw, make_float3(d->normals[3ull * vi], d->normals[3ull * vi + 1], d->normals[3ull * vi + 2])));
          fv[3 * t + c] = make_float4(p.x, p.y, p.z, 0.0f);
          fn[3 * t + c] = make_float4(nn.x, nn.y, nn.z, 0.0f);
        }
        fpacked[t] = r.prim_offset + lt;
        fowner[t] = internal_of[i];
      }
    }
    OLC_CUDA(cudaMemcpyAsync(sp.tri_verts.as<float4>() + 3ull * total_t, fv.data(), fv.size() * sizeof(float4),
                             cudaMemcpyHostToDevice, st));
    OLC_CUDA(cudaMemcpyAsync(sp.tri_normals.as<float4>() + 3ull * total_t, fn.data(), fn.size() * sizeof(float4),
                             cudaMemcpyHostToDevice, st));
    OLC_CUDA(cudaMemcpyAsync(sp.tri_index.as<uint32_t>() + total_t, fpacked.data(), fpacked.size() * 4,
                             cudaMemcpyHostToDevice, st));
    OLC_CUDA(cudaMemcpyAsync(sp.tri_owner.as<uint32_t>() + total_t, fowner.data(), fowner.size() * 4,
                             cudaMemcpyHostToDevice, st));
    OLC_CUDA(cudaStreamSynchronize(st));  // the host staging vectors go out of scope
    // identity record that hits on direct triangles report as their instance
    const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    InstanceRec& r = inst[pseudo];
    fill_record(r, identity);
    r.blas_root = 0;
    r.material = 0;
    r.prim_offset = 0;
    r.instance_id = 0xffffffffu;
    r.flags = OLC_INSTANCE_FLATTENED;
  }
  upload(sp.instances, inst.data(), n_records, st, bytes);
  upload(sp.o2w, o2w.data(), 12ull * std::max<uint32_t>(pseudo, 1), st, bytes);
  std::vector<uint2> ranges(std::max<uint32_t>(pseudo, 1));
  for (uint32_t k = 0; k < pseudo; ++k) {
    const uint32_t m = d->instance_mesh[order[k]];
    ranges[k] = make_uint2(d->mesh_triangle_offset[m], d->mesh_triangle_offset[m + 1]);
  }
  DeviceBuffer dranges;
  uint64_t scratch_bytes = 0;
  upload(dranges, ranges.data(), pseudo, st, scratch_bytes);
  uint32_t tlas_root = build_tlas(sp.o2w.as<float>(), dranges.as<uint2>(), pseudo, sp.tri_verts.as<float4>(),
                                  sp.tri_verts.as<float4>() + 3ull * total_t, (uint32_t)flat_tris, ctx->scratch,
                                  sp.nodes.as<BvhNode>(), tlas_base, st);
  OLC_CUDA(cudaStreamSynchronize(st));  // dranges goes out of scope
  sp.flattened_instances = flat_count;
  sp.tlas_instances = tlas_members;
  // materials
  std::vector<MaterialRec> mats(d->num_materials);
  std::vector<MaterialAux> aux(d->num_materials);
  for (uint32_t k = 0; k < d->num_materials; ++k) {
    const float* p = d->materials + 16ull * k;
    mats[k].base_rough = make_float4(p[0], p[1], p[2], p[3]);
    mats[k].emit_metal = make_float4(p[4], p[5], p[6], p[7]);
    aux[k].two_sided = p[8] > 0.5f ? 1u : 0u;
    uint32_t mid;
    std::memcpy(&mid, &p[9], 4);
    aux[k].material_id = mid;
    aux[k].pad0 = aux[k].pad1 = 0;
  }
  upload(sp.materials, mats.data(), mats.size(), st, bytes);
  upload(sp.material_aux, aux.data(), aux.size(), st, bytes);
  {
    std::vector<EmitterRec> em;
    std::vector<AliasEntry> alias;
    build_emitters(d, em, alias);
    upload(sp.emitters, em.data(), em.size(), st, bytes);
    upload(sp.emitter_alias, alias.data(), alias.size(), st, bytes);
  }
  upload(sp.lights, reinterpret_cast<const LightRec*>(d->lights), d->num_lights, st, bytes);
  size_t env_count = d->environment_kind == OLC_ENV_EQUIRECT ? 3ull * d->environment_width * d->environment_height : 0;
  if (d->environment_kind == OLC_ENV_EQUIRECT && (!d->environment_image || env_count == 0))
    throw Error(OLC_ERR_VALUE, "equirect environment needs an image");
  upload(sp.env_image, d->environment_image, env_count, st, bytes);
  size_t vol_count = d->volume_present ? (size_t)d->volume_dims[0] * d->volume_dims[1] * d->volume_dims[2] : 0;
  upload(sp.volume, d->volume_density, vol_count, st, bytes);

  SceneView& v = sp.view;
  v.nodes = sp.nodes.as<BvhNode>();
  v.tri_verts = sp.tri_verts.as<float4>();
  v.tri_normals = sp.tri_normals.as<float4>();
  v.tri_index = sp.tri_index.as<uint32_t>();
  v.tri_owner = sp.tri_owner.as<uint32_t>();
  v.instances = sp.instances.as<InstanceRec>();
  v.materials = sp.materials.as<MaterialRec>();
  v.material_aux = sp.material_aux.as<MaterialAux>();
  v.emitters = sp.emitters.as<EmitterRec>();
  v.emitter_alias = sp.emitter_alias.as<AliasEntry>();
  v.lights = sp.lights.as<LightRec>();
  v.env_image = sp.env_image.as<float>();
  v.volume = sp.volume.as<float>();
  v.tlas_root = tlas_root;
  v.num_instances = tlas_members;
  v.tlas_instances = pseudo;
  v.flat_slot_base = total_t;
  v.flat_instance = pseudo;
  v.num_emitters = d->num_emitters;
  v.num_lights = d->num_lights;
  v.emissive_weight = d->emissive_weight;
  v.env_kind = d->environment_kind;
  v.env_color = make_float3(d->environment_color[0], d->environment_color[1], d->environment_color[2]);
  v.env_rotation = d->environment_rotation;
  v.env_w = d->environment_width;
  v.env_h = d->environment_height;
  v.volume_present = d->volume_present;
  v.vol_nx = d->volume_dims[0];
  v.vol_ny = d->volume_dims[1];
  v.vol_nz = d->volume_dims[2];
  const float* vb = d->volume_world_to_box;
  v.vol_world_to_box.r0 = make_float4(vb[0], vb[1], vb[2], vb[3]);
  v.vol_world_to_box.r1 = make_float4(vb[4], vb[5], vb[6], vb[7]);
  v.vol_world_to_box.r2 = make_float4(vb[8], vb[9], vb[10], vb[11]);
  v.vol_sigma_t_scale = d->volume_sigma_t_scale;
  v.vol_albedo = d->volume_albedo;
  v.vol_max_density = d->volume_max_density;
  OLC_CUDA(cudaStreamSynchronize(st));
  sp.total_triangles = total_t;
  sp.blas_nodes = tlas_base;
  sp.tlas_nodes = tlas_nodes;
  sp.blas_count = nm;
  sp.bytes = bytes;
  sp.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  sp.valid = true;
}

void ensure_wavefront(olc_context* ctx, uint32_t capacity, uint32_t npix) {
  if (capacity > ctx->capacity) {
    size_t c = capacity;
    ctx->q0_o.allocate(c * 16);
    ctx->q0_d.allocate(c * 16);
    ctx->q0_p.allocate(c * 4);
    ctx->q1_o.allocate(c * 16);
    ctx->q1_d.allocate(c * 16);
    ctx->q1_p.allocate(c * 4);
    ctx->hit_tuv.allocate(c * 16);
    ctx->hit_inst.allocate(c * 4);
    ctx->sh_o.allocate(c * 16);
    ctx->sh_d.allocate(c * 16);
    ctx->sh_c.allocate(c * 16);
    ctx->ps_tp.allocate(c * 16);
    ctx->ps_rad.allocate(c * 16);
    ctx->ps_meta.allocate(c * 16);
    ctx->capacity = capacity;
    drop_graphs(ctx);
  }
  if (npix > ctx->npix_capacity) {
    size_t n = npix;
    ctx->accum.allocate(n * 3 * 8);
    ctx->out_dev.allocate(n * 16);
    ctx->prod_depth.allocate(n * 4);
    ctx->prod_normal.allocate(n * 16);
    ctx->prod_inst.allocate(n * 4);
    ctx->prod_mat.allocate(n * 4);
    ctx->prod_prim.allocate(n * 4);
    ctx->npix_capacity = npix;
    drop_graphs(ctx);
  }
  if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
  if (!ctx->fp_dev.get()) ctx->fp_dev.allocate(sizeof(FrameParams));
}

void ensure_host_counters(olc_context* ctx, uint32_t chunks) {
  if (chunks <= ctx->counters_host_chunks) return;
  if (ctx->counters_host) cudaFreeHost(ctx->counters_host);
  ctx->counters_host = nullptr;
  OLC_CUDA(cudaMallocHost(&ctx->counters_host, sizeof(Counters) * chunks));
  ctx->counters_host_chunks = chunks;
  drop_graphs(ctx);
}

void fill_frame(olc_context* ctx, const olc_camera* cam, uint32_t w, uint32_t h, uint32_t spp, uint32_t frame_index) {
  FrameParams& f = *ctx->fp_host;
  f.cam_pos = make_float4(cam->position[0], cam->position[1], cam->position[2], 0.0f);
  f.cam_forward = make_float4(cam->forward[0], cam->forward[1], cam->forward[2], 0.0f);
  f.cam_right = make_float4(cam->right[0], cam->right[1], cam->right[2], 0.0f);
  f.cam_up = make_float4(cam->up[0], cam->up[1], cam->up[2], 0.0f);
  if (cam->projection == OLC_PROJECTION_PANORAMIC) {
    f.cam_pos.w = cam->horizontal_half;
    f.cam_forward.w = cam->vertical_half;
  } else {
    f.cam_pos.w = (float)((double)w / (double)h * (double)cam->half_height);
    f.cam_forward.w = cam->half_height;
  }
  f.projection = cam->projection;
  f.width = w;
  f.height = h;
  f.spp = spp;
  f.frame = ctx->cfg.seed + frame_index;
  f.npix = w * h;
  f.max_bounces = ctx->cfg.max_bounces;
  f.mode = ctx->cfg.mode;
  f.rr_start = ctx->cfg.mode == OLC_MODE_PRODUCTION ? ctx->cfg.russian_roulette_start : 0u;
  f.rr_min_survival = ctx->cfg.russian_roulette_min_survival;
  f.restir = ctx->cfg.restir;
  f.nee = ctx->cfg.disable_nee ? 0u : 1u;
}

struct Timing {
  bool on = false;
  cudaEvent_t ev[8] = {};
  float ms[7] = {};
};

// Record the device work of one frame into ctx->stream.
void record_frame(olc_context* ctx, uint32_t w, uint32_t h, uint32_t spp, bool products) {
  cudaStream_t st = ctx->stream;
  const uint32_t npix = w * h;
  const uint64_t total = (uint64_t)npix * spp;
  const uint32_t cap = ctx->capacity;
  const uint32_t chunks = (uint32_t)((total + cap - 1) / cap);
  const SceneView& s = ctx->scene.view;
  const FrameParams* fp = ctx->fp_dev.as<FrameParams>();
  Counters* cnt = ctx->counters.as<Counters>();
  RayQueue qa{ctx->q0_o.as<float4>(), ctx->q0_d.as<float4>(), ctx->q0_p.as<uint32_t>()};
  RayQueue qb{ctx->q1_o.as<float4>(), ctx->q1_d.as<float4>(), ctx->q1_p.as<uint32_t>()};
  HitBuf hb{ctx->hit_tuv.as<float4>(), ctx->hit_inst.as<uint32_t>()};
  ShadowQueue sq{ctx->sh_o.as<float4>(), ctx->sh_d.as<float4>(), ctx->sh_c.as<float4>()};
  PathState ps{ctx->ps_tp.as<float4>(), ctx->ps_rad.as<float4>(), ctx->ps_meta.as<uint4>()};
  ProductPtrs prod;
  if (products) {
    prod.depth = ctx->prod_depth.as<float>();
    prod.normal = ctx->prod_normal.as<float4>();
    prod.instance_id = ctx->prod_inst.as<uint32_t>();
    prod.material_id = ctx->prod_mat.as<uint32_t>();
    prod.primitive_id = ctx->prod_prim.as<uint32_t>();
  }
  const float t_min = ctx->cfg.mode == OLC_MODE_REFERENCE_COMPATIBLE ? 1e-4f : 0.001f;
  OLC_CUDA(cudaMemsetAsync(ctx->accum.get(), 0, (size_t)npix * 3 * 8, st));
  tl_begin(ctx);
  for (uint32_t c = 0; c < chunks; ++c) {
    uint64_t begin = (uint64_t)c * cap;
    uint32_t count = (uint32_t)std::min<uint64_t>(cap, total - begin);
    OLC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(Counters), st));
    launch_raygen(ctx->ls, fp, begin, count, qa, ps, cnt, t_min, st);
    tl_mark(ctx, OLC_STAGE_RAYGEN, 0, c);
    RayQueue* qin = &qa;
    RayQueue* qout = &qb;
    for (uint32_t b = 0; b < ctx->cfg.max_bounces; ++b) {
      launch_trace_closest(ctx->ls, s, *qin, hb, cnt, b, st);
      tl_mark(ctx, OLC_STAGE_TRACE, b, c);
      const uint4* restir = nullptr;
      if (b == 0 && ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION && s.num_emitters > 0) {
        restir = restir_run(ctx->restir, ctx->cfg, ctx->ls, s, fp, *qin, hb, ps, cnt, begin, count, npix, st);
        tl_mark(ctx, OLC_STAGE_RESTIR, b, c);
      }
      launch_shade(ctx->ls, ctx->cfg.mode, fp, s, *qin, hb, *qout, sq, ps, cnt, b, cap,
                   (products && c == 0) ? prod : ProductPtrs{}, restir, st);
      tl_mark(ctx, OLC_STAGE_SHADE, b, c);
      launch_trace_shadow(ctx->ls, s, sq, ps, cnt, b, st);
      tl_mark(ctx, OLC_STAGE_SHADOW, b, c);
      std::swap(qin, qout);
    }
    launch_accumulate(ctx->ls, ps, count, ctx->accum.as<unsigned long long>(), cnt, st);
    tl_mark(ctx, OLC_STAGE_ACCUMULATE, 0, c);
    OLC_CUDA(cudaMemcpyAsync(ctx->counters_host + c, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
  }
  launch_resolve(ctx->ls, ctx->accum.as<unsigned long long>(), npix, spp, ctx->out_dev.as<float4>(), st);
  tl_mark(ctx, OLC_STAGE_RESOLVE, 0, 0);
}

uint32_t choose_capacity(olc_context* ctx, uint32_t npix, uint32_t spp) {
  uint64_t total = (uint64_t)npix * spp;
  uint64_t cap = ctx->cfg.chunk_paths ? ctx->cfg.chunk_paths : (1ull << 24);
  if (ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION) {
    // whole sample streams per chunk (spatial reuse reads neighbours)
    uint64_t streams = std::max<uint64_t>(1, cap / npix);
    cap = streams * npix;
  }
  cap = std::min<uint64_t>(cap, total);
  if (cap > 0xffffffffull) cap = 0xffffffffull;
  return (uint32_t)cap;
}

}  // namespace

namespace olc {
void set_thread_error(const std::string& message) { g_thread_error = message; }
}  // namespace olc

extern "C" {

int olc_abi_version(void) { return OLC_ABI_VERSION; }

const char* olc_last_error(const olc_context* ctx) {
  if (ctx) return ctx->error.c_str();
  return g_thread_error.c_str();
}

int olc_create(const olc_config* cfg, olc_context** out) {
  if (!cfg || !out) return fail(nullptr, OLC_ERR_VALUE, "config and output pointer are required");
  *out = nullptr;
  std::unique_ptr<olc_context> ctx(new olc_context());
  int rc = guarded(nullptr, [&] {
    validate_config(*cfg);
    int n = 0;
    OLC_CUDA(cudaGetDeviceCount(&n));
    if (cfg->device < 0 || cfg->device >= n) throw Error(OLC_ERR_VALUE, "CUDA device ordinal out of range");
    ctx->cfg = *cfg;
    ctx->device = cfg->device;
    OLC_CUDA(cudaSetDevice(ctx->device));
    cudaDeviceProp prop;
    OLC_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    ctx->sm_count = prop.multiProcessorCount;
    OLC_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    OLC_CUDA(cudaEventCreate(&ctx->ev_begin));
    OLC_CUDA(cudaEventCreate(&ctx->ev_end));
    OLC_CUDA(cudaMallocHost(&ctx->fp_host, sizeof(FrameParams)));
    std::memset(ctx->fp_host, 0, sizeof(FrameParams));
    configure_trace_kernels();
    apply_launch_shape(ctx.get());
  });
  if (rc != OLC_OK) {
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    return rc;
  }
  *out = ctx.release();
  return OLC_OK;
}

int olc_destroy(olc_context* ctx) {
  if (!ctx) return OLC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  drop_graphs(ctx);
  restir_release(ctx->restir);
  if (ctx->fp_host) cudaFreeHost(ctx->fp_host);
  if (ctx->counters_host) cudaFreeHost(ctx->counters_host);
  for (cudaEvent_t e : ctx->tl_events) cudaEventDestroy(e);
  if (ctx->ev_begin) cudaEventDestroy(ctx->ev_begin);
  if (ctx->ev_end) cudaEventDestroy(ctx->ev_end);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return OLC_OK;
}

int olc_reconfigure(olc_context* ctx, const olc_config* cfg) {
  if (!ctx || !cfg) return fail(ctx, OLC_ERR_VALUE, "context and config are required");
  return guarded(ctx, [&] {
    validate_config(*cfg);
    if (cfg->device != ctx->cfg.device) throw Error(OLC_ERR_RUNTIME, "changing the device requires a new renderer");
    bool restir_changed = cfg->restir != ctx->cfg.restir || cfg->restir_candidates != ctx->cfg.restir_candidates;
    ctx->cfg = *cfg;
    apply_launch_shape(ctx);
    drop_graphs(ctx);
    if (restir_changed) restir_reset(ctx->restir);
  });
}

int olc_upload_scene(olc_context* ctx, const olc_scene_desc* scene) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    ScenePack fresh;
    build_scene(ctx, scene, fresh);   // throws before touching the resident scene
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->scene = std::move(fresh);
    drop_graphs(ctx);
    restir_reset(ctx->restir);
  });
}

int olc_scene_bytes(const olc_context* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  *bytes = ctx->scene.bytes;
  return OLC_OK;
}

int olc_render(olc_context* ctx, const olc_camera* camera, uint32_t width, uint32_t height, uint32_t spp,
               uint32_t frame_index, float* out_rgba, int out_is_device, olc_render_stats* stats) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (!camera) throw Error(OLC_ERR_VALUE, "camera is required");
    if (width == 0 || height == 0) throw Error(OLC_ERR_VALUE, "width and height must be positive");
    if ((uint64_t)width * height > (1ull << 28)) throw Error(OLC_ERR_VALUE, "image is too large");
    if (spp < 1 || spp > 65536) throw Error(OLC_ERR_VALUE, "samples must be between 1 and 65536");
    if (camera->projection > 2) throw Error(OLC_ERR_VALUE, "unknown camera projection");
    if (!ctx->scene.valid) throw Error(OLC_ERR_RUNTIME, "no scene is resident; upload a scene first");
    if (!out_rgba) throw Error(OLC_ERR_VALUE, "output pointer is required");
    const uint32_t npix = width * height;
    uint32_t cap = choose_capacity(ctx, npix, spp);
    ensure_wavefront(ctx, cap, npix);
    uint64_t total = (uint64_t)npix * spp;
    uint32_t chunks = (uint32_t)((total + ctx->capacity - 1) / ctx->capacity);
    ensure_host_counters(ctx, chunks);
    fill_frame(ctx, camera, width, height, spp, frame_index);
    if (ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION)
      restir_prepare(ctx->restir, ctx->cfg, width, height, spp, frame_index, ctx->capacity, *ctx->fp_host);
    cudaStream_t st = ctx->stream;
    OLC_CUDA(cudaMemcpyAsync(ctx->fp_dev.get(), ctx->fp_host, sizeof(FrameParams), cudaMemcpyHostToDevice, st));
    bool products = true;
    OLC_CUDA(cudaEventRecord(ctx->ev_begin, st));
    bool use_graph = ctx->cfg.use_graphs != 0 && !(ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION);
    if (use_graph) {
      GraphKey key{width, height, spp};
      auto it = ctx->graphs.find(key);
      if (it == ctx->graphs.end()) {
        cudaGraph_t g;
        OLC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        ctx->capturing = true;
        try {
          record_frame(ctx, width, height, spp, products);
        } catch (...) {
          ctx->capturing = false;
          cudaStreamEndCapture(st, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        ctx->capturing = false;
        OLC_CUDA(cudaStreamEndCapture(st, &g));
        cudaGraphExec_t exec;
        cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        OLC_CUDA(e);
        it = ctx->graphs.emplace(key, exec).first;
        ctx->graph_timelines[key] = ctx->tl_entries;
      }
      ctx->tl_entries = ctx->graph_timelines[key];
      OLC_CUDA(cudaGraphLaunch(it->second, st));
    } else {
      record_frame(ctx, width, height, spp, products);
    }
    OLC_CUDA(cudaEventRecord(ctx->ev_end, st));
    if (out_is_device) {
      OLC_CUDA(cudaMemcpyAsync(out_rgba, ctx->out_dev.get(), (size_t)npix * 16, cudaMemcpyDeviceToDevice, st));
    } else {
      OLC_CUDA(cudaMemcpyAsync(out_rgba, ctx->out_dev.get(), (size_t)npix * 16, cudaMemcpyDeviceToHost, st));
    }
    OLC_CUDA(cudaStreamSynchronize(st));
    ctx->last_w = width;
    ctx->last_h = height;
    if (ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION) restir_finish(ctx->restir);
    // per-launch device timeline
    ctx->last_profile.clear();
    float stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
    for (size_t k = 0; k < ctx->tl_entries.size(); ++k) {
      const TimelineEntry& e = ctx->tl_entries[k];
      olc_launch_record r{};
      r.stage = e.stage;
      r.bounce = e.bounce;
      r.chunk = e.chunk;
      OLC_CUDA(cudaEventElapsedTime(&r.ms, ctx->tl_events[k], ctx->tl_events[k + 1]));
      const Counters& kc = ctx->counters_host[std::min<uint32_t>(e.chunk, chunks - 1)];
      uint64_t chunk_count = std::min<uint64_t>(ctx->capacity, total - (uint64_t)e.chunk * ctx->capacity);
      switch (e.stage) {
        case OLC_STAGE_RAYGEN: case OLC_STAGE_ACCUMULATE: r.items = chunk_count; break;
        case OLC_STAGE_TRACE: case OLC_STAGE_SHADE: case OLC_STAGE_RESTIR:
          r.items = kc.queue_count[e.bounce];
          r.misses = kc.miss_count[e.bounce];
          break;
        case OLC_STAGE_SHADOW: r.items = kc.shadow_count[e.bounce]; break;
        default: r.items = npix; break;
      }
      stage_ms[e.stage] += r.ms;
      ctx->last_profile.push_back(r);
    }
    if (stats) {
      std::memset(stats, 0, sizeof(*stats));
      stats->raygen_ms = stage_ms[OLC_STAGE_RAYGEN];
      stats->trace_ms = stage_ms[OLC_STAGE_TRACE];
      stats->restir_ms = stage_ms[OLC_STAGE_RESTIR];
      stats->shade_ms = stage_ms[OLC_STAGE_SHADE];
      stats->shadow_ms = stage_ms[OLC_STAGE_SHADOW];
      stats->accumulate_ms = stage_ms[OLC_STAGE_ACCUMULATE] + stage_ms[OLC_STAGE_RESOLVE];
      for (uint32_t c = 0; c < chunks; ++c) {
        const Counters& k = ctx->counters_host[c];
        stats->camera_rays += k.queue_count[0];
        for (uint32_t b = 1; b < ctx->cfg.max_bounces; ++b) stats->extension_rays += k.queue_count[b];
        for (uint32_t b = 0; b < ctx->cfg.max_bounces; ++b) stats->shadow_rays += k.shadow_count[b];
        stats->overflow += k.overflow;
        stats->traversal_errors += k.traversal_errors;
      }
      OLC_CUDA(cudaEventElapsedTime(&stats->gpu_ms, ctx->ev_begin, ctx->ev_end));
      stats->chunks = chunks;
      stats->restir_history_used = ctx->restir.history_used ? 1u : 0u;
    }
  });
}

int olc_frame_profile(const olc_context* ctx, olc_launch_record* records, uint32_t capacity, uint32_t* count) {
  if (!ctx || !count) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and count are required");
  *count = (uint32_t)ctx->last_profile.size();
  if (records) {
    uint32_t n = std::min<uint32_t>(capacity, *count);
    std::memcpy(records, ctx->last_profile.data(), sizeof(olc_launch_record) * n);
  }
  return OLC_OK;
}

int olc_stream(const olc_context* ctx, void** stream) {
  if (!ctx || !stream) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  *stream = (void*)ctx->stream;
  return OLC_OK;
}

int olc_read_products(olc_context* ctx, uint32_t width, uint32_t height, float* depth, float* normal,
                      uint32_t* instance_id, uint32_t* material_id, uint32_t* primitive_id) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (width != ctx->last_w || height != ctx->last_h)
      throw Error(OLC_ERR_VALUE, "products are available only for the size of the last render");
    const size_t n = (size_t)width * height;
    cudaStream_t st = ctx->stream;
    if (depth) OLC_CUDA(cudaMemcpyAsync(depth, ctx->prod_depth.get(), n * 4, cudaMemcpyDeviceToHost, st));
    if (instance_id) OLC_CUDA(cudaMemcpyAsync(instance_id, ctx->prod_inst.get(), n * 4, cudaMemcpyDeviceToHost, st));
    if (material_id) OLC_CUDA(cudaMemcpyAsync(material_id, ctx->prod_mat.get(), n * 4, cudaMemcpyDeviceToHost, st));
    if (primitive_id) OLC_CUDA(cudaMemcpyAsync(primitive_id, ctx->prod_prim.get(), n * 4, cudaMemcpyDeviceToHost, st));
    std::vector<float4> nrm;
    if (normal) {
      nrm.resize(n);
      OLC_CUDA(cudaMemcpyAsync(nrm.data(), ctx->prod_normal.get(), n * 16, cudaMemcpyDeviceToHost, st));
    }
    OLC_CUDA(cudaStreamSynchronize(st));
    if (normal)
      for (size_t i = 0; i < n; ++i) {
        normal[3 * i + 0] = nrm[i].x;
        normal[3 * i + 1] = nrm[i].y;
        normal[3 * i + 2] = nrm[i].z;
      }
  });
}

int olc_reset_history(olc_context* ctx) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] { restir_reset(ctx->restir); });
}

int olc_trace_closest(olc_context* ctx, uint32_t n, const float* origins, const float* directions, float t_min,
                      uint32_t* instance_id, int32_t* primitive, float* t, float* barycentrics) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (!ctx->scene.valid) throw Error(OLC_ERR_RUNTIME, "no scene is resident");
    if (n == 0) return;
    if (!origins || !directions) throw Error(OLC_ERR_VALUE, "origins and directions are required");
    if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
    OLC_CUDA(cudaMemsetAsync(ctx->counters.get(), 0, sizeof(Counters), ctx->stream));
    launch_trace_rays(ctx->ls, ctx->scene.view, n, origins, directions, t_min, instance_id, primitive, t,
                      barycentrics, ctx->counters.as<Counters>(), ctx->stream);
    Counters h;
    OLC_CUDA(cudaMemcpyAsync(&h, ctx->counters.get(), sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h.traversal_errors) throw Error(OLC_ERR_RUNTIME, "traversal stack overflow");
  });
}

int olc_trace_occluded(olc_context* ctx, uint32_t n, const float* origins, const float* directions, float t_min,
                       const float* t_max, uint8_t* occluded) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (!ctx->scene.valid) throw Error(OLC_ERR_RUNTIME, "no scene is resident");
    if (n == 0) return;
    if (!origins || !directions || !t_max || !occluded) throw Error(OLC_ERR_VALUE, "all arrays are required");
    if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
    OLC_CUDA(cudaMemsetAsync(ctx->counters.get(), 0, sizeof(Counters), ctx->stream));
    launch_occluded_rays(ctx->ls, ctx->scene.view, n, origins, directions, t_min, t_max, occluded,
                         ctx->counters.as<Counters>(), ctx->stream);
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int olc_camera_rays(olc_context* ctx, const olc_camera* camera, uint32_t width, uint32_t height, uint32_t sample,
                    uint32_t frame_index, const float* jitter_override, float* origins, float* directions) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (!camera || !origins || !directions) throw Error(OLC_ERR_VALUE, "camera and outputs are required");
    if (width == 0 || height == 0) throw Error(OLC_ERR_VALUE, "width and height must be positive");
    if (!ctx->fp_dev.get()) ctx->fp_dev.allocate(sizeof(FrameParams));
    fill_frame(ctx, camera, width, height, 1, frame_index);
    OLC_CUDA(cudaMemcpyAsync(ctx->fp_dev.get(), ctx->fp_host, sizeof(FrameParams), cudaMemcpyHostToDevice,
                             ctx->stream));
    launch_camera_rays(ctx->ls, ctx->fp_dev.as<FrameParams>(), sample, jitter_override, origins, directions,
                       ctx->stream);
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int olc_morton_codes(olc_context* ctx, uint32_t n, const float* tri_vertices, uint32_t* codes) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (n == 0) return;
    if (!tri_vertices || !codes) throw Error(OLC_ERR_VALUE, "arrays are required");
    ctx->scratch.ensure(n);
    triangle_centers_flat(tri_vertices, n, ctx->scratch.boxes_lo.as<float4>(), ctx->scratch.boxes_hi.as<float4>(),
                          ctx->scratch.centers.as<float4>(), ctx->stream);
    morton_codes(ctx->scratch.centers.as<float4>(), n, ctx->scratch.bounds.as<uint32_t>(), codes, ctx->stream);
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int olc_radix_sort_pairs(olc_context* ctx, uint32_t n, uint32_t key_bits, uint32_t* keys, uint32_t* values) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (key_bits < 1 || key_bits > 32) throw Error(OLC_ERR_VALUE, "key_bits must be between 1 and 32");
    if (n == 0) return;
    if (!keys || !values) throw Error(OLC_ERR_VALUE, "arrays are required");
    ctx->scratch.ensure(n);
    radix_sort_pairs(keys, values, ctx->scratch.keys_alt.as<uint32_t>(), ctx->scratch.vals_alt.as<uint32_t>(),
                     ctx->scratch.hist.as<uint32_t>(), n, key_bits, ctx->stream);
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int olc_bvh_info_get(const olc_context* ctx, olc_bvh_info* info) {
  if (!ctx || !info) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  std::memset(info, 0, sizeof(*info));
  info->blas_count = ctx->scene.blas_count;
  info->blas_nodes = ctx->scene.blas_nodes;
  info->tlas_nodes = ctx->scene.tlas_nodes;
  info->triangles = ctx->scene.total_triangles;
  info->build_ms = ctx->scene.build_ms;
  return OLC_OK;
}

int olc_bvh_validate(olc_context* ctx, uint64_t* bad) {
  if (!ctx || !bad) return fail(ctx, OLC_ERR_VALUE, "context and output are required");
  return guarded(ctx, [&] {
    if (!ctx->scene.valid) throw Error(OLC_ERR_RUNTIME, "no scene is resident");
    *bad = validate_bvh(ctx->scene.view, ctx->scene.blas_ranges, ctx->stream);
  });
}

}  // extern "C"
