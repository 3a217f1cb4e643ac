// C ABI of libolcuda: context, the resident scene pool, and the chunked
// wavefront executor that plain frames, batches and served requests share.
//
// Work is organised in jobs (one image of one scene) and chunks (at most
// `capacity` paths resident at once).  A job's path has the job-local index
// sample * npix + pixel.  A chunk is a list of segments, each a contiguous
// run of one job's paths, so one chunk can hold paths of many jobs and
// scenes.  Segments of ReSTIR jobs hold whole sample streams, because
// spatial reuse reads the stream's neighbouring pixels.  Per chunk: raygen,
// then per bounce trace_closest -> [ReSTIR at bounce 0] -> shade ->
// trace_shadow, then accumulate into the job's pixels in fixed point (order
// independent), so the bits of a job do not depend on how its paths are
// chunked or mixed with other jobs.
//
// A run is a sequence of chunks planned on the host.  All chunk tables reach
// the device in one copy, and the run's launches are captured into a CUDA
// graph keyed by the run's signature (each chunk's bounce count and ReSTIR
// flag plus every buffer address the launches see); later runs with the same
// signature replay it.  A plain frame is one run over one job, a batch one
// run over all its jobs, a serving step one run of one chunk over the queued
// jobs (continuous batching: jobs submitted between steps join the next
// chunk).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "olcuda.h"
#include "olc_refvolume.cuh"
#include "olc_internal.h"
#include "olc_motion.h"
#include "olc_restir.h"
#include "olc_wavefront.h"

using namespace olc;

namespace {

thread_local std::string g_thread_error;

// Instances of meshes with at most this many triangles are baked into
// world-space triangles referenced by the TLAS, up to kFlattenMaxTotal baked
// triangles per scene.
constexpr uint32_t kFlattenMaxTriangles = 64;
// Triangles per BLAS leaf.  One triangle per leaf: the parent's child box
// then bounds exactly that triangle, so a ray tests a triangle only when it
// enters its box (measured per 1080p frame against 2 / 3 / 4 / 8 per leaf:
// traversal 12 % faster than 4 on the instanced scene, 22 % on the terrain).
constexpr uint32_t kBlasLeafTriangles = 1;
constexpr uint64_t kFlattenMaxTotal = 1ull << 24;
constexpr size_t kMaxGraphs = 16;
constexpr uint64_t kDefaultChunkPaths = 1ull << 24;
constexpr uint32_t kNoScene = 0xffffffffu;

// First-fit allocator of element ranges in [0, capacity).
class RangeAllocator {
 public:
  bool allocate(uint64_t n, uint64_t& off) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      off = it->first;
      const uint64_t rest = it->second - n;
      free_.erase(it);
      if (rest) free_.emplace(off + n, rest);
      used_ += n;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t n) {
    if (n == 0) return;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  void grow(uint64_t new_capacity) {
    if (new_capacity <= capacity_) return;
    const uint64_t old = capacity_;
    capacity_ = new_capacity;
    used_ += new_capacity - old;  // release() below takes it off again
    release(old, new_capacity - old);
  }
  // Free elements at the end of the range (a growth extends them).
  uint64_t tail_free() const {
    if (free_.empty()) return 0;
    auto last = std::prev(free_.end());
    return last->first + last->second == capacity_ ? last->second : 0;
  }
  uint64_t capacity() const { return capacity_; }
  uint64_t used() const { return used_; }

 private:
  std::map<uint64_t, uint64_t> free_;  // offset -> size
  uint64_t capacity_ = 0, used_ = 0;
};

struct Range {
  uint64_t off = 0, n = 0;
};

// Device arrays indexed by one range allocator (for example the four
// per-slot triangle arrays).  Growing copies the old contents into the new
// allocation, so indices held by resident scenes and queued jobs stay valid;
// only base addresses change.
struct PoolGroup {
  std::vector<size_t> elem;  // bytes per element of each array
  std::vector<DeviceBuffer> bufs;
  RangeAllocator ranges;
  uint32_t min_capacity = 1024;

  PoolGroup(std::initializer_list<size_t> sizes, uint32_t min_cap) : elem(sizes), bufs(sizes.size()),
                                                                      min_capacity(min_cap) {}

  Range acquire(uint64_t n, cudaStream_t st) {
    Range r;
    r.n = n;
    if (n == 0) return r;
    if (ranges.allocate(n, r.off)) return r;
    const uint64_t cap = ranges.capacity();
    const uint64_t need = cap + n - ranges.tail_free();
    const uint64_t new_cap = std::max<uint64_t>({need, cap + cap / 2, (uint64_t)min_capacity});
    for (size_t k = 0; k < bufs.size(); ++k) {
      DeviceBuffer nb(new_cap * elem[k]);
      if (cap)
        OLC_CUDA(cudaMemcpyAsync(nb.get(), bufs[k].get(), cap * elem[k], cudaMemcpyDeviceToDevice, st));
      OLC_CUDA(cudaStreamSynchronize(st));
      bufs[k] = std::move(nb);
    }
    ranges.grow(new_cap);
    if (!ranges.allocate(n, r.off)) throw Error(OLC_ERR_RUNTIME, "pool allocation failed after growth");
    return r;
  }
  void release(Range& r) {
    ranges.release(r.off, r.n);
    r = Range{};
  }
  template <class T>
  T* at(size_t k, uint64_t off = 0) const {
    return reinterpret_cast<T*>(bufs[k].as<char>() + off * elem[k]);
  }
  uint64_t range_bytes(const Range& r) const {
    uint64_t b = 0;
    for (size_t e : elem) b += r.n * e;
    return b;
  }
  uint64_t bytes() const {
    uint64_t b = 0;
    for (const DeviceBuffer& d : bufs) b += d.bytes();
    return b;
  }
};

// One resident scene: its ranges of the pool and its own image and volume.
// Placement of a scene description in the pool: which instances are baked
// into world-space triangles, the scene-local instance order (TLAS members
// first, then the baked originals, whose records hold material and Mesh.id),
// and where each mesh's BLAS nodes and the TLAS go in the scene's node range.
struct SceneLayout {
  uint32_t nm = 0, ni = 0, total_v = 0, total_t = 0;
  std::vector<uint8_t> flat;
  uint64_t flat_tris = 0;
  uint32_t flat_count = 0;
  std::vector<uint32_t> order;       // member instances (not baked)
  std::vector<uint32_t> local_of;    // scene-local record of each instance
  uint32_t members = 0;
  std::vector<uint8_t> mesh_used;    // a BLAS is built for the mesh
  std::vector<uint32_t> node_local;  // first node of each built BLAS
  uint32_t tlas_local = 0, tlas_nodes = 0, node_count = 0;
  uint64_t slot_count = 0;
  // what an in-place update must find unchanged
  std::vector<uint32_t> mesh_vertex_offset, mesh_triangle_offset, instance_mesh;
  std::vector<uint32_t> instance_prim_offset;   // packed triangle base of each instance
  uint64_t packed_triangles = 0;                // Scene.triangles() length
};

struct ResidentScene {
  Range nodes, slots, instances, materials, emitters, lights;
  DeviceBuffer env_image, volume;
  DeviceBuffer tex_words, tex_bindings, tex_attr, mat_tex;   // textured scenes only
  DeviceBuffer ref_vol_recs, ref_vol_grid, ref_vol_lut;      // volumes in the reference's model
  SceneRec rec{};
  SceneLayout layout;
  std::vector<BlasRange> blas_ranges;
  std::vector<uint32_t> blas_root;   // per mesh (0 where no BLAS is built)
  uint32_t triangles = 0, blas_count = 0, blas_nodes = 0, tlas_nodes = 0, flattened = 0;
  uint64_t bytes = 0;
  double build_ms = 0.0;
};

// A job waiting for (or in) the wavefront.
struct QueuedJob {
  uint64_t ticket = 0;
  JobRec rec{};              // seg_* filled per segment
  uint64_t total = 0;        // npix * spp
  uint64_t issued = 0;       // paths handed to chunks
  Range pixels;              // accumulator / output arena range
  float* out = nullptr;
  bool out_device = false;
  bool out_staged = false;   // pageable host output: copied through the run's pinned staging
  uint64_t* sums = nullptr;  // optional fixed-point sums output (same memory kind as out)
  // ReSTIR reservoirs at job-local indices (reservoir_base 0), where the next
  // plain frame's temporal pass finds them; otherwise chunk-local ones
  bool job_local_reservoirs = false;
  bool textured = false;     // its scene has textures (the run uses the textured kernels)
  bool ref_volumes = false;  // reference-compatible job whose scene has volumes (their ray march runs)
  bool media = false;        // production job whose scene has a participating medium
  uint32_t age = 0;          // serving steps since it was queued
};

struct ChunkPlan {
  uint32_t count = 0;
  uint32_t bounces = 0;
  bool restir = false;
  bool textures = false;     // its jobs' scenes have textures (all or none of them)
  bool ref_volumes = false;  // some job marches reference volumes
  bool media = false;        // some job tracks a participating medium (the shading kernel with media)
  std::vector<JobRec> segs;
};

struct RunPlan {
  std::vector<ChunkPlan> chunks;
  std::vector<QueuedJob*> finished;  // jobs whose last paths are in this run
  uint32_t max_segments = 0;
  uint32_t max_count = 0;
  bool restir = false;               // some chunk runs ReSTIR
  bool chunk_reservoirs = false;     // some ReSTIR segment uses chunk-local reservoirs
};

// One timed stage of a run: its events (indices into the run slot's event
// list) bracket it on the stream it ran on.
struct TimelineEntry {
  uint32_t stage, bounce, chunk;
  uint32_t start, end;
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  std::vector<TimelineEntry> timeline;
  uint64_t last_used = 0;
};

// Host-visible state of one run: its tables (pinned staging and device
// copy), the counters it copies back, its launch timeline and bracketing
// events, and its plan.  Two slots let a serving step launch the next chunk
// before it waits for the previous one.
struct RunSlot {
  DeviceBuffer table_dev;
  char* table_host = nullptr;        // pinned
  size_t table_capacity = 0;
  size_t table_bytes = 0;            // bytes staged for the current run
  Counters* counters_host = nullptr; // pinned, one per chunk
  uint32_t counters_chunks = 0;
  std::vector<cudaEvent_t> events;   // events[k] .. events[k+1] brackets launch k
  std::vector<TimelineEntry> entries;
  cudaEvent_t begin = nullptr, end = nullptr, done = nullptr;
  // Pageable host outputs are copied into this pinned staging buffer by the
  // device and from it by the host when the run is collected, so the
  // device-to-host copy is asynchronous and overlaps the next run.
  float4* staging = nullptr;
  size_t staging_pixels = 0;
  std::vector<std::pair<QueuedJob*, size_t>> staged;   // job, first staging pixel
  RunPlan plan;
  bool busy = false;
};

}  // namespace

struct olc_context {
  olc_config cfg{};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  // any-hit traversal of a bounce's shadow rays runs on a second stream,
  // beside the later bounces' traversal and shading.  Shadow queues
  // alternate between two buffers by bounce parity, so shading waits only
  // for the shadow rays of two bounces back (which read the queue it
  // refills); accumulation waits for all of them
  cudaStream_t side = nullptr;
  cudaEvent_t fork_event = nullptr, join_event[2] = {nullptr, nullptr};
  bool side_pending[2] = {false, false};
  uint32_t side_last = 0;   // parity of the latest shadow launch
  uint32_t tl_next = 0, tl_last = 0;   // next event index; last event on the main stream
  std::string error;
  BuildScratch scratch;
  LaunchShape ls;
  // scene pool
  PoolGroup nodes{{sizeof(BvhNode), sizeof(BvhNode4)}, 4096};
  PoolGroup slots{{3 * sizeof(float4), 3 * sizeof(float4), sizeof(uint32_t), sizeof(uint32_t)}, 4096};
  PoolGroup instances{{sizeof(InstanceRec)}, 256};
  PoolGroup materials{{sizeof(MaterialRec), sizeof(MaterialAux)}, 64};
  PoolGroup emitters{{sizeof(EmitterRec), sizeof(AliasEntry)}, 256};
  PoolGroup lights{{sizeof(LightRec)}, 16};
  Range identity_instance;
  std::vector<std::unique_ptr<ResidentScene>> scenes;  // index = handle
  DeviceBuffer scene_table;                              // SceneRec per handle
  uint32_t default_scene = kNoScene;
  // wavefront buffers
  uint32_t capacity = 0;
  DeviceBuffer q0_o, q0_d, q0_p, q1_o, q1_d, q1_p, q2_o, q2_d, q2_p, hit_tuv, hit_inst, sh_o, sh_d, sh_c, sh1_o,
      sh1_d, sh1_c, ps_tp, ps_rad, ps_shadow, ps_meta, ps_ior, ps_cone, sort_keys, sort_bins;
  DeviceBuffer counters, job_dev;
  DeviceBuffer prod_depth, prod_normal, prod_inst, prod_mat, prod_prim, prod_pos, prod_bary, prod_signals,
      prod_secondary;
  uint32_t prod_pixels = 0;
  DeviceBuffer srgb_lut;           // 256 sRGB-to-linear values for texture decoding
  DeviceBuffer motion_prev;        // world-space triangles of the motion history frame (3 float4 each)
  uint32_t motion_prev_count = 0;  // packed triangles in it; 0: none captured
  DeviceBuffer sample_lum;         // per-sample luminance of the last plain render (sample_variance)
  uint32_t lum_spp = 0;            // its samples; 0: none kept
  PoolGroup pixels{{3 * sizeof(unsigned long long), sizeof(float4)}, 1 << 16};
  // run tables (chunk headers + segments, then the resolve list) per slot
  RunSlot runs[2];
  RunSlot* cur = nullptr;            // slot being recorded
  int inflight = -1;                 // serving run launched but not yet finished
  uint32_t seg_capacity = 64;
  RestirState restir;
  std::map<std::vector<uint64_t>, GraphEntry> graphs;
  uint64_t graph_clock = 0;
  bool capturing = false;
  std::vector<olc_launch_record> last_profile;
  std::vector<uint32_t> last_chunk_counts;
  uint32_t last_w = 0, last_h = 0;
  // served jobs in submission order
  std::deque<std::unique_ptr<QueuedJob>> served;
  uint64_t next_ticket = 1;
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
  if (c.trace_block != 0 && c.trace_block != 64 && c.trace_block != 128 && c.trace_block != 256)
    throw Error(OLC_ERR_VALUE, "trace_block must be 64, 128 or 256");
  if (c.russian_roulette_min_survival < 0.0f || c.russian_roulette_min_survival > 1.0f)
    throw Error(OLC_ERR_VALUE, "russian_roulette_min_survival must be in [0, 1]");
}

void apply_launch_shape(olc_context* ctx) {
  ctx->ls.block = ctx->cfg.block_size ? ctx->cfg.block_size : 256;
  // traversal and shading: 64, 128 or 256 threads; 1,536 threads per SM of
  // grid keeps the persistent kernels' work cursors busy on every SM
  const uint32_t tb = ctx->cfg.trace_block ? ctx->cfg.trace_block : 128;
  ctx->ls.trace_block = tb;
  ctx->ls.stack_depth = ctx->cfg.stack_depth ? ctx->cfg.stack_depth : 24;
  ctx->ls.scheduler = ctx->cfg.trace_scheduler;
  ctx->ls.sort_rays = ctx->cfg.ray_sort ? 1u : 0u;
  ctx->ls.grid_simple = ctx->sm_count * 8;
  ctx->ls.grid_shade = ctx->sm_count * (1536 / tb);
  ctx->ls.grid_trace = ctx->sm_count * (1536 / tb);
}

void drop_graphs(olc_context* ctx) {
  if (!ctx->graphs.empty()) cudaStreamSynchronize(ctx->stream);   // none may still run
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
}

// Record the next timeline event on `stream`; returns its index.
uint32_t tl_record(olc_context* ctx, cudaStream_t stream) {
  RunSlot& sl = *ctx->cur;
  const uint32_t index = ctx->tl_next++;
  while (sl.events.size() <= index) {
    cudaEvent_t e;
    OLC_CUDA(cudaEventCreate(&e));
    sl.events.push_back(e);
  }
  if (ctx->capturing)
    OLC_CUDA(cudaEventRecordWithFlags(sl.events[index], stream, cudaEventRecordExternal));
  else
    OLC_CUDA(cudaEventRecord(sl.events[index], stream));
  return index;
}

void tl_begin(olc_context* ctx) {
  ctx->cur->entries.clear();
  ctx->side_pending[0] = ctx->side_pending[1] = false;
  ctx->tl_next = 0;
  ctx->tl_last = tl_record(ctx, ctx->stream);
}

// A stage that just ran on the main stream.
void tl_mark(olc_context* ctx, uint32_t stage, uint32_t bounce, uint32_t chunk) {
  const uint32_t end = tl_record(ctx, ctx->stream);
  ctx->cur->entries.push_back(TimelineEntry{stage, bounce, chunk, ctx->tl_last, end});
  ctx->tl_last = end;
}

// Wait on the main stream for the side stream's shadow launches of one
// bounce parity (and, the side stream being in order, for every one before).
void side_wait(olc_context* ctx, uint32_t parity) {
  if (!ctx->side_pending[parity]) return;
  OLC_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->join_event[parity], 0));
  ctx->side_pending[parity] = false;
  if (parity == ctx->side_last) ctx->side_pending[parity ^ 1u] = false;
  ctx->tl_last = tl_record(ctx, ctx->stream);   // later stages start after the wait
}

// Wait on the main stream for all of the side stream's pending work.
void side_join(olc_context* ctx) {
  if (ctx->side_pending[ctx->side_last]) side_wait(ctx, ctx->side_last);
  else if (ctx->side_pending[ctx->side_last ^ 1u]) side_wait(ctx, ctx->side_last ^ 1u);
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

template <class T>
void upload_to(T* dst, const T* host, size_t count, cudaStream_t stream) {
  if (count) OLC_CUDA(cudaMemcpyAsync(dst, host, count * sizeof(T), cudaMemcpyHostToDevice, stream));
}

SceneView pool_view(const olc_context* ctx) {
  SceneView v{};
  v.nodes = ctx->nodes.at<BvhNode>(0);
  v.wide = ctx->nodes.at<BvhNode4>(1);
  v.tri_verts = ctx->slots.at<float4>(0);
  v.tri_normals = ctx->slots.at<float4>(1);
  v.tri_index = ctx->slots.at<uint32_t>(2);
  v.tri_owner = ctx->slots.at<uint32_t>(3);
  v.instances = ctx->instances.at<InstanceRec>(0);
  v.materials = ctx->materials.at<MaterialRec>(0);
  v.material_aux = ctx->materials.at<MaterialAux>(1);
  v.emitters = ctx->emitters.at<EmitterRec>(0);
  v.emitter_alias = ctx->emitters.at<AliasEntry>(1);
  v.lights = ctx->lights.at<LightRec>(0);
  v.scenes = ctx->scene_table.as<SceneRec>();
  return v;
}

// Emitter records for sampling from the reference layout (a, b, c, emission +
// area, cdf/pdf/two-sided; Scene.emissive_triangle_data), plus a Vose alias
// table over the pdfs (M. D. Vose, "A linear algorithm for generating random
// numbers with a given distribution", IEEE TSE 1991).  Alias entries are
// scene-local indices.
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
    em[i].normal = make_float4(nrm.x, nrm.y, nrm.z, pdf / fmaxf(r[15], 1e-12f));
    const float area = fmaxf(r[15], 1e-12f);
    em[i].emission = make_float4(r[12], r[13], r[14], pdf > 0.0f ? area / pdf : 0.0f);
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

void fill_instance(InstanceRec& r, const float* m) {
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
}

void release_scene_ranges(olc_context* ctx, ResidentScene& rs) {
  ctx->nodes.release(rs.nodes);
  ctx->slots.release(rs.slots);
  ctx->instances.release(rs.instances);
  ctx->materials.release(rs.materials);
  ctx->emitters.release(rs.emitters);
  ctx->lights.release(rs.lights);
}

void check_scene_desc(const olc_scene_desc* d) {
  if (!d) throw Error(OLC_ERR_VALUE, "scene description is null");
  const uint32_t nm = d->num_meshes, ni = d->num_instances;
  if (nm && (!d->mesh_vertex_offset || !d->mesh_triangle_offset))
    throw Error(OLC_ERR_VALUE, "mesh offsets are required");
  uint32_t total_t = nm ? d->mesh_triangle_offset[nm] : 0;
  if (total_t >= (1u << 28)) throw Error(OLC_ERR_VALUE, "scene exceeds 2^28 triangles");
  for (uint32_t m = 0; m < nm; ++m) {
    if (d->mesh_vertex_offset[m + 1] < d->mesh_vertex_offset[m] ||
        d->mesh_triangle_offset[m + 1] < d->mesh_triangle_offset[m])
      throw Error(OLC_ERR_VALUE, "mesh offsets must be non-decreasing");
    const uint32_t nv = d->mesh_vertex_offset[m + 1] - d->mesh_vertex_offset[m];
    const uint64_t k0 = 3ull * d->mesh_triangle_offset[m], k1 = 3ull * d->mesh_triangle_offset[m + 1];
    if (k1 == k0) continue;
    uint32_t largest = 0;  // a max reduction vectorises; an early exit would not
    for (uint64_t k = k0; k < k1; ++k) largest = std::max(largest, d->indices[k]);
    if (largest >= nv) throw Error(OLC_ERR_VALUE, "an index refers to a vertex that does not exist");
  }
  for (uint32_t i = 0; i < ni; ++i) {
    if (d->instance_mesh[i] >= nm) throw Error(OLC_ERR_VALUE, "instance refers to a missing mesh");
    if (d->instance_material[i] >= d->num_materials) throw Error(OLC_ERR_VALUE, "instance refers to a missing material");
    const float* m = d->instance_object_to_world + 12ull * i;
    for (int k = 0; k < 12; ++k)
      if (!std::isfinite(m[k])) throw Error(OLC_ERR_VALUE, "instance transform must be finite");
  }
  if (d->environment_kind > OLC_ENV_EQUIRECT) throw Error(OLC_ERR_VALUE, "unknown environment kind");
  if (d->environment_kind == OLC_ENV_EQUIRECT &&
      (!d->environment_image || d->environment_width == 0 || d->environment_height == 0))
    throw Error(OLC_ERR_VALUE, "equirect environment needs an image");
}

uint32_t mesh_triangles(const olc_scene_desc* d, uint32_t m) {
  return d->mesh_triangle_offset[m + 1] - d->mesh_triangle_offset[m];
}

SceneLayout plan_scene(const olc_context* ctx, const olc_scene_desc* d) {
  SceneLayout L;
  const uint32_t nm = d->num_meshes, ni = d->num_instances;
  L.nm = nm;
  L.ni = ni;
  L.total_v = nm ? d->mesh_vertex_offset[nm] : 0;
  L.total_t = nm ? d->mesh_triangle_offset[nm] : 0;
  L.flat.assign(ni, 0);
  for (uint32_t i = 0; i < ni; ++i) {
    uint32_t nt = mesh_triangles(d, d->instance_mesh[i]);
    if (nt > 0 && nt <= kFlattenMaxTriangles) {
      L.flat[i] = 1;
      L.flat_tris += nt;
      ++L.flat_count;
    }
  }
  if (!ctx->cfg.flatten_instances || L.flat_count < 2 || L.flat_tris > kFlattenMaxTotal) {
    std::fill(L.flat.begin(), L.flat.end(), 0);
    L.flat_tris = 0;
    L.flat_count = 0;
  }
  for (uint32_t i = 0; i < ni; ++i)
    if (!L.flat[i]) L.order.push_back(i);
  L.members = (uint32_t)L.order.size();
  L.local_of.assign(ni, 0);
  for (uint32_t k = 0; k < L.members; ++k) L.local_of[L.order[k]] = k;
  {
    uint32_t k = L.members;
    for (uint32_t i = 0; i < ni; ++i)
      if (L.flat[i]) L.local_of[i] = k++;
  }
  L.mesh_used.assign(nm, 0);
  for (uint32_t k = 0; k < L.members; ++k) L.mesh_used[d->instance_mesh[L.order[k]]] = 1;
  L.node_local.assign(nm, 0);
  uint32_t node_count = 0;
  for (uint32_t m = 0; m < nm; ++m) {
    L.node_local[m] = node_count;
    if (L.mesh_used[m]) node_count += blas_node_count(mesh_triangles(d, m));
  }
  L.tlas_local = node_count;
  const uint64_t tlas_prims = (uint64_t)L.members + L.flat_tris;
  L.tlas_nodes = tlas_prims > 1 ? (uint32_t)(tlas_prims - 1) : 1;
  L.node_count = node_count + L.tlas_nodes;
  L.slot_count = (uint64_t)L.total_t + L.flat_tris;
  if (nm) {
    L.mesh_vertex_offset.assign(d->mesh_vertex_offset, d->mesh_vertex_offset + nm + 1);
    L.mesh_triangle_offset.assign(d->mesh_triangle_offset, d->mesh_triangle_offset + nm + 1);
  }
  L.instance_mesh.assign(d->instance_mesh, d->instance_mesh + ni);
  L.instance_prim_offset.assign(d->instance_primitive_offset, d->instance_primitive_offset + ni);
  for (uint32_t i = 0; i < ni; ++i)
    L.packed_triangles =
        std::max<uint64_t>(L.packed_triangles, (uint64_t)d->instance_primitive_offset[i] + mesh_triangles(d, d->instance_mesh[i]));
  return L;
}

bool same_layout(const SceneLayout& a, const SceneLayout& b) {
  return a.flat == b.flat && a.mesh_vertex_offset == b.mesh_vertex_offset &&
         a.mesh_triangle_offset == b.mesh_triangle_offset && a.instance_mesh == b.instance_mesh;
}

// Texture data of a scene: the texture words, bindings, per-material binding
// records and per-slot vertex attributes (texcoords, tangents), validated
// so that no device lookup can leave its array.  Member instances' slots
// take their corners from the mesh arrays in BLAS slot order; baked
// triangles get texcoords and world-space tangents (Mesh.world_tangents,
// scene/_core.py:702-714) in packed order.
void write_textures(olc_context* ctx, const olc_scene_desc* d, ResidentScene& rs, uint64_t& own) {
  for (DeviceBuffer* b : {&rs.tex_words, &rs.tex_bindings, &rs.tex_attr, &rs.mat_tex}) b->release();
  if (d->num_texture_bindings == 0) return;
  cudaStream_t st = ctx->stream;
  const SceneLayout& L = rs.layout;
  if (!d->texture_words || !d->texture_bindings || !d->material_textures || !d->texcoords || !d->tangents)
    throw Error(OLC_ERR_VALUE, "a textured scene needs texture words, bindings, material textures, texcoords and tangents");
  const uint32_t nw = d->num_texture_words;
  if (nw < 1 || (uint64_t)1 + 8ull * d->texture_words[0] > nw) throw Error(OLC_ERR_VALUE, "texture header is truncated");
  const uint32_t ntex = d->texture_words[0];
  for (uint32_t t = 0; t < ntex; ++t) {
    const uint32_t* m = d->texture_words + 1 + 8ull * t;
    const uint64_t w = m[2], h = m[3], levels = m[5];
    if (w == 0 || h == 0 || levels == 0 || levels > 32) throw Error(OLC_ERR_VALUE, "texture size or level count is invalid");
    uint64_t words = 0, lw = w, lh = h;
    for (uint64_t l = 0; l < levels; ++l) {
      words += lw * lh;
      lw = std::max<uint64_t>((lw + 1) / 2, 1);
      lh = std::max<uint64_t>((lh + 1) / 2, 1);
    }
    if ((uint64_t)m[0] + words > nw || (uint64_t)m[1] + words > nw) throw Error(OLC_ERR_VALUE, "texture data is truncated");
  }
  const uint32_t nb = d->num_texture_bindings;
  for (uint32_t b = 0; b < nb; ++b) {
    const float t = d->texture_bindings[8ull * b];
    if (!(t == -1.0f || (t >= 0.0f && t < (float)ntex && t == std::floor(t))))
      throw Error(OLC_ERR_VALUE, "a texture binding refers to a missing texture");
    for (int k = 0; k < 8; ++k)
      if (!std::isfinite(d->texture_bindings[8ull * b + k])) throw Error(OLC_ERR_VALUE, "texture bindings must be finite");
  }
  for (uint32_t mi = 0; mi < d->num_materials; ++mi)
    for (int k = 0; k < 6; ++k) {
      const float v = d->material_textures[12ull * mi + k];
      if (!(v < 0.0f || (v < (float)nb && v == std::floor(v))))
        throw Error(OLC_ERR_VALUE, "a material refers to a missing texture binding");
    }
  uint64_t staging = 0;
  upload(rs.tex_words, d->texture_words, nw, st, own);
  upload(rs.tex_bindings, d->texture_bindings, 8ull * nb, st, own);
  upload(rs.mat_tex, d->material_textures, 12ull * std::max<uint32_t>(d->num_materials, 1), st, own);
  const uint64_t slots = std::max<uint64_t>(L.slot_count, 1);
  rs.tex_attr.allocate(slots * 6 * sizeof(float4));
  own += rs.tex_attr.bytes();
  const uint32_t slot0 = (uint32_t)rs.slots.off;
  DeviceBuffer duv, dtan, di;
  upload(duv, d->texcoords, 4ull * L.total_v, st, staging);
  upload(dtan, d->tangents, 4ull * L.total_v, st, staging);
  upload(di, d->indices, 3ull * L.total_t, st, staging);
  const uint32_t* tri_index = ctx->slots.at<uint32_t>(2);
  for (uint32_t m = 0; m < L.nm; ++m) {
    if (!L.mesh_used[m]) continue;
    slot_attributes(duv.as<float4>(), dtan.as<float4>(), di.as<uint32_t>() + 3ull * d->mesh_triangle_offset[m],
                    mesh_triangles(d, m), d->mesh_vertex_offset[m], tri_index, slot0 + d->mesh_triangle_offset[m],
                    slot0, rs.tex_attr.as<float4>(), st);
  }
  if (L.flat_tris) {
    std::vector<float4> fa(6ull * L.flat_tris);
    uint64_t t = 0;
    for (uint32_t i = 0; i < L.ni; ++i) {
      if (!L.flat[i]) continue;
      const float* x = d->instance_object_to_world + 12ull * i;
      const double lin[3][3] = {{x[0], x[1], x[2]}, {x[4], x[5], x[6]}, {x[8], x[9], x[10]}};
      const double det = lin[0][0] * (lin[1][1] * lin[2][2] - lin[1][2] * lin[2][1]) -
                         lin[0][1] * (lin[1][0] * lin[2][2] - lin[1][2] * lin[2][0]) +
                         lin[0][2] * (lin[1][0] * lin[2][1] - lin[1][1] * lin[2][0]);
      double inv[3][3];   // inverse transpose: normals to world space
      inv[0][0] = (lin[1][1] * lin[2][2] - lin[1][2] * lin[2][1]) / det;
      inv[0][1] = (lin[1][2] * lin[2][0] - lin[1][0] * lin[2][2]) / det;
      inv[0][2] = (lin[1][0] * lin[2][1] - lin[1][1] * lin[2][0]) / det;
      inv[1][0] = (lin[0][2] * lin[2][1] - lin[0][1] * lin[2][2]) / det;
      inv[1][1] = (lin[0][0] * lin[2][2] - lin[0][2] * lin[2][0]) / det;
      inv[1][2] = (lin[0][1] * lin[2][0] - lin[0][0] * lin[2][1]) / det;
      inv[2][0] = (lin[0][1] * lin[1][2] - lin[0][2] * lin[1][1]) / det;
      inv[2][1] = (lin[0][2] * lin[1][0] - lin[0][0] * lin[1][2]) / det;
      inv[2][2] = (lin[0][0] * lin[1][1] - lin[0][1] * lin[1][0]) / det;
      const uint32_t m = d->instance_mesh[i];
      const uint32_t v0 = d->mesh_vertex_offset[m];
      for (uint32_t lt = 0; lt < mesh_triangles(d, m); ++lt, ++t) {
        for (int c = 0; c < 3; ++c) {
          const uint64_t vi = v0 + d->indices[3ull * (d->mesh_triangle_offset[m] + lt) + c];
          const float* uv = d->texcoords + 4 * vi;
          const float* tg = d->tangents + 4 * vi;
          const float* nm = d->normals + 3 * vi;
          double tw[3], nw3[3];
          for (int r = 0; r < 3; ++r) {
            tw[r] = lin[r][0] * tg[0] + lin[r][1] * tg[1] + lin[r][2] * tg[2];
            nw3[r] = inv[r][0] * nm[0] + inv[r][1] * nm[1] + inv[r][2] * nm[2];
          }
          const double nl = std::sqrt(nw3[0] * nw3[0] + nw3[1] * nw3[1] + nw3[2] * nw3[2]);
          for (double& v : nw3) v /= (nl > 0 ? nl : 1.0);
          const double dn = tw[0] * nw3[0] + tw[1] * nw3[1] + tw[2] * nw3[2];
          for (int r = 0; r < 3; ++r) tw[r] -= nw3[r] * dn;
          const double tl = std::sqrt(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
          for (double& v : tw) v /= (tl > 0 ? tl : 1.0);
          fa[6 * t + 2 * c] = make_float4(uv[0], uv[1], uv[2], uv[3]);
          fa[6 * t + 2 * c + 1] = make_float4((float)tw[0], (float)tw[1], (float)tw[2], det < 0.0 ? -tg[3] : tg[3]);
        }
      }
    }
    upload_to(rs.tex_attr.as<float4>() + 6ull * L.total_t, fa.data(), fa.size(), st);
  }
  OLC_CUDA(cudaStreamSynchronize(st));
}

// The reference-model volume records index the concatenated grids and
// transfer tables on the device: every offset, size and parameter is checked
// here, before upload.
void check_ref_volumes(const olc_scene_desc* d) {
  if (d->num_ref_volumes == 0) return;
  if (d->num_ref_volumes > kMaxRefVolumes) throw Error(OLC_ERR_VALUE, "at most 8 visible volumes per scene");
  if (!d->ref_volume_records || !d->ref_volume_grids || !d->ref_volume_luts)
    throw Error(OLC_ERR_VALUE, "volume records, grids and transfer tables are required");
  for (uint32_t k = 0; k < d->num_ref_volumes; ++k) {
    RefVolume v;
    std::memcpy(&v, d->ref_volume_records + 72ull * k, sizeof(RefVolume));
    if (v.nx < 2 || v.ny < 2 || v.nz < 2) throw Error(OLC_ERR_VALUE, "volume grids need at least 2 samples per axis");
    if ((uint64_t)v.grid_off + (uint64_t)v.nx * v.ny * v.nz > d->ref_grid_values)
      throw Error(OLC_ERR_VALUE, "a volume grid lies outside the grid values");
    if (v.lut_len < 1 || (uint64_t)v.lut_off + v.lut_len > d->ref_lut_entries)
      throw Error(OLC_ERR_VALUE, "a transfer function lies outside the transfer entries");
    if (v.address > 2 || v.num_clip > 8 || v.orders < 1 || v.orders > 8)
      throw Error(OLC_ERR_VALUE, "invalid volume addressing, clip-plane count or scattering orders");
    if (!(v.step_size > 0.0f) || !std::isfinite(v.step_size) || !(v.density_scale >= 0.0f) ||
        !(v.emission_scale >= 0.0f) || !(v.scattering_scale >= 0.0f))
      throw Error(OLC_ERR_VALUE, "volume step size must be positive and scales non-negative");
  }
}

// Everything of a resident scene besides its BLAS: instance records, the
// baked world-space triangles, the TLAS, materials, emitters, lights,
// environment, volume and the SceneRec.  Runs at upload and at every
// in-place update (a transform, material or light change rewrites all of
// it; only the TLAS build costs more than a copy).
void write_scene_records(olc_context* ctx, const olc_scene_desc* d, ResidentScene& rs, uint64_t& own) {
  cudaStream_t st = ctx->stream;
  const SceneLayout& L = rs.layout;
  const uint32_t ni = L.ni;
  const uint32_t slot0 = (uint32_t)rs.slots.off, inst0 = (uint32_t)rs.instances.off;
  const uint32_t node0 = (uint32_t)rs.nodes.off, mat0 = (uint32_t)rs.materials.off;
  const uint32_t flat_slot0 = slot0 + L.total_t;
  BvhNode* nodes = ctx->nodes.at<BvhNode>(0);
  float4* tri_verts = ctx->slots.at<float4>(0);
  float4* tri_normals = ctx->slots.at<float4>(1);
  uint32_t* tri_index = ctx->slots.at<uint32_t>(2);
  uint32_t* tri_owner = ctx->slots.at<uint32_t>(3);
  uint64_t staging = 0;

  // ---- instance records (global indices)
  std::vector<InstanceRec> inst(ni);
  std::vector<float> o2w(12ull * std::max<uint32_t>(L.members, 1), 0.0f);
  for (uint32_t i = 0; i < ni; ++i) {
    const float* m = d->instance_object_to_world + 12ull * i;
    const uint32_t k = L.local_of[i];
    InstanceRec& r = inst[k];
    fill_instance(r, m);
    r.blas_root = rs.blas_root[d->instance_mesh[i]];
    r.material = mat0 + d->instance_material[i];
    r.prim_offset = d->instance_primitive_offset[i];
    r.instance_id = d->instance_id[i];
    if (k < L.members)
      for (int c = 0; c < 12; ++c) o2w[12ull * k + c] = m[c];
  }
  // world-space triangles of the baked instances, in packed order; the
  // TLAS references their slots directly and hits report the identity
  // record, whose tri_owner entries name the original instances
  std::vector<float4> fv(3ull * L.flat_tris), fn(3ull * L.flat_tris);
  std::vector<uint32_t> fpacked(L.flat_tris), fowner(L.flat_tris);
  {
    uint64_t t = 0;
    for (uint32_t i = 0; i < ni; ++i) {
      if (!L.flat[i]) continue;
      const InstanceRec& r = inst[L.local_of[i]];
      Affine mo{r.o2w0, r.o2w1, r.o2w2}, mw{r.w2o0, r.w2o1, r.w2o2};
      const uint32_t m = d->instance_mesh[i];
      const uint32_t v0 = d->mesh_vertex_offset[m];
      for (uint32_t lt = 0; lt < mesh_triangles(d, m); ++lt, ++t) {
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
        fowner[t] = inst0 + L.local_of[i];
      }
    }
  }
  upload_to(tri_verts + 3ull * flat_slot0, fv.data(), fv.size(), st);
  upload_to(tri_normals + 3ull * flat_slot0, fn.data(), fn.size(), st);
  upload_to(tri_index + flat_slot0, fpacked.data(), fpacked.size(), st);
  upload_to(tri_owner + flat_slot0, fowner.data(), fowner.size(), st);
  upload_to(ctx->instances.at<InstanceRec>(0, inst0), inst.data(), inst.size(), st);

  // ---- TLAS over the member instances and the baked triangles
  std::vector<uint2> ranges(std::max<uint32_t>(L.members, 1));
  uint32_t max_tris = 0;
  for (uint32_t k = 0; k < L.members; ++k) {
    const uint32_t m = d->instance_mesh[L.order[k]];
    ranges[k] = make_uint2(slot0 + d->mesh_triangle_offset[m], slot0 + d->mesh_triangle_offset[m + 1]);
    max_tris = std::max(max_tris, mesh_triangles(d, m));
  }
  DeviceBuffer d_o2w, d_ranges;
  upload(d_o2w, o2w.data(), o2w.size(), st, staging);
  upload(d_ranges, ranges.data(), L.members, st, staging);
  const uint32_t tlas_root =
      build_tlas(d_o2w.as<float>(), d_ranges.as<uint2>(), L.members, max_tris, inst0, tri_verts, tri_verts + 3ull * flat_slot0,
                 (uint32_t)L.flat_tris, flat_slot0, ctx->scratch, nodes, node0 + L.tlas_local, st);
  // traversal reads the BVH4 form of every BLAS and of the TLAS
  build_bvh4(nodes, ctx->nodes.at<BvhNode4>(1), node0, (uint32_t)rs.nodes.n, st);

  // ---- materials, emitters, lights
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
    if (!(p[10] >= 0.0f && p[10] <= 1.0f)) throw Error(OLC_ERR_VALUE, "material transmission must be in [0, 1]");
    if (p[10] > 0.001f && !(p[11] > 0.0f && std::isfinite(p[11])))
      throw Error(OLC_ERR_VALUE, "a transmissive material needs a positive index of refraction");
    aux[k].transmission = p[10];
    aux[k].ior = p[11];
  }
  upload_to(ctx->materials.at<MaterialRec>(0, mat0), mats.data(), mats.size(), st);
  upload_to(ctx->materials.at<MaterialAux>(1, mat0), aux.data(), aux.size(), st);
  std::vector<EmitterRec> em;
  std::vector<AliasEntry> alias;
  build_emitters(d, em, alias);
  upload_to(ctx->emitters.at<EmitterRec>(0, rs.emitters.off), em.data(), em.size(), st);
  upload_to(ctx->emitters.at<AliasEntry>(1, rs.emitters.off), alias.data(), alias.size(), st);
  if (d->num_lights && !d->lights) throw Error(OLC_ERR_VALUE, "light records are required");
  upload_to(ctx->lights.at<LightRec>(0, rs.lights.off), reinterpret_cast<const LightRec*>(d->lights),
            d->num_lights, st);
  size_t env_count =
      d->environment_kind == OLC_ENV_EQUIRECT ? 3ull * d->environment_width * d->environment_height : 0;
  upload(rs.env_image, d->environment_image, env_count, st, own);
  size_t vol_count = d->volume_present ? (size_t)d->volume_dims[0] * d->volume_dims[1] * d->volume_dims[2] : 0;
  if (d->volume_present && (!d->volume_density || vol_count == 0))
    throw Error(OLC_ERR_VALUE, "a volume needs a density grid");
  upload(rs.volume, d->volume_density, vol_count, st, own);
  check_ref_volumes(d);
  upload(rs.ref_vol_recs, reinterpret_cast<const RefVolume*>(d->ref_volume_records), d->num_ref_volumes, st, own);
  upload(rs.ref_vol_grid, d->ref_volume_grids, d->num_ref_volumes ? d->ref_grid_values : 0, st, own);
  upload(rs.ref_vol_lut, reinterpret_cast<const float4*>(d->ref_volume_luts),
         d->num_ref_volumes ? d->ref_lut_entries : 0, st, own);
  OLC_CUDA(cudaStreamSynchronize(st));  // host staging vectors go out of scope

  SceneRec& v = rs.rec;
  std::memset(&v, 0, sizeof(v));
  v.tlas_root = tlas_root;
  v.emitter_base = (uint32_t)rs.emitters.off;
  v.num_emitters = d->num_emitters;
  v.emissive_weight = d->emissive_weight;
  v.light_base = (uint32_t)rs.lights.off;
  v.num_lights = d->num_lights;
  v.env_kind = d->environment_kind;
  v.env_rotation = d->environment_rotation;
  v.env_color = make_float4(d->environment_color[0], d->environment_color[1], d->environment_color[2], 0.0f);
  v.env_image = rs.env_image.as<float>();
  v.env_w = d->environment_width;
  v.env_h = d->environment_height;
  v.volume = rs.volume.as<float>();
  v.volume_present = d->volume_present;
  v.vol_nx = d->volume_dims[0];
  v.vol_ny = d->volume_dims[1];
  v.vol_nz = d->volume_dims[2];
  const float* vb = d->volume_world_to_box;
  v.vol_w2b0 = make_float4(vb[0], vb[1], vb[2], vb[3]);
  v.vol_w2b1 = make_float4(vb[4], vb[5], vb[6], vb[7]);
  v.vol_w2b2 = make_float4(vb[8], vb[9], vb[10], vb[11]);
  v.vol_sigma_t_scale = d->volume_sigma_t_scale;
  v.vol_albedo = d->volume_albedo;
  v.vol_max_density = d->volume_max_density;
  write_textures(ctx, d, rs, own);
  v.tex_words = rs.tex_words.as<uint32_t>();
  v.tex_bindings = rs.tex_bindings.as<float4>();
  v.tex_attr = rs.tex_attr.as<float4>();
  v.mat_tex = rs.mat_tex.as<float4>();
  v.srgb_lut = ctx->srgb_lut.as<float>();
  v.slot_base = (uint32_t)rs.slots.off;
  v.material_base = (uint32_t)rs.materials.off;
  v.ref_vols = rs.ref_vol_recs.as<RefVolume>();
  v.ref_grid = rs.ref_vol_grid.as<float>();
  v.ref_lut = rs.ref_vol_lut.as<float4>();
  v.num_ref_vols = d->num_ref_volumes;
}

BlasDesc mesh_blas_desc(const olc_scene_desc* d, uint32_t m, const DeviceBuffer& dv, const DeviceBuffer& dn,
                        const DeviceBuffer& di) {
  BlasDesc bd;
  const uint32_t v0 = d->mesh_vertex_offset[m], t0 = d->mesh_triangle_offset[m];
  bd.vertices = dv.as<float>() + 3ull * v0;
  bd.normals = dn.as<float>() + 3ull * v0;
  bd.indices = di.as<uint32_t>() + 3ull * t0;
  bd.num_vertices = d->mesh_vertex_offset[m + 1] - v0;
  bd.num_triangles = mesh_triangles(d, m);
  return bd;
}

// Build one scene into the pool.  Every range is acquired before any data is
// written (a growth moves the arrays), and all of them are released again if
// the build fails.
void build_scene(olc_context* ctx, const olc_scene_desc* d, ResidentScene& rs) {
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = ctx->stream;
  check_scene_desc(d);
  rs.layout = plan_scene(ctx, d);
  const SceneLayout& L = rs.layout;
  const uint32_t nm = L.nm;
  try {
    // ---- pool ranges (acquire everything first)
    rs.nodes = ctx->nodes.acquire(L.node_count, st);
    rs.slots = ctx->slots.acquire(std::max<uint64_t>(L.slot_count, 1), st);
    rs.instances = ctx->instances.acquire(L.ni, st);
    rs.materials = ctx->materials.acquire(d->num_materials, st);
    rs.emitters = ctx->emitters.acquire(d->num_emitters, st);
    rs.lights = ctx->lights.acquire(d->num_lights, st);
    if (rs.slots.off + rs.slots.n >= (1ull << 28)) throw Error(OLC_ERR_MEMORY, "scene pool exceeds 2^28 triangle slots");
    if (rs.instances.off + rs.instances.n >= (1ull << 28)) throw Error(OLC_ERR_MEMORY, "scene pool exceeds 2^28 instances");
    if (rs.nodes.off + rs.nodes.n >= 0x7fffffffull) throw Error(OLC_ERR_MEMORY, "scene pool exceeds 2^31 nodes");
    const uint32_t slot0 = (uint32_t)rs.slots.off, node0 = (uint32_t)rs.nodes.off;
    BvhNode* nodes = ctx->nodes.at<BvhNode>(0);
    float4* tri_verts = ctx->slots.at<float4>(0);
    float4* tri_normals = ctx->slots.at<float4>(1);
    uint32_t* tri_index = ctx->slots.at<uint32_t>(2);
    uint32_t* tri_owner = ctx->slots.at<uint32_t>(3);
    OLC_CUDA(cudaMemsetAsync(tri_owner + slot0, 0, rs.slots.n * sizeof(uint32_t), st));

    // ---- geometry staging and BLAS builds
    uint64_t staging = 0;
    DeviceBuffer dv, dn, di;
    upload(dv, d->vertices, 3ull * L.total_v, st, staging);
    upload(dn, d->normals, 3ull * L.total_v, st, staging);
    upload(di, d->indices, 3ull * L.total_t, st, staging);
    rs.blas_ranges.clear();
    rs.blas_root.assign(nm, 0);
    for (uint32_t m = 0; m < nm; ++m) {
      if (!L.mesh_used[m]) continue;
      const BlasDesc bd = mesh_blas_desc(d, m, dv, dn, di);
      const uint32_t first_slot = slot0 + d->mesh_triangle_offset[m];
      rs.blas_root[m] = build_blas(bd, ctx->scratch, nodes, node0 + L.node_local[m], tri_verts, tri_normals,
                                   tri_index, first_slot, kBlasLeafTriangles, st);
      rs.blas_ranges.push_back({rs.blas_root[m], first_slot, first_slot + bd.num_triangles});
    }
    uint64_t own = 0;
    write_scene_records(ctx, d, rs, own);

    rs.triangles = L.total_t;
    rs.blas_count = (uint32_t)rs.blas_ranges.size();
    rs.blas_nodes = L.tlas_local;
    rs.tlas_nodes = L.tlas_nodes;
    rs.flattened = L.flat_count;
    rs.bytes = ctx->nodes.range_bytes(rs.nodes) + ctx->slots.range_bytes(rs.slots) +
               ctx->instances.range_bytes(rs.instances) + ctx->materials.range_bytes(rs.materials) +
               ctx->emitters.range_bytes(rs.emitters) + ctx->lights.range_bytes(rs.lights) + own;
    rs.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  } catch (...) {
    cudaStreamSynchronize(st);
    release_scene_ranges(ctx, rs);
    throw;
  }
}

// Update a resident scene in place from a description with the same layout
// (_try_update_window_scene, ordinarylight/targets/vulkan/core.py:4696-4868):
// the flagged meshes get their triangle slots rewritten and their BLAS
// refit (_refit_scene_blases, targets/vulkan/scene.py:1217-1281); records,
// baked triangles, the TLAS (_rebuild_scene_tlas, scene.py:1299-1330),
// materials, emitters, lights, environment and volume are rewritten.  A
// material, emitter or light table of another length moves to a new pool
// range (a pool growth then invalidates the captured graphs).  Returns
// false, with nothing changed, when the layout differs.
bool update_scene(olc_context* ctx, ResidentScene& rs, const olc_scene_desc* d, const uint8_t* mesh_changed,
                  uint32_t* refitted) {
  auto t0 = std::chrono::steady_clock::now();
  cudaStream_t st = ctx->stream;
  check_scene_desc(d);
  const SceneLayout L = plan_scene(ctx, d);
  if (!same_layout(L, rs.layout)) return false;
  const uint32_t env_old = rs.rec.env_kind == OLC_ENV_EQUIRECT ? 3u * rs.rec.env_w * rs.rec.env_h : 0u;
  const uint32_t env_new =
      d->environment_kind == OLC_ENV_EQUIRECT ? 3u * d->environment_width * d->environment_height : 0u;
  if (env_old != env_new) return false;
  OLC_CUDA(cudaStreamSynchronize(st));  // no run reads the scene while it changes
  {
    // new ranges first (an allocation failure leaves the scene as it was)
    Range mats = rs.materials, ems = rs.emitters, lts = rs.lights;
    const void* bases[3] = {ctx->materials.bufs[0].get(), ctx->emitters.bufs[0].get(), ctx->lights.bufs[0].get()};
    try {
      if (d->num_materials != mats.n) mats = ctx->materials.acquire(d->num_materials, st);
      if (d->num_emitters != ems.n) ems = ctx->emitters.acquire(d->num_emitters, st);
      if (d->num_lights != lts.n) lts = ctx->lights.acquire(d->num_lights, st);
    } catch (...) {
      if (mats.off != rs.materials.off || mats.n != rs.materials.n) ctx->materials.release(mats);
      if (ems.off != rs.emitters.off || ems.n != rs.emitters.n) ctx->emitters.release(ems);
      throw;
    }
    auto swap_in = [](PoolGroup& pool, Range& held, const Range& next) {
      if (next.off == held.off && next.n == held.n) return;
      pool.release(held);
      held = next;
    };
    swap_in(ctx->materials, rs.materials, mats);
    swap_in(ctx->emitters, rs.emitters, ems);
    swap_in(ctx->lights, rs.lights, lts);
    if (bases[0] != ctx->materials.bufs[0].get() || bases[1] != ctx->emitters.bufs[0].get() ||
        bases[2] != ctx->lights.bufs[0].get())
      drop_graphs(ctx);
  }
  const uint32_t slot0 = (uint32_t)rs.slots.off, node0 = (uint32_t)rs.nodes.off;
  BvhNode* nodes = ctx->nodes.at<BvhNode>(0);
  float4* tri_verts = ctx->slots.at<float4>(0);
  float4* tri_normals = ctx->slots.at<float4>(1);
  const uint32_t* tri_index = ctx->slots.at<uint32_t>(2);
  uint32_t count = 0;
  bool any = false;
  for (uint32_t m = 0; m < L.nm; ++m) any = any || (L.mesh_used[m] && (!mesh_changed || mesh_changed[m]));
  if (any) {
    uint64_t staging = 0;
    DeviceBuffer dv, dn, di;
    upload(dv, d->vertices, 3ull * L.total_v, st, staging);
    upload(dn, d->normals, 3ull * L.total_v, st, staging);
    upload(di, d->indices, 3ull * L.total_t, st, staging);
    for (uint32_t m = 0; m < L.nm; ++m) {
      if (!L.mesh_used[m] || (mesh_changed && !mesh_changed[m])) continue;
      const BlasDesc bd = mesh_blas_desc(d, m, dv, dn, di);
      refit_blas(bd, ctx->scratch, nodes, node0 + L.node_local[m], blas_node_count(bd.num_triangles), tri_verts,
                 tri_normals, tri_index, slot0 + d->mesh_triangle_offset[m], st);
      ++count;
    }
    OLC_CUDA(cudaStreamSynchronize(st));
  }
  uint64_t own = 0;
  write_scene_records(ctx, d, rs, own);
  rs.bytes = ctx->nodes.range_bytes(rs.nodes) + ctx->slots.range_bytes(rs.slots) +
             ctx->instances.range_bytes(rs.instances) + ctx->materials.range_bytes(rs.materials) +
             ctx->emitters.range_bytes(rs.emitters) + ctx->lights.range_bytes(rs.lights) + own;
  if (refitted) *refitted = count;
  rs.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

// Upload the scene table (one SceneRec per handle).
void sync_scene_table(olc_context* ctx) {
  const size_t n = std::max<size_t>(ctx->scenes.size(), 1);
  std::vector<SceneRec> recs(n);
  std::memset(recs.data(), 0, n * sizeof(SceneRec));
  for (size_t i = 0; i < ctx->scenes.size(); ++i)
    if (ctx->scenes[i]) recs[i] = ctx->scenes[i]->rec;
  if (ctx->scene_table.bytes() < n * sizeof(SceneRec)) {
    ctx->scene_table.allocate(std::max<size_t>(n, 16) * sizeof(SceneRec));
  }
  OLC_CUDA(cudaMemcpyAsync(ctx->scene_table.get(), recs.data(), n * sizeof(SceneRec), cudaMemcpyHostToDevice,
                           ctx->stream));
  OLC_CUDA(cudaStreamSynchronize(ctx->stream));
}

uint32_t add_scene(olc_context* ctx, const olc_scene_desc* desc) {
  std::unique_ptr<ResidentScene> rs(new ResidentScene());
  build_scene(ctx, desc, *rs);
  uint32_t handle = 0;
  while (handle < ctx->scenes.size() && ctx->scenes[handle]) ++handle;
  if (handle == ctx->scenes.size()) ctx->scenes.emplace_back();
  ctx->scenes[handle] = std::move(rs);
  sync_scene_table(ctx);
  drop_graphs(ctx);
  return handle;
}

void remove_scene(olc_context* ctx, uint32_t handle) {
  if (handle >= ctx->scenes.size() || !ctx->scenes[handle]) throw Error(OLC_ERR_VALUE, "unknown scene handle");
  for (const auto& j : ctx->served)
    if (j->rec.scene == handle) throw Error(OLC_ERR_RUNTIME, "a queued job still renders this scene");
  OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  release_scene_ranges(ctx, *ctx->scenes[handle]);
  ctx->scenes[handle].reset();
  if (ctx->default_scene == handle) ctx->default_scene = kNoScene;
  if (ctx->restir.hist_scene == handle) restir_reset(ctx->restir);
  sync_scene_table(ctx);
  drop_graphs(ctx);
}

const ResidentScene& scene_of(const olc_context* ctx, uint32_t handle) {
  if (handle >= ctx->scenes.size() || !ctx->scenes[handle]) throw Error(OLC_ERR_VALUE, "unknown scene handle");
  return *ctx->scenes[handle];
}

const ResidentScene& default_scene(const olc_context* ctx) {
  if (ctx->default_scene == kNoScene) throw Error(OLC_ERR_RUNTIME, "no scene is resident; upload a scene first");
  return *ctx->scenes[ctx->default_scene];
}

// ---- jobs -----------------------------------------------------------------

void check_camera(const olc_camera* cam) {
  if (!cam) throw Error(OLC_ERR_VALUE, "camera is required");
  if (cam->projection > 2) throw Error(OLC_ERR_VALUE, "unknown camera projection");
}

void check_size(uint32_t w, uint32_t h, uint32_t spp) {
  if (w == 0 || h == 0) throw Error(OLC_ERR_VALUE, "width and height must be positive");
  if ((uint64_t)w * h > (1ull << 28)) throw Error(OLC_ERR_VALUE, "image is too large");
  // the accumulator's clamp keeps a pixel's sum below 2^63 up to this many samples
  if (spp < 1 || spp > OLC_MAX_FRAME_SAMPLES) throw Error(OLC_ERR_VALUE, "samples must be between 1 and 65536");
}

JobRec make_job(const olc_context* ctx, const olc_camera* cam, uint32_t w, uint32_t h, uint32_t spp,
                uint32_t frame_index, uint32_t max_bounces, uint32_t scene) {
  JobRec f;
  std::memset(&f, 0, sizeof(f));
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
  f.max_bounces = max_bounces ? max_bounces : ctx->cfg.max_bounces;
  f.mode = ctx->cfg.mode;
  f.rr_start = ctx->cfg.mode == OLC_MODE_PRODUCTION ? ctx->cfg.russian_roulette_start : 0u;
  f.rr_min_survival = ctx->cfg.russian_roulette_min_survival;
  f.nee = ctx->cfg.disable_nee ? 0u : 1u;
  f.scene = scene;
  f.lum_base = ~0ull;
  const bool restir = ctx->cfg.restir && ctx->cfg.mode == OLC_MODE_PRODUCTION &&
                      scene < ctx->scenes.size() && ctx->scenes[scene] && ctx->scenes[scene]->rec.num_emitters > 0;
  f.restir = restir ? 1u : 0u;
  return f;
}

// Reserve the job's accumulator pixels and clear them (stream ordered, before
// any of its chunks).
void admit_job(olc_context* ctx, QueuedJob& j) {
  j.pixels = ctx->pixels.acquire(j.rec.npix, ctx->stream);
  j.rec.pixel_base = j.pixels.off;
  OLC_CUDA(cudaMemsetAsync(ctx->pixels.at<unsigned long long>(0, j.pixels.off), 0,
                           (size_t)j.rec.npix * ctx->pixels.elem[0], ctx->stream));
}

uint64_t plan_capacity(const olc_context* ctx, const std::vector<QueuedJob*>& jobs) {
  uint64_t cap = ctx->cfg.chunk_paths ? ctx->cfg.chunk_paths : kDefaultChunkPaths;
  for (const QueuedJob* j : jobs)
    if (j->rec.restir) cap = std::max<uint64_t>(cap, j->rec.npix);  // a whole stream per ReSTIR segment
  return std::min<uint64_t>(cap, 0xffffffffull);
}

// Split the jobs' remaining paths into at most max_chunks chunks of at most
// cap paths, in job order.  A ReSTIR segment holds whole sample streams; a
// stream that does not fit leaves room for later jobs' paths.  Chunk-local
// reservoirs start after the first reservoir_region entries (the job-local
// reservoirs of a plain frame).
void plan_run(std::vector<QueuedJob*>& jobs, uint64_t cap, uint32_t max_chunks, uint64_t reservoir_region,
              RunPlan& plan) {
  struct Take {
    QueuedJob* job;
    uint64_t first, count;
  };
  for (uint32_t c = 0; c < max_chunks; ++c) {
    // choose the chunk's segments in job order
    std::vector<Take> takes;
    uint64_t fill = 0;
    for (QueuedJob* j : jobs) {
      if (j->issued >= j->total) continue;
      // textured and untextured jobs never share a chunk: each chunk runs
      // one kernel variant, so a job's bits do not depend on its company
      if (!takes.empty() && j->textured != takes.front().job->textured) continue;
      const uint64_t left = cap - fill;
      if (left == 0) break;
      uint64_t take;
      if (j->rec.restir) {
        const uint64_t streams = std::min<uint64_t>(left / j->rec.npix, (j->total - j->issued) / j->rec.npix);
        take = streams * j->rec.npix;
        if (take == 0) continue;
      } else {
        take = std::min<uint64_t>(left, j->total - j->issued);
      }
      takes.push_back(Take{j, j->issued, take});
      fill += take;
      j->issued += take;
      if (j->issued == j->total) plan.finished.push_back(j);
    }
    if (fill == 0) break;
    // lay the segments out grouped by scene: the persistent kernels walk the
    // queue in order, so the SMs then work on few hierarchies at a time and
    // more of each stays in L2 (the layout changes no image)
    std::stable_sort(takes.begin(), takes.end(),
                     [](const Take& a, const Take& b) { return a.job->rec.scene < b.job->rec.scene; });
    ChunkPlan ch;
    uint64_t at = 0;
    for (const Take& t : takes) {
      JobRec seg = t.job->rec;
      seg.seg_begin = at;
      seg.seg_first = t.first;
      if (seg.restir && !t.job->job_local_reservoirs) {
        // chunk-local reservoirs: index = reservoir_region + chunk path index
        seg.reservoir_base = reservoir_region + at - t.first;  // modulo 2^64
        plan.chunk_reservoirs = true;
      }
      ch.segs.push_back(seg);
      ch.bounces = std::max(ch.bounces, seg.max_bounces);
      ch.restir = ch.restir || seg.restir;
      ch.ref_volumes = ch.ref_volumes || t.job->ref_volumes;
      ch.media = ch.media || t.job->media;
      at += t.count;
    }
    ch.count = (uint32_t)fill;
    ch.textures = takes.front().job->textured;
    plan.restir = plan.restir || ch.restir;
    plan.max_segments = std::max<uint32_t>(plan.max_segments, (uint32_t)ch.segs.size());
    plan.max_count = std::max<uint32_t>(plan.max_count, ch.count);
    plan.chunks.push_back(std::move(ch));
  }
}

void ensure_wavefront(olc_context* ctx, uint32_t capacity) {
  if (capacity <= ctx->capacity) return;
  size_t c = capacity;
  ctx->q0_o.allocate(c * 16);
  ctx->q0_d.allocate(c * 16);
  ctx->q0_p.allocate(c * 4);
  ctx->q1_o.allocate(c * 16);
  ctx->q1_d.allocate(c * 16);
  ctx->q1_p.allocate(c * 4);
  ctx->q2_o.allocate(c * 16);
  ctx->q2_d.allocate(c * 16);
  ctx->q2_p.allocate(c * 4);
  ctx->sort_keys.allocate(c * 4);
  if (!ctx->sort_bins.get()) ctx->sort_bins.allocate(sort_bins_bytes());
  ctx->hit_tuv.allocate(c * 16);
  ctx->hit_inst.allocate(c * 4);
  ctx->sh_o.allocate(c * 16);
  ctx->sh_d.allocate(c * 16);
  ctx->sh_c.allocate(c * 16);
  ctx->sh1_o.allocate(c * 16);
  ctx->sh1_d.allocate(c * 16);
  ctx->sh1_c.allocate(c * 16);
  ctx->ps_tp.allocate(c * 16);
  ctx->ps_rad.allocate(c * 16);
  ctx->ps_shadow.allocate(c * 16);
  ctx->ps_ior.allocate(c * 64);
  ctx->ps_cone.allocate(c * 8);
  ctx->ps_meta.allocate(c * 16);
  ctx->capacity = capacity;
  drop_graphs(ctx);
}

void ensure_products(olc_context* ctx, uint32_t npix) {
  if (npix <= ctx->prod_pixels) return;
  size_t n = npix;
  ctx->prod_depth.allocate(n * 4);
  ctx->prod_normal.allocate(n * 16);
  ctx->prod_inst.allocate(n * 4);
  ctx->prod_mat.allocate(n * 4);
  ctx->prod_prim.allocate(n * 4);
  ctx->prod_pos.allocate(n * 16);
  ctx->prod_bary.allocate(n * 8);
  ctx->prod_signals.allocate(n * 16);
  ctx->prod_secondary.allocate(n * 16);
  ctx->prod_pixels = npix;
  drop_graphs(ctx);
}

size_t chunk_stride(uint32_t seg_capacity) { return sizeof(ChunkHeader) + (size_t)seg_capacity * sizeof(JobRec); }

void ensure_host_counters(olc_context* ctx, RunSlot& sl, uint32_t chunks) {
  if (chunks <= sl.counters_chunks) return;
  if (sl.counters_host) cudaFreeHost(sl.counters_host);
  sl.counters_host = nullptr;
  sl.counters_chunks = 0;
  OLC_CUDA(cudaMallocHost(&sl.counters_host, sizeof(Counters) * chunks));
  sl.counters_chunks = chunks;
  drop_graphs(ctx);
}

void ensure_table(olc_context* ctx, RunSlot& sl, size_t bytes) {
  if (bytes <= sl.table_capacity) return;
  size_t b = std::max<size_t>(bytes, 64 * 1024);
  sl.table_dev.allocate(b);
  if (sl.table_host) cudaFreeHost(sl.table_host);
  sl.table_host = nullptr;
  sl.table_capacity = 0;
  OLC_CUDA(cudaMallocHost(&sl.table_host, b));
  sl.table_capacity = b;
  drop_graphs(ctx);
}

void release_slot(RunSlot& sl) {
  if (sl.table_host) cudaFreeHost(sl.table_host);
  if (sl.counters_host) cudaFreeHost(sl.counters_host);
  if (sl.staging) cudaFreeHost(sl.staging);
  sl.table_host = nullptr;
  sl.counters_host = nullptr;
  sl.staging = nullptr;
  sl.staging_pixels = 0;
  for (cudaEvent_t e : sl.events) cudaEventDestroy(e);
  sl.events.clear();
  for (cudaEvent_t* e : {&sl.begin, &sl.end, &sl.done})
    if (*e) cudaEventDestroy(*e);
  sl.table_dev.release();
}

struct RunBuffers {
  RayQueue qa, qb, qc;
  HitBuf hb;
  ShadowQueue sq[2];   // by bounce parity
  PathState ps;
  ProductPtrs prod;
  Counters* cnt;
  unsigned long long* accum;
  float4* out;
  float* sample_lum;
  const char* table;
  size_t stride;
  size_t resolve_offset;
};

RunBuffers run_buffers(olc_context* ctx, const RunSlot& sl, size_t stride, size_t resolve_offset) {
  RunBuffers b;
  b.qa = RayQueue{ctx->q0_o.as<float4>(), ctx->q0_d.as<float4>(), ctx->q0_p.as<uint32_t>()};
  b.qb = RayQueue{ctx->q1_o.as<float4>(), ctx->q1_d.as<float4>(), ctx->q1_p.as<uint32_t>()};
  b.qc = RayQueue{ctx->q2_o.as<float4>(), ctx->q2_d.as<float4>(), ctx->q2_p.as<uint32_t>()};
  b.hb = HitBuf{ctx->hit_tuv.as<float4>(), ctx->hit_inst.as<uint32_t>()};
  b.sq[0] = ShadowQueue{ctx->sh_o.as<float4>(), ctx->sh_d.as<float4>(), ctx->sh_c.as<float4>()};
  b.sq[1] = ShadowQueue{ctx->sh1_o.as<float4>(), ctx->sh1_d.as<float4>(), ctx->sh1_c.as<float4>()};
  b.ps = PathState{ctx->ps_tp.as<float4>(), ctx->ps_rad.as<float4>(), ctx->ps_meta.as<uint4>(),
                   ctx->ps_ior.as<float4>(), ctx->ps_cone.as<float2>(), ctx->ps_shadow.as<float4>()};
  b.prod.depth = ctx->prod_depth.as<float>();
  b.prod.normal = ctx->prod_normal.as<float4>();
  b.prod.instance_id = ctx->prod_inst.as<uint32_t>();
  b.prod.material_id = ctx->prod_mat.as<uint32_t>();
  b.prod.primitive_id = ctx->prod_prim.as<uint32_t>();
  b.prod.position = ctx->prod_pos.as<float4>();
  b.prod.barycentric = ctx->prod_bary.as<float2>();
  b.prod.signals = ctx->prod_signals.as<float4>();
  b.prod.secondary = ctx->prod_secondary.as<float4>();
  b.cnt = ctx->counters.as<Counters>();
  b.accum = ctx->pixels.at<unsigned long long>(0);
  b.out = ctx->pixels.at<float4>(1);
  b.sample_lum = ctx->sample_lum.as<float>();
  b.table = sl.table_dev.as<char>();
  b.stride = stride;
  b.resolve_offset = resolve_offset;
  return b;
}

// Record the device work of one run into ctx->stream.
void record_run(olc_context* ctx, const RunPlan& plan, const RunBuffers& rb) {
  cudaStream_t st = ctx->stream;
  const SceneView s = pool_view(ctx);
  const SceneRec* scenes = ctx->scene_table.as<SceneRec>();
  tl_begin(ctx);
  for (uint32_t c = 0; c < plan.chunks.size(); ++c) {
    const ChunkPlan& ch = plan.chunks[c];
    const ChunkHeader* hdr = reinterpret_cast<const ChunkHeader*>(rb.table + c * rb.stride);
    const JobRec* jobs = reinterpret_cast<const JobRec*>(rb.table + c * rb.stride + sizeof(ChunkHeader));
    OLC_CUDA(cudaMemsetAsync(rb.cnt, 0, sizeof(Counters), st));
    const RayQueue* qin = &rb.qa;
    const RayQueue* qout = &rb.qb;
    const RayQueue* spare = &rb.qc;
    for (uint32_t b = 0; b < ch.bounces; ++b) {
      if (b > 0 && ctx->ls.sort_rays) {
        launch_sort_rays(ctx->ls, s, *qin, *spare, rb.cnt, b, ctx->sort_keys.as<uint32_t>(),
                         ctx->sort_bins.as<uint32_t>(), st);
        tl_mark(ctx, OLC_STAGE_SORT, b, c);
        std::swap(qin, spare);
      }
      HitListOut hl;
      if (b == 0 && ch.restir) {
        // the primary hits of the chunk's ReSTIR jobs, listed by the traversal
        hl.jobs = jobs;
        hl.meta = rb.ps.meta;
        hl.list = ctx->restir.hit_list.as<uint32_t>();
        hl.count = ctx->restir.hit_count.as<uint32_t>();
        OLC_CUDA(cudaMemsetAsync(hl.count, 0, 32, st));   // count and the passes' cursors
      }
      // bounce 0 generates the chunk's camera rays as it traces them
      const CameraPaths cam{hdr, jobs, scenes, rb.ps};
      launch_trace_closest(ctx->ls, s, *qin, rb.hb, rb.cnt, b, hl, b == 0 ? &cam : nullptr, st);
      tl_mark(ctx, OLC_STAGE_TRACE, b, c);
      const uint4* restir = nullptr;
      if (b == 0 && ch.restir) {
        restir = restir_run(ctx->restir, ctx->cfg, ctx->ls, s, hdr, jobs, *qin, rb.hb, rb.ps, ch.textures, st);
        tl_mark(ctx, OLC_STAGE_RESTIR, b, c);
      }
      // shading refills the shadow queue of its bounce's parity: the shadow
      // rays of two bounces back, which read it, must be done
      side_wait(ctx, b & 1u);
      if (ch.ref_volumes) {
        // reference-compatible paths cross their scene's volumes before shading
        launch_ref_volumes(ctx->ls, jobs, s, *qin, rb.hb, rb.ps, rb.cnt, b, st);
        tl_mark(ctx, OLC_STAGE_SHADE, b, c);
      }
      launch_shade(ctx->ls, jobs, s, *qin, rb.hb, *qout, rb.sq[b & 1u], rb.ps, rb.cnt, b, ctx->capacity, rb.prod,
                   restir, ch.textures, ch.media, b == 0 && !ch.ref_volumes, st);
      tl_mark(ctx, OLC_STAGE_SHADE, b, c);
      // this bounce's shadow rays on the side stream: they read only their
      // queue and add only to the paths' shadow sums, so the later bounces'
      // traversal and shading run beside them and fill their tail
      OLC_CUDA(cudaEventRecord(ctx->fork_event, st));
      OLC_CUDA(cudaStreamWaitEvent(ctx->side, ctx->fork_event, 0));
      const uint32_t side_start = tl_record(ctx, ctx->side);
      launch_trace_shadow(ctx->ls, s, rb.sq[b & 1u], rb.ps, rb.cnt, b, ctx->side);
      const uint32_t side_end = tl_record(ctx, ctx->side);
      ctx->cur->entries.push_back(TimelineEntry{OLC_STAGE_SHADOW, b, c, side_start, side_end});
      OLC_CUDA(cudaEventRecord(ctx->join_event[b & 1u], ctx->side));
      ctx->side_pending[b & 1u] = true;
      ctx->side_last = b & 1u;
      std::swap(qin, qout);
    }
    side_join(ctx);
    launch_accumulate(ctx->ls, hdr, jobs, rb.ps, rb.accum, rb.sample_lum, rb.cnt, st);
    tl_mark(ctx, OLC_STAGE_ACCUMULATE, 0, c);
    OLC_CUDA(cudaMemcpyAsync(ctx->cur->counters_host + c, rb.cnt, sizeof(Counters), cudaMemcpyDeviceToHost, st));
  }
  const uint32_t* num_entries = reinterpret_cast<const uint32_t*>(rb.table + rb.resolve_offset);
  const ResolveEntry* entries = reinterpret_cast<const ResolveEntry*>(rb.table + rb.resolve_offset + 16);
  launch_resolve(ctx->ls, entries, num_entries, rb.accum, rb.out, st);
  tl_mark(ctx, OLC_STAGE_RESOLVE, 0, 0);
}

// Everything the recorded launches depend on besides the device tables.
std::vector<uint64_t> run_signature(const olc_context* ctx, const RunPlan& plan, const RunBuffers& rb) {
  std::vector<uint64_t> k;
  k.push_back(plan.chunks.size());
  for (const ChunkPlan& c : plan.chunks)
    k.push_back(((uint64_t)c.bounces << 4) | (c.media ? 8u : 0u) | (c.ref_volumes ? 4u : 0u) |
                (c.textures ? 2u : 0u) | (c.restir ? 1u : 0u));
  auto ptr = [&](const void* p) { k.push_back((uint64_t)(uintptr_t)p); };
  const SceneView s = pool_view(ctx);
  const void* const* sv = reinterpret_cast<const void* const*>(&s);
  for (size_t i = 0; i < sizeof(SceneView) / sizeof(void*); ++i) ptr(sv[i]);
  for (const void* p : std::initializer_list<const void*>{(const void*)rb.qa.origin_tmin, (const void*)rb.qa.dir_root, (const void*)rb.qa.path,
                        (const void*)rb.qb.origin_tmin, (const void*)rb.qb.dir_root, (const void*)rb.qb.path,
                        (const void*)rb.qc.origin_tmin, (const void*)rb.qc.dir_root, (const void*)rb.qc.path,
                        ctx->sort_keys.get(), ctx->sort_bins.get(),
                        (const void*)rb.hb.tuv_slot, (const void*)rb.hb.instance, (const void*)rb.sq[0].origin_tmax,
                        (const void*)rb.sq[0].dir_path, (const void*)rb.sq[0].contrib_root,
                        (const void*)rb.sq[1].origin_tmax, (const void*)rb.sq[1].dir_path,
                        (const void*)rb.sq[1].contrib_root, (const void*)rb.ps.throughput,
                        (const void*)rb.ps.radiance, (const void*)rb.ps.shadow, (const void*)rb.ps.meta, (const void*)rb.ps.ior_stack, (const void*)rb.ps.cone, (const void*)rb.prod.depth,
                        (const void*)rb.prod.normal, (const void*)rb.prod.instance_id, (const void*)rb.prod.material_id,
                        (const void*)rb.prod.primitive_id, (const void*)rb.prod.position,
                        (const void*)rb.prod.barycentric, (const void*)rb.prod.signals,
                        (const void*)rb.prod.secondary, (const void*)rb.cnt, (const void*)rb.accum,
                        (const void*)rb.out, (const void*)rb.sample_lum, (const void*)rb.table, (const void*)ctx->cur->counters_host,
                        (const void*)ctx->cur,
                        ctx->restir.res_a0.get(), ctx->restir.res_a1.get(), ctx->restir.res_a2.get(),
                        ctx->restir.res_b0.get(), ctx->restir.res_b1.get(), ctx->restir.res_b2.get(),
                        ctx->restir.hist0.get(), ctx->restir.hist1.get(), ctx->restir.hist2.get(),
                        ctx->restir.selected.get(), ctx->restir.hit_list.get(), ctx->restir.hit_count.get(),
                        ctx->restir.pool0.get(), ctx->restir.pool1.get(), ctx->restir.pool2.get()})
    ptr(p);
  k.push_back(rb.stride);
  k.push_back(rb.resolve_offset);
  k.push_back(ctx->capacity);
  const LaunchShape& ls = ctx->ls;
  for (uint32_t v : {ls.block, ls.trace_block, ls.grid_simple, ls.grid_trace, ls.grid_shade, ls.stack_depth,
                     ls.scheduler})
    k.push_back(v);
  const olc_config& c = ctx->cfg;
  for (uint32_t v : {c.restir_candidates, c.restir_spatial, c.restir_neighbours, c.restir_max_history})
    k.push_back(v);
  uint32_t radius;
  std::memcpy(&radius, &c.restir_radius, 4);
  k.push_back(radius);
  return k;
}

// Launch a run: from a cached graph, a newly captured one, or directly.
void launch_run(olc_context* ctx, const RunPlan& plan, const RunBuffers& rb) {
  cudaStream_t st = ctx->stream;
  if (!ctx->cfg.use_graphs) {
    record_run(ctx, plan, rb);
    return;
  }
  std::vector<uint64_t> key = run_signature(ctx, plan, rb);
  auto it = ctx->graphs.find(key);
  if (it == ctx->graphs.end()) {
    if (ctx->graphs.size() >= kMaxGraphs) {
      auto oldest = ctx->graphs.begin();
      for (auto g = ctx->graphs.begin(); g != ctx->graphs.end(); ++g)
        if (g->second.last_used < oldest->second.last_used) oldest = g;
      cudaGraphExecDestroy(oldest->second.exec);
      ctx->graphs.erase(oldest);
    }
    cudaGraph_t g = nullptr;
    OLC_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    ctx->capturing = true;
    try {
      record_run(ctx, plan, rb);
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
    GraphEntry ge;
    ge.exec = exec;
    ge.timeline = ctx->cur->entries;
    it = ctx->graphs.emplace(std::move(key), std::move(ge)).first;
  }
  it->second.last_used = ++ctx->graph_clock;
  ctx->cur->entries = it->second.timeline;
  OLC_CUDA(cudaGraphLaunch(it->second.exec, st));
}

// Stage a planned run into slot `sl` and launch it with the output copies of
// the jobs it completes; returns without waiting.
void launch_planned(olc_context* ctx, RunSlot& sl, RunPlan&& plan) {
  cudaStream_t st = ctx->stream;
  const uint32_t nchunks = (uint32_t)plan.chunks.size();
  if (nchunks == 0) throw Error(OLC_ERR_RUNTIME, "a run without paths");
  if (plan.max_segments > ctx->seg_capacity) {
    uint32_t s = ctx->seg_capacity;
    while (s < plan.max_segments) s *= 2;
    ctx->seg_capacity = s;
    drop_graphs(ctx);
  }
  ensure_wavefront(ctx, std::max<uint32_t>(plan.max_count, 1));
  ensure_host_counters(ctx, sl, std::max<uint32_t>(nchunks, 1));
  if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
  for (cudaEvent_t* e : {&sl.begin, &sl.end, &sl.done})
    if (!*e) OLC_CUDA(cudaEventCreate(e));
  const size_t stride = chunk_stride(ctx->seg_capacity);
  const size_t resolve_offset = stride * nchunks;
  const size_t bytes = resolve_offset + 16 + sizeof(ResolveEntry) * plan.finished.size();
  ensure_table(ctx, sl, bytes);
  sl.table_bytes = bytes;
  // host staging of all chunk tables and the resolve list
  for (uint32_t c = 0; c < nchunks; ++c) {
    const ChunkPlan& ch = plan.chunks[c];
    ChunkHeader* h = reinterpret_cast<ChunkHeader*>(sl.table_host + c * stride);
    h->count = ch.count;
    h->num_segments = (uint32_t)ch.segs.size();
    h->stamp = plan.restir ? ctx->restir.run_first + c : 0u;
    h->history_first = ctx->restir.hist_first;
    h->history_last = ctx->restir.hist_last;
    h->pad[0] = h->pad[1] = h->pad[2] = 0;
    std::memcpy(sl.table_host + c * stride + sizeof(ChunkHeader), ch.segs.data(), ch.segs.size() * sizeof(JobRec));
  }
  {
    uint32_t* n = reinterpret_cast<uint32_t*>(sl.table_host + resolve_offset);
    n[0] = (uint32_t)plan.finished.size();
    n[1] = n[2] = n[3] = 0;
    ResolveEntry* e = reinterpret_cast<ResolveEntry*>(sl.table_host + resolve_offset + 16);
    for (size_t k = 0; k < plan.finished.size(); ++k) {
      e[k].pixel_base = plan.finished[k]->rec.pixel_base;
      e[k].npix = plan.finished[k]->rec.npix;
      e[k].spp = plan.finished[k]->rec.spp;
    }
  }
  OLC_CUDA(cudaMemcpyAsync(sl.table_dev.get(), sl.table_host, bytes, cudaMemcpyHostToDevice, st));
  const RunBuffers rb = run_buffers(ctx, sl, stride, resolve_offset);
  ctx->cur = &sl;
  OLC_CUDA(cudaEventRecord(sl.begin, st));
  launch_run(ctx, plan, rb);
  OLC_CUDA(cudaEventRecord(sl.end, st));
  size_t staged_pixels = 0;
  for (QueuedJob* j : plan.finished)
    if (j->out && j->out_staged) staged_pixels += j->rec.npix;
  if (staged_pixels > sl.staging_pixels) {
    // page locking is slow: grow geometrically from 4 Mpixel (64 MB)
    const size_t want = std::max<size_t>({staged_pixels, 2 * sl.staging_pixels, (size_t)1 << 22});
    if (sl.staging) cudaFreeHost(sl.staging);
    sl.staging = nullptr;
    sl.staging_pixels = 0;
    OLC_CUDA(cudaMallocHost(&sl.staging, want * sizeof(float4)));
    sl.staging_pixels = want;
  }
  sl.staged.clear();
  size_t at = 0;
  for (QueuedJob* j : plan.finished) {
    if (!j->out) continue;
    const size_t bytes = (size_t)j->rec.npix * sizeof(float4);
    if (j->out_staged) {
      OLC_CUDA(cudaMemcpyAsync(sl.staging + at, rb.out + j->rec.pixel_base, bytes, cudaMemcpyDeviceToHost, st));
      sl.staged.emplace_back(j, at);
      at += j->rec.npix;
    } else {
      OLC_CUDA(cudaMemcpyAsync(j->out, rb.out + j->rec.pixel_base, bytes,
                               j->out_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    }
  }
  for (QueuedJob* j : plan.finished) {
    if (!j->sums) continue;
    OLC_CUDA(cudaMemcpyAsync(j->sums, rb.accum + 3ull * j->rec.pixel_base, (size_t)j->rec.npix * 3 * sizeof(uint64_t),
                             j->out_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
  }
  OLC_CUDA(cudaEventRecord(sl.done, st));
  sl.plan = std::move(plan);
  sl.busy = true;
}

// Wait for the run in slot `sl` (outputs included) and gather its timeline
// and statistics.
void finish_run(olc_context* ctx, RunSlot& sl, olc_render_stats* stats) {
  OLC_CUDA(cudaEventSynchronize(sl.done));
  sl.busy = false;
  for (const auto& js : sl.staged)
    std::memcpy(js.first->out, sl.staging + js.second, (size_t)js.first->rec.npix * sizeof(float4));
  sl.staged.clear();
  const RunPlan& plan = sl.plan;
  const uint32_t nchunks = (uint32_t)plan.chunks.size();
  ctx->last_profile.clear();
  ctx->last_chunk_counts.clear();
  for (const ChunkPlan& ch : plan.chunks) ctx->last_chunk_counts.push_back(ch.count);
  float stage_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint64_t resolved_pixels = 0;
  for (const QueuedJob* j : plan.finished) resolved_pixels += j->rec.npix;
  for (size_t k = 0; k < sl.entries.size(); ++k) {
    const TimelineEntry& e = sl.entries[k];
    olc_launch_record r{};
    r.stage = e.stage;
    r.bounce = e.bounce;
    r.chunk = e.chunk;
    OLC_CUDA(cudaEventElapsedTime(&r.ms, sl.events[e.start], sl.events[e.end]));
    const Counters& kc = sl.counters_host[std::min<uint32_t>(e.chunk, nchunks - 1)];
    switch (e.stage) {
      case OLC_STAGE_RAYGEN: case OLC_STAGE_ACCUMULATE: r.items = plan.chunks[e.chunk].count; break;
      case OLC_STAGE_TRACE: case OLC_STAGE_SHADE: case OLC_STAGE_RESTIR:
        r.items = kc.queue_count[e.bounce];
        r.misses = kc.miss_count[e.bounce];
        break;
      case OLC_STAGE_SHADOW: r.items = kc.shadow_count[e.bounce]; break;
      case OLC_STAGE_SORT: r.items = kc.queue_count[e.bounce]; break;
      default: r.items = resolved_pixels; break;
    }
    stage_ms[e.stage] += r.ms;
    ctx->last_profile.push_back(r);
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->raygen_ms = stage_ms[OLC_STAGE_RAYGEN];
    stats->trace_ms = stage_ms[OLC_STAGE_TRACE] + stage_ms[OLC_STAGE_SORT];
    stats->restir_ms = stage_ms[OLC_STAGE_RESTIR];
    stats->shade_ms = stage_ms[OLC_STAGE_SHADE];
    stats->shadow_ms = stage_ms[OLC_STAGE_SHADOW];
    stats->accumulate_ms = stage_ms[OLC_STAGE_ACCUMULATE] + stage_ms[OLC_STAGE_RESOLVE];
    for (uint32_t c = 0; c < nchunks; ++c) {
      const Counters& k = sl.counters_host[c];
      stats->camera_rays += k.queue_count[0];
      for (uint32_t b = 1; b < plan.chunks[c].bounces; ++b) stats->extension_rays += k.queue_count[b];
      for (uint32_t b = 0; b < plan.chunks[c].bounces; ++b) stats->shadow_rays += k.shadow_count[b];
      stats->overflow += k.overflow;
      stats->traversal_errors += k.traversal_errors;
    }
    OLC_CUDA(cudaEventElapsedTime(&stats->gpu_ms, sl.begin, sl.end));
    stats->chunks = nchunks;
    stats->jobs_completed = (uint32_t)plan.finished.size();
    stats->h2d_bytes = sl.table_bytes;
    stats->d2h_bytes = (uint64_t)nchunks * sizeof(Counters);
    for (const QueuedJob* j : plan.finished)
      if (j->out && !j->out_device) stats->d2h_bytes += (uint64_t)j->rec.npix * sizeof(float4);
  }
}

// A slot no run occupies (plain frames and batches run beside an in-flight
// serving step).
RunSlot& free_slot(olc_context* ctx) { return ctx->runs[0].busy ? ctx->runs[1] : ctx->runs[0]; }

// Launch and wait: plain frames and batches.
void execute_run(olc_context* ctx, RunPlan& plan, olc_render_stats* stats) {
  RunSlot& sl = free_slot(ctx);
  launch_planned(ctx, sl, std::move(plan));
  finish_run(ctx, sl, stats);
}

// Render the given jobs to completion as one run (plain frames and batches).
void run_to_completion(olc_context* ctx, std::vector<QueuedJob*>& jobs, olc_render_stats* stats) {
  uint64_t job_local = 0;
  for (const QueuedJob* j : jobs)
    if (j->rec.restir && j->job_local_reservoirs) job_local = std::max<uint64_t>(job_local, j->total);
  RunPlan plan;
  plan_run(jobs, plan_capacity(ctx, jobs), 0xffffffffu, job_local, plan);
  if (plan.restir)
    restir_prepare(ctx->restir, job_local + (plan.chunk_reservoirs ? plan.max_count : 0),
                   std::max<uint32_t>(plan.max_count, 1), (uint32_t)plan.chunks.size(), plan.max_segments);
  execute_run(ctx, plan, stats);
}

void release_job(olc_context* ctx, QueuedJob& j) { ctx->pixels.release(j.pixels); }

// Page-locked (or registered) host memory takes asynchronous copies directly.
bool is_pinned(const void* p) {
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return attr.type == cudaMemoryTypeHost;
}

// Fill an olc_job into a queued job (validated; not yet admitted).
void job_from_desc(olc_context* ctx, const olc_job* d, QueuedJob& q) {
  if (!d) throw Error(OLC_ERR_VALUE, "job is required");
  check_camera(&d->camera);
  check_size(d->width, d->height, d->samples_per_pixel);
  if (d->max_bounces > OLC_MAX_BOUNCES) throw Error(OLC_ERR_VALUE, "max_bounces must be between 1 and 64");
  scene_of(ctx, d->scene);
  if (!d->out_rgba && !d->out_sums) throw Error(OLC_ERR_VALUE, "an output pointer is required");
  if ((uint64_t)d->first_sample + d->samples_per_pixel > 0xffffffffull)
    throw Error(OLC_ERR_VALUE, "first_sample + samples_per_pixel exceeds 2^32");
  q.rec = make_job(ctx, &d->camera, d->width, d->height, d->samples_per_pixel, d->frame_index, d->max_bounces,
                   d->scene);
  q.rec.sample_base = d->first_sample;
  q.textured = scene_of(ctx, d->scene).rec.tex_words != nullptr;
  q.ref_volumes = q.rec.mode == OLC_MODE_REFERENCE_COMPATIBLE && scene_of(ctx, d->scene).rec.num_ref_vols > 0u;
  q.media = q.rec.mode != OLC_MODE_REFERENCE_COMPATIBLE && scene_of(ctx, d->scene).rec.volume_present != 0u;
  q.total = (uint64_t)q.rec.npix * q.rec.spp;
  q.out = d->out_rgba;
  q.sums = d->out_sums;
  q.out_device = d->out_is_device != 0;
  q.out_staged = q.out && !q.out_device && !is_pinned(q.out);
}

bool same_camera(const JobRec& a, const JobRec& b) {
  auto same = [](const float4& x, const float4& y) { return x.x == y.x && x.y == y.y && x.z == y.z && x.w == y.w; };
  return same(a.cam_pos, b.cam_pos) && same(a.cam_forward, b.cam_forward) && same(a.cam_right, b.cam_right) &&
         same(a.cam_up, b.cam_up) && a.projection == b.projection;
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
    OLC_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    OLC_CUDA(cudaEventCreateWithFlags(&ctx->fork_event, cudaEventDisableTiming));
    OLC_CUDA(cudaEventCreateWithFlags(&ctx->join_event[0], cudaEventDisableTiming));
    OLC_CUDA(cudaEventCreateWithFlags(&ctx->join_event[1], cudaEventDisableTiming));
    configure_trace_kernels();
    apply_launch_shape(ctx.get());
    // pool record 0: the identity instance that baked triangles report
    ctx->identity_instance = ctx->instances.acquire(1, ctx->stream);
    if (ctx->identity_instance.off != OLC_IDENTITY_INSTANCE) throw Error(OLC_ERR_RUNTIME, "instance pool is not empty");
    InstanceRec id;
    const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    fill_instance(id, identity);
    id.blas_root = 0;
    id.material = 0;
    id.prim_offset = 0;
    id.instance_id = 0xffffffffu;
    id.flags = OLC_INSTANCE_FLATTENED;
    upload_to(ctx->instances.at<InstanceRec>(0, OLC_IDENTITY_INSTANCE), &id, 1, ctx->stream);
    ctx->srgb_lut.allocate(256 * sizeof(float));
    srgb_table(ctx->srgb_lut.as<float>(), ctx->stream);
    sync_scene_table(ctx.get());
  });
  if (rc != OLC_OK) {
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->fork_event) cudaEventDestroy(ctx->fork_event);
    for (cudaEvent_t e : ctx->join_event)
      if (e) cudaEventDestroy(e);
    ctx->stream = nullptr;
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
  for (RunSlot& sl : ctx->runs) release_slot(sl);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  cudaStream_t st = ctx->stream, side = ctx->side;
  cudaEvent_t fork = ctx->fork_event, join0 = ctx->join_event[0], join1 = ctx->join_event[1];
  delete ctx;  // device buffers are freed here
  if (st) cudaStreamDestroy(st);
  if (side) cudaStreamDestroy(side);
  if (fork) cudaEventDestroy(fork);
  if (join0) cudaEventDestroy(join0);
  if (join1) cudaEventDestroy(join1);
  return OLC_OK;
}

int olc_reconfigure(olc_context* ctx, const olc_config* cfg) {
  if (!ctx || !cfg) return fail(ctx, OLC_ERR_VALUE, "context and config are required");
  return guarded(ctx, [&] {
    validate_config(*cfg);
    if (cfg->device != ctx->cfg.device) throw Error(OLC_ERR_RUNTIME, "changing the device requires a new renderer");
    if (!ctx->served.empty() && (cfg->mode != ctx->cfg.mode || cfg->restir != ctx->cfg.restir))
      throw Error(OLC_ERR_RUNTIME, "mode and ReSTIR cannot change while served jobs are queued");
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
    const uint32_t old = ctx->default_scene;
    if (old != kNoScene)
      for (const auto& j : ctx->served)
        if (j->rec.scene == old) throw Error(OLC_ERR_RUNTIME, "a queued job still renders the current scene");
    const uint32_t handle = add_scene(ctx, scene);  // throws before touching the resident scene
    ctx->default_scene = handle;
    if (old != kNoScene) remove_scene(ctx, old);
    restir_reset(ctx->restir);
  });
}

int olc_scene_bytes(const olc_context* ctx, uint64_t* bytes) {
  if (!ctx || !bytes) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  *bytes = ctx->default_scene == kNoScene ? 0 : ctx->scenes[ctx->default_scene]->bytes;
  return OLC_OK;
}

int olc_add_scene(olc_context* ctx, const olc_scene_desc* scene, uint32_t* handle) {
  if (!ctx || !handle) return fail(ctx, OLC_ERR_VALUE, "context and handle output are required");
  return guarded(ctx, [&] { *handle = add_scene(ctx, scene); });
}

int olc_remove_scene(olc_context* ctx, uint32_t handle) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] { remove_scene(ctx, handle); });
}

int olc_update_scene(olc_context* ctx, uint32_t handle, const olc_scene_desc* scene, const uint8_t* mesh_changed,
                     int32_t* applied, uint32_t* refitted) {
  if (!ctx || !applied) return fail(ctx, OLC_ERR_VALUE, "context and applied output are required");
  return guarded(ctx, [&] {
    *applied = 0;
    if (refitted) *refitted = 0;
    if (handle == OLC_DEFAULT_SCENE) {
      if (ctx->default_scene == kNoScene) throw Error(OLC_ERR_RUNTIME, "no scene is resident; upload a scene first");
      handle = ctx->default_scene;
    }
    if (handle >= ctx->scenes.size() || !ctx->scenes[handle]) throw Error(OLC_ERR_VALUE, "unknown scene handle");
    for (const auto& j : ctx->served)
      if (j->rec.scene == handle) throw Error(OLC_ERR_RUNTIME, "a queued job still renders this scene");
    ResidentScene& rs = *ctx->scenes[handle];
    if (!update_scene(ctx, rs, scene, mesh_changed, refitted)) return;
    sync_scene_table(ctx);
    if (ctx->restir.hist_scene == handle) restir_reset(ctx->restir);
    *applied = 1;
  });
}

int olc_scene_stats_get(const olc_context* ctx, uint32_t handle, olc_scene_stats* stats) {
  if (!ctx || !stats) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  return guarded(const_cast<olc_context*>(ctx), [&] {
    const ResidentScene& rs = scene_of(ctx, handle);
    std::memset(stats, 0, sizeof(*stats));
    stats->bytes = rs.bytes;
    stats->triangles = rs.triangles;
    stats->blas_count = rs.blas_count;
    stats->blas_nodes = rs.blas_nodes;
    stats->tlas_nodes = rs.tlas_nodes;
    stats->flattened_instances = rs.flattened;
    stats->build_ms = rs.build_ms;
  });
}

int olc_pool_info_get(const olc_context* ctx, olc_pool_info* info) {
  if (!ctx || !info) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and output are required");
  std::memset(info, 0, sizeof(*info));
  for (const auto& s : ctx->scenes)
    if (s) {
      ++info->resident_scenes;
      info->scene_bytes += s->bytes;
    }
  info->queued_jobs = (uint32_t)ctx->served.size();
  info->pool_bytes = ctx->nodes.bytes() + ctx->slots.bytes() + ctx->instances.bytes() + ctx->materials.bytes() +
                     ctx->emitters.bytes() + ctx->lights.bytes() + ctx->scene_table.bytes();
  uint64_t wf = 0;
  for (const DeviceBuffer* b : {&ctx->q0_o, &ctx->q0_d, &ctx->q0_p, &ctx->q1_o, &ctx->q1_d, &ctx->q1_p, &ctx->q2_o,
                                &ctx->q2_d, &ctx->q2_p, &ctx->sort_keys, &ctx->sort_bins,
                                &ctx->hit_tuv, &ctx->hit_inst, &ctx->sh_o, &ctx->sh_d, &ctx->sh_c, &ctx->sh1_o,
                                &ctx->sh1_d, &ctx->sh1_c, &ctx->ps_tp, &ctx->ps_rad, &ctx->ps_shadow, &ctx->ps_meta, &ctx->ps_ior, &ctx->ps_cone, &ctx->runs[0].table_dev, &ctx->runs[1].table_dev,
                                &ctx->prod_depth, &ctx->prod_normal,
                                &ctx->prod_inst, &ctx->prod_mat, &ctx->prod_prim, &ctx->prod_pos, &ctx->prod_bary,
                                &ctx->prod_signals, &ctx->prod_secondary,
                                &ctx->sample_lum, &ctx->motion_prev, &ctx->restir.res_a0,
                                &ctx->restir.res_a1, &ctx->restir.res_a2, &ctx->restir.res_b0, &ctx->restir.res_b1,
                                &ctx->restir.res_b2, &ctx->restir.hist0, &ctx->restir.hist1, &ctx->restir.hist2,
                                &ctx->restir.selected, &ctx->restir.hit_list})
    wf += b->bytes();
  info->wavefront_bytes = wf;
  info->pixel_bytes = ctx->pixels.bytes();
  info->pixel_bytes_used = ctx->pixels.ranges.used() * (ctx->pixels.elem[0] + ctx->pixels.elem[1]);
  return OLC_OK;
}

int olc_render(olc_context* ctx, const olc_camera* camera, uint32_t width, uint32_t height, uint32_t spp,
               uint32_t frame_index, float* out_rgba, int out_is_device, olc_render_stats* stats) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    check_camera(camera);
    check_size(width, height, spp);
    const ResidentScene& rs = default_scene(ctx);
    if (!out_rgba) throw Error(OLC_ERR_VALUE, "output pointer is required");
    QueuedJob job;
    job.rec = make_job(ctx, camera, width, height, spp, frame_index, 0, ctx->default_scene);
    job.rec.products = 1;
    job.textured = rs.rec.tex_words != nullptr;
    job.ref_volumes = job.rec.mode == OLC_MODE_REFERENCE_COMPATIBLE && rs.rec.num_ref_vols > 0u;
    job.media = job.rec.mode != OLC_MODE_REFERENCE_COMPATIBLE && rs.rec.volume_present != 0u;
    job.total = (uint64_t)job.rec.npix * spp;
    job.out = out_rgba;
    job.out_device = out_is_device != 0;
    job.out_staged = !job.out_device && !is_pinned(out_rgba);
    const bool restir = job.rec.restir != 0;
    // the frame's reservoirs live at job-local indices, where the next frame's
    // temporal pass finds them; the history survives only if the reservoir
    // buffers need not grow for this frame
    RestirState& rst = ctx->restir;
    const bool history = restir && ctx->cfg.restir_temporal && rst.history_valid && rst.hist_w == width &&
                         rst.hist_h == height && rst.hist_spp == spp && rst.hist_frame + 1u == frame_index &&
                         rst.hist_scene == ctx->default_scene && same_camera(job.rec, rst.hist_camera) &&
                         job.total <= rst.reservoirs;
    job.job_local_reservoirs = restir;
    job.rec.history = history ? 1u : 0u;
    job.rec.reservoir_base = 0;
    job.rec.history_base = 0;
    ensure_products(ctx, job.rec.npix);
    ctx->lum_spp = 0;
    if (ctx->cfg.sample_variance) {
      const size_t bytes = (size_t)job.total * sizeof(float);
      if (bytes > ctx->sample_lum.bytes()) {
        ctx->sample_lum.allocate(bytes);
        drop_graphs(ctx);
      }
      job.rec.lum_base = 0;
    }
    admit_job(ctx, job);
    std::vector<QueuedJob*> jobs{&job};
    try {
      run_to_completion(ctx, jobs, stats);
    } catch (...) {
      release_job(ctx, job);
      throw;
    }
    release_job(ctx, job);
    ctx->last_w = width;
    ctx->last_h = height;
    ctx->lum_spp = ctx->cfg.sample_variance ? spp : 0u;
    if (restir) {
      restir_finish(rst);
      rst.history_valid = true;
      rst.history_used = history;
      rst.hist_w = width;
      rst.hist_h = height;
      rst.hist_spp = spp;
      rst.hist_frame = frame_index;
      rst.hist_scene = ctx->default_scene;
      rst.hist_camera = job.rec;
    }
    if (stats) stats->restir_history_used = (restir && rst.history_used) ? 1u : 0u;
  });
}

int olc_render_batch(olc_context* ctx, const olc_job* jobs, uint32_t num_jobs, olc_render_stats* stats) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (num_jobs == 0) {
      if (stats) std::memset(stats, 0, sizeof(*stats));
      return;
    }
    if (!jobs) throw Error(OLC_ERR_VALUE, "jobs are required");
    std::vector<QueuedJob> q(num_jobs);
    for (uint32_t i = 0; i < num_jobs; ++i) job_from_desc(ctx, &jobs[i], q[i]);
    std::vector<QueuedJob*> ptrs;
    try {
      for (QueuedJob& j : q) {
        admit_job(ctx, j);
        ptrs.push_back(&j);
      }
      // jobs of one scene next to each other: a chunk then touches fewer
      // hierarchies, which keeps more of each in L2 (the order changes no image)
      std::stable_sort(ptrs.begin(), ptrs.end(),
                       [](const QueuedJob* a, const QueuedJob* b) { return a->rec.scene < b->rec.scene; });
      run_to_completion(ctx, ptrs, stats);
    } catch (...) {
      for (QueuedJob* j : ptrs) release_job(ctx, *j);
      throw;
    }
    for (QueuedJob* j : ptrs) release_job(ctx, *j);
  });
}

int olc_job_bytes(const olc_context* ctx, const olc_job* job, uint64_t* bytes) {
  if (!ctx || !job || !bytes) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "arguments are required");
  *bytes = (uint64_t)job->width * job->height * (ctx->pixels.elem[0] + ctx->pixels.elem[1]);
  return OLC_OK;
}

int olc_submit(olc_context* ctx, const olc_job* job, uint64_t* ticket) {
  if (!ctx || !ticket) return fail(ctx, OLC_ERR_VALUE, "context and ticket output are required");
  return guarded(ctx, [&] {
    std::unique_ptr<QueuedJob> q(new QueuedJob());
    job_from_desc(ctx, job, *q);
    admit_job(ctx, *q);
    q->ticket = ctx->next_ticket++;
    *ticket = q->ticket;
    ctx->served.push_back(std::move(q));
  });
}

int olc_cancel(olc_context* ctx, uint64_t ticket) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    for (auto it = ctx->served.begin(); it != ctx->served.end(); ++it) {
      if ((*it)->ticket != ticket) continue;
      QueuedJob* job = it->get();
      if (ctx->inflight >= 0) {
        // the in-flight chunk may hold its paths: let it finish, and keep it
        // from reporting the job
        RunSlot& sl = ctx->runs[ctx->inflight];
        OLC_CUDA(cudaEventSynchronize(sl.done));
        auto& fin = sl.plan.finished;
        fin.erase(std::remove(fin.begin(), fin.end(), job), fin.end());
      }
      release_job(ctx, *job);
      ctx->served.erase(it);
      return;
    }
    throw Error(OLC_ERR_VALUE, "unknown or completed ticket");
  });
}

int olc_serve_step(olc_context* ctx, uint64_t* done, uint32_t done_capacity, uint32_t* num_done,
                   olc_render_stats* stats) {
  if (!ctx || !num_done) return fail(ctx, OLC_ERR_VALUE, "context and num_done are required");
  return guarded(ctx, [&] {
    *num_done = 0;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    RunSlot* prev = ctx->inflight >= 0 ? &ctx->runs[ctx->inflight] : nullptr;
    if (prev && prev->plan.finished.size() > done_capacity)
      throw Error(OLC_ERR_VALUE, "done_capacity is smaller than the number of jobs the step completes");
    // 1. plan and launch the next chunk so the device stays busy while the
    //    previous one is collected
    std::vector<QueuedJob*> jobs;
    std::vector<uint64_t> issued_before;
    for (auto& j : ctx->served) {
      jobs.push_back(j.get());
      issued_before.push_back(j->issued);
    }
    // Shortest remaining work first, so small requests finish inside the
    // chunks of large ones instead of queueing behind them; jobs queued for
    // serve_aging_steps steps or more go first, oldest first, which bounds
    // how long large ones wait.  The order changes no image.
    const uint32_t aging = ctx->cfg.serve_aging_steps ? ctx->cfg.serve_aging_steps : 0xffffffffu;
    std::stable_sort(jobs.begin(), jobs.end(), [aging](const QueuedJob* a, const QueuedJob* b) {
      const bool sa = a->age >= aging, sb = b->age >= aging;
      if (sa != sb) return sa;
      if (sa) return a->ticket < b->ticket;
      return a->total - a->issued < b->total - b->issued;
    });
    RunPlan plan;
    plan_run(jobs, plan_capacity(ctx, jobs), 1, 0, plan);
    int launched = -1;
    if (!plan.chunks.empty()) {
      RunSlot& sl = prev == &ctx->runs[0] ? ctx->runs[1] : ctx->runs[0];
      try {
        if (plan.restir)
          restir_prepare(ctx->restir, plan.max_count, std::max<uint32_t>(plan.max_count, 1),
                         (uint32_t)plan.chunks.size(), plan.max_segments);
        launch_planned(ctx, sl, std::move(plan));
      } catch (...) {
        // the chunk's jobs hold partial samples of a failed chunk: drop them
        cudaStreamSynchronize(ctx->stream);
        size_t k = 0;
        for (auto it = ctx->served.begin(); it != ctx->served.end(); ++k) {
          if ((*it)->issued != issued_before[k]) {
            release_job(ctx, **it);
            it = ctx->served.erase(it);
          } else {
            ++it;
          }
        }
        throw;
      }
      launched = (int)(&sl - ctx->runs);
    }
    for (auto& j : ctx->served) ++j->age;
    ctx->inflight = launched;
    // 2. collect the previous chunk: its finished jobs are complete
    if (prev) {
      finish_run(ctx, *prev, stats);
      for (QueuedJob* j : prev->plan.finished) done[(*num_done)++] = j->ticket;
      for (QueuedJob* j : prev->plan.finished) {
        auto it = std::find_if(ctx->served.begin(), ctx->served.end(),
                               [&](const std::unique_ptr<QueuedJob>& q) { return q.get() == j; });
        release_job(ctx, *j);
        ctx->served.erase(it);
      }
      prev->plan = RunPlan{};
    }
  });
}

int olc_queued_jobs(const olc_context* ctx, uint64_t* tickets, uint32_t capacity, uint32_t* count) {
  if (!ctx || !count) return fail(const_cast<olc_context*>(ctx), OLC_ERR_VALUE, "context and count are required");
  *count = (uint32_t)ctx->served.size();
  if (tickets) {
    uint32_t n = 0;
    for (const auto& j : ctx->served) {
      if (n == capacity) break;
      tickets[n++] = j->ticket;
    }
  }
  return OLC_OK;
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
    if (width != ctx->last_w || height != ctx->last_h || ctx->last_w == 0)
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

int olc_read_variance(olc_context* ctx, uint32_t width, uint32_t height, float* variance, int out_is_device) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (width != ctx->last_w || height != ctx->last_h || ctx->last_w == 0)
      throw Error(OLC_ERR_VALUE, "products are available only for the size of the last render");
    if (ctx->lum_spp == 0)
      throw Error(OLC_ERR_RUNTIME, "the last render kept no sample luminance (enable sample_variance)");
    if (!variance) throw Error(OLC_ERR_VALUE, "output pointer is required");
    const uint32_t npix = width * height;
    cudaStream_t st = ctx->stream;
    DeviceBuffer staging;
    float* dst = variance;
    if (!out_is_device) {
      staging.allocate((size_t)npix * sizeof(float));
      dst = staging.as<float>();
    }
    launch_sample_variance(ctx->ls, ctx->sample_lum.as<float>(), npix, ctx->lum_spp, dst, st);
    if (!out_is_device)
      OLC_CUDA(cudaMemcpyAsync(variance, dst, (size_t)npix * sizeof(float), cudaMemcpyDeviceToHost, st));
    OLC_CUDA(cudaStreamSynchronize(st));
  });
}

int olc_read_hit_geometry(olc_context* ctx, uint32_t width, uint32_t height, float* position, float* barycentric) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (width != ctx->last_w || height != ctx->last_h || ctx->last_w == 0)
      throw Error(OLC_ERR_VALUE, "products are available only for the size of the last render");
    const size_t n = (size_t)width * height;
    cudaStream_t st = ctx->stream;
    std::vector<float4> pos;
    if (position) {
      pos.resize(n);
      OLC_CUDA(cudaMemcpyAsync(pos.data(), ctx->prod_pos.get(), n * 16, cudaMemcpyDeviceToHost, st));
    }
    if (barycentric) OLC_CUDA(cudaMemcpyAsync(barycentric, ctx->prod_bary.get(), n * 8, cudaMemcpyDeviceToHost, st));
    OLC_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < pos.size(); ++i) {
      position[3 * i + 0] = pos[i].x;
      position[3 * i + 1] = pos[i].y;
      position[3 * i + 2] = pos[i].z;
    }
  });
}

int olc_read_path_signals(olc_context* ctx, uint32_t width, uint32_t height, float* signals, float* secondary) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (width != ctx->last_w || height != ctx->last_h || ctx->last_w == 0)
      throw Error(OLC_ERR_VALUE, "products are available only for the size of the last render");
    const size_t n = (size_t)width * height;
    cudaStream_t st = ctx->stream;
    if (signals) OLC_CUDA(cudaMemcpyAsync(signals, ctx->prod_signals.get(), n * 16, cudaMemcpyDeviceToHost, st));
    if (secondary) OLC_CUDA(cudaMemcpyAsync(secondary, ctx->prod_secondary.get(), n * 16, cudaMemcpyDeviceToHost, st));
    OLC_CUDA(cudaStreamSynchronize(st));
  });
}

int olc_capture_motion_state(olc_context* ctx) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    const ResidentScene& rs = default_scene(ctx);
    const SceneLayout& L = rs.layout;
    cudaStream_t st = ctx->stream;
    std::vector<MotionSegment> segs;
    std::vector<uint32_t> prefix;
    uint32_t total = 0;
    for (uint32_t k = 0; k < L.members; ++k) {
      const uint32_t i = L.order[k], m = L.instance_mesh[i];
      const uint32_t nt = L.mesh_triangle_offset[m + 1] - L.mesh_triangle_offset[m];
      if (nt == 0) continue;
      segs.push_back({total, (uint32_t)rs.slots.off + L.mesh_triangle_offset[m], (uint32_t)rs.instances.off + k,
                      L.instance_prim_offset[i]});
      prefix.push_back(total);
      total += nt;
    }
    if (L.flat_tris) {
      segs.push_back({total, (uint32_t)rs.slots.off + L.total_t, 0u, 0xffffffffu});
      prefix.push_back(total);
      total += (uint32_t)L.flat_tris;
    }
    const uint32_t packed = (uint32_t)L.packed_triangles;
    ctx->motion_prev.ensure(std::max<size_t>((size_t)packed * 48, 48));
    OLC_CUDA(cudaMemsetAsync(ctx->motion_prev.get(), 0, std::max<size_t>((size_t)packed * 48, 48), st));
    DeviceBuffer d_segs, d_prefix;
    uint64_t staging = 0;
    upload(d_segs, segs.data(), segs.size(), st, staging);
    upload(d_prefix, prefix.data(), prefix.size(), st, staging);
    world_triangles(pool_view(ctx), d_segs.as<MotionSegment>(), d_prefix.as<uint32_t>(), (uint32_t)segs.size(), total,
                    packed, ctx->motion_prev.as<float4>(), st);
    OLC_CUDA(cudaStreamSynchronize(st));
    ctx->motion_prev_count = packed;
  });
}

int olc_read_motion(olc_context* ctx, uint32_t width, uint32_t height, const olc_motion_mesh* meshes,
                    uint32_t num_meshes, const olc_motion_camera* now, const olc_motion_camera* before,
                    float* motion) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (width != ctx->last_w || height != ctx->last_h || ctx->last_w == 0)
      throw Error(OLC_ERR_VALUE, "products are available only for the size of the last render");
    if (!motion || !now || !before) throw Error(OLC_ERR_VALUE, "cameras and output are required");
    if (num_meshes && !meshes) throw Error(OLC_ERR_VALUE, "mesh table is required");
    std::vector<MotionMesh> table(num_meshes);
    for (uint32_t k = 0; k < num_meshes; ++k) {
      const olc_motion_mesh& m = meshes[k];
      if (k && m.first < meshes[k - 1].first) throw Error(OLC_ERR_VALUE, "motion meshes must be sorted by first");
      uint32_t prev = m.previous_first;
      if (prev != 0xffffffffu && (uint64_t)prev + m.count > ctx->motion_prev_count)
        throw Error(OLC_ERR_VALUE, "a motion mesh lies outside the captured frame");
      table[k] = MotionMesh{m.first, m.count, prev, 0u};
    }
    auto cam = [](const olc_motion_camera* c) {
      MotionCamera r;
      for (int k = 0; k < 3; ++k) {
        r.origin[k] = c->origin[k];
        r.forward[k] = c->forward[k];
        r.right[k] = c->right[k];
        r.up[k] = c->up[k];
      }
      r.scale = c->scale;
      return r;
    };
    const size_t n = (size_t)width * height;
    cudaStream_t st = ctx->stream;
    DeviceBuffer d_table, d_out(n * sizeof(float2));
    uint64_t staging = 0;
    upload(d_table, table.data(), table.size(), st, staging);
    motion_vectors(ctx->prod_prim.as<uint32_t>(), ctx->prod_pos.as<float4>(), ctx->prod_bary.as<float2>(), width,
                   height, d_table.as<MotionMesh>(), ctx->motion_prev_count ? num_meshes : 0u,
                   ctx->motion_prev.as<float4>(), cam(now), cam(before), d_out.as<float2>(), st);
    OLC_CUDA(cudaMemcpyAsync(motion, d_out.get(), n * sizeof(float2), cudaMemcpyDeviceToHost, st));
    OLC_CUDA(cudaStreamSynchronize(st));
  });
}

int olc_sample_texture(olc_context* ctx, uint32_t handle, int32_t binding, uint32_t n, const float* uv0,
                       const float* uv1, const float* fp0, const float* fp1, int srgb, float* out) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    if (handle == OLC_DEFAULT_SCENE) handle = ctx->default_scene;
    const ResidentScene& rs = scene_of(ctx, handle);
    if (!rs.rec.tex_words) throw Error(OLC_ERR_VALUE, "the scene has no textures");
    if (binding < -1 || binding >= (int32_t)(rs.tex_bindings.bytes() / 32)) throw Error(OLC_ERR_VALUE, "unknown texture binding");
    if (n == 0) return;
    if (!uv0 || !uv1 || !fp0 || !fp1 || !out) throw Error(OLC_ERR_VALUE, "inputs and output are required");
    cudaStream_t st = ctx->stream;
    uint64_t staging = 0;
    DeviceBuffer d0, d1, f0, f1, dout(n * sizeof(float4));
    upload(d0, uv0, 2ull * n, st, staging);
    upload(d1, uv1, 2ull * n, st, staging);
    upload(f0, fp0, n, st, staging);
    upload(f1, fp1, n, st, staging);
    launch_sample_textures(ctx->ls, ctx->scene_table.as<SceneRec>(), handle, (float)binding, n, d0.as<float2>(),
                           d1.as<float2>(), f0.as<float>(), f1.as<float>(), srgb, dout.as<float4>(), st);
    OLC_CUDA(cudaMemcpyAsync(out, dout.get(), n * sizeof(float4), cudaMemcpyDeviceToHost, st));
    OLC_CUDA(cudaStreamSynchronize(st));
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
    const ResidentScene& rs = default_scene(ctx);
    if (n == 0) return;
    if (!origins || !directions) throw Error(OLC_ERR_VALUE, "origins and directions are required");
    if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
    OLC_CUDA(cudaMemsetAsync(ctx->counters.get(), 0, sizeof(Counters), ctx->stream));
    launch_trace_rays(ctx->ls, pool_view(ctx), rs.rec.tlas_root, n, origins, directions, t_min, instance_id,
                      primitive, t, barycentrics, ctx->counters.as<Counters>(), ctx->stream);
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
    const ResidentScene& rs = default_scene(ctx);
    if (n == 0) return;
    if (!origins || !directions || !t_max || !occluded) throw Error(OLC_ERR_VALUE, "all arrays are required");
    if (!ctx->counters.get()) ctx->counters.allocate(sizeof(Counters));
    OLC_CUDA(cudaMemsetAsync(ctx->counters.get(), 0, sizeof(Counters), ctx->stream));
    launch_occluded_rays(ctx->ls, pool_view(ctx), rs.rec.tlas_root, n, origins, directions, t_min, t_max, occluded,
                         ctx->counters.as<Counters>(), ctx->stream);
    OLC_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int olc_camera_rays(olc_context* ctx, const olc_camera* camera, uint32_t width, uint32_t height, uint32_t sample,
                    uint32_t frame_index, const float* jitter_override, float* origins, float* directions) {
  if (!ctx) return fail(nullptr, OLC_ERR_VALUE, "context is required");
  return guarded(ctx, [&] {
    check_camera(camera);
    if (!origins || !directions) throw Error(OLC_ERR_VALUE, "camera and outputs are required");
    if (width == 0 || height == 0) throw Error(OLC_ERR_VALUE, "width and height must be positive");
    if (!ctx->job_dev.get()) ctx->job_dev.allocate(sizeof(JobRec));
    JobRec job = make_job(ctx, camera, width, height, 1, frame_index, 0, kNoScene);
    OLC_CUDA(cudaMemcpyAsync(ctx->job_dev.get(), &job, sizeof(JobRec), cudaMemcpyHostToDevice, ctx->stream));
    launch_camera_rays(ctx->ls, ctx->job_dev.as<JobRec>(), sample, jitter_override, origins, directions, ctx->stream);
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
  if (ctx->default_scene == kNoScene) return OLC_OK;
  const ResidentScene& rs = *ctx->scenes[ctx->default_scene];
  info->blas_count = rs.blas_count;
  info->blas_nodes = rs.blas_nodes;
  info->tlas_nodes = rs.tlas_nodes;
  info->triangles = rs.triangles;
  info->build_ms = rs.build_ms;
  return OLC_OK;
}

int olc_bvh_validate(olc_context* ctx, uint64_t* bad) {
  if (!ctx || !bad) return fail(ctx, OLC_ERR_VALUE, "context and output are required");
  return guarded(ctx, [&] {
    const ResidentScene& rs = default_scene(ctx);
    *bad = validate_bvh(pool_view(ctx), rs.blas_ranges, ctx->stream);
  });
}

}  // extern "C"
