// Host-side internals shared by the translation units of libolcuda.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "olc_common.cuh"

namespace olc {

// Error carrying an olc_status code across the C++ layers; the C ABI
// converts it into a return code plus last-error string.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

// Message returned by olc_last_error(NULL) on this thread.
void set_thread_error(const std::string& message);

inline void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? 5 /*OLC_ERR_MEMORY*/ : 4 /*OLC_ERR_CUDA*/;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define OLC_CUDA(call) ::olc::check_cuda((call), #call)
#define OLC_LAUNCH_CHECK(name) ::olc::check_cuda(cudaGetLastError(), name)

// Owning device allocation.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { allocate(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) { o.ptr_ = nullptr; o.bytes_ = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) { release(); ptr_ = o.ptr_; bytes_ = o.bytes_; o.ptr_ = nullptr; o.bytes_ = 0; }
    return *this;
  }
  void allocate(size_t bytes) {
    release();
    if (bytes == 0) return;
    OLC_CUDA(cudaMalloc(&ptr_, bytes));
    bytes_ = bytes;
  }
  // Grow-only reallocation (contents are not preserved).
  void ensure(size_t bytes) { if (bytes > bytes_) allocate(bytes); }
  void release() {
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(ptr_); }
  void* get() const { return ptr_; }
  size_t bytes() const { return bytes_; }

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

// ---- LBVH construction (olc_bvh.cu) --------------------------------------

// Scratch for one LBVH build of up to n primitives.
struct BuildScratch {
  DeviceBuffer boxes_lo, boxes_hi;   // float4 per primitive (unsorted)
  DeviceBuffer centers;              // float4 per primitive
  DeviceBuffer bounds;               // 6 ordered uints
  DeviceBuffer keys, vals, keys_alt, vals_alt, hist;
  DeviceBuffer sorted_lo, sorted_hi; // float4 per leaf in sorted order
  DeviceBuffer left, right, first, last, parent, leaf_parent, flags;
  DeviceBuffer node_lo, node_hi;     // float4 per internal node
  size_t capacity = 0;
  void ensure(size_t n);
};

// Compute 30-bit Morton codes of box centres (exposed for tests too).
void morton_codes(const float4* centers, uint32_t n, uint32_t* bounds_scratch, uint32_t* codes,
                  cudaStream_t stream);
// Centres of triangle AABBs from a flat [n*9] array (tests).
void triangle_centers_flat(const float* tri, uint32_t n, float4* lo, float4* hi, float4* centers,
                           cudaStream_t stream);
// Stable LSD radix sort of pairs; result lands in keys/vals.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      uint32_t* hist, uint32_t n, uint32_t key_bits, cudaStream_t stream);
size_t radix_sort_hist_words(uint32_t n);

struct BlasDesc {
  const float* vertices;      // device [nv*3]
  const float* normals;       // device [nv*3]
  const uint32_t* indices;    // device [nt*3]
  uint32_t num_vertices;
  uint32_t num_triangles;
};

// Build one BLAS.  Writes nodes at nodes[node_base ...] and triangle data at
// slot range [slot_base, slot_base + nt).  Returns the root node index.
uint32_t build_blas(const BlasDesc& d, BuildScratch& scratch, BvhNode* nodes, uint32_t node_base,
                    float4* tri_verts, float4* tri_normals, uint32_t* tri_index, uint32_t slot_base,
                    uint32_t leaf_max, cudaStream_t stream);
inline uint32_t blas_node_count(uint32_t nt) { return nt > 1 ? nt - 1 : 1; }

// Texture attributes of one mesh's BLAS slots [first_slot, +nt) into
// attr[6 * (slot - scene_slot0) ...] (texcoords / tangents: float4 per vertex
// of the concatenated mesh arrays, mesh_indices: the mesh's index triples).
void slot_attributes(const float4* texcoords, const float4* tangents, const uint32_t* mesh_indices, uint32_t nt,
                     uint32_t vertex_base, const uint32_t* tri_index, uint32_t first_slot, uint32_t scene_slot0,
                     float4* attr, cudaStream_t stream);
// The 256-entry sRGB decode table.
void srgb_table(float* out, cudaStream_t stream);

// Refit one BLAS in place for new positions of the same triangles: rewrite
// its slots [slot_base, +nt) from d and recompute the boxes of its
// node_count nodes at node_base bottom-up.  The hierarchy is unchanged.
void refit_blas(const BlasDesc& d, BuildScratch& scratch, BvhNode* nodes, uint32_t node_base, uint32_t node_count,
                float4* tri_verts, float4* tri_normals, const uint32_t* tri_index, uint32_t slot_base,
                cudaStream_t stream);

// Build the TLAS over n instances (world boxes computed from BLAS roots) and
// n_flat world-space triangles referenced directly (flat_verts: 3 float4 per
// triangle, the same data as pool slots [flat_slot_base, +n_flat)).  Build
// primitive p < n becomes an instance leaf of global instance
// instance_base + p; p >= n a triangle leaf of global slot
// flat_slot_base + p - n.  slot_ranges[i] = triangle slot range of instance
// i's BLAS (its world box is the transformed bounds of those vertices);
// max_instance_triangles is the largest of those ranges.
uint32_t build_tlas(const float* object_to_world, const uint2* slot_ranges, uint32_t n,
                    uint32_t max_instance_triangles, uint32_t instance_base, const float4* tri_verts,
                    const float4* flat_verts, uint32_t n_flat, uint32_t flat_slot_base, BuildScratch& scratch,
                    BvhNode* nodes, uint32_t node_base, cudaStream_t stream);

// The BVH4 form (BvhNode4) of BVH2 nodes [begin, begin + count): wide[i]
// holds up to four descendants of nodes[i] (greedy surface-area collapse).
// Run after every build or refit that wrote those nodes.
void build_bvh4(const BvhNode* nodes, BvhNode4* wide, uint32_t begin, uint32_t count, cudaStream_t stream);

// One built bottom-level structure: its root node and triangle slot range.
struct BlasRange {
  uint32_t root, slot_begin, slot_end;
};

// Count structural violations of the resident BVH: every slot of every built
// BLAS reached exactly once from its root, child boxes inside parent boxes.
uint64_t validate_bvh(const SceneView& s, const std::vector<BlasRange>& blas, cudaStream_t stream);

}  // namespace olc
