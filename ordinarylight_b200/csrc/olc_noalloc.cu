// Allocation-free radix sort entry point.
//
// Some callers cannot allocate device memory at the moment they need a sort:
// code that runs while a CUDA stream is being captured into a graph (an
// allocation there is either an error or silently leaves the graph), serving
// loops that admit work against a fixed HBM budget and must not grow their
// footprint per request, and embedders whose allocator is owned by another
// runtime.  olc_radix_sort_pairs_noalloc gives them the stable LSD radix sort
// of the LBVH build with its scratch (ping-pong key/value arrays and the
// digit histogram) in one file-scope device array instead of memory from
// cudaMalloc.
//
// Properties a caller must know:
// * At most kNoAllocMaxPairs pairs per call; larger requests are rejected
//   with OLC_ERR_VALUE before any device work.
// * The scratch array exists once per device that loads the library and is
//   held until the process exits.
// * The first call on a device looks up the array's device address
//   (cudaGetSymbolAddress) with that device current; make that first call
//   before any stream capture on the device.  The address is cached per
//   CUDA context, so after the context is torn down (cudaDeviceReset) the
//   next call on that device looks it up again instead of reusing a
//   dangling address; make that call, too, outside any capture.
// * Every call on a device shares the one array and it keeps the last call's
//   contents.  Nothing in it needs to start at zero: the histogram and both
//   ping-pong arrays are fully rewritten by each pass before they are read.
//   Calls whose device work overlaps (different streams, or different host
//   threads without ordering) race on the array; order them on one stream.
#include <mutex>

#include "olcuda.h"
#include "olc_internal.h"

namespace {

constexpr uint32_t kNoAllocMaxPairs = 1u << 20;
// ping-pong keys, ping-pong values, histogram (256 digits x blocks of 2048)
constexpr size_t kNoAllocHistWords = 256u * ((kNoAllocMaxPairs + 2047u) / 2048u);
constexpr size_t kNoAllocWords = 2u * kNoAllocMaxPairs + kNoAllocHistWords;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_lock;
struct ScratchAddress {
  void* context = nullptr;      // the CUDA context the address belongs to
  uint32_t* address = nullptr;
};
ScratchAddress g_scratch[kMaxDevices];

// cuCtxGetCurrent, reached through the runtime so that the library does not
// link the driver library itself (it must load on machines without a GPU).
using CtxGetCurrentFn = int (*)(void**);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* entry = nullptr;
    cudaDriverEntryPointQueryResult found;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &entry, cudaEnableDefault, &found) != cudaSuccess ||
        found != cudaDriverEntryPointSuccess)
      entry = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(entry);
  }();
  return fn;
}

// Device address of the scratch array in the current device's context,
// looked up once per device and context.  A thread on which the runtime has
// not yet made a context current gets one from the symbol lookup itself
// (cudaGetSymbolAddress initialises the device's primary context).
uint32_t* scratch_on_current_device() {
  int device = 0;
  OLC_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kMaxDevices) throw olc::Error(OLC_ERR_VALUE, "device ordinal out of range");
  CtxGetCurrentFn get = ctx_get_current();
  if (!get) throw olc::Error(OLC_ERR_CUDA, "cuCtxGetCurrent is not available from the CUDA driver");
  std::lock_guard<std::mutex> lock(g_setup_lock);
  void* context = nullptr;
  if (get(&context) != 0) throw olc::Error(OLC_ERR_CUDA, "the current CUDA context could not be determined");
  ScratchAddress& entry = g_scratch[device];
  if (!context || entry.context != context || !entry.address) {
    void* ptr = nullptr;
    OLC_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    if (get(&context) != 0 || !context)
      throw olc::Error(OLC_ERR_CUDA, "the current CUDA context could not be determined");
    entry.context = context;
    entry.address = static_cast<uint32_t*>(ptr);
  }
  return entry.address;
}

}  // namespace

extern "C" int olc_radix_sort_pairs_noalloc(uint32_t n, uint32_t key_bits, uint32_t* keys, uint32_t* values,
                                            void* stream) {
  try {
    if (key_bits < 1 || key_bits > 32) throw olc::Error(OLC_ERR_VALUE, "key_bits must be between 1 and 32");
    if (n > kNoAllocMaxPairs)
      throw olc::Error(OLC_ERR_VALUE, "olc_radix_sort_pairs_noalloc sorts at most 1048576 pairs per call; got " +
                                          std::to_string(n));
    if (n == 0) return OLC_OK;
    if (!keys || !values) throw olc::Error(OLC_ERR_VALUE, "keys and values are required");
    uint32_t* scratch = scratch_on_current_device();
    uint32_t* keys_alt = scratch;
    uint32_t* vals_alt = scratch + kNoAllocMaxPairs;
    uint32_t* hist = scratch + 2u * kNoAllocMaxPairs;
    olc::radix_sort_pairs(keys, values, keys_alt, vals_alt, hist, n, key_bits, static_cast<cudaStream_t>(stream));
    return OLC_OK;
  } catch (const olc::Error& e) {
    olc::set_thread_error(e.what());
    return e.code;
  } catch (const std::exception& e) {
    olc::set_thread_error(e.what());
    return OLC_ERR_RUNTIME;
  }
}
