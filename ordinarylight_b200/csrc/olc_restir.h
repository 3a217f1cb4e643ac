// ReSTIR DI at the primary vertex: interface used by the frame driver.
#pragma once

#include "olcuda.h"
#include "olc_internal.h"
#include "olc_wavefront.h"

namespace olc {

// Reservoir storage of one frame and the previous frame's history.
struct RestirState {
  DeviceBuffer res_a0, res_a1;     // current reservoirs (two uint4 words each)
  DeviceBuffer res_b0, res_b1;     // spatial ping-pong
  DeviceBuffer hist0, hist1;       // previous frame's final reservoirs
  DeviceBuffer selected;           // per path slot: light, bary, W
  DeviceBuffer hit_list;           // path slots whose primary ray hit
  DeviceBuffer hit_count;
  uint32_t stamp = 0;              // validity stamp of this frame's reservoirs
  uint32_t prev_stamp = 0;
  uint64_t reservoirs = 0;         // npix * spp capacity
  uint32_t slots = 0;              // path slot capacity
  // frame continuity of the history
  bool history_valid = false;
  bool history_used = false;
  uint32_t hist_w = 0, hist_h = 0, hist_spp = 0, hist_frame = 0;
  FrameParams hist_camera{};
  uint32_t cur_w = 0, cur_h = 0, cur_spp = 0, cur_frame = 0;
  bool final_in_b = false;
};

// Size buffers and decide whether last frame's reservoirs are a valid
// temporal history for (w, h, spp, frame_index, camera).
void restir_prepare(RestirState& st, const olc_config& cfg, uint32_t w, uint32_t h, uint32_t spp,
                    uint32_t frame_index, uint32_t slots, const FrameParams& camera);
// Run initial RIS + temporal + spatial reuse for one chunk; returns the
// per-path-slot selected sample buffer consumed by k_shade at bounce 0.
const uint4* restir_run(RestirState& st, const olc_config& cfg, const LaunchShape& ls, const SceneView& s,
                        const FrameParams* fp, const RayQueue& q, const HitBuf& hits, const PathState& ps,
                        Counters* cnt, uint64_t chunk_begin, uint32_t chunk_count, uint32_t npix,
                        cudaStream_t stream);
// Promote this frame's final reservoirs to history.
void restir_finish(RestirState& st);
void restir_reset(RestirState& st);
void restir_release(RestirState& st);

}  // namespace olc
