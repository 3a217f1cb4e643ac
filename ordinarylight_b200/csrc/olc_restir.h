// ReSTIR DI at the primary vertex: interface used by the frame driver.
#pragma once

#include "olcuda.h"
#include "olc_internal.h"
#include "olc_wavefront.h"

namespace olc {

// Reservoir storage of one wavefront and the previous plain frame's history.
struct RestirState {
  DeviceBuffer res_a0, res_a1, res_a2;   // current reservoirs (three uint4 words each)
  DeviceBuffer res_b0, res_b1, res_b2;   // spatial ping-pong
  DeviceBuffer hist0, hist1, hist2;      // previous frame's final reservoirs
  DeviceBuffer selected;           // per path slot: light, bary, W
  DeviceBuffer pool0, pool1, pool2;  // light pool of each chunk segment (k_restir_pool)
  DeviceBuffer hit_list;           // path slots whose primary ray hit (ReSTIR jobs only)
  DeviceBuffer hit_count;
  uint64_t reservoirs = 0;         // reservoir capacity (pixel-samples of ReSTIR jobs)
  uint32_t slots = 0;              // path slot capacity
  uint32_t pool_segments = 0;      // chunk segments the light pool has room for
  uint32_t next_stamp = 1;         // stamp of the next chunk (0 never marks a valid reservoir)
  uint32_t run_first = 0, run_last = 0;    // stamps of this run's chunks
  uint32_t hist_first = 0, hist_last = 0;  // stamps of the history's chunks (set by restir_finish)
  bool final_in_b = false;
  // continuity key of the history (a plain frame: one job)
  bool history_valid = false;
  bool history_used = false;
  uint32_t hist_w = 0, hist_h = 0, hist_spp = 0, hist_frame = 0, hist_scene = 0;
  JobRec hist_camera{};
};

// Size buffers for `reservoirs` pixel-samples, `slots` path slots and light
// pools for `segments` chunk segments, and reserve one stamp per chunk of the
// run (chunk c of the run gets st.run_first + c; the caller stores it and the
// history's stamp range in each chunk header).
void restir_prepare(RestirState& st, uint64_t reservoirs, uint32_t slots, uint32_t chunks, uint32_t segments);
// Run initial RIS (+ temporal for jobs with history) + spatial reuse for one
// chunk over the primary hits the bounce-0 traversal listed in hit_list /
// hit_count; returns the per-path-slot selected sample buffer consumed by the
// bounce-0 shading pass.  Every host-side input is a pointer or a configuration value,
// so the launches can be captured in a graph and replayed.
const uint4* restir_run(RestirState& st, const olc_config& cfg, const LaunchShape& ls, const SceneView& s,
                        const ChunkHeader* hdr, const JobRec* jobs, const RayQueue& q, const HitBuf& hits,
                        const PathState& ps, bool textures, cudaStream_t stream);
// Promote this wavefront's final reservoirs to history (plain frames only).
void restir_finish(RestirState& st);
void restir_reset(RestirState& st);
void restir_release(RestirState& st);

}  // namespace olc
