// Host-only harness of the binned SAH builder (ordinarylight_b200/csrc/olc_sah.h)
// for the CPU tests: the tree as flat arrays.
#include <cstring>

#include "olc_sah.h"

extern "C" int sah_build_flat(uint32_t n, const float* lo, const float* hi, const float* centre, int32_t* child,
                              float* boxes, uint32_t* order) {
  std::vector<olc::sah::Node> nodes;
  std::vector<uint32_t> ord;
  olc::sah::build(n, lo, hi, centre, 3, nodes, ord);
  for (size_t i = 0; i < nodes.size(); ++i) {
    for (int s = 0; s < 2; ++s) {
      child[2 * i + s] = nodes[i].child[s];
      std::memcpy(boxes + 12 * i + 6 * s, nodes[i].box[s].lo, 3 * sizeof(float));
      std::memcpy(boxes + 12 * i + 6 * s + 3, nodes[i].box[s].hi, 3 * sizeof(float));
    }
  }
  std::memcpy(order, ord.data(), n * sizeof(uint32_t));
  return (int)nodes.size();
}
