// Binned SAH hierarchy over primitive boxes, built on the host (plain C++,
// no CUDA types: the device builder in olc_bvh.cu converts the result to its
// BVH2 node layout, and a host-only harness tests it on the CPU).
//
// Top-down, one primitive per leaf; each split is the best of 3 axes x
// (kSahBins - 1) planes between centroid bins by the surface area heuristic
// A(L) n(L) + A(R) n(R) (Wald, "On fast Construction of SAH-based Bounding
// Volume Hierarchies", IEEE Symposium on Interactive Ray Tracing 2007); a
// median split where no axis has a usable centroid extent (coincident
// centroids, or an extent so small that the bin scale overflows).
//
// Output: n - 1 internal nodes, node 0 the root, each child of an internal
// node created after it (indices grow downwards).  A child reference c >= 0
// is internal node c; c < 0 is the leaf at sorted position ~c, and order[k]
// is the primitive of sorted position k.  Every node's primitives are a
// contiguous range of sorted positions.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace olc {
namespace sah {

constexpr int kSahBins = 16;

struct Box {
  float lo[3] = {INFINITY, INFINITY, INFINITY};
  float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  void grow(const float* l, const float* h) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], l[a]);
      hi[a] = std::max(hi[a], h[a]);
    }
  }
  void grow(const Box& b) { grow(b.lo, b.hi); }
  double area() const {
    const double e0 = std::max(0.0, (double)hi[0] - lo[0]), e1 = std::max(0.0, (double)hi[1] - lo[1]);
    const double e2 = std::max(0.0, (double)hi[2] - lo[2]);
    return 2.0 * (e0 * e1 + e1 * e2 + e2 * e0);
  }
};

struct Node {
  Box box[2];        // child boxes
  int32_t child[2];  // >= 0: internal node; < 0: ~(sorted leaf position)
};

// lo, hi, centre: n records of `stride` floats each (x, y, z first), e.g.
// float4 arrays with stride 4.
inline void build(uint32_t n, const float* lo, const float* hi, const float* centre, uint32_t stride,
                  std::vector<Node>& nodes, std::vector<uint32_t>& order) {
  order.resize(n);
  for (uint32_t p = 0; p < n; ++p) order[p] = p;
  nodes.assign(n > 1 ? n - 1 : 0, Node{});
  if (n < 2) return;
  auto box_of = [&](uint32_t p) {
    Box b;
    b.grow(lo + (size_t)p * stride, hi + (size_t)p * stride);
    return b;
  };
  auto cen = [&](uint32_t p, int a) { return centre[(size_t)p * stride + a]; };
  // bin of centre coordinate c along an axis; the same expression serves the
  // binning and the partition, so both see the same bins
  auto bin_of = [](float c, float base, float scale) {
    const float x = (c - base) * scale;
    return x >= (float)(kSahBins - 1) ? kSahBins - 1 : (x > 0.0f ? (int)x : 0);
  };
  struct Task {
    uint32_t begin, end, node;
  };
  std::vector<Task> tasks{{0, n, 0}};
  uint32_t next = 1;
  while (!tasks.empty()) {
    const Task t = tasks.back();
    tasks.pop_back();
    Box cb;
    for (uint32_t k = t.begin; k < t.end; ++k) {
      const float c[3] = {cen(order[k], 0), cen(order[k], 1), cen(order[k], 2)};
      cb.grow(c, c);
    }
    double best = INFINITY;
    int best_axis = -1, best_plane = 0;
    float best_scale = 0.0f;
    for (int a = 0; a < 3; ++a) {
      const float extent = cb.hi[a] - cb.lo[a];
      const float scale = (float)kSahBins / extent;
      if (!(extent > 0.0f) || !std::isfinite(scale)) continue;
      Box bins[kSahBins];
      uint32_t counts[kSahBins] = {};
      for (uint32_t k = t.begin; k < t.end; ++k) {
        const uint32_t p = order[k];
        const int b = bin_of(cen(p, a), cb.lo[a], scale);
        bins[b].grow(box_of(p));
        ++counts[b];
      }
      double right_area[kSahBins] = {};
      uint32_t right_count[kSahBins] = {};
      Box acc;
      uint32_t cnt = 0;
      for (int b = kSahBins - 1; b > 0; --b) {
        acc.grow(bins[b]);
        cnt += counts[b];
        right_area[b] = acc.area();
        right_count[b] = cnt;
      }
      acc = Box();
      cnt = 0;
      for (int b = 0; b < kSahBins - 1; ++b) {
        acc.grow(bins[b]);
        cnt += counts[b];
        if (cnt == 0 || right_count[b + 1] == 0) continue;
        const double cost = acc.area() * cnt + right_area[b + 1] * right_count[b + 1];
        if (cost < best) {
          best = cost;
          best_axis = a;
          best_plane = b + 1;
          best_scale = scale;
        }
      }
    }
    uint32_t mid = t.begin + (t.end - t.begin) / 2;   // coincident centroids: median
    if (best_axis >= 0) {
      const int axis = best_axis, plane = best_plane;
      const float base = cb.lo[axis], scale = best_scale;
      mid = (uint32_t)(std::stable_partition(order.begin() + t.begin, order.begin() + t.end,
                                             [&](uint32_t p) { return bin_of(cen(p, axis), base, scale) < plane; }) -
                       order.begin());
    }
    const uint32_t range[2][2] = {{t.begin, mid}, {mid, t.end}};
    Node& nd = nodes[t.node];
    for (int s = 0; s < 2; ++s) {
      Box b;
      for (uint32_t k = range[s][0]; k < range[s][1]; ++k) b.grow(box_of(order[k]));
      nd.box[s] = b;
      if (range[s][1] - range[s][0] == 1) {
        nd.child[s] = ~(int32_t)range[s][0];
      } else {
        const uint32_t c = next++;
        nd.child[s] = (int32_t)c;
        tasks.push_back(Task{range[s][0], range[s][1], c});
      }
    }
  }
}

}  // namespace sah
}  // namespace olc
