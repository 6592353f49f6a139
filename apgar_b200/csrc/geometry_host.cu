// C ABI of the GPU geometry compile (geometry.cu): the exact swept-trace
// clearance predicate and the legal-edge masks of a set of lattice nodes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "apgar_b200.h"
#include "geometry_common.cuh"
#include "host_common.h"

namespace apgar_b200 {

cudaError_t launch_swept_cases(const int64_t* cases, uint64_t count, uint32_t* out, cudaStream_t stream);
cudaError_t launch_legal_edges(const GeometryLaunch& g, cudaStream_t stream);

namespace {

constexpr int64_t kLimit = 1000000000000ll;
constexpr int64_t kBin = 16;  // nodes per bin side

struct NodeKey {
  uint32_t layer;
  int64_t x, y;
  bool operator==(const NodeKey& o) const { return layer == o.layer && x == o.x && y == o.y; }
};
struct NodeKeyHash {
  size_t operator()(const NodeKey& k) const {
    uint64_t h = static_cast<uint64_t>(k.x) * 0x9E3779B97F4A7C15ull;
    h ^= static_cast<uint64_t>(k.y) * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
    return static_cast<size_t>(h ^ (static_cast<uint64_t>(k.layer) << 32));
  }
};

int64_t floor_div(__int128 a, int64_t b) {
  __int128 q = a / b;
  if ((a % b != 0) && ((a < 0) != (b < 0))) --q;
  return static_cast<int64_t>(q);
}

}  // namespace
}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" int apgar_b200_swept_clearance(const int64_t* cases, uint64_t count, uint32_t* out) {
  if (count > 0 && (cases == nullptr || out == nullptr)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "swept clearance received a null argument");
  }
  DeviceBuffer<int64_t> d_cases;
  DeviceBuffer<uint32_t> d_out;
  APGAR_B200_CUDA("cudaMalloc(cases)", d_cases.ensure(std::max<uint64_t>(10 * count, 1)));
  APGAR_B200_CUDA("cudaMalloc(verdicts)", d_out.ensure(std::max<uint64_t>(2 * count, 1)));
  if (count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(cases)", cudaMemcpy(d_cases.get(), cases, 80 * count, cudaMemcpyHostToDevice));
  }
  APGAR_B200_CUDA("swept clearance launch", launch_swept_cases(d_cases.get(), count, d_out.get(), nullptr));
  if (count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(verdicts)", cudaMemcpy(out, d_out.get(), 8 * count, cudaMemcpyDeviceToHost));
  }
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_compile_legal_edges(const apgar_b200_edge_rules* rules,
                                              const apgar_b200_obstacle_box* obstacles,
                                              uint64_t obstacle_count, const int64_t* lattice_xy,
                                              const uint32_t* layers, uint32_t node_count,
                                              uint8_t* legal_edges) {
  if (rules == nullptr || (obstacle_count > 0 && obstacles == nullptr) ||
      (node_count > 0 && (lattice_xy == nullptr || layers == nullptr || legal_edges == nullptr))) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "legal-edge compile received a null argument");
  }
  const int64_t step = rules->lattice_step, w = rules->nominal_width, c = rules->clearance;
  if (step <= 0 || step > kLimit || w <= 0 || w > kLimit || c < 0 || c > kLimit) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice step, trace width or clearance out of range");
  }
  try {
    // node points inside the exact coordinate envelope
    std::unordered_map<NodeKey, uint32_t, NodeKeyHash> index;
    index.reserve(node_count * 2ull + 1);
    for (uint32_t i = 0; i < node_count; ++i) {
      const __int128 px = static_cast<__int128>(rules->lattice_origin_x) + static_cast<__int128>(lattice_xy[2 * i]) * step;
      const __int128 py = static_cast<__int128>(rules->lattice_origin_y) + static_cast<__int128>(lattice_xy[2 * i + 1]) * step;
      if (px < -kLimit || px > kLimit || py < -kLimit || py > kLimit) {
        return set_error(APGAR_B200_INTERNAL_INVARIANT, "a lattice node lies outside the exact coordinate envelope");
      }
      if (!index.emplace(NodeKey{layers[i], lattice_xy[2 * i], lattice_xy[2 * i + 1]}, i).second) {
        return set_error(APGAR_B200_INTERNAL_INVARIANT, "a lattice node is given twice");
      }
    }
    static const int dx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
    static const int dy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
    std::vector<uint32_t> neighbor(8ull * node_count, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < node_count; ++i) {
      for (int d = 0; d < 8; ++d) {
        const auto it = index.find(NodeKey{layers[i], lattice_xy[2 * i] + dx[d], lattice_xy[2 * i + 1] + dy[d]});
        if (it != index.end()) neighbor[8ull * i + d] = it->second;
      }
    }
    for (uint64_t k = 0; k < obstacle_count; ++k) {
      const apgar_b200_obstacle_box& o = obstacles[k];
      if (o.min_x > o.max_x || o.min_y > o.max_y || o.min_x < -kLimit || o.max_x > kLimit ||
          o.min_y < -kLimit || o.max_y > kLimit) {
        return set_error(APGAR_B200_INTERNAL_INVARIANT, "an obstacle box is not normalized or leaves the envelope");
      }
    }
    // per-layer bins over the nodes' lattice extent
    struct LayerBins {
      int64_t x0 = 0, y0 = 0, x1 = -1, y1 = -1;
      int64_t bw = 0, bh = 0;
      size_t first = 0;
    };
    std::unordered_map<uint32_t, LayerBins> bins;
    for (uint32_t i = 0; i < node_count; ++i) {
      auto [it, fresh] = bins.try_emplace(layers[i]);
      LayerBins& b = it->second;
      const int64_t x = lattice_xy[2 * i], y = lattice_xy[2 * i + 1];
      if (fresh) {
        b.x0 = b.x1 = x;
        b.y0 = b.y1 = y;
      } else {
        b.x0 = std::min(b.x0, x); b.x1 = std::max(b.x1, x);
        b.y0 = std::min(b.y0, y); b.y1 = std::max(b.y1, y);
      }
    }
    size_t total_bins = 0;
    for (auto& [layer, b] : bins) {
      b.bw = (b.x1 - b.x0) / kBin + 1;
      b.bh = (b.y1 - b.y0) / kBin + 1;
      b.first = total_bins;
      total_bins += static_cast<size_t>(b.bw * b.bh);
    }
    // a box can fail a move that starts within w / 2 + c + 2 steps of it
    const __int128 expand = static_cast<__int128>(w) / 2 + c + 2 * static_cast<__int128>(step);
    std::vector<std::vector<uint32_t>> lists(total_bins);
    for (uint64_t k = 0; k < obstacle_count; ++k) {
      const apgar_b200_obstacle_box& o = obstacles[k];
      if (o.owned_by_net != 0u) continue;
      const auto it = bins.find(o.layer);
      if (it == bins.end()) continue;
      const LayerBins& b = it->second;
      const int64_t lx0 = floor_div(o.min_x - expand - rules->lattice_origin_x, step);
      const int64_t lx1 = floor_div(o.max_x + expand - rules->lattice_origin_x, step) + 1;
      const int64_t ly0 = floor_div(o.min_y - expand - rules->lattice_origin_y, step);
      const int64_t ly1 = floor_div(o.max_y + expand - rules->lattice_origin_y, step) + 1;
      const int64_t bx0 = std::max<int64_t>(0, (std::max(lx0, b.x0) - b.x0) / kBin);
      const int64_t bx1 = std::min<int64_t>(b.bw - 1, (std::min(lx1, b.x1) - b.x0) / kBin);
      const int64_t by0 = std::max<int64_t>(0, (std::max(ly0, b.y0) - b.y0) / kBin);
      const int64_t by1 = std::min<int64_t>(b.bh - 1, (std::min(ly1, b.y1) - b.y0) / kBin);
      if (lx1 < b.x0 || lx0 > b.x1 || ly1 < b.y0 || ly0 > b.y1) continue;
      for (int64_t by = by0; by <= by1; ++by) {
        for (int64_t bx = bx0; bx <= bx1; ++bx) lists[b.first + by * b.bw + bx].push_back(static_cast<uint32_t>(k));
      }
    }
    std::vector<uint32_t> bin_offset(total_bins + 1, 0);
    for (size_t i = 0; i < total_bins; ++i) bin_offset[i + 1] = bin_offset[i] + static_cast<uint32_t>(lists[i].size());
    std::vector<uint32_t> bin_boxes(std::max<uint32_t>(bin_offset[total_bins], 1));
    for (size_t i = 0; i < total_bins; ++i) std::copy(lists[i].begin(), lists[i].end(), bin_boxes.begin() + bin_offset[i]);
    std::vector<uint32_t> node_start(std::max<uint32_t>(node_count, 1)), node_len(std::max<uint32_t>(node_count, 1));
    for (uint32_t i = 0; i < node_count; ++i) {
      const LayerBins& b = bins.at(layers[i]);
      const size_t bin = b.first + static_cast<size_t>(((lattice_xy[2 * i + 1] - b.y0) / kBin) * b.bw +
                                                       (lattice_xy[2 * i] - b.x0) / kBin);
      node_start[i] = bin_offset[bin];
      node_len[i] = bin_offset[bin + 1] - bin_offset[bin];
    }
    std::vector<int64_t> boxes(std::max<uint64_t>(4 * obstacle_count, 4));
    for (uint64_t k = 0; k < obstacle_count; ++k) {
      boxes[4 * k] = obstacles[k].min_x;
      boxes[4 * k + 1] = obstacles[k].min_y;
      boxes[4 * k + 2] = obstacles[k].max_x;
      boxes[4 * k + 3] = obstacles[k].max_y;
    }
    DeviceBuffer<int64_t> d_xy, d_box;
    DeviceBuffer<uint32_t> d_layer, d_nb, d_start, d_len, d_bins;
    DeviceBuffer<uint8_t> d_legal;
    const size_t n = std::max<uint32_t>(node_count, 1);
    APGAR_B200_CUDA("cudaMalloc(nodes)", d_xy.ensure(2 * n));
    APGAR_B200_CUDA("cudaMalloc(layers)", d_layer.ensure(n));
    APGAR_B200_CUDA("cudaMalloc(neighbours)", d_nb.ensure(8 * n));
    APGAR_B200_CUDA("cudaMalloc(bins)", d_start.ensure(n));
    APGAR_B200_CUDA("cudaMalloc(bins)", d_len.ensure(n));
    APGAR_B200_CUDA("cudaMalloc(bin boxes)", d_bins.ensure(bin_boxes.size()));
    APGAR_B200_CUDA("cudaMalloc(boxes)", d_box.ensure(boxes.size()));
    APGAR_B200_CUDA("cudaMalloc(legal)", d_legal.ensure(n));
    if (node_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(nodes)", cudaMemcpy(d_xy.get(), lattice_xy, 16ull * node_count, cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(layers)", cudaMemcpy(d_layer.get(), layers, 4ull * node_count, cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(neighbours)", cudaMemcpy(d_nb.get(), neighbor.data(), 32ull * node_count, cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(bins)", cudaMemcpy(d_start.get(), node_start.data(), 4ull * node_count, cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(bins)", cudaMemcpy(d_len.get(), node_len.data(), 4ull * node_count, cudaMemcpyHostToDevice));
    }
    APGAR_B200_CUDA("cudaMemcpy(bin boxes)", cudaMemcpy(d_bins.get(), bin_boxes.data(), 4 * bin_boxes.size(), cudaMemcpyHostToDevice));
    APGAR_B200_CUDA("cudaMemcpy(boxes)", cudaMemcpy(d_box.get(), boxes.data(), 8 * boxes.size(), cudaMemcpyHostToDevice));
    GeometryLaunch g{};
    g.xy = d_xy.get();
    g.layer = d_layer.get();
    g.neighbor = d_nb.get();
    g.node_count = node_count;
    g.box = d_box.get();
    g.bin_start = d_start.get();
    g.bin_count = d_len.get();
    g.bin_boxes = d_bins.get();
    g.origin_x = rules->lattice_origin_x;
    g.origin_y = rules->lattice_origin_y;
    g.step = step;
    g.required = w + 2 * c;
    g.heading_mask = rules->heading_mask;
    g.legal = d_legal.get();
    APGAR_B200_CUDA("legal-edge launch", launch_legal_edges(g, nullptr));
    if (node_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(legal)", cudaMemcpy(legal_edges, d_legal.get(), node_count, cudaMemcpyDeviceToHost));
    }
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during the legal-edge compile");
  }
}
