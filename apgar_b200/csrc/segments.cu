// Route reconstruction on the GPU: reverse paths -> exact points -> segments.
//
// One warp per path.  The path is read in forward order (start to goal; the
// stored paths are goal first).  Point j maps to exact board coordinates
// origin + lattice index * step (LatticeIndexToExactPoint,
// src/geometry_compiler/compiled_board.cc:219-238); a point outside the exact
// coordinate envelope (|v| > 10^12, board_ir::kMaxAbsDbCoord) fails the path.
// A segment starts at point 0 and wherever the step between consecutive
// points (dx, dy, dlayer) changes, as in routing::CoalesceSegments
// (src/routing/planar_route.cc:188-215, which is planar; the layer step is the
// extension for vias).  Lane s handles step s (points s - 1 -> s): a ballot of
// the steps that start a segment gives every segment its index, the lane that
// starts segment k writes its start and the end of segment k - 1.
#include <cuda_runtime.h>

#include <cstdint>

#include "apgar_b200.h"

namespace apgar_b200 {
namespace {

constexpr int64_t kMaxAbsCoord = 1000000000000ll;

struct ExactPoint {
  int64_t x, y;
  uint32_t layer;
  bool ok;
};

__device__ __forceinline__ ExactPoint exact_point(int64_t ox, int64_t oy, int64_t step, int64_t ix,
                                                  int64_t iy, uint32_t layer) {
  const __int128 x = static_cast<__int128>(ox) + static_cast<__int128>(ix) * step;
  const __int128 y = static_cast<__int128>(oy) + static_cast<__int128>(iy) * step;
  ExactPoint p;
  p.ok = x >= -kMaxAbsCoord && x <= kMaxAbsCoord && y >= -kMaxAbsCoord && y <= kMaxAbsCoord;
  p.x = static_cast<int64_t>(x);
  p.y = static_cast<int64_t>(y);
  p.layer = layer;
  return p;
}

// Coalesces the n forward points given by point_at(j) into out[0 ..); returns
// the segment count (uniform over the warp), or APGAR_B200_SEGMENT_FAILURE.
template <class PointAt>
__device__ uint32_t coalesce_warp(uint32_t n, const PointAt& point_at, apgar_b200_segment* out) {
  const int lane = threadIdx.x & 31;
  if (n < 2) return 0u;
  uint32_t carry = 0;
  bool bad = false;
  for (uint32_t base = 1; base < n; base += 32) {
    const uint32_t s = base + static_cast<uint32_t>(lane);
    const bool valid = s < n;
    bool boundary = false;
    ExactPoint prev{};
    if (valid) {
      prev = point_at(s - 1);
      const ExactPoint cur = point_at(s);
      bad = bad || !prev.ok || !cur.ok;
      if (s == 1) {
        boundary = true;
      } else {
        const ExactPoint pp = point_at(s - 2);
        bad = bad || !pp.ok;
        boundary = (cur.x - prev.x) != (prev.x - pp.x) || (cur.y - prev.y) != (prev.y - pp.y) ||
                   (static_cast<int64_t>(cur.layer) - prev.layer) !=
                       (static_cast<int64_t>(prev.layer) - pp.layer);
      }
    }
    const unsigned ballot = __ballot_sync(0xFFFFFFFFu, boundary);
    if (boundary) {
      const uint32_t k = carry + __popc(ballot & ((1u << lane) - 1u));
      out[k].layer0 = prev.layer;
      out[k].x0 = prev.x;
      out[k].y0 = prev.y;
      if (k > 0) {
        out[k - 1].layer1 = prev.layer;
        out[k - 1].x1 = prev.x;
        out[k - 1].y1 = prev.y;
      }
    }
    carry += __popc(ballot);
  }
  if (__any_sync(0xFFFFFFFFu, bad)) return APGAR_B200_SEGMENT_FAILURE;
  if (lane == 0) {
    const ExactPoint last = point_at(n - 1);
    out[carry - 1].layer1 = last.layer;
    out[carry - 1].x1 = last.x;
    out[carry - 1].y1 = last.y;
  }
  return carry;
}

// V1 compact paths: state = node * 9 + heading, goal first.
__global__ void path_segments_kernel(const apgar_b200_node_v1* __restrict__ nodes, uint32_t node_count,
                                     int64_t ox, int64_t oy, int64_t step,
                                     const apgar_b200_compact_path_v1* __restrict__ paths,
                                     const uint32_t* __restrict__ states, uint64_t state_count,
                                     uint32_t count, apgar_b200_segment* __restrict__ segments,
                                     uint32_t* __restrict__ segment_counts) {
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < count; i += warps) {
    const apgar_b200_compact_path_v1 p = paths[i];
    uint32_t result;
    if (p.state_offset > state_count || p.state_count > state_count - p.state_offset) {
      result = APGAR_B200_SEGMENT_FAILURE;
    } else {
      const uint32_t n = p.state_count;
      const uint32_t* rev = states + p.state_offset;
      const auto point_at = [&](uint32_t j) {
        const uint32_t node = rev[n - 1 - j] / 9u;
        if (node >= node_count) return ExactPoint{0, 0, 0, false};
        const apgar_b200_node_v1 nd = nodes[node];
        return exact_point(ox, oy, step, nd.lattice_x, nd.lattice_y, nd.layer);
      };
      result = coalesce_warp(n, point_at, segments + p.state_offset);
    }
    if ((threadIdx.x & 31) == 0) segment_counts[i] = result;
  }
}

// Lattice packed paths: global cell ids (layer * H + y) * W + x, goal first.
__global__ void lattice_segments_kernel(const apgar_b200_lattice_result* __restrict__ results,
                                        const uint32_t* __restrict__ paths, uint32_t count,
                                        uint32_t width, uint32_t height, int64_t ox, int64_t oy,
                                        int64_t step, apgar_b200_segment* __restrict__ segments,
                                        uint32_t* __restrict__ segment_counts) {
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < count; i += warps) {
    const apgar_b200_lattice_result r = results[i];
    uint32_t result = 0;
    if (r.completion == APGAR_B200_COMPLETION_REACHED) {
      const uint32_t n = r.path_len;
      const uint32_t* rev = paths + r.path_offset;
      const auto point_at = [&](uint32_t j) {
        const uint32_t c = rev[n - 1 - j];
        const uint32_t x = c % width, y = (c / width) % height, l = c / width / height;
        return exact_point(ox, oy, step, x, y, l);
      };
      result = coalesce_warp(n, point_at, segments + r.path_offset);
    }
    if ((threadIdx.x & 31) == 0) segment_counts[i] = result;
  }
}

unsigned warp_blocks(uint32_t count) {
  const uint32_t blocks = (count + 7u) / 8u;  // 8 warps per block
  return blocks < 148u * 32u ? blocks : 148u * 32u;
}

}  // namespace

cudaError_t launch_path_segments(const apgar_b200_node_v1* nodes, uint32_t node_count, int64_t ox,
                                 int64_t oy, int64_t step, const apgar_b200_compact_path_v1* paths,
                                 const uint32_t* states, uint64_t state_count, uint32_t count,
                                 apgar_b200_segment* segments, uint32_t* segment_counts,
                                 cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  path_segments_kernel<<<warp_blocks(count), 256, 0, stream>>>(nodes, node_count, ox, oy, step, paths,
                                                              states, state_count, count, segments,
                                                              segment_counts);
  return cudaGetLastError();
}

cudaError_t launch_lattice_segments(const apgar_b200_lattice_result* results, const uint32_t* paths,
                                    uint32_t count, uint32_t width, uint32_t height, int64_t ox,
                                    int64_t oy, int64_t step, apgar_b200_segment* segments,
                                    uint32_t* segment_counts, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  lattice_segments_kernel<<<warp_blocks(count), 256, 0, stream>>>(results, paths, count, width, height,
                                                                 ox, oy, step, segments,
                                                                 segment_counts);
  return cudaGetLastError();
}

}  // namespace apgar_b200
