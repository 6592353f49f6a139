// Exact edge legality of the geometry compile, on the GPU.
//
// A one-step lattice move from node a to node b (8 headings) is legal when
// the heading is in the compiler's mask, b is a represented node on the same
// layer, and the swept trace of width w around the centreline keeps clearance
// c from every obstacle box on the layer that the routed net does not own
// (CompileBoard's edge loop, src/geometry_compiler/compiled_board.cc:427-476,
// over geometry::ValidateMovement, src/geometry/exact.cc:364-409).
//
// The clearance test is exact integer geometry on doubled coordinates, so the
// required distance d = w + 2c stays integral (exact.cc:165-216, :325-360):
// the move clears the box when their bounding boxes are at least d apart on
// one axis; it fails when an endpoint lies in the closed box, when the
// centreline touches a box edge, or when any endpoint of either lies closer
// than d to the other segment.  Products of doubled coordinates fit 128 bits;
// the one squared-distance comparison that does not (cross^2 against
// d^2 * |v|^2) is done in 256 bits.
//
// Obstacles are binned per layer on the host into 16 x 16-node bins over
// the layer's nodes; a box is listed in every bin whose nodes can start a
// move within w / 2 + c of it.  One thread handles one node and its eight
// moves, reading only its bin's boxes.
#include <cuda_runtime.h>

#include <cstdint>

#include "apgar_b200.h"
#include "geometry_common.cuh"

namespace apgar_b200 {


namespace {

using i128 = __int128;
using u128 = unsigned __int128;

struct Pt {
  i128 x, y;
};

__device__ __forceinline__ i128 orient(Pt a, Pt b, Pt c) {
  return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x);
}

__device__ __forceinline__ int sgn(i128 v) { return (v > 0) - (v < 0); }

__device__ __forceinline__ bool within(i128 v, i128 a, i128 b) {
  return v >= (a < b ? a : b) && v <= (a < b ? b : a);
}

__device__ __forceinline__ bool collinear_on(Pt a, Pt b, Pt p) {
  return within(p.x, a.x, b.x) && within(p.y, a.y, b.y);
}

// closed segments ab and cd share a point
__device__ bool touch(Pt a, Pt b, Pt c, Pt d) {
  const i128 o1 = orient(a, b, c), o2 = orient(a, b, d), o3 = orient(c, d, a), o4 = orient(c, d, b);
  if (sgn(o1) * sgn(o2) < 0 && sgn(o3) * sgn(o4) < 0) return true;
  return (o1 == 0 && collinear_on(a, b, c)) || (o2 == 0 && collinear_on(a, b, d)) ||
         (o3 == 0 && collinear_on(c, d, a)) || (o4 == 0 && collinear_on(c, d, b));
}

__device__ __forceinline__ u128 mag(i128 v) { return v < 0 ? static_cast<u128>(-v) : static_cast<u128>(v); }

// a * b as 256 bits (hi, lo)
__device__ void mul_wide(u128 a, u128 b, u128& hi, u128& lo) {
  const uint64_t a0 = static_cast<uint64_t>(a), a1 = static_cast<uint64_t>(a >> 64);
  const uint64_t b0 = static_cast<uint64_t>(b), b1 = static_cast<uint64_t>(b >> 64);
  const u128 p00 = static_cast<u128>(a0) * b0, p01 = static_cast<u128>(a0) * b1;
  const u128 p10 = static_cast<u128>(a1) * b0, p11 = static_cast<u128>(a1) * b1;
  const u128 mid = (p00 >> 64) + static_cast<uint64_t>(p01) + static_cast<uint64_t>(p10);
  lo = static_cast<uint64_t>(p00) | (mid << 64);
  hi = p11 + (p01 >> 64) + (p10 >> 64) + (mid >> 64);
}

__device__ __forceinline__ bool length_at_least(i128 x, i128 y, i128 d) {
  const u128 mx = mag(x), my = mag(y), md = static_cast<u128>(d);
  return mx * mx + my * my >= md * md;
}

// the distance from p to segment ab is at least d
__device__ bool point_segment_at_least(Pt p, Pt a, Pt b, i128 d) {
  const i128 vx = b.x - a.x, vy = b.y - a.y, wx = p.x - a.x, wy = p.y - a.y;
  const u128 len2 = mag(vx) * mag(vx) + mag(vy) * mag(vy);
  if (len2 == 0) return length_at_least(wx, wy, d);
  const i128 proj = wx * vx + wy * vy;
  if (proj <= 0) return length_at_least(wx, wy, d);
  if (static_cast<u128>(proj) >= len2) return length_at_least(p.x - b.x, p.y - b.y, d);
  const u128 cross = mag(vx * wy - vy * wx);
  u128 lh, ll, rh, rl;
  mul_wide(cross, cross, lh, ll);
  const u128 md = static_cast<u128>(d);
  mul_wide(md * md, len2, rh, rl);
  return lh > rh || (lh == rh && ll >= rl);
}

// doubled coordinates; d = w + 2c > 0
__device__ bool clears_box(Pt s, Pt e, Pt lo, Pt hi, i128 d) {
  const i128 sx0 = s.x < e.x ? s.x : e.x, sx1 = s.x < e.x ? e.x : s.x;
  const i128 sy0 = s.y < e.y ? s.y : e.y, sy1 = s.y < e.y ? e.y : s.y;
  if (sx1 <= lo.x - d || sx0 >= hi.x + d || sy1 <= lo.y - d || sy0 >= hi.y + d) return true;
  const auto inside = [&](Pt p) { return p.x >= lo.x && p.x <= hi.x && p.y >= lo.y && p.y <= hi.y; };
  if (inside(s) || inside(e)) return false;
  const Pt corner[4] = {lo, Pt{hi.x, lo.y}, hi, Pt{lo.x, hi.y}};
  for (int k = 0; k < 4; ++k) {
    const Pt c = corner[k], f = corner[(k + 1) & 3];
    if (touch(s, e, c, f)) return false;
    if (!point_segment_at_least(s, c, f, d) || !point_segment_at_least(e, c, f, d) ||
        !point_segment_at_least(c, s, e, d) || !point_segment_at_least(f, s, e, d)) {
      return false;
    }
  }
  return true;
}

constexpr int64_t kLimit = 1000000000000ll;

__device__ __forceinline__ bool coord_ok(int64_t v) { return v >= -kLimit && v <= kLimit; }

// error code (0 ok, 1 coordinate out of range, 2 invalid box, 3 invalid
// distance) and verdict of one segment against one box
__device__ uint32_t swept_case(const int64_t* c, uint32_t* satisfied) {
  *satisfied = 0;
  for (int i = 0; i < 8; ++i) {
    if (!coord_ok(c[i])) return 1u;
  }
  if (c[4] > c[6] || c[5] > c[7]) return 2u;
  const int64_t w = c[8], cl = c[9];
  if (w <= 0 || w > kLimit || cl < 0 || cl > kLimit) return 3u;
  const i128 d = static_cast<i128>(w) + 2 * static_cast<i128>(cl);
  const Pt s{2 * static_cast<i128>(c[0]), 2 * static_cast<i128>(c[1])};
  const Pt e{2 * static_cast<i128>(c[2]), 2 * static_cast<i128>(c[3])};
  const Pt lo{2 * static_cast<i128>(c[4]), 2 * static_cast<i128>(c[5])};
  const Pt hi{2 * static_cast<i128>(c[6]), 2 * static_cast<i128>(c[7])};
  *satisfied = clears_box(s, e, lo, hi, d) ? 1u : 0u;
  return 0u;
}

__global__ void swept_cases_kernel(const int64_t* __restrict__ cases, uint64_t count,
                                   uint32_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t sat;
    const uint32_t err = swept_case(cases + 10 * i, &sat);
    out[2 * i] = err;
    out[2 * i + 1] = sat;
  }
}

__constant__ int kDx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
__constant__ int kDy[8] = {0, 1, 1, 1, 0, -1, -1, -1};

__global__ void legal_edges_kernel(GeometryLaunch g) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.node_count; i += gridDim.x * blockDim.x) {
    const int64_t x = g.xy[2 * i], y = g.xy[2 * i + 1];
    const Pt s{2 * (static_cast<i128>(g.origin_x) + static_cast<i128>(x) * g.step),
               2 * (static_cast<i128>(g.origin_y) + static_cast<i128>(y) * g.step)};
    const uint32_t first = g.bin_start[i], n = g.bin_count[i];
    uint32_t mask = 0;
    for (int d = 0; d < 8; ++d) {
      const uint32_t heading = (d == 0 || d == 4) ? 1u : ((d == 2 || d == 6) ? 2u : 4u);
      if ((g.heading_mask & heading) == 0 || g.neighbor[8ull * i + d] == 0xFFFFFFFFu) continue;
      const Pt e{s.x + 2 * static_cast<i128>(kDx[d]) * g.step, s.y + 2 * static_cast<i128>(kDy[d]) * g.step};
      bool ok = true;
      for (uint32_t k = 0; k < n && ok; ++k) {
        const int64_t* b = g.box + 4ull * g.bin_boxes[first + k];
        ok = clears_box(s, e, Pt{2 * static_cast<i128>(b[0]), 2 * static_cast<i128>(b[1])},
                        Pt{2 * static_cast<i128>(b[2]), 2 * static_cast<i128>(b[3])}, g.required);
      }
      if (ok) mask |= 1u << d;
    }
    g.legal[i] = static_cast<uint8_t>(mask);
  }
}

}  // namespace

cudaError_t launch_swept_cases(const int64_t* cases, uint64_t count, uint32_t* out, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  const uint64_t blocks = (count + 255) / 256;
  swept_cases_kernel<<<static_cast<unsigned>(blocks < 4096 ? blocks : 4096), 256, 0, stream>>>(cases, count, out);
  return cudaGetLastError();
}

cudaError_t launch_legal_edges(const GeometryLaunch& g, cudaStream_t stream) {
  if (g.node_count == 0) return cudaSuccess;
  const uint32_t blocks = (g.node_count + 255) / 256;
  legal_edges_kernel<<<blocks < 148u * 64u ? blocks : 148u * 64u, 256, 0, stream>>>(g);
  return cudaGetLastError();
}

}  // namespace apgar_b200
