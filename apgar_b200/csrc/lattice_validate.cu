// Validation of untrusted lattice-mode results on the device: the lattice
// counterpart of the structural stage of ValidateAndReconstructCompactGpuPath
// (src/gpu/planar_router.cc:969-1067), for the packed reverse paths of global
// cell ids (goal first) that a lattice route returns.
//
// Per reached net, in this order: the path lies inside the packed array and
// holds at least one cell; it starts at the goal and ends at the start; every
// cell lies in the lattice and in the net's window; every consecutive pair is
// one legal move, re-derived from the blocked and via bits (not from the
// search's precomputed move map): an orthogonal move needs both cells free, a
// diagonal one both cells and both side cells free, a via the same column on
// the adjacent layer with both cells free and the via bit set; and the move
// costs sum to the reported cost.  The first failing cell (counted from the
// start, like the reference's forward index) is reported.
//
// One warp per net; lane j checks the moves j, j + 32, ... of the path, and a
// warp reduction gives the cost sum and the first failure.
#include <cuda_runtime.h>

#include <cstdint>

#include "apgar_b200.h"
#include "lattice_common.cuh"

namespace apgar_b200 {
namespace {

__device__ __forceinline__ bool free_at(const LatticeDeviceView& lat, int l, int x, int y) {
  const uint32_t w =
      __ldg(lat.blocked + (static_cast<size_t>(l) * lat.height + y) * lat.words + (x >> 5));
  return ((w >> (x & 31)) & 1u) == 0u;
}

__device__ __forceinline__ bool via_bit(const LatticeDeviceView& lat, int lower, int x, int y) {
  if (lat.via_ok == nullptr) return true;
  const uint32_t w =
      __ldg(lat.via_ok + (static_cast<size_t>(lower) * lat.height + y) * lat.words + (x >> 5));
  return ((w >> (x & 31)) & 1u) != 0u;
}

struct Cell {
  int l, x, y;
};

__device__ __forceinline__ Cell cell_of(const LatticeDeviceView& lat, uint32_t c) {
  const uint32_t w = static_cast<uint32_t>(lat.width), h = static_cast<uint32_t>(lat.height);
  return Cell{static_cast<int>(c / w / h), static_cast<int>(c % w), static_cast<int>((c / w) % h)};
}

// cost of the legal move a -> b, or 0 if it is not one
__device__ __forceinline__ uint32_t move_cost(const LatticeDeviceView& lat, Cell a, Cell b) {
  const int dx = b.x - a.x, dy = b.y - a.y, dl = b.l - a.l;
  if (dl != 0) {
    if (dx != 0 || dy != 0 || (dl != 1 && dl != -1)) return 0u;
    const int lower = dl > 0 ? a.l : b.l;
    return (free_at(lat, a.l, a.x, a.y) && free_at(lat, b.l, b.x, b.y) &&
            via_bit(lat, lower, a.x, a.y))
               ? lat.via
               : 0u;
  }
  if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || (dx == 0 && dy == 0)) return 0u;
  if (!free_at(lat, a.l, a.x, a.y) || !free_at(lat, b.l, b.x, b.y)) return 0u;
  if (dx != 0 && dy != 0) {
    if (!free_at(lat, a.l, b.x, a.y) || !free_at(lat, a.l, a.x, b.y)) return 0u;
    return lat.diag;
  }
  return lat.orth;
}

__global__ void lattice_validate_kernel(LatticeDeviceView lat, const apgar_b200_lattice_net* nets,
                                        const apgar_b200_lattice_result* results,
                                        const uint32_t* paths, uint64_t path_count, uint32_t count,
                                        apgar_b200_path_verdict* out) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  const uint64_t cells = static_cast<uint64_t>(lat.layers) * lat.height * lat.width;
  for (uint32_t i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); i < count; i += warps) {
    const apgar_b200_lattice_result r = results[i];
    const apgar_b200_lattice_net n = nets[i];
    apgar_b200_path_verdict v{};
    if (r.completion != APGAR_B200_COMPLETION_REACHED) {
      v.code = APGAR_B200_PATH_NOT_REACHED;
    } else if (r.path_len == 0 || r.path_offset > path_count || r.path_len > path_count - r.path_offset) {
      v.code = APGAR_B200_PATH_BOUNDS;
    } else {
      const uint32_t len = r.path_len;
      const uint32_t* rev = paths + r.path_offset;
      const uint32_t goal = (n.goal_layer * static_cast<uint32_t>(lat.height) + n.goal_y) *
                                static_cast<uint32_t>(lat.width) + n.goal_x;
      const uint32_t start = (n.start_layer * static_cast<uint32_t>(lat.height) + n.start_y) *
                                 static_cast<uint32_t>(lat.width) + n.start_x;
      // forward index f = len - 1 - (reverse index); lane work: forward
      // index f checks cell f (bounds) and the move f - 1 -> f
      uint64_t first_bad = ~0ull;
      uint32_t bad_code = 0;
      uint64_t sum = 0;
      for (uint32_t f = lane; f < len; f += 32) {
        const uint32_t c = rev[len - 1 - f];
        uint32_t code = 0;
        if (c >= cells) {
          code = APGAR_B200_PATH_BOUNDS;
        } else {
          const Cell b = cell_of(lat, c);
          if (b.x < static_cast<int>(n.win_x0) || b.x >= static_cast<int>(n.win_x0 + n.win_w) ||
              b.y < static_cast<int>(n.win_y0) || b.y >= static_cast<int>(n.win_y0 + n.win_h)) {
            code = APGAR_B200_PATH_BOUNDS;
          } else if (f > 0) {
            const uint32_t p = rev[len - f];
            if (p >= cells) {
              code = APGAR_B200_PATH_BOUNDS;
            } else {
              const uint32_t cost = move_cost(lat, cell_of(lat, p), b);
              if (cost == 0u) code = APGAR_B200_PATH_EDGE;
              sum += cost;
            }
          }
        }
        if (code != 0u && f < first_bad) {
          first_bad = f;
          bad_code = code;
        }
      }
      // the first failure over the warp (smallest forward index)
      uint64_t best = first_bad;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) best = min(best, __shfl_xor_sync(0xFFFFFFFFu, best, s));
      const unsigned owner = __ballot_sync(0xFFFFFFFFu, first_bad == best && best != ~0ull);
      const uint32_t code = __shfl_sync(0xFFFFFFFFu, bad_code, owner ? __ffs(owner) - 1 : 0);
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, s);
      if (rev[len - 1] != start || rev[0] != goal) {
        v.code = APGAR_B200_PATH_ENDPOINT;
        v.failing_index = rev[len - 1] != start ? 0u : len - 1u;
      } else if (best != ~0ull) {
        v.code = code;
        v.failing_index = best;
      } else if (sum != r.cost) {
        v.code = APGAR_B200_PATH_COST;
        v.total_cost = sum;
      } else {
        v.total_cost = sum;
      }
    }
    if (lane == 0) out[i] = v;
  }
}

}  // namespace

cudaError_t launch_lattice_validate(const LatticeDeviceView& lat, const apgar_b200_lattice_net* nets,
                                    const apgar_b200_lattice_result* results, const uint32_t* paths,
                                    uint64_t path_count, uint32_t count,
                                    apgar_b200_path_verdict* out, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  const uint32_t blocks = (count + 7u) / 8u;  // 8 warps per block
  lattice_validate_kernel<<<blocks < 148u * 32u ? blocks : 148u * 32u, 256, 0, stream>>>(
      lat, nets, results, paths, path_count, count, out);
  return cudaGetLastError();
}

}  // namespace apgar_b200
