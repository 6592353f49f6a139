// Structural validation of untrusted compact reverse paths on the device: the
// device-view checks of the reference's ValidateAndReconstructCompactGpuPath
// (src/gpu/planar_router.cc:969-1067), in its order, one thread per query.
// The exact-geometry stage that follows them in the reference (lattice points,
// coalesced segments, obstacle clearance) stays on the host.
//
// Per query: first the compact path's envelope (schema version 1, the
// query's id and workspace owner, a slice inside the state array, non-empty
// exactly when reached; src/gpu/planar_router.cc:1789-1805), then a reached
// completion and a path of 1..9N states; the goal state
// first and the canonical start state (start node, heading 8) last; every
// state below 9N; then in forward order: no repeated state (a visited bit per
// state), the start-only heading sentinel, one adjacent compiled legal edge
// (same layer, the lattice delta of the heading, the neighbour slot and the
// legal bit), no banned resource, and a checked finite cost sum.
#include <cuda_runtime.h>

#include <cstdint>

#include "graph_common.cuh"

namespace apgar_b200 {
namespace {

__device__ __forceinline__ bool add_finite(uint64_t a, uint64_t b, uint64_t* out) {
  constexpr uint64_t kMaxFinite = kGraphInf - 1u;
  if (a > kMaxFinite || b > kMaxFinite - a) return false;
  *out = a + b;
  return true;
}

__device__ __forceinline__ uint64_t adjustment(const apgar_b200_policy_edge_v1* pol, uint32_t count,
                                               uint32_t edge) {
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2u;
    if (pol[mid].physical_edge_index < edge) {
      lo = mid + 1u;
    } else {
      hi = mid;
    }
  }
  return (lo < count && pol[lo].physical_edge_index == edge) ? pol[lo].adjustment : 0ull;
}

__global__ void validate_paths_kernel(PathCheckLaunch p) {
  constexpr int kDx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
  constexpr int kDy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  const uint64_t states = static_cast<uint64_t>(p.node_count) * 9u;
  const uint64_t words = (states + 63u) / 64u;
  for (uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x; qi < p.query_count;
       qi += gridDim.x * blockDim.x) {
    apgar_b200_path_verdict v{};
    const apgar_b200_batch_result_v1 r = p.results[qi];
    const apgar_b200_batch_query_v1 q = p.queries[qi];
    const apgar_b200_compact_path_v1 c = p.compact[qi];
    uint64_t* visited = p.visited + static_cast<uint64_t>(qi) * words;
    const uint32_t start_state = q.start_node * 9u + 8u;
    const uint32_t* rev = p.states + c.state_offset;
    const uint64_t len = c.state_count;
    const bool reached = r.completion == APGAR_B200_COMPLETION_REACHED;
    const uint64_t end = c.state_offset + static_cast<uint64_t>(c.state_count);
    if (c.schema_version != 1u || c.query_id != q.query_id ||
        c.workspace_owner != q.workspace_owner || end < c.state_offset || end > p.state_count ||
        (reached ? c.state_count == 0u : c.state_count != 0u)) {
      // the compact path envelope (src/gpu/planar_router.cc:1789-1805)
      v.code = APGAR_B200_PATH_BOUNDS;
    } else if (!reached) {
      v.code = APGAR_B200_PATH_NOT_REACHED;
    } else if (len == 0 || len > states || c.state_offset > p.state_count ||
               len > p.state_count - c.state_offset) {
      v.code = APGAR_B200_PATH_BOUNDS;
    } else if (rev[0] != r.goal_state || rev[len - 1] != start_state ||
               r.goal_state / 9u != q.goal_node || r.goal_state % 9u >= 8u) {
      v.code = APGAR_B200_PATH_ENDPOINT;
    } else {
      for (uint64_t i = 0; i < len && v.code == 0; ++i) {
        if (rev[i] >= states) {
          v.code = APGAR_B200_PATH_BOUNDS;
        } else {
          visited[rev[i] / 64u] = 0;  // clear only the words this path touches
        }
      }
      uint64_t total = 0;
      const apgar_b200_policy_edge_v1* pol = p.policy + q.policy_offset;
      for (uint64_t index = 0; index < len && v.code == 0; ++index) {
        const uint64_t ri = len - 1u - index;
        const uint32_t state = rev[ri];
        v.failing_index = index;
        const uint64_t bit = 1ull << (state % 64u);
        if (visited[state / 64u] & bit) {
          v.code = APGAR_B200_PATH_CYCLE;
          break;
        }
        visited[state / 64u] |= bit;
        const uint32_t node = state / 9u;
        if (index == 0) {
          if (state != start_state) v.code = APGAR_B200_PATH_ENDPOINT;
          continue;
        }
        const uint32_t pred_state = rev[ri + 1u];
        const uint32_t pred = pred_state / 9u;
        const uint32_t incoming = state % 9u, pred_heading = pred_state % 9u;
        if (incoming >= 8u || (pred_heading == 8u && pred_state != start_state)) {
          v.code = APGAR_B200_PATH_HEADING;
          break;
        }
        const apgar_b200_node_v1& a = p.nodes[pred];
        const apgar_b200_node_v1& b = p.nodes[node];
        if (a.layer != b.layer || b.lattice_x - a.lattice_x != kDx[incoming] ||
            b.lattice_y - a.lattice_y != kDy[incoming] || a.neighbors[incoming] != node ||
            (a.legal_edges & (1u << incoming)) == 0) {
          v.code = APGAR_B200_PATH_EDGE;
          break;
        }
        // canonical physical edge: forward directions from the source, the
        // other four from the neighbour (the same resource either way)
        const uint32_t edge = incoming < 4u ? pred * 8u + incoming : node * 8u + incoming - 4u;
        const uint64_t adj = adjustment(pol, q.policy_count, edge);
        if (adj == kGraphInf) {
          v.code = APGAR_B200_PATH_BANNED;
          break;
        }
        const uint64_t step = (incoming & 1u) ? static_cast<uint64_t>(p.diag) : p.orth;
        const uint64_t sur = (incoming & 1u) ? q.diagonal_step_surcharge : q.orthogonal_step_surcharge;
        uint64_t t;
        bool ok = add_finite(step, sur, &t);
        if (ok && pred_heading != 8u && pred_heading != incoming) {
          ok = add_finite(t, static_cast<uint64_t>(p.bend), &t) && add_finite(t, q.bend_surcharge, &t);
        }
        ok = ok && add_finite(t, adj, &t) && add_finite(total, t, &total);
        if (!ok) {
          v.code = APGAR_B200_PATH_EDGE;
          break;
        }
      }
      if (v.code == 0) {
        v.total_cost = total;
        v.failing_index = 0;
      }
    }
    p.out[qi] = v;
  }
}

}  // namespace

cudaError_t launch_validate_paths(const PathCheckLaunch& launch, cudaStream_t stream) {
  if (launch.query_count == 0) return cudaSuccess;
  const uint32_t blocks = (launch.query_count + 127u) / 128u;
  validate_paths_kernel<<<blocks, 128, 0, stream>>>(launch);
  return cudaGetLastError();
}

}  // namespace apgar_b200
