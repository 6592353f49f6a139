// Reachability under policy bans, for the confirmation of DISCONNECTED
// results (the device counterpart of ConfirmDisconnectedWithCpuOracle,
// src/gpu/planar_router.cc:629-667).
//
// The CPU A* (src/routing/cpu_astar.cc:413-512) expands states (node,
// incoming heading); a move is taken when the node's compiled legal mask has
// its direction and the policy does not ban its canonical edge resource.
// Headings only change costs, so its queue empties without the goal exactly
// when the goal node is unreachable from the start node over those moves.
//
// One CTA per query, level-synchronous breadth-first search: a visited bit
// per node (atomicOr decides which thread queues a node), the level's nodes
// in a global list, the next level's count in shared memory.  Every node is
// queued at most once, so each list holds at most `nodes` entries.  The
// search stops early when it queues the goal.
#include <cuda_runtime.h>

#include <cstdint>

#include "graph_common.cuh"

namespace apgar_b200 {
namespace {

__device__ __forceinline__ bool banned(const apgar_b200_policy_edge_v1* pol, uint32_t count,
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
  return lo < count && pol[lo].physical_edge_index == edge && pol[lo].adjustment == kGraphInf;
}

__global__ void __launch_bounds__(256) reach_kernel(ReachLaunch p) {
  __shared__ uint32_t next_count, found;
  const uint32_t n_nodes = p.node_count;
  const uint64_t words = (static_cast<uint64_t>(n_nodes) + 31u) / 32u;
  for (uint32_t k = blockIdx.x; k < p.count; k += gridDim.x) {
    const apgar_b200_batch_query_v1 q = p.queries[p.selected[k]];
    const apgar_b200_policy_edge_v1* pol = p.policy + q.policy_offset;
    uint32_t* visited = p.visited + static_cast<uint64_t>(k) * words;
    uint32_t* cur = p.queues + static_cast<uint64_t>(k) * 2u * n_nodes;
    uint32_t* nxt = cur + n_nodes;
    for (uint64_t i = threadIdx.x; i < words; i += blockDim.x) visited[i] = 0u;
    __syncthreads();
    if (threadIdx.x == 0) {
      visited[q.start_node / 32u] = 1u << (q.start_node % 32u);
      cur[0] = q.start_node;
      found = q.start_node == q.goal_node ? 1u : 0u;
    }
    __syncthreads();
    uint32_t n = 1;
    uint64_t total = 1;
    while (n > 0 && found == 0u) {  // uniform: both read after a barrier
      if (threadIdx.x == 0) next_count = 0u;
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t u = cur[i];
        const uint32_t mask = p.legal[u];
        for (uint32_t d = 0; d < 8u; ++d) {
          if ((mask & (1u << d)) == 0u) continue;
          const uint32_t v = p.neighbors[static_cast<uint64_t>(d) * n_nodes + u];
          // canonical physical edge: forward directions from the source, the
          // other four from the neighbour
          const uint32_t edge = d < 4u ? u * 8u + d : v * 8u + d - 4u;
          if (banned(pol, q.policy_count, edge)) continue;
          const uint32_t bit = 1u << (v % 32u);
          if ((atomicOr(&visited[v / 32u], bit) & bit) != 0u) continue;
          nxt[atomicAdd(&next_count, 1u)] = v;
          if (v == q.goal_node) found = 1u;
        }
      }
      __syncthreads();
      n = next_count;
      total += n;
      uint32_t* t = cur;
      cur = nxt;
      nxt = t;
      __syncthreads();  // next_count read by all before it is reset
    }
    if (threadIdx.x == 0) {
      p.reached[k] = found;
      p.reach_nodes[k] = total;
    }
    __syncthreads();
  }
}

}  // namespace

cudaError_t launch_reach(const ReachLaunch& launch, cudaStream_t stream) {
  if (launch.count == 0) return cudaSuccess;
  const uint32_t blocks = launch.count < 148u * 8u ? launch.count : 148u * 8u;
  reach_kernel<<<blocks, 256, 0, stream>>>(launch);
  return cudaGetLastError();
}

}  // namespace apgar_b200
