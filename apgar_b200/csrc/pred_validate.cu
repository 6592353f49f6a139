// Validation of untrusted full-workspace results (labels and predecessors of
// every heading state) on the device: the checks of ValidateAllPredecessors
// (src/gpu/planar_router.cc:492-611) for every state of every query at once.
//
// The reference walks the states in index order and returns at the first
// failure.  Here one thread checks one state; a failing state records
// ((state + 1) << 32 | code) with a 64-bit atomicMin, so the query keeps the
// reference's first failure.  The start-state check runs before the walk in
// the reference, so its failure records key 0 and wins over every state.
//
// Per state other than the start, in the reference's order: a heading-8 state
// (no incoming heading) must be unreachable with no predecessor; an
// unreachable state must have no predecessor; a reachable state with no
// predecessor passes under partial validation (a bounded search may have
// improved it last); the predecessor must be in bounds, not the state itself,
// one adjacent compiled legal edge in the state's heading, not a heading-8
// state other than the start, reachable, not over a banned resource, and its
// label plus the transition cost (checked add) must equal the label (exact)
// or not exceed it (partial).
#include <cuda_runtime.h>

#include <cstdint>

#include "graph_common.cuh"

namespace apgar_b200 {
namespace {

__device__ __forceinline__ bool add_checked(uint64_t a, uint64_t b, uint64_t* out) {
  constexpr uint64_t kMaxFinite = kGraphInf - 1u;
  if (a > kMaxFinite || b > kMaxFinite - a) return false;
  *out = a + b;
  return true;
}

// adjustment of one physical edge in a sorted policy slice (0 if absent)
__device__ __forceinline__ uint64_t edge_adjustment(const apgar_b200_policy_edge_v1* pol,
                                                    uint32_t count, uint32_t edge) {
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

__global__ void validate_predecessors_kernel(PredCheckLaunch p) {
  constexpr int kDx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
  constexpr int kDy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  const uint64_t states = static_cast<uint64_t>(p.node_count) * 9u;
  const uint64_t total = states * p.query_count;
  for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    const uint32_t qi = static_cast<uint32_t>(t / states);
    const uint32_t state = static_cast<uint32_t>(t % states);
    const apgar_b200_batch_query_v1 q = p.queries[qi];
    const uint64_t* labels = p.labels + static_cast<uint64_t>(qi) * states;
    const uint32_t* preds = p.predecessors + static_cast<uint64_t>(qi) * states;
    const bool partial = p.partial != nullptr && p.partial[qi] != 0u;
    uint32_t code = 0;
    if (q.start_node >= p.node_count) {
      if (state == 0u) atomicMin(&p.first[qi], static_cast<unsigned long long>(APGAR_B200_PRED_START));
      continue;
    }
    const uint32_t start_state = q.start_node * 9u + 8u;
    const uint64_t label = labels[state];
    const uint32_t pred = preds[state];
    const uint32_t incoming = state % 9u;
    if (state == start_state) {
      if (label != 0u || pred != kInvalid32) {
        atomicMin(&p.first[qi], static_cast<unsigned long long>(APGAR_B200_PRED_START));
      }
      continue;
    }
    if (incoming == 8u) {
      if (label != kGraphInf || pred != kInvalid32) code = APGAR_B200_PRED_NO_HEADING;
    } else if (label == kGraphInf) {
      if (pred != kInvalid32) code = APGAR_B200_PRED_UNREACHABLE;
    } else if (pred == kInvalid32 && partial) {
      code = 0;
    } else if (pred >= states) {
      code = APGAR_B200_PRED_BOUNDS;
    } else if (pred == state) {
      code = APGAR_B200_PRED_SELF_REFERENCE;
    } else {
      const uint32_t node = state / 9u, pnode = pred / 9u;
      const apgar_b200_node_v1& a = p.nodes[pnode];
      const apgar_b200_node_v1& b = p.nodes[node];
      const uint32_t pheading = pred % 9u;
      if (a.layer != b.layer || b.lattice_x - a.lattice_x != kDx[incoming] ||
          b.lattice_y - a.lattice_y != kDy[incoming] || a.neighbors[incoming] != node ||
          (a.legal_edges & (1u << incoming)) == 0) {
        code = APGAR_B200_PRED_EDGE;
      } else if (pheading == 8u && pred != start_state) {
        code = APGAR_B200_PRED_SENTINEL;
      } else if (labels[pred] == kGraphInf) {
        code = APGAR_B200_PRED_INFINITE;
      } else {
        // canonical physical edge: forward directions from the predecessor,
        // the other four from the state's node
        const uint32_t edge = incoming < 4u ? pnode * 8u + incoming : node * 8u + incoming - 4u;
        const uint64_t adj =
            edge_adjustment(p.policy + q.policy_offset, q.policy_count, edge);
        if (adj == kGraphInf) {
          code = APGAR_B200_PRED_BANNED;
        } else {
          // StepCostUnderPolicy (src/routing/candidate_policy.cc:419-438)
          const bool diag = (incoming & 1u) != 0u;
          unsigned __int128 t = diag ? static_cast<unsigned __int128>(p.diag) + q.diagonal_step_surcharge
                                     : static_cast<unsigned __int128>(p.orth) + q.orthogonal_step_surcharge;
          if (pheading != 8u && pheading != incoming) {
            t += static_cast<unsigned __int128>(p.bend) + q.bend_surcharge;
          }
          t += adj;
          uint64_t expected = 0;
          const bool ok = t < static_cast<unsigned __int128>(kGraphInf) &&
                          add_checked(labels[pred], static_cast<uint64_t>(t), &expected);
          if (!ok || (partial ? expected > label : expected != label)) code = APGAR_B200_PRED_COST;
        }
      }
    }
    if (code != 0u) {
      atomicMin(&p.first[qi], ((static_cast<unsigned long long>(state) + 1ull) << 32) | code);
    }
  }
}

}  // namespace

cudaError_t launch_validate_predecessors(const PredCheckLaunch& launch, cudaStream_t stream) {
  const uint64_t total = static_cast<uint64_t>(launch.node_count) * 9u * launch.query_count;
  if (total == 0) return cudaSuccess;
  const uint64_t blocks = (total + 255u) / 256u;
  validate_predecessors_kernel<<<static_cast<unsigned>(blocks < 148u * 64u ? blocks : 148u * 64u), 256,
                                 0, stream>>>(launch);
  return cudaGetLastError();
}

}  // namespace apgar_b200
