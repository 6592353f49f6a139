// Shared definitions for the drop-in (reference device-view) engine.
//
// States are node*9 + incoming heading (planar_router.h:261-272); labels are
// uint64 with UINT64_MAX as the unreachable sentinel and every sum checked
// against it (planar_router.cu:332-340).
#pragma once

#include <cstdint>

#include "apgar_b200.h"

namespace apgar_b200 {

constexpr uint64_t kGraphInf = ~0ull;
constexpr uint32_t kInvalid32 = 0xFFFFFFFFu;

struct GraphDeviceView {
  const uint32_t* neighbors;  // [8][nodes], kInvalid32 where no edge
  const uint8_t* legal;       // [nodes] legal-edge masks
  uint32_t node_count;
  uint32_t orth, diag, bend;
  // association fields repeated into every result header
  uint32_t compiler_version;
  uint64_t source_board_content_hash, compiler_profile_fingerprint, rule_bucket_identity;
  uint64_t device_view_fingerprint;
};

struct GraphLaunch {
  GraphDeviceView g;
  const apgar_b200_batch_query_v1* queries;
  uint32_t query_count;
  const apgar_b200_policy_edge_v1* policy;
  uint64_t* labels;         // [Q][9N]
  uint32_t* queues;         // [Q][2][N] node frontier queues
  uint32_t* stamps;         // [Q][N] enqueue round stamps
  apgar_b200_batch_result_v1* results;   // [Q]
  apgar_b200_compact_path_v1* compact;   // [Q] (compact mode)
  uint32_t* path_stage;     // [Q][9N] reverse paths before packing (compact mode)
  uint32_t* predecessors;   // [Q][9N] (workspace mode)
  uint64_t* state_owners;   // [Q][9N] (workspace mode)
  uint64_t* predecessor_owners;  // [Q][9N] (workspace mode)
  uint32_t maximum_rounds;
  uint8_t generator;
  uint8_t workspace_mode;   // 1: converge fully and emit predecessors; 0: compact path
  const volatile uint32_t* cancel;  // host-mapped flag or nullptr
  uint32_t max_policy_edges;  // the largest policy_count of the batch
  uint32_t policy_smem_offset;  // where a query's edges are staged in shared memory, or ~0u
  uint32_t nbr_smem_offset;     // where the neighbour table is staged in shared memory, or ~0u
};

struct PathCheckLaunch {
  const apgar_b200_node_v1* nodes;
  uint32_t node_count;
  uint32_t orth, diag, bend;
  const apgar_b200_batch_query_v1* queries;
  const apgar_b200_policy_edge_v1* policy;
  const apgar_b200_batch_result_v1* results;
  const apgar_b200_compact_path_v1* compact;
  const uint32_t* states;
  uint64_t state_count;
  uint64_t* visited;  // [query][ceil(9N / 64)] scratch bits
  apgar_b200_path_verdict* out;
  uint32_t query_count;
};

// Full-workspace predecessor validation of a batch (labels and predecessors
// [query][9 * nodes], as read back).
struct PredCheckLaunch {
  const apgar_b200_node_v1* nodes;
  uint32_t node_count;
  uint32_t orth, diag, bend;
  const apgar_b200_batch_query_v1* queries;
  const apgar_b200_policy_edge_v1* policy;
  const uint64_t* labels;
  const uint32_t* predecessors;
  const uint8_t* partial;  // [query] 1 = partial (lower-bound) cost validation, or nullptr
  unsigned long long* first;  // [query] least (state + 1) << 32 | code; ~0 when valid
  uint32_t query_count;
};

// Reachability of each selected query's goal under its policy bans.
struct ReachLaunch {
  const uint32_t* neighbors;  // [8][nodes]
  const uint8_t* legal;       // [nodes]
  uint32_t node_count;
  const apgar_b200_batch_query_v1* queries;
  const apgar_b200_policy_edge_v1* policy;
  const uint32_t* selected;   // [count] query indices
  uint32_t count;
  uint32_t* visited;          // [count][ceil(nodes / 32)] scratch bits
  uint32_t* queues;           // [count][2][nodes] scratch
  uint32_t* reached;          // [count] 1 when the goal was reached
  uint64_t* reach_nodes;      // [count] nodes reached
};

}  // namespace apgar_b200
