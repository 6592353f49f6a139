/*
 * apgar_b200 — C ABI of the B200 search backend.
 *
 * Plain pointers and sizes only.  Every entry point returns an
 * apgar_b200_status; apgar_b200_last_error() returns the detail string of the
 * calling thread's last failure.  Host buffers are ordinary (pageable or
 * pinned) memory; `*_device` entry points take device pointers and a CUDA
 * stream handle passed as void*.
 *
 * Two families of entry points:
 *
 *  A. The drop-in seam for the reference's IPlanarRouteBackend
 *     (include/apgar/gpu/planar_router.h:543-560).  Records are bit-identical
 *     to the reference V1 layouts (DeviceCompiledHeaderV1 :170-188,
 *     DeviceLayerRangeV1 :190-201, DeviceNodeV1 :203-213, DeviceRunV1 :215-223,
 *     DeviceCandidatePolicyEdgeV1 :340-348, DeviceCandidateBatchQueryV1 :352-377,
 *     DeviceCandidateBatchResultV1 :381-407, DeviceCandidateCompactPathV1
 *     :413-423).  Status codes map 1:1 onto BackendErrorCode (:475-480).
 *
 *  B. Lattice mode: dense bit-packed multi-layer lattices with vias, per-net
 *     windows and uint32 costs (no reference counterpart; the reference is
 *     planar-only and whole-board).
 */
#ifndef APGAR_B200_H_
#define APGAR_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define APGAR_B200_API __attribute__((visibility("default")))
#else
#define APGAR_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define APGAR_B200_ABI_VERSION 1u

/* Mirrors BackendErrorCode (planar_router.h:475-480) with 0 = success. */
typedef enum apgar_b200_status {
  APGAR_B200_OK = 0,
  APGAR_B200_UNSUPPORTED = 1,        /* BackendErrorCode::kUnsupported */
  APGAR_B200_RESOURCE_EXHAUSTED = 2, /* BackendErrorCode::kResourceExhausted */
  APGAR_B200_BACKEND_FAILURE = 3,    /* BackendErrorCode::kBackendFailure */
  APGAR_B200_INTERNAL_INVARIANT = 4  /* BackendErrorCode::kInternalInvariant */
} apgar_b200_status;

/* Per-query outcome; values 0..3 equal KernelCompletion (planar_router.h:294-299). */
enum {
  APGAR_B200_COMPLETION_REACHED = 0,
  APGAR_B200_COMPLETION_DISCONNECTED = 1,
  APGAR_B200_COMPLETION_BUDGET_EXHAUSTED = 2,
  APGAR_B200_COMPLETION_CANCELLED = 3,
  /* lattice mode only: the net was not admitted (cost domain, width or path
   * arena bound) and carries no result */
  APGAR_B200_COMPLETION_REJECTED = 4
};

#define APGAR_B200_UNREACHABLE 0xFFFFFFFFu

APGAR_B200_API uint32_t apgar_b200_abi_version(void);

/* Copies the calling thread's last error detail (NUL-terminated, truncated to
 * capacity) and returns its full length. */
APGAR_B200_API size_t apgar_b200_last_error(char* buffer, size_t capacity);

/* Replaces BackendMetadata discovery (planar_router.h:281-292,
 * gpu/cuda/planar_router.cu:2006-2046) for the current CUDA device. */
typedef struct apgar_b200_metadata {
  char device_name[256];
  char device_uuid[40];
  uint32_t compute_capability_major;
  uint32_t compute_capability_minor;
  uint32_t runtime_version;
  uint32_t driver_version;
  uint64_t global_memory_bytes;
  uint32_t multiprocessor_count;
  uint32_t reserved;
} apgar_b200_metadata;

APGAR_B200_API int apgar_b200_query_metadata(apgar_b200_metadata* out);

/* =================== A. drop-in seam (reference V1 records) =================== */

/* Generator values of PlanarGenerator (planar_router.h:42-45) plus the two
 * values this backend adds for its own persistent engine (the reference's
 * extension mechanism: a new enumerator with its own descriptor,
 * schemas/device_candidate_batch/v1.md:21-25).
 *
 * The persistent generators search a whole batch on the device with no
 * host-chunked rounds.  B200_PERSISTENT returns compact paths (3 launches:
 * search, path-offset scan, packing); B200_PERSISTENT_WORKSPACE returns the
 * full workspace (1 launch).  Their descriptor (the reference's
 * DescribePlanarGenerator, planar_router.h:56-100): workspace kSweep or
 * kFrontier by readback form, chunk_rounds = 1, 8 examined work per round and
 * per node, 8 turn relaxations per examined work, no per-round kernels,
 * fixed_launches = 2 or 0, and host_chunked = false, a flag the descriptor
 * gains with these values.  The batch reports 0 blocking status readbacks,
 * its last launch as the finalization launch, dispatched_rounds = the most
 * rounds any query ran, and device bytes
 * Q*(120 + 120 + 32) + E*16 + Q*S*8 + Q*N*12 + Q*S*4 (+ Q*S*16 for the full
 * workspace) + 16, for Q queries, E policy edges, N nodes and S = 9N states.
 * apgar_b200/adapter/reference_generator.patch is that change to the
 * reference's host code.  The two stock generators keep their descriptors;
 * this engine serves them with the same launches and reports its own
 * counts, which their host-chunked descriptors do not describe. */
enum {
  APGAR_B200_GENERATOR_BUCKETED_FRONTIER = 0,          /* PlanarGenerator::kBucketedFrontier */
  APGAR_B200_GENERATOR_HEADING_SWEEP = 1,              /* PlanarGenerator::kHeadingAwareSweep */
  APGAR_B200_GENERATOR_B200_PERSISTENT = 2,            /* added: compact paths */
  APGAR_B200_GENERATOR_B200_PERSISTENT_WORKSPACE = 3   /* added: full workspace */
};

/* DeviceCompiledHeaderV1 (planar_router.h:170-188), 112 bytes. */
typedef struct apgar_b200_compiled_header_v1 {
  uint32_t schema_version;
  uint32_t compiler_version;
  uint64_t source_board_content_hash;
  uint64_t compiler_profile_fingerprint;
  uint64_t rule_bucket_identity;
  uint64_t device_view_fingerprint;
  uint64_t represented_nodes;
  uint64_t represented_states;
  uint64_t estimated_persistent_device_bytes;
  int64_t lattice_origin_x, lattice_origin_y;
  int64_t lattice_step;
  uint32_t orthogonal_step, diagonal_step, bend; /* DeterministicCosts */
  uint8_t heading_mask;
  uint8_t reserved[7];
  uint8_t padding[4];
} apgar_b200_compiled_header_v1;

/* DeviceLayerRangeV1 (planar_router.h:190-201), 48 bytes. */
typedef struct apgar_b200_layer_range_v1 {
  uint32_t layer, node_offset, node_count, padding;
  int64_t minimum_lattice_x, maximum_lattice_x, minimum_lattice_y, maximum_lattice_y;
} apgar_b200_layer_range_v1;

/* DeviceNodeV1 (planar_router.h:203-213), 56 bytes. */
typedef struct apgar_b200_node_v1 {
  int64_t lattice_x, lattice_y;
  uint32_t layer;
  uint8_t legal_edges;
  uint8_t reserved[3];
  uint32_t neighbors[8];
} apgar_b200_node_v1;

/* DeviceRunV1 (planar_router.h:215-223), 12 bytes. */
typedef struct apgar_b200_run_v1 {
  uint32_t node_offset, node_count;
  uint8_t direction;
  uint8_t reserved[3];
} apgar_b200_run_v1;

/* DeviceCandidatePolicyEdgeV1 (planar_router.h:340-348), 16 bytes. */
typedef struct apgar_b200_policy_edge_v1 {
  uint32_t physical_edge_index;
  uint32_t reserved;
  uint64_t adjustment; /* UINT64_MAX = banned */
} apgar_b200_policy_edge_v1;

/* DeviceCandidateBatchQueryV1 (planar_router.h:352-377), 120 bytes. */
typedef struct apgar_b200_batch_query_v1 {
  uint32_t schema_version, input_ordinal;
  uint64_t batch_id, query_id, workspace_owner, policy_identity, routing_profile_fingerprint;
  uint32_t start_node, goal_node, policy_offset, policy_count;
  uint64_t workspace_offset, workspace_state_count, frontier_state_capacity;
  uint64_t orthogonal_step_surcharge, diagonal_step_surcharge, bend_surcharge;
  uint32_t maximum_rounds;
  uint8_t generator;
  uint8_t reserved[3];
} apgar_b200_batch_query_v1;

/* DeviceCandidateBatchResultV1 (planar_router.h:381-407), 120 bytes. */
typedef struct apgar_b200_batch_result_v1 {
  uint32_t schema_version, compiler_version, input_ordinal, start_node, goal_node, goal_state, rounds;
  uint8_t generator, completion; /* completion: APGAR_B200_COMPLETION_* (0..3) */
  uint8_t reserved[2];
  uint64_t batch_id, query_id, workspace_owner, policy_identity, routing_profile_fingerprint;
  uint64_t source_board_content_hash, compiler_profile_fingerprint, rule_bucket_identity;
  uint64_t device_view_fingerprint, examined_work, heading_turn_relaxations;
} apgar_b200_batch_result_v1;

/* DeviceCandidateCompactPathV1 (planar_router.h:413-423), 32 bytes. */
typedef struct apgar_b200_compact_path_v1 {
  uint32_t schema_version, state_count;
  uint64_t query_id, workspace_owner, state_offset;
} apgar_b200_compact_path_v1;

/* DeviceRouteResultHeaderV1 (planar_router.h:225-241), 64 bytes. */
typedef struct apgar_b200_route_result_header_v1 {
  uint32_t schema_version, compiler_version, start_node, goal_node;
  uint64_t source_board_content_hash, compiler_profile_fingerprint, routing_profile_fingerprint;
  uint64_t rule_bucket_identity, device_view_fingerprint;
  uint8_t generator;
  uint8_t reserved[7];
} apgar_b200_route_result_header_v1;

/* The non-vector fields of BackendCandidateBatchExecutionRequest
 * (planar_router.h:425-437). */
typedef struct apgar_b200_batch_request {
  uint32_t schema_version;
  uint8_t generator;
  uint8_t reserved[3];
  uint64_t batch_id;
  uint32_t maximum_rounds;
  uint32_t padding;
  uint64_t maximum_workspace_states_per_query;
  uint64_t maximum_frontier_states_per_query;
  uint64_t maximum_device_bytes;
  uint64_t maximum_host_bytes;
} apgar_b200_batch_request;

/* CandidateBatchTelemetry (planar_router.h:127-147) as produced by this
 * backend: launches and readbacks are this engine's own counts. */
typedef struct apgar_b200_batch_telemetry {
  uint64_t persistent_device_bytes;
  uint64_t batch_device_bytes;
  uint64_t workspace_capacity_device_bytes;
  uint64_t peak_device_bytes;
  uint64_t device_to_host_readback_bytes;
  uint64_t kernel_launch_count;
  uint64_t blocking_status_readback_count;
  uint32_t dispatched_rounds;
  uint32_t finalization_launch_count;
  double kernel_milliseconds;
} apgar_b200_batch_telemetry;

/* UploadCompiledView (planar_router.h:548; gpu/cuda/planar_router.cu:1951-2003):
 * validates the flattened view (the checks of planar_router.cu:1256-1451 that
 * guard device memory safety and the cost bound) and uploads it to the
 * current device. */
APGAR_B200_API int apgar_b200_view_upload(const apgar_b200_compiled_header_v1* header,
                                          const apgar_b200_layer_range_v1* layers,
                                          uint64_t layer_count,
                                          const apgar_b200_node_v1* nodes, uint64_t node_count,
                                          const apgar_b200_run_v1* runs, uint64_t run_count,
                                          const uint32_t* run_nodes, uint64_t run_node_count,
                                          void** out_view);
APGAR_B200_API int apgar_b200_view_release(void* view);

/* ExecuteCandidateBatch (planar_router.h:556-557; planar_router.cu:2183-2625):
 * validates the batch (ordering, ownership, workspace and policy bounds, the
 * cost-sentinel bound of planar_router.cu:1731-1909), then searches every
 * query on the device.  `cancel` (optional, host memory) is sampled on the
 * host while the batch runs. */
APGAR_B200_API int apgar_b200_execute_batch(void* view, const apgar_b200_batch_request* request,
                                            const apgar_b200_batch_query_v1* queries,
                                            uint32_t query_count,
                                            const apgar_b200_policy_edge_v1* policy_edges,
                                            uint64_t policy_edge_count,
                                            const volatile uint8_t* cancel, void** out_pending);

/* ReadbackCandidateBatch (planar_router.h:558-559; planar_router.cu:2627-2792),
 * compact form: result headers, compact path headers and the packed reverse
 * state paths (state = node*9 + incoming heading, goal first). */
APGAR_B200_API int apgar_b200_readback_batch(void* pending, apgar_b200_batch_result_v1* results,
                                             apgar_b200_compact_path_v1* compact_paths,
                                             uint32_t* path_states, uint64_t path_capacity,
                                             uint64_t* path_state_count,
                                             apgar_b200_batch_telemetry* telemetry);

/* Full-workspace form (the frontier generator's readback): query-major labels
 * (uint64, UINT64_MAX unreachable), canonical predecessors (UINT32_MAX none)
 * and the owner stamps of every state.  Arrays hold query_count * 9 * nodes. */
APGAR_B200_API int apgar_b200_readback_batch_workspace(void* pending, uint64_t* labels,
                                                       uint32_t* predecessors,
                                                       uint64_t* state_owners,
                                                       uint64_t* predecessor_owners);
APGAR_B200_API int apgar_b200_release_batch(void* pending);

/* ExecuteRoute / ReadbackRoute (planar_router.h:549-551; planar_router.cu:2049-2181,
 * :2794-2853): one query without a policy; readback returns the result header,
 * completion, goal state and the full label / predecessor arrays (9 * nodes). */
APGAR_B200_API int apgar_b200_execute_route(void* view, uint8_t generator, uint32_t start_node,
                                            uint32_t goal_node,
                                            uint64_t routing_profile_fingerprint,
                                            uint32_t maximum_rounds,
                                            uint64_t maximum_device_bytes,
                                            const volatile uint8_t* cancel, void** out_pending);
APGAR_B200_API int apgar_b200_readback_route(void* pending,
                                             apgar_b200_route_result_header_v1* header,
                                             uint8_t* completion, uint32_t* goal_state,
                                             uint64_t* labels, uint32_t* predecessors,
                                             apgar_b200_batch_telemetry* telemetry);
APGAR_B200_API int apgar_b200_release_route(void* pending);

/* Structural validation of untrusted compact paths on the device: the
 * compact path envelope of the readback (schema version, query id, workspace
 * owner, slice bounds, non-empty exactly when reached;
 * src/gpu/planar_router.cc:1789-1805), then the device-view checks of
 * ValidateAndReconstructCompactGpuPath (src/gpu/planar_router.cc:969-1067),
 * in the reference's order, for every query of a batch at once.  The exact-geometry stage that follows them in
 * the reference (src/gpu/planar_router.cc:1069-1111) stays with the host.
 * Codes name the reference's invariant ids. */
enum {
  APGAR_B200_PATH_OK = 0,
  APGAR_B200_PATH_BOUNDS = 1,    /* gpu.batch.compact_path.bounds.v1 */
  APGAR_B200_PATH_ENDPOINT = 2,  /* gpu.batch.compact_path.endpoint.v1 */
  APGAR_B200_PATH_CYCLE = 3,     /* gpu.batch.compact_path.cycle.v1 */
  APGAR_B200_PATH_HEADING = 4,   /* gpu.batch.compact_path.heading.v1 */
  APGAR_B200_PATH_EDGE = 5,      /* gpu.batch.compact_path.edge.v1 */
  APGAR_B200_PATH_BANNED = 6,    /* gpu.policy.banned_predecessor.v1 */
  APGAR_B200_PATH_NOT_REACHED = 7, /* the query did not reach its goal: not validated */
  APGAR_B200_PATH_COST = 8         /* lattice mode: the move costs do not sum to the reported cost */
};
typedef struct apgar_b200_path_verdict {
  uint32_t code;          /* APGAR_B200_PATH_* */
  uint32_t reserved;
  uint64_t failing_index; /* forward index (from the start) of the first failing state */
  uint64_t total_cost;    /* the path's cost under the query's policy when code == OK */
} apgar_b200_path_verdict;

/* Validates the compact paths of a batch (host arrays, as read back) against
 * an uploaded view and the batch's own queries and policy edges; writes one
 * verdict per query. */
APGAR_B200_API int apgar_b200_validate_compact_paths(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count,
    const apgar_b200_batch_result_v1* results, const apgar_b200_compact_path_v1* compact_paths,
    const uint32_t* path_states, uint64_t path_state_count, apgar_b200_path_verdict* verdicts);

/* Validation of untrusted full-workspace results on the device: the checks of
 * ValidateAllPredecessors (src/gpu/planar_router.cc:492-611) over every
 * heading state of every query, in the reference's order, reporting each
 * query's first failure (state index in failing_index).  `labels` [query][9N]
 * uint64 and `predecessors` [query][9N] uint32 are host arrays as read back
 * (apgar_b200_readback_batch_workspace, or one query of
 * apgar_b200_readback_route); `partial` [query] selects the lower-bound cost
 * check of bounded results (1) instead of the exact one (0), or is NULL (all
 * exact).  Codes: */
enum {
  APGAR_B200_PRED_OK = 0,
  APGAR_B200_PRED_START = 1,          /* start state not labelled 0 without predecessor */
  APGAR_B200_PRED_NO_HEADING = 2,     /* a heading-8 state away from the start is reachable */
  APGAR_B200_PRED_UNREACHABLE = 3,    /* an unreachable state carries a predecessor */
  APGAR_B200_PRED_BOUNDS = 4,         /* predecessor index out of bounds */
  APGAR_B200_PRED_SELF_REFERENCE = 5, /* gpu.predecessor.self_reference.v1 */
  APGAR_B200_PRED_EDGE = 6,           /* not one adjacent compiled legal edge */
  APGAR_B200_PRED_SENTINEL = 7,       /* predecessor uses heading 8 away from the start */
  APGAR_B200_PRED_INFINITE = 8,       /* reachable state after an unreachable predecessor */
  APGAR_B200_PRED_BANNED = 9,         /* gpu.policy.banned_predecessor.v1 */
  APGAR_B200_PRED_COST = 10           /* label does not reconstruct the scalar cost */
};
APGAR_B200_API int apgar_b200_validate_predecessors(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count, const uint8_t* partial,
    const uint64_t* labels, const uint32_t* predecessors, apgar_b200_path_verdict* verdicts);

/* Confirmation of DISCONNECTED results on the device, in place of the CPU A*
 * rerun of ConfirmDisconnectedWithCpuOracle (src/gpu/planar_router.cc:629-667).
 * The CPU A* (src/routing/cpu_astar.cc:323-512) reports kDisconnected exactly
 * when its queue empties without the goal: every state reachable from the
 * start through compiled legal edges whose resource the query's policy does
 * not ban has been expanded.  A per-query breadth-first search over the same
 * edges decides that reachability.  The CPU search can instead fail with
 * kResourceExhausted when a reachable state's cost plus a transition leaves
 * the finite range; that cannot happen when (8 * reachable nodes + 1) times
 * the query's largest finite transition stays below UINT64_MAX, and a query
 * past that bound gets the code UNBOUNDED (confirm it on the CPU). */
enum {
  APGAR_B200_DISCONNECT_CONFIRMED = 0,   /* no path under the query's bans */
  APGAR_B200_DISCONNECT_REACHABLE = 1,   /* gpu.disconnected.cpu_reachable.v1 */
  APGAR_B200_DISCONNECT_UNBOUNDED = 2,   /* unreachable, but the cost bound cannot rule out
                                            the CPU search's overflow failure */
  APGAR_B200_DISCONNECT_NOT_CLAIMED = 3  /* the result is not DISCONNECTED: not checked */
};
typedef struct apgar_b200_disconnect_verdict {
  uint32_t code;             /* APGAR_B200_DISCONNECT_* */
  uint32_t reserved;
  uint64_t reachable_nodes;  /* nodes reached from the start (a REACHABLE search stops at the goal) */
} apgar_b200_disconnect_verdict;

/* Confirms every DISCONNECTED result of a batch (host arrays, as read back)
 * against an uploaded view and the batch's own queries and policy edges
 * (each query's slice sorted by physical_edge_index); writes one verdict per
 * query. */
APGAR_B200_API int apgar_b200_confirm_disconnected(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count,
    const apgar_b200_batch_result_v1* results, apgar_b200_disconnect_verdict* verdicts);

/* ======================= B. lattice mode ======================= */

typedef struct apgar_b200_lattice_desc {
  int32_t layers;          /* 1..8 */
  int32_t height, width;   /* width is a multiple of 32 */
  const uint32_t* blocked; /* host: [layers][height][width/32], bit x%32 of word x/32 */
  const uint32_t* via_ok;  /* host: [layers-1][height][width/32] or NULL (all vias allowed) */
  uint32_t orth, diag, via;
} apgar_b200_lattice_desc;

typedef struct apgar_b200_lattice_net {
  uint32_t start_layer, start_x, start_y;
  uint32_t goal_layer, goal_x, goal_y;
  uint32_t win_x0, win_y0, win_w, win_h; /* window in lattice cells, all layers */
} apgar_b200_lattice_net;

typedef struct apgar_b200_lattice_result {
  uint32_t cost;         /* APGAR_B200_UNREACHABLE unless reached */
  uint32_t completion;   /* APGAR_B200_COMPLETION_* */
  uint32_t sweeps;       /* row sweeps executed (including the final quiet one) */
  uint32_t path_len;     /* cells in the reverse path (goal first) */
  uint64_t path_offset;  /* into the packed path array */
  uint64_t arena_offset; /* internal staging offset; zero once results are packed */
  uint32_t row_steps;    /* window rows processed (all layers of a row = 1) */
  uint32_t row_stores;   /* layer rows written back */
  uint32_t row_loads;    /* layer rows read (current and re-read predecessor rows) */
  uint32_t reserved;
} apgar_b200_lattice_result;

/* Validates lattice route results on the device, the lattice counterpart of
 * the structural checks of ValidateAndReconstructCompactGpuPath
 * (src/gpu/planar_router.cc:969-1067).  `results` and `paths` are untrusted
 * host arrays as read back from a lattice route or plan (packed reverse paths
 * of global cell ids, goal first); `nets` are the nets they answer.  Per
 * reached net: path bounds (BOUNDS), the start and goal endpoints (ENDPOINT),
 * every cell inside the lattice and the net's window (BOUNDS), every step one
 * legal move re-derived from the blocked and via masks (EDGE), and the move
 * costs summing to the reported cost (COST; unpriced costs).  One verdict per
 * net: failing_index counts cells from the start; total_cost is the sum.
 * Unreached nets get NOT_REACHED. */
APGAR_B200_API int apgar_b200_lattice_validate(void* lattice, const apgar_b200_lattice_net* nets,
                                               uint32_t count,
                                               const apgar_b200_lattice_result* results,
                                               const uint32_t* paths, uint64_t path_count,
                                               apgar_b200_path_verdict* verdicts);

/* Uploads the lattice masks to the current device (the prepared view). */
APGAR_B200_API int apgar_b200_lattice_upload(const apgar_b200_lattice_desc* desc, void** out_lattice);
APGAR_B200_API int apgar_b200_lattice_release(void* lattice);

/* End-to-end batch on host buffers: copies the nets in, searches every net in
 * its window, and copies results and packed reverse paths (global cell ids
 * (layer*height + y)*width + x, goal first) out.  `paths` may be NULL to skip
 * the path copy; *path_total receives the number of path cells.  `cancel`
 * (optional) is polled between sweeps; non-zero cancels unfinished nets. */
APGAR_B200_API int apgar_b200_lattice_route(void* lattice, const apgar_b200_lattice_net* nets, uint32_t count,
                             uint32_t max_sweeps, const volatile uint32_t* cancel,
                             apgar_b200_lattice_result* results, uint32_t* paths,
                             uint64_t path_capacity, uint64_t* path_total);

/* Allocation-free form of apgar_b200_lattice_route.  No counterpart in the
 * reference: it is an addition for callers that must not allocate device
 * memory while they route, such as a process whose device memory is already
 * held by another allocator (a caching allocator or a fixed serving budget,
 * where cudaMalloc fails), or a router sharing the GPU with work on other
 * streams that cannot take the device-wide synchronisation cudaMalloc and
 * cudaFree imply.
 *
 * Same admission, search, results and packed paths as
 * apgar_b200_lattice_route, with these differences:
 *  - Its label slabs, plan records, result records and path arena live in one
 *    fixed device array of APGAR_B200_NOALLOC_SCRATCH_BYTES per device.  It
 *    calls no cudaMalloc or cudaFree and creates no stream, event or pinned
 *    buffer.  The host-side plan is staged in fixed arrays.
 *  - A batch that needs more than the scratch holds, or has more than
 *    APGAR_B200_NOALLOC_MAX_NETS nets, fails with
 *    APGAR_B200_RESOURCE_EXHAUSTED and a message giving the bytes it needed.
 *  - Its copies and launches go to `stream` (NULL: the legacy default
 *    stream).  Width classes run one after another on that stream.  The call
 *    synchronises only that stream before it returns.
 *  - It takes no cancel flag.
 *  - Every call looks up the array's device address (cudaGetSymbolAddress,
 *    which allocates nothing) with the lattice's device current.  The first
 *    call on a device also loads the module there, so it should come before
 *    any stream capture on that device.  Do not call it across a device
 *    reset of the lattice's device.
 *  - The array is part of the library's device image: every process that
 *    loads the library holds APGAR_B200_NOALLOC_SCRATCH_BYTES on each device
 *    where it uses the library, until exit, whether or not it calls this
 *    entry point.
 *  - The scratch is shared by every call on a device and the host staging by
 *    every call of the process.  Calls therefore take one process-wide lock
 *    from admission to the final stream synchronisation, so calls from
 *    several host threads, on one device or several, run one after another.
 *    Overlapping calls would race on the scratch and the staging; a plan
 *    uploaded beside another call's nets could make the sweep write outside
 *    its slabs and fault the GPU, not just corrupt results.  The scratch
 *    keeps the last call's contents; each call clears what must start at
 *    zero. */
#define APGAR_B200_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
#define APGAR_B200_NOALLOC_MAX_NETS 4096u
APGAR_B200_API int apgar_b200_lattice_route_noalloc(void* lattice, const apgar_b200_lattice_net* nets,
                                     uint32_t count, uint32_t max_sweeps, void* stream,
                                     apgar_b200_lattice_result* results, uint32_t* paths,
                                     uint64_t path_capacity, uint64_t* path_total);

/* Resident form for repeated launches: plan once (host planning, workspace
 * allocation, nets copied to the device), then execute on a stream (launches
 * only; capturable in a CUDA graph), then read back. */
APGAR_B200_API int apgar_b200_lattice_plan(void* lattice, const apgar_b200_lattice_net* nets, uint32_t count,
                            uint32_t max_sweeps, void** out_plan);
APGAR_B200_API int apgar_b200_lattice_execute(void* plan, void* stream);
APGAR_B200_API int apgar_b200_lattice_readback(void* plan, apgar_b200_lattice_result* results, uint32_t* paths,
                                uint64_t path_capacity, uint64_t* path_total);
/* Device pointers of the plan's result records and packed paths. */
APGAR_B200_API int apgar_b200_lattice_device_results(void* plan, const apgar_b200_lattice_result** results,
                                      const uint32_t** paths);
typedef struct apgar_b200_plan_info {
  uint32_t net_count;
  uint32_t kernel_launches;     /* launches per execute */
  uint32_t class_count;         /* width classes launched */
  uint32_t reserved;
  uint64_t workspace_bytes;     /* label slabs + arena + records */
  uint64_t label_cells;         /* sum of layers*rows*pitch over nets */
  uint64_t path_arena_capacity; /* cells */
} apgar_b200_plan_info;
APGAR_B200_API int apgar_b200_lattice_plan_info(void* plan, apgar_b200_plan_info* out);

/* Search generators of lattice mode, the counterpart of the reference's
 * PlanarGenerator choice (include/apgar/gpu/planar_router.h:56-100).  Both
 * give the same costs and the same canonical reverse paths.
 *  SWEEP:    alternating row sweeps to the full-window fixed point.  Result
 *            counters: sweeps, row_steps, row_stores, row_loads.
 *  FRONTIER: bucketed, label-correcting A* (key = label + octile-plus-via
 *            bound) in key levels of `bucket_width`.  One warp group per net,
 *            persistent and work-stealing, largest windows first.  It stops
 *            once every cell with key <= the goal label is final.  Result
 *            counters: sweeps = rounds, row_steps = cell expansions,
 *            row_stores = key levels opened, row_loads = 0.  Rounds and
 *            expansions depend on the order of concurrent relaxations;
 *            costs and paths do not. */
#define APGAR_B200_LATTICE_SWEEP 0u
#define APGAR_B200_LATTICE_FRONTIER 1u
typedef struct apgar_b200_lattice_options {
  uint32_t generator;      /* APGAR_B200_LATTICE_* */
  uint32_t max_iterations; /* sweeps (SWEEP, 1..30000) or rounds (FRONTIER, 1..2^30) */
  uint32_t bucket_width;   /* FRONTIER: key width of a level; raised to at least twice
                              the largest move cost (0 = that minimum) */
  uint32_t chain;          /* FRONTIER: 0 = the default per width class; n >= 1 = every
                              queued cell is followed within its round by up to n - 1
                              chained expansions of the least-key cell it queued
                              (1 = none); at most 16.  Results do not depend on it. */
  uint32_t class_bounds;   /* FRONTIER: width classes of 1, 2, 4, 8 and 16 warps per net;
                              byte k (k = 0..3) is log2 of the largest window (cells over
                              all layers) of the 2^k-warp class, strictly increasing in
                              1..31; larger windows take 16 warps.  0 = the default
                              0x13110F0C (2^12, 2^15, 2^17, 2^19).  Results do not
                              depend on it. */
  uint32_t wide_bucket_width; /* FRONTIER: key width of the 16-warp class's levels (its
                                 nets are the batch's longest searches, so its schedule
                                 is tuned apart); 0 = bucket_width; raised like it */
  uint32_t wide_chain;        /* FRONTIER: chain of the 16-warp class, meaning as chain;
                                 0 = chain.  Results depend on neither. */
} apgar_b200_lattice_options;

/* Per-cell entry prices for a FRONTIER plan (no reference counterpart at this
 * level: it carries the negotiated-congestion snapshot cost of
 * src/allocator/cpu_sequential_negotiated_routing.cc:299-505 per lattice cell).
 * `cell_costs` is a device array [layers][height][width] of uint32, read by
 * every later execute until replaced; NULL removes it.  A move into cell c
 * then costs its move cost plus cell_costs[c].  A net whose path costs reach
 * 2^31 - 1 comes back REJECTED instead of with a wrong cost. */
APGAR_B200_API int apgar_b200_lattice_plan_set_cell_costs(void* plan, const uint32_t* cell_costs);

/* Corridor mode of a FRONTIER plan (no reference counterpart: the learned
 * corridor with its exact certificate).  `corridor_bits` is device memory,
 * 128 uint32 words per net of the plan: a 64 x 64 bitmap of coarse cells over
 * the net's window, bit cx of word 2 * cy + cx / 32 for coarse cell (cx, cy).
 * A coarse cell covers 2^s x 2^s window cells on every layer, where s is the
 * least value >= 2 with ceil(max(win_w, win_h) / 2^s) <= 63.  Each net first
 * searches its corridor only.  The result is kept when its cost is strictly
 * below the least key (label + move + admissible bound) over every legal
 * move leaving the corridor that the search expanded, which proves it equal
 * to the full-window result, path included.  Otherwise the net is searched
 * again over the whole window, so results never depend on the corridor.
 * NULL detaches the corridors.  Not combined with per-cell prices. */
enum {
  APGAR_B200_CORRIDOR_NONE = 0,               /* no corridors, or the net's bitmap is empty */
  APGAR_B200_CORRIDOR_CERTIFIED = 1,          /* the corridor result, certified */
  APGAR_B200_CORRIDOR_FALLBACK_EXIT = 2,      /* reached, but an exit key was <= its cost */
  APGAR_B200_CORRIDOR_FALLBACK_UNREACHED = 3  /* a terminal outside, or goal not reached */
};
APGAR_B200_API int apgar_b200_lattice_plan_set_corridors(void* plan, const uint32_t* corridor_bits);
/* Waits for the device and copies the per-net APGAR_B200_CORRIDOR_* outcomes
 * of the last corridor-mode execution (one byte per net) to host memory. */
APGAR_B200_API int apgar_b200_lattice_plan_corridor_status(void* plan, uint8_t* out);

/* apgar_b200_lattice_plan / apgar_b200_lattice_route with a generator choice. */
APGAR_B200_API int apgar_b200_lattice_plan_ex(void* lattice, const apgar_b200_lattice_net* nets,
                               uint32_t count, const apgar_b200_lattice_options* options,
                               void** out_plan);
APGAR_B200_API int apgar_b200_lattice_route_ex(void* lattice, const apgar_b200_lattice_net* nets,
                                uint32_t count, const apgar_b200_lattice_options* options,
                                const volatile uint32_t* cancel,
                                apgar_b200_lattice_result* results, uint32_t* paths,
                                uint64_t path_capacity, uint64_t* path_total);
APGAR_B200_API int apgar_b200_lattice_plan_release(void* plan);

/* =================== F. route reconstruction =================== */

/* One segment of a reconstructed route, in exact board coordinates (origin +
 * lattice index * step, LatticeIndexToExactPoint,
 * src/geometry_compiler/compiled_board.cc:219-238).  layer0 == layer1 for a
 * planar run (routing::LayerSegment, include/apgar/routing/planar_route.h:32);
 * a run of vias has layer0 != layer1 and equal end points.  40 bytes. */
typedef struct apgar_b200_segment {
  uint32_t layer0, layer1;
  int64_t x0, y0, x1, y1;
} apgar_b200_segment;
/* segment count of a path that failed reconstruction (a state outside the
 * view, or a point outside the exact coordinate envelope |v| <= 10^12) */
#define APGAR_B200_SEGMENT_FAILURE 0xFFFFFFFFu

/* Coalesces V1 compact paths (reverse states, goal first) into segments on
 * the GPU: a segment starts at the start point and wherever the step between
 * consecutive points changes (routing::CoalesceSegments,
 * src/routing/planar_route.cc:188-215, applied by the reference to every
 * host-validated GPU path, src/gpu/planar_router.cc:1085-1105).  Host
 * buffers: path i's segments are written at segments + paths[i].state_offset
 * (segment_capacity >= path_state_count), its count at segment_counts[i]. */
APGAR_B200_API int apgar_b200_path_segments(void* view, const apgar_b200_compact_path_v1* paths,
                             uint32_t path_count, const uint32_t* path_states,
                             uint64_t path_state_count, apgar_b200_segment* segments,
                             uint64_t segment_capacity, uint32_t* segment_counts);
/* The same for the packed paths of a lattice plan's last execution, on
 * device memory and `stream`: net i's segments at segments +
 * results[i].path_offset (capacity: the plan's packed path cells), its count
 * at segment_counts[i] (0 when not reached).  Lattice index (x, y) maps to
 * (origin_x + x * step, origin_y + y * step); a via run splits segments. */
APGAR_B200_API int apgar_b200_lattice_segments(void* plan, int64_t origin_x, int64_t origin_y, int64_t step,
                                apgar_b200_segment* segments, uint32_t* segment_counts,
                                void* stream);

/* =================== G. geometry compile (edge legality) =================== */

/* An obstacle box in board units (board_ir::Obstacle, its layer and whether
 * the routed net owns it; owned boxes never block).  40 bytes. */
typedef struct apgar_b200_obstacle_box {
  int64_t min_x, min_y, max_x, max_y;
  uint32_t layer, owned_by_net;
} apgar_b200_obstacle_box;

/* The compile rules of edge legality: the routing profile's trace width and
 * clearance, the compiler's lattice placement and heading mask (bit 0
 * horizontal, 1 vertical, 2 diagonal 45; board_ir::Heading).  48 bytes. */
typedef struct apgar_b200_edge_rules {
  int64_t nominal_width, clearance;
  int64_t lattice_origin_x, lattice_origin_y, lattice_step;
  uint32_t heading_mask, reserved;
} apgar_b200_edge_rules;

/* Exact swept-trace clearance of one-step centrelines against boxes, on the
 * GPU (geometry::SweptTraceClearanceAtLeast, src/geometry/exact.cc:325-360):
 * cases are 10 int64 each (start x, y, end x, y, box min x, y, max x, y,
 * width, clearance); out receives (error, satisfied) per case, error 0 ok,
 * 1 coordinate out of range, 2 box not normalized, 3 width or clearance out
 * of range (geometry::ExactGeometryErrorCode order).  Host buffers. */
APGAR_B200_API int apgar_b200_swept_clearance(const int64_t* cases, uint64_t count, uint32_t* out);

/* The legal-edge masks of the geometry compile for the given lattice nodes
 * (CompileBoard's edge loop, src/geometry_compiler/compiled_board.cc:427-476):
 * bit d (geometry_compiler::Direction order E, NE, N, NW, W, SW, S, SE) is set
 * when the neighbour in direction d is one of the given nodes on the same
 * layer, the heading is in rules->heading_mask, and the move clears every
 * obstacle on the layer not owned by the net.  lattice_xy holds (x, y) per
 * node.  Host buffers; the exact tests run on the GPU over per-layer
 * obstacle bins. */
APGAR_B200_API int apgar_b200_compile_legal_edges(const apgar_b200_edge_rules* rules,
                                   const apgar_b200_obstacle_box* obstacles,
                                   uint64_t obstacle_count, const int64_t* lattice_xy,
                                   const uint32_t* layers, uint32_t node_count,
                                   uint8_t* legal_edges);

/* ===================== E. learned corridor (CNN) =====================
 * No reference counterpart.  A 6-layer 3x3 CNN (layers 1-5: 16 -> 32 -> ... ->
 * 32 channels, bias, ReLU, bf16 weights and activations, f32 accumulation on
 * the tensor cores; layer 6: 32 -> 1 logit, f32) over each net's 64 x 64
 * coarse raster (the corridor bitmap's grid).  Raster channels: 0 blocked
 * fraction over all layers, 1 fraction blocked on every layer, 2 congestion
 * (mean entry price / 1024, capped at 8; 0 without prices), 3 start, 4 goal,
 * 5 inside the window, 6-9 coarse offsets to start and goal / 32, 10 distance
 * to the start-goal segment / 8 (capped at 4), 11-15 zero.
 * Tensors are device memory: rasters bf16 [count][66][64][16]; activations
 * bf16 [count][66][64][32] (grid row y stored at row y + 1).  The producers
 * write the rows that in-window outputs read, with the cells outside each
 * net's window as zeros: the pad row above the grid and grid rows 0 .. ch
 * (coarse height ch; row ch is all zeros).  Rows below are left as they are:
 * they reach only cells outside the window, whose outputs are written as
 * zeros, and the gradients read inputs inside the window only.  So are the
 * convolutions' columns 32 .. 63 of a window at most 31 coarse columns wide,
 * whose tiles cover columns 0 .. 31 only (the rasters write all 64);
 * logits and dlogit f32 [count][64][64]; labels u8
 * [count][64][64]; dims u32 [count] (coarse width | height << 8 | scale << 16).
 * params f32 [apgar_b200_cnn_param_count()]: per layer l w[32][9][cin_l] then
 * b[32], then the head w6[9][32] and b6 (tap = (dy + 1) * 3 + dx + 1);
 * operands bf16 [apgar_b200_cnn_operand_count()] (apgar_b200_cnn_prepare). */
enum { APGAR_B200_CNN_TIMEOUT = 1u }; /* a tensor-core completion wait ran out */
APGAR_B200_API uint32_t apgar_b200_cnn_param_count(void);
APGAR_B200_API uint32_t apgar_b200_cnn_operand_count(void);
/* Coarse rasters and dims of every net of a FRONTIER plan; `cell_costs` is
 * the plan's optional price array (device, [layers][height][width]) or NULL. */
APGAR_B200_API int apgar_b200_corridor_rasters(void* plan, const uint32_t* cell_costs, void* rasters,
                                uint32_t* dims, void* stream);
/* Coarse labels (1 where the net's path of the plan's last execution has a
 * cell) for training. */
APGAR_B200_API int apgar_b200_corridor_labels(void* plan, const uint32_t* dims, uint8_t* labels,
                               void* stream);
/* The plan's corridor bitmaps (128 words per net) from logits: coarse cells
 * with logit > threshold, dilated by `dilate` coarse cells, plus both
 * terminals.  A net whose window holds more than `max_window_cells` cells
 * (all layers; 0 = no limit) gets an empty bitmap: no corridor is proposed,
 * its whole window is searched at once, and its status is NONE. */
APGAR_B200_API int apgar_b200_corridor_from_logits(void* plan, const float* logits, const uint32_t* dims,
                                    float threshold, int32_t dilate, uint64_t max_window_cells,
                                    uint32_t* bits, void* stream);
/* bf16 operand layouts of the current params (after every update). */
APGAR_B200_API int apgar_b200_cnn_prepare(const float* params, void* operands, void* stream);
/* Forward pass; acts holds five activation buffers (they may alternate
 * between two for inference).  `error` receives APGAR_B200_CNN_* bits. */
APGAR_B200_API int apgar_b200_cnn_forward(const float* params, const void* operands, const void* rasters,
                           const uint32_t* dims, uint32_t count, void* const acts[5], float* logits,
                           uint32_t* error, void* stream);
/* Backward pass of the weighted cross-entropy (positives weighted by
 * pos_weight, mean over each net's window cells, then over nets) after a
 * forward pass with five distinct activation buffers.  Overwrites grads
 * (f32, params layout) and adds the loss to *loss (device f32).  scratch0 and
 * scratch1 are activation-sized; dlogit is logits-sized. */
APGAR_B200_API int apgar_b200_cnn_backward(const float* params, const void* operands, const void* rasters,
                            const uint32_t* dims, uint32_t count, void* const acts[5],
                            const float* logits, const uint8_t* labels, float pos_weight,
                            float* dlogit, void* scratch0, void* scratch1, float* grads,
                            float* loss, uint32_t* error, void* stream);
/* One Adam step (step counts from 1) on params with f32 moments m and v. */
APGAR_B200_API int apgar_b200_cnn_adam(float* params, const float* grads, float* m, float* v,
                        uint32_t step, float lr, float beta1, float beta2, float eps,
                        void* stream);

/* ======================= C. congestion prices ======================= */

/* Integer negotiated-congestion price schedule.  Combines the allocator epoch
 * update (NegotiatedPriceUpdatePolicyV1 and the per-resource update of
 * src/allocator/negotiated_regeneration_plan.cc:430-442, :676-760) with the
 * CS-RR-v1 history update and next-pass query snapshot cost
 * (src/allocator/cpu_sequential_negotiated_routing.cc:299-505, :1300-1330);
 * overuse = max(0, usage - capacity) as in resource_accounting.cc:212-213. */
typedef struct apgar_b200_price_policy {
  uint64_t initial_present_factor;     /* 100 in the reference default */
  uint64_t present_factor_increment;   /* 100 */
  uint64_t historical_price_increment; /* 10 */
  uint64_t capacity;                   /* capacity units per resource */
  uint64_t maximum_value;              /* bound on histories and snapshot costs */
} apgar_b200_price_policy;

/* status bits written by the price update */
enum { APGAR_B200_PRICE_OVERFLOW = 1u, APGAR_B200_PRICE_BOUND = 2u };

/* One fused pass over `count` resources with usage counts `usage`, for price
 * epoch `epoch` (factor = initial + epoch * increment):
 *   overuse > 0:  present = factor * overuse, history += increment * overuse,
 *   otherwise:    present = 0, history unchanged;
 *   total = present + history;
 *   next_cost (optional) = history + factor(epoch + 1) * max(0, usage + 1 - capacity),
 * the CS-RR snapshot cost a query pays in the next pass.  All arithmetic is
 * checked uint64; *status receives APGAR_B200_PRICE_* bits (0 = clean).
 * Device pointers, stream-ordered; `status` is a device word. */
APGAR_B200_API int apgar_b200_price_update_device(uint32_t count, const uint32_t* usage,
                                                  const apgar_b200_price_policy* policy,
                                                  uint64_t epoch, uint64_t* present,
                                                  uint64_t* history, uint64_t* total,
                                                  uint64_t* next_cost, uint32_t* status,
                                                  void* stream);
/* Same on host arrays (copies in, runs on the current device, copies out). */
APGAR_B200_API int apgar_b200_price_update(uint32_t count, const uint32_t* usage,
                                           const apgar_b200_price_policy* policy, uint64_t epoch,
                                           uint64_t* present, uint64_t* history, uint64_t* total,
                                           uint64_t* next_cost, uint32_t* status);

/* Adds one usage unit per path cell of a lattice plan's packed paths
 * (cell resources, usage indexed by global cell id; `cell_count` bounds the
 * array).  Device pointer, stream-ordered. */
APGAR_B200_API int apgar_b200_lattice_accumulate_usage(void* plan, uint32_t* usage,
                                                       uint64_t cell_count, void* stream);

/* ================= D. negotiated-congestion rounds ================= */

/* Batched rip-up and reroute on a FRONTIER plan: the reference's negotiated
 * loop (RouteCpuSequentialNegotiated, src/allocator/
 * cpu_sequential_negotiated_routing.cc:993-1330) with the GPU batched search
 * as its engine and one resource per lattice cell.  Round r reroutes every
 * net of the plan against the frozen snapshot prices, counts per-cell usage
 * of the reached paths, and runs the fused price pass at epoch r: history
 * += increment * overuse; next snapshot = history + factor(r + 1) *
 * max(0, usage + 1 - capacity).  From round 1 on, a net pays for the cells
 * of its own previous route the snapshot of the other nets' usage (usage - 1
 * in place of usage), as the reference rips the incumbent route up before
 * pricing a query (cpu_sequential_negotiated_routing.cc:1023-1034).  Rounds
 * are Jacobi (all nets against one snapshot), while the reference's loop is
 * Gauss-Seidel (net by net), so the two give different routings by design;
 * every round is exact for its snapshot. */
typedef struct apgar_b200_negotiation_round {
  uint64_t overused_cells; /* cells with usage > capacity after the round */
  uint64_t total_overuse;  /* sum of max(0, usage - capacity) */
  uint32_t price_status;   /* APGAR_B200_PRICE_* bits of the round's price pass */
  uint32_t reserved;
} apgar_b200_negotiation_round;

/* Binds a negotiation to a FRONTIER plan (the plan must outlive it; the
 * negotiation sets the plan's cell prices while it runs). */
APGAR_B200_API int apgar_b200_negotiation_create(void* plan, const apgar_b200_price_policy* policy,
                                  void** out_negotiation);
/* Runs a whole negotiation from zero history and zero prices: `rounds`
 * rounds, stream-ordered after `stream`.  With use_graph != 0 the rounds
 * are captured once as one CUDA graph (re-captured when `rounds` changes)
 * and replayed; the first call with a given round count does the capture.
 * The plan's results and paths hold the last round's routing. */
APGAR_B200_API int apgar_b200_negotiation_run(void* negotiation, uint32_t rounds, uint32_t use_graph,
                               void* stream);
/* Flags of apgar_b200_negotiation_run_ex. */
#define APGAR_B200_NEGOTIATE_GRAPH 1u   /* capture the rounds once as one CUDA graph */
#define APGAR_B200_NEGOTIATE_PARTIAL 2u /* partial rip-up: from round 1 on, reroute only the
                                           nets whose route crosses an overused cell (or
                                           did not reach its goal); the others keep theirs */
/* apgar_b200_negotiation_run with flags (run == run_ex with GRAPH or 0). */
APGAR_B200_API int apgar_b200_negotiation_run_ex(void* negotiation, uint32_t rounds, uint32_t flags,
                                  void* stream);
/* Split-round form, for one rank of a multi-GPU negotiation whose plan holds
 * that rank's share of the segments.  Round r is two steps: ROUTE reroutes
 * the plan's nets against the current snapshot and counts their per-cell
 * usage (round 0's ROUTE first zeroes history and prices); the caller then
 * sums the usage buffer over all ranks in place (one integer all-reduce);
 * PRICE runs the fused price pass over the summed usage, identically on every
 * rank.  Rounds are Jacobi, so R ranks give exactly the single-plan results.
 * Steps alternate ROUTE, PRICE in round order from round 0 (rounds 0..999);
 * flags: APGAR_B200_NEGOTIATE_PARTIAL only.  Work is ordered after `stream`
 * and `stream` after the work. */
enum { APGAR_B200_NEGOTIATE_ROUTE = 0, APGAR_B200_NEGOTIATE_PRICE = 1 };
APGAR_B200_API int apgar_b200_negotiation_step(void* negotiation, uint32_t round, uint32_t phase,
                                               uint32_t flags, void* stream);
/* Makes the negotiation count usage into the caller's device buffer (one
 * uint32 per lattice cell, on the plan's device), so that a collective can
 * sum it in place between ROUTE and PRICE; NULL returns to the negotiation's
 * own buffer. */
APGAR_B200_API int apgar_b200_negotiation_set_usage_buffer(void* negotiation, uint32_t* usage_device);
/* Waits for the negotiation; copies the last round's usage, the history,
 * the next snapshot prices (each optional, layers*height*width cells) and
 * per-round statistics. */
APGAR_B200_API int apgar_b200_negotiation_readback(void* negotiation, uint32_t* usage, uint64_t* history,
                                    uint32_t* cell_costs, apgar_b200_negotiation_round* rounds,
                                    uint32_t round_count);
/* Device pointer of the negotiation's current snapshot prices (one uint32 per
 * lattice cell, on the plan's device), written by each round's PRICE step
 * and read by the next ROUTE: for instance the congestion raster of a
 * learned corridor proposal between the two (stream-ordered after the
 * PRICE step's `stream`).  Valid while the negotiation lives. */
APGAR_B200_API int apgar_b200_negotiation_device_prices(void* negotiation, const uint32_t** cell_costs);
APGAR_B200_API int apgar_b200_negotiation_release(void* negotiation);

#ifdef __cplusplus
}
#endif

#endif /* APGAR_B200_H_ */
