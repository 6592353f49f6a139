// Host side of the drop-in seam: device-view upload with validation,
// candidate-batch admission, execution on the device engine
// (graph_search.cu) and readback in the reference V1 record formats.  No CPU
// search fallback exists: every admitted query is searched on the GPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "graph_common.cuh"
#include "host_common.h"

static_assert(sizeof(apgar_b200_compiled_header_v1) == 112, "DeviceCompiledHeaderV1 layout");
static_assert(sizeof(apgar_b200_layer_range_v1) == 48, "DeviceLayerRangeV1 layout");
static_assert(sizeof(apgar_b200_node_v1) == 56, "DeviceNodeV1 layout");
static_assert(sizeof(apgar_b200_run_v1) == 12, "DeviceRunV1 layout");
static_assert(sizeof(apgar_b200_policy_edge_v1) == 16, "DeviceCandidatePolicyEdgeV1 layout");
static_assert(sizeof(apgar_b200_batch_query_v1) == 120, "DeviceCandidateBatchQueryV1 layout");
static_assert(sizeof(apgar_b200_batch_result_v1) == 120, "DeviceCandidateBatchResultV1 layout");
static_assert(sizeof(apgar_b200_compact_path_v1) == 32, "DeviceCandidateCompactPathV1 layout");
static_assert(sizeof(apgar_b200_route_result_header_v1) == 64, "DeviceRouteResultHeaderV1 layout");

namespace apgar_b200 {

cudaError_t launch_graph_search(const GraphLaunch& launch, cudaStream_t stream);
cudaError_t launch_validate_paths(const PathCheckLaunch& launch, cudaStream_t stream);
cudaError_t launch_reach(const ReachLaunch& launch, cudaStream_t stream);
cudaError_t launch_validate_predecessors(const PredCheckLaunch& launch, cudaStream_t stream);
cudaError_t launch_path_segments(const apgar_b200_node_v1* nodes, uint32_t node_count, int64_t ox,
                                 int64_t oy, int64_t step, const apgar_b200_compact_path_v1* paths,
                                 const uint32_t* states, uint64_t state_count, uint32_t count,
                                 apgar_b200_segment* segments, uint32_t* segment_counts,
                                 cudaStream_t stream);
cudaError_t launch_graph_pack(apgar_b200_compact_path_v1* compact, uint32_t count,
                              uint64_t states_per_query, const uint32_t* stage, uint32_t* packed,
                              unsigned long long* total, int sm_count, cudaStream_t stream);

namespace {

using U128 = unsigned __int128;
constexpr uint64_t kMaximumRepresentedNodes = 10'000'000;  // compiled_board.h:21
constexpr uint64_t kMaximumPolicyEntries = 1'000'000;      // candidate_policy.h:18
constexpr int kDx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
constexpr int kDy[8] = {0, 1, 1, 1, 0, -1, -1, -1};

int invariant(const std::string& detail) { return set_error(APGAR_B200_INTERNAL_INVARIANT, detail); }

// One execution at a time per view, from execute until release (the
// reference's prepared-view execution lease), independent of the thread.
struct Lease {
  std::mutex m;
  std::condition_variable cv;
  bool busy = false;
  void acquire() {
    std::unique_lock<std::mutex> lock(m);
    cv.wait(lock, [&] { return !busy; });
    busy = true;
  }
  void release() {
    {
      std::lock_guard<std::mutex> lock(m);
      busy = false;
    }
    cv.notify_one();
  }
};

struct Workspace {
  DeviceBuffer<apgar_b200_batch_query_v1> queries;
  DeviceBuffer<apgar_b200_policy_edge_v1> policy;
  DeviceBuffer<apgar_b200_batch_result_v1> results;
  DeviceBuffer<apgar_b200_compact_path_v1> compact;
  DeviceBuffer<uint64_t> labels;
  DeviceBuffer<uint32_t> queues;
  DeviceBuffer<uint32_t> stamps;
  DeviceBuffer<uint32_t> stage;  // compact: staged paths; workspace: predecessors
  DeviceBuffer<uint64_t> owners;
  DeviceBuffer<uint64_t> pred_owners;
  DeviceBuffer<unsigned long long> counters;
  uint64_t bytes() const {
    return queries.bytes() + policy.bytes() + results.bytes() + compact.bytes() + labels.bytes() +
           queues.bytes() + stamps.bytes() + stage.bytes() + owners.bytes() + pred_owners.bytes() +
           counters.bytes();
  }
};

// Page-locked host staging, grown on demand and kept with its view: a batch's
// inputs go up and its results come back through it in one asynchronous copy
// per buffer, with a single synchronisation per direction.
struct PinnedStage {
  uint8_t* p = nullptr;
  size_t cap = 0;
  ~PinnedStage() {
    if (p != nullptr) cudaFreeHost(p);
  }
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p != nullptr) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    void* q = nullptr;
    const cudaError_t e = cudaHostAlloc(&q, n, cudaHostAllocDefault);
    if (e != cudaSuccess) return e;
    p = static_cast<uint8_t*>(q);
    cap = n;
    return cudaSuccess;
  }
};

inline size_t round16(size_t n) { return (n + 15) & ~static_cast<size_t>(15); }

struct ViewObject {
  int device = -1;
  int sm_count = 0;
  apgar_b200_compiled_header_v1 header{};
  std::vector<uint8_t> legal;  // host copy for policy-edge admission
  uint64_t persistent_bytes = 0;
  DeviceBuffer<uint32_t> neighbors;
  DeviceBuffer<uint8_t> legal_dev;
  DeviceBuffer<apgar_b200_node_v1> nodes_dev;  // full records, for path validation
  Lease lease;
  Workspace ws;
  PinnedStage host_stage;
  uint32_t* cancel_host = nullptr;
  uint32_t* cancel_dev = nullptr;
  ~ViewObject() {
    if (cancel_host != nullptr) cudaFreeHost(cancel_host);
  }
  GraphDeviceView device_view() const {
    GraphDeviceView g{};
    g.neighbors = neighbors.get();
    g.legal = legal_dev.get();
    g.node_count = static_cast<uint32_t>(legal.size());
    g.orth = header.orthogonal_step;
    g.diag = header.diagonal_step;
    g.bend = header.bend;
    g.compiler_version = header.compiler_version;
    g.source_board_content_hash = header.source_board_content_hash;
    g.compiler_profile_fingerprint = header.compiler_profile_fingerprint;
    g.rule_bucket_identity = header.rule_bucket_identity;
    g.device_view_fingerprint = header.device_view_fingerprint;
    return g;
  }
};

struct PendingBatch {
  ViewObject* view = nullptr;
  bool leased = false;
  bool workspace_mode = false;
  uint8_t generator = 0;
  uint32_t query_count = 0;
  uint64_t states = 0;
  uint64_t batch_bytes = 0;
  float kernel_ms = 0.0f;
  uint64_t launches = 0;
  ~PendingBatch() {
    if (leased && view != nullptr) view->lease.release();
  }
};

struct PendingRoute {
  std::unique_ptr<PendingBatch> batch;
  apgar_b200_route_result_header_v1 header{};
};

int check_device(int expected) {
  int current = -1;
  APGAR_B200_CUDA("cudaGetDevice", cudaGetDevice(&current));
  if (current != expected) {
    return set_error(APGAR_B200_BACKEND_FAILURE,
                     "current CUDA device differs from the device the view was uploaded on");
  }
  return APGAR_B200_OK;
}

// Memory-safety and cost-domain checks of the reference upload validation
// (gpu/cuda/planar_router.cu:1256-1451).  The FNV view fingerprint is not
// recomputed here; the C++ adapter recomputes it with the reference routine.
int validate_view(const apgar_b200_compiled_header_v1& h, const apgar_b200_layer_range_v1* layers,
                  uint64_t layer_count, const apgar_b200_node_v1* nodes, uint64_t n,
                  const apgar_b200_run_v1* runs, uint64_t run_count, const uint32_t* run_nodes,
                  uint64_t run_node_count) {
  if (h.schema_version != 1u || n == 0 || n > kMaximumRepresentedNodes || n >= 0xFFFFFFFFull ||
      h.represented_nodes != n || 9ull * n >= 0xFFFFFFFFull || h.represented_states != 9ull * n) {
    return invariant("upload rejected inconsistent schema or node/state count bounds");
  }
  if (h.lattice_step <= 0 || h.orthogonal_step == 0 || h.diagonal_step == 0 ||
      h.heading_mask == 0 || (h.heading_mask & ~0x7u) != 0 ||
      std::any_of(h.reserved, h.reserved + 7, [](uint8_t b) { return b != 0; })) {
    return invariant("upload rejected invalid lattice, cost, heading-mask or reserved header fields");
  }
  const U128 max_transition =
      static_cast<U128>(std::max(h.orthogonal_step, h.diagonal_step)) + h.bend;
  if (max_transition * n * 8u >= static_cast<U128>(~0ull)) {
    return invariant("upload rejected costs that exceed or collide with the finite route-cost bound");
  }
  if (layer_count == 0 || layers == nullptr) return invariant("upload rejected an empty layer partition");
  uint64_t expected = 0;
  for (uint64_t li = 0; li < layer_count; ++li) {
    const apgar_b200_layer_range_v1& L = layers[li];
    const uint64_t end = static_cast<uint64_t>(L.node_offset) + L.node_count;
    if (L.node_count == 0 || L.node_offset != expected || end > n ||
        L.minimum_lattice_x > L.maximum_lattice_x || L.minimum_lattice_y > L.maximum_lattice_y ||
        (li != 0 && layers[li - 1].layer >= L.layer)) {
      return invariant("upload rejected an invalid or non-canonical layer range");
    }
    int64_t mnx = nodes[L.node_offset].lattice_x, mxx = mnx;
    int64_t mny = nodes[L.node_offset].lattice_y, mxy = mny;
    for (uint64_t i = L.node_offset; i < end; ++i) {
      if (nodes[i].layer != L.layer) return invariant("upload rejected a node outside its layer range");
      mnx = std::min(mnx, nodes[i].lattice_x);
      mxx = std::max(mxx, nodes[i].lattice_x);
      mny = std::min(mny, nodes[i].lattice_y);
      mxy = std::max(mxy, nodes[i].lattice_y);
    }
    if (mnx != L.minimum_lattice_x || mxx != L.maximum_lattice_x || mny != L.minimum_lattice_y ||
        mxy != L.maximum_lattice_y) {
      return invariant("upload rejected inexact layer bounds");
    }
    expected = end;
  }
  if (expected != n) return invariant("upload rejected a layer partition that does not cover all nodes");
  for (uint64_t i = 0; i < n; ++i) {
    const apgar_b200_node_v1& node = nodes[i];
    if (node.reserved[0] | node.reserved[1] | node.reserved[2]) {
      return invariant("upload rejected nonzero reserved node fields");
    }
    for (int d = 0; d < 8; ++d) {
      const bool legal = (node.legal_edges >> d) & 1u;
      const uint32_t nb = node.neighbors[d];
      const uint8_t heading = d % 4 == 0 ? 1u : (d % 4 == 2 ? 2u : 4u);  // H, V, 45
      if (legal != (nb != 0xFFFFFFFFu) || (legal && ((h.heading_mask & heading) == 0 || nb >= n))) {
        return invariant("upload rejected a legal mask and neighbor-index disagreement");
      }
      if (!legal) continue;
      const apgar_b200_node_v1& other = nodes[nb];
      if (other.layer != node.layer || other.lattice_x != node.lattice_x + kDx[d] ||
          other.lattice_y != node.lattice_y + kDy[d]) {
        return invariant("upload rejected a non-adjacent neighbor index");
      }
      const int od = (d + 4) % 8;
      if (((other.legal_edges >> od) & 1u) == 0 || other.neighbors[od] != i) {
        return invariant("upload rejected an edge without its exact reverse edge");
      }
    }
  }
  // directional runs: bounds, direction, and exact coverage of legal edges
  std::vector<uint8_t> covered(n, 0);
  uint64_t run_offset = 0;
  for (uint64_t ri = 0; ri < run_count; ++ri) {
    const apgar_b200_run_v1& r = runs[ri];
    const uint64_t end = static_cast<uint64_t>(r.node_offset) + r.node_count;
    if (r.direction >= 8 || r.node_count < 2 || r.node_offset != run_offset || end > run_node_count ||
        r.reserved[0] | r.reserved[1] | r.reserved[2]) {
      return invariant("upload rejected invalid directional-run bounds or direction");
    }
    for (uint64_t k = r.node_offset; k + 1 < end; ++k) {
      const uint32_t a = run_nodes[k], b = run_nodes[k + 1];
      if (a >= n || b >= n || nodes[a].neighbors[r.direction] != b) {
        return invariant("upload rejected an invalid directed run edge");
      }
      if (covered[a] & (1u << r.direction)) return invariant("upload rejected a duplicated run edge");
      covered[a] |= static_cast<uint8_t>(1u << r.direction);
    }
    run_offset = end;
  }
  if (run_offset != run_node_count) return invariant("upload rejected unowned run-node storage");
  for (uint64_t i = 0; i < n; ++i) {
    if (covered[i] != nodes[i].legal_edges) {
      return invariant("upload rejected incomplete directional-run edge coverage");
    }
  }
  const U128 bytes = 112u + static_cast<U128>(layer_count) * 48u + static_cast<U128>(n) * 56u +
                     static_cast<U128>(run_count) * 12u + static_cast<U128>(run_node_count) * 4u;
  if (bytes != h.estimated_persistent_device_bytes) {
    return invariant("upload rejected inconsistent persistent-memory accounting");
  }
  return APGAR_B200_OK;
}

// Candidate-batch admission (gpu/cuda/planar_router.cu:1731-1909): ordering,
// ownership, associations, workspace bounds, policy encoding and the
// cost-sentinel bound.
// Generators whose readback is the full workspace (labels, predecessors and
// owners of every state) rather than compact paths.
bool full_workspace_generator(uint8_t generator) {
  return generator == APGAR_B200_GENERATOR_BUCKETED_FRONTIER ||
         generator == APGAR_B200_GENERATOR_B200_PERSISTENT_WORKSPACE;
}

int validate_batch(const ViewObject& v, const apgar_b200_batch_request& req,
                   const apgar_b200_batch_query_v1* queries, uint32_t count,
                   const apgar_b200_policy_edge_v1* edges, uint64_t edge_count) {
  const uint64_t n = v.legal.size();
  const uint64_t S = 9ull * n;
  if (req.schema_version != 1u || req.batch_id == 0 || count == 0 ||
      edge_count > kMaximumPolicyEntries || req.maximum_rounds == 0 ||
      req.generator > APGAR_B200_GENERATOR_B200_PERSISTENT_WORKSPACE) {
    return invariant("candidate batch has invalid schema, identity, policy size, generator or rounds");
  }
  if (req.maximum_workspace_states_per_query < S) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "batch exceeds the per-query workspace-state capacity");
  }
  const bool frontier = full_workspace_generator(req.generator);
  if (frontier && req.maximum_frontier_states_per_query < S) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "batch exceeds the per-query frontier-state capacity");
  }
  if (static_cast<U128>(S) * count > static_cast<U128>(1ull << 40)) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "batch query-major state space is too large");
  }
  std::set<uint64_t> owners;
  uint64_t expected_policy = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const apgar_b200_batch_query_v1& q = queries[i];
    const uint64_t pend = static_cast<uint64_t>(q.policy_offset) + q.policy_count;
    if (q.schema_version != 1u || q.batch_id != req.batch_id || q.query_id == 0 ||
        q.workspace_owner == 0 || q.generator != req.generator ||
        q.maximum_rounds != req.maximum_rounds || q.start_node >= n || q.goal_node >= n ||
        q.start_node == q.goal_node || q.workspace_offset != i * S || q.workspace_state_count != S ||
        q.frontier_state_capacity != (frontier ? S : 0) || q.policy_offset != expected_policy ||
        pend > 0xFFFFFFFFull || pend > edge_count || (q.reserved[0] | q.reserved[1] | q.reserved[2]) ||
        (i != 0 && queries[i - 1].query_id >= q.query_id) || !owners.insert(q.workspace_owner).second) {
      return invariant("candidate batch query ordering, ownership, association, endpoint, policy or "
                       "workspace bounds are invalid");
    }
    uint64_t max_penalty = 0;
    for (uint64_t e = q.policy_offset; e < pend; ++e) {
      const apgar_b200_policy_edge_v1& pe = edges[e];
      const uint32_t node = pe.physical_edge_index / 8u, dir = pe.physical_edge_index % 8u;
      if (pe.reserved != 0 || node >= n || dir >= 4 || ((v.legal[node] >> dir) & 1u) == 0 ||
          (e != q.policy_offset && edges[e - 1].physical_edge_index >= pe.physical_edge_index)) {
        return invariant("candidate batch policy edge encoding is invalid or non-canonical");
      }
      if (pe.adjustment != ~0ull) max_penalty = std::max(max_penalty, pe.adjustment);
    }
    const U128 orth = static_cast<U128>(v.header.orthogonal_step) + q.orthogonal_step_surcharge;
    const U128 diag = static_cast<U128>(v.header.diagonal_step) + q.diagonal_step_surcharge;
    const U128 bend = static_cast<U128>(v.header.bend) + q.bend_surcharge;
    const U128 max_t = std::max(orth, diag) + bend + max_penalty;
    const U128 inf = static_cast<U128>(~0ull);
    if (orth >= inf || diag >= inf || bend >= inf || max_t * n * 8u >= inf) {
      return invariant("candidate batch policy cost bound collides with the unreachable sentinel");
    }
    expected_policy = pend;
  }
  if (expected_policy != edge_count) return invariant("candidate batch contains unowned policy-edge storage");
  return APGAR_B200_OK;
}

int run_batch(ViewObject* v, const apgar_b200_batch_request& req,
              const apgar_b200_batch_query_v1* queries, uint32_t count,
              const apgar_b200_policy_edge_v1* edges, uint64_t edge_count,
              const volatile uint8_t* cancel, PendingBatch* pending) {
  const uint64_t n = v->legal.size();
  const uint64_t S = 9ull * n;
  const bool workspace_mode = full_workspace_generator(req.generator);
  Workspace& w = v->ws;
  const uint64_t Q = count;
  // deterministic workspace bytes for this batch (checked against the budget
  // before allocating)
  const U128 need = static_cast<U128>(Q) * (120u + 120u + 32u) + static_cast<U128>(edge_count) * 16u +
                    static_cast<U128>(Q) * S * 8u + static_cast<U128>(Q) * n * 12u +
                    static_cast<U128>(Q) * S * 4u +
                    (workspace_mode ? static_cast<U128>(Q) * S * 16u : 0u) + 16u;
  if (v->persistent_bytes > req.maximum_device_bytes ||
      need > static_cast<U128>(req.maximum_device_bytes - v->persistent_bytes)) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "batch exceeds the device-memory budget");
  }
  APGAR_B200_CUDA("cudaMalloc(queries)", w.queries.ensure(Q));
  // no policy buffer without policy edges (the kernel reads none), so a
  // fresh workspace holds exactly the bytes `need` accounts for
  APGAR_B200_CUDA("cudaMalloc(policy)", w.policy.ensure(edge_count));
  APGAR_B200_CUDA("cudaMalloc(results)", w.results.ensure(Q));
  APGAR_B200_CUDA("cudaMalloc(compact)", w.compact.ensure(Q));
  APGAR_B200_CUDA("cudaMalloc(labels)", w.labels.ensure(Q * S));
  APGAR_B200_CUDA("cudaMalloc(queues)", w.queues.ensure(Q * 2 * n));
  APGAR_B200_CUDA("cudaMalloc(stamps)", w.stamps.ensure(Q * n));
  APGAR_B200_CUDA("cudaMalloc(stage)", w.stage.ensure(Q * S));
  if (workspace_mode) {
    APGAR_B200_CUDA("cudaMalloc(owners)", w.owners.ensure(Q * S));
    APGAR_B200_CUDA("cudaMalloc(pred owners)", w.pred_owners.ensure(Q * S));
  }
  APGAR_B200_CUDA("cudaMalloc(counters)", w.counters.ensure(2));
  // queries and policy edges through the pinned stage, copied in stream order
  // before the search (the view's lease keeps the stage to this batch)
  const size_t qbytes = Q * sizeof(*queries), ebytes = edge_count * sizeof(*edges);
  APGAR_B200_CUDA("cudaHostAlloc(staging)", v->host_stage.ensure(round16(qbytes) + ebytes));
  std::memcpy(v->host_stage.p, queries, qbytes);
  if (ebytes > 0) std::memcpy(v->host_stage.p + round16(qbytes), edges, ebytes);
  APGAR_B200_CUDA("cudaMemcpyAsync(queries)",
                  cudaMemcpyAsync(w.queries.get(), v->host_stage.p, qbytes, cudaMemcpyHostToDevice, nullptr));
  if (ebytes > 0) {
    APGAR_B200_CUDA("cudaMemcpyAsync(policy)",
                    cudaMemcpyAsync(w.policy.get(), v->host_stage.p + round16(qbytes), ebytes,
                                    cudaMemcpyHostToDevice, nullptr));
  }
  if (v->cancel_host == nullptr) {
    void* h = nullptr;
    APGAR_B200_CUDA("cudaHostAlloc(cancel flag)", cudaHostAlloc(&h, sizeof(uint32_t), cudaHostAllocMapped));
    v->cancel_host = static_cast<uint32_t*>(h);
    void* d = nullptr;
    APGAR_B200_CUDA("cudaHostGetDevicePointer(cancel flag)", cudaHostGetDevicePointer(&d, h, 0));
    v->cancel_dev = static_cast<uint32_t*>(d);
  }
  *reinterpret_cast<volatile uint32_t*>(v->cancel_host) = 0u;

  GraphLaunch L{};
  L.g = v->device_view();
  L.queries = w.queries.get();
  L.query_count = count;
  L.policy = w.policy.get();
  L.labels = w.labels.get();
  L.queues = w.queues.get();
  L.stamps = w.stamps.get();
  L.results = w.results.get();
  L.compact = w.compact.get();
  L.path_stage = w.stage.get();
  L.predecessors = w.stage.get();
  L.state_owners = w.owners.get();
  L.predecessor_owners = w.pred_owners.get();
  L.maximum_rounds = req.maximum_rounds;
  L.generator = req.generator;
  L.workspace_mode = workspace_mode ? 1 : 0;
  L.cancel = v->cancel_dev;
  for (uint64_t i = 0; i < Q; ++i) L.max_policy_edges = std::max(L.max_policy_edges, queries[i].policy_count);

  cudaEvent_t t0 = nullptr, t1 = nullptr;
  APGAR_B200_CUDA("cudaEventCreate", cudaEventCreate(&t0));
  APGAR_B200_CUDA("cudaEventCreate", cudaEventCreate(&t1));
  std::unique_ptr<CUevent_st, decltype(&cudaEventDestroy)> g0(t0, cudaEventDestroy);
  std::unique_ptr<CUevent_st, decltype(&cudaEventDestroy)> g1(t1, cudaEventDestroy);
  APGAR_B200_CUDA("cudaEventRecord", cudaEventRecord(t0, nullptr));
  APGAR_B200_CUDA("graph search launch", launch_graph_search(L, nullptr));
  uint64_t launches = 1;
  if (!workspace_mode) {
    // packed states reuse the label slab, dead once every path is staged
    APGAR_B200_CUDA("graph pack launch",
                    launch_graph_pack(w.compact.get(), count, S, w.stage.get(),
                                      reinterpret_cast<uint32_t*>(w.labels.get()),
                                      w.counters.get(), v->sm_count, nullptr));
    launches += 2;
  }
  APGAR_B200_CUDA("cudaEventRecord", cudaEventRecord(t1, nullptr));
  // The caller's flag is sampled here and forwarded through the view's
  // mapped flag, which the kernel polls once per round.
  for (;;) {
    const cudaError_t q = cudaEventQuery(t1);
    if (q == cudaSuccess) break;
    if (q != cudaErrorNotReady) return cuda_failure("graph search", q);
    if (cancel != nullptr && *cancel != 0u) *reinterpret_cast<volatile uint32_t*>(v->cancel_host) = 1u;
    std::this_thread::yield();
  }
  float ms = 0.0f;
  APGAR_B200_CUDA("cudaEventElapsedTime", cudaEventElapsedTime(&ms, t0, t1));
  pending->view = v;
  pending->workspace_mode = workspace_mode;
  pending->generator = req.generator;
  pending->query_count = count;
  pending->states = S;
  pending->batch_bytes = static_cast<uint64_t>(need);
  pending->kernel_ms = ms;
  pending->launches = launches;
  return APGAR_B200_OK;
}

void fill_telemetry(const PendingBatch& p, uint64_t readback_bytes, uint32_t max_rounds,
                    apgar_b200_batch_telemetry* t) {
  if (t == nullptr) return;
  std::memset(t, 0, sizeof(*t));
  t->persistent_device_bytes = p.view->persistent_bytes;
  t->batch_device_bytes = p.batch_bytes;
  t->workspace_capacity_device_bytes = std::max<uint64_t>(p.view->ws.bytes(), p.batch_bytes);
  t->peak_device_bytes = t->persistent_device_bytes + t->workspace_capacity_device_bytes;
  t->device_to_host_readback_bytes = readback_bytes;
  t->kernel_launch_count = p.launches;
  t->blocking_status_readback_count = 0;  // no host round trip during the search
  t->dispatched_rounds = max_rounds;
  // The persistent generators' descriptor counts the batch's last launch
  // (path packing, or the single search launch of the full workspace, which
  // writes every final result header) as its finalization launch.
  t->finalization_launch_count = p.generator >= APGAR_B200_GENERATOR_B200_PERSISTENT ? 1u : 0u;
  t->kernel_milliseconds = p.kernel_ms;
}

}  // namespace
}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" int apgar_b200_view_upload(const apgar_b200_compiled_header_v1* header,
                                      const apgar_b200_layer_range_v1* layers, uint64_t layer_count,
                                      const apgar_b200_node_v1* nodes, uint64_t node_count,
                                      const apgar_b200_run_v1* runs, uint64_t run_count,
                                      const uint32_t* run_nodes, uint64_t run_node_count,
                                      void** out_view) {
  if (header == nullptr || nodes == nullptr || out_view == nullptr ||
      (run_count > 0 && runs == nullptr) || (run_node_count > 0 && run_nodes == nullptr)) {
    return invariant("view upload received a null argument");
  }
  try {
    if (int rc = validate_view(*header, layers, layer_count, nodes, node_count, runs, run_count,
                               run_nodes, run_node_count);
        rc != APGAR_B200_OK) {
      return rc;
    }
    auto v = std::make_unique<ViewObject>();
    APGAR_B200_CUDA("cudaGetDevice", cudaGetDevice(&v->device));
    APGAR_B200_CUDA("cudaDeviceGetAttribute",
                    cudaDeviceGetAttribute(&v->sm_count, cudaDevAttrMultiProcessorCount, v->device));
    v->header = *header;
    v->persistent_bytes = header->estimated_persistent_device_bytes;
    v->legal.resize(node_count);
    std::vector<uint32_t> soa(8 * node_count);
    for (uint64_t i = 0; i < node_count; ++i) {
      v->legal[i] = nodes[i].legal_edges;
      for (int d = 0; d < 8; ++d) soa[static_cast<uint64_t>(d) * node_count + i] = nodes[i].neighbors[d];
    }
    APGAR_B200_CUDA("cudaMalloc(neighbors)", v->neighbors.ensure(soa.size()));
    APGAR_B200_CUDA("cudaMemcpy(neighbors)", cudaMemcpy(v->neighbors.get(), soa.data(),
                                                        soa.size() * 4, cudaMemcpyHostToDevice));
    APGAR_B200_CUDA("cudaMalloc(legal)", v->legal_dev.ensure(node_count));
    APGAR_B200_CUDA("cudaMemcpy(legal)", cudaMemcpy(v->legal_dev.get(), v->legal.data(), node_count,
                                                    cudaMemcpyHostToDevice));
    APGAR_B200_CUDA("cudaMalloc(nodes)", v->nodes_dev.ensure(node_count));
    APGAR_B200_CUDA("cudaMemcpy(nodes)", cudaMemcpy(v->nodes_dev.get(), nodes,
                                                    node_count * sizeof(apgar_b200_node_v1),
                                                    cudaMemcpyHostToDevice));
    *out_view = v.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during upload");
  }
}

extern "C" int apgar_b200_view_release(void* view) {
  delete static_cast<ViewObject*>(view);
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_execute_batch(void* view, const apgar_b200_batch_request* request,
                                        const apgar_b200_batch_query_v1* queries,
                                        uint32_t query_count,
                                        const apgar_b200_policy_edge_v1* policy_edges,
                                        uint64_t policy_edge_count, const volatile uint8_t* cancel,
                                        void** out_pending) {
  if (view == nullptr || request == nullptr || out_pending == nullptr ||
      (query_count > 0 && queries == nullptr) || (policy_edge_count > 0 && policy_edges == nullptr)) {
    return invariant("candidate batch received a null argument");
  }
  auto* v = static_cast<ViewObject*>(view);
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  try {
    auto pending = std::make_unique<PendingBatch>();
    v->lease.acquire();
    pending->view = v;
    pending->leased = true;
    if (int rc = validate_batch(*v, *request, queries, query_count, policy_edges, policy_edge_count);
        rc != APGAR_B200_OK) {
      return rc;
    }
    if (int rc = run_batch(v, *request, queries, query_count, policy_edges, policy_edge_count, cancel,
                           pending.get());
        rc != APGAR_B200_OK) {
      return rc;
    }
    *out_pending = pending.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during execution");
  }
}

extern "C" int apgar_b200_readback_batch(void* pending, apgar_b200_batch_result_v1* results,
                                         apgar_b200_compact_path_v1* compact_paths,
                                         uint32_t* path_states, uint64_t path_capacity,
                                         uint64_t* path_state_count,
                                         apgar_b200_batch_telemetry* telemetry) {
  if (pending == nullptr || results == nullptr) return invariant("readback received a null argument");
  auto* p = static_cast<PendingBatch*>(pending);
  if (int rc = check_device(p->view->device); rc != APGAR_B200_OK) return rc;
  Workspace& w = p->view->ws;
  PinnedStage& stage = p->view->host_stage;
  const uint64_t Q = p->query_count;
  // results, the path-state total and the compact records in one round trip
  const size_t rbytes = Q * sizeof(*results), cbytes = Q * sizeof(*compact_paths);
  const size_t off_total = round16(rbytes), off_compact = off_total + 16;
  APGAR_B200_CUDA("cudaHostAlloc(staging)", stage.ensure(off_compact + cbytes));
  APGAR_B200_CUDA("cudaMemcpyAsync(results)",
                  cudaMemcpyAsync(stage.p, w.results.get(), rbytes, cudaMemcpyDeviceToHost, nullptr));
  const bool compact = !p->workspace_mode;
  if (compact) {
    APGAR_B200_CUDA("cudaMemcpyAsync(path total)",
                    cudaMemcpyAsync(stage.p + off_total, w.counters.get(), sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, nullptr));
    if (compact_paths != nullptr) {
      APGAR_B200_CUDA("cudaMemcpyAsync(compact paths)",
                      cudaMemcpyAsync(stage.p + off_compact, w.compact.get(), cbytes, cudaMemcpyDeviceToHost,
                                      nullptr));
    }
  }
  APGAR_B200_CUDA("cudaStreamSynchronize(readback)", cudaStreamSynchronize(nullptr));
  std::memcpy(results, stage.p, rbytes);
  uint64_t bytes = rbytes;
  uint32_t max_rounds = 0;
  for (uint64_t i = 0; i < Q; ++i) max_rounds = std::max(max_rounds, results[i].rounds);
  uint64_t total = 0;
  if (compact) {
    unsigned long long t = 0;
    std::memcpy(&t, stage.p + off_total, sizeof(t));
    total = t;
    if (compact_paths != nullptr) {
      std::memcpy(compact_paths, stage.p + off_compact, cbytes);
      bytes += cbytes;
    }
    if (path_states != nullptr && total > 0) {
      if (total > path_capacity) {
        return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "compact path buffer is too small");
      }
      APGAR_B200_CUDA("cudaMemcpy(path states)",
                      cudaMemcpy(path_states, w.labels.get(), total * 4, cudaMemcpyDeviceToHost));
      bytes += total * 4;
    }
  }
  if (path_state_count != nullptr) *path_state_count = total;
  fill_telemetry(*p, bytes, max_rounds, telemetry);
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_readback_batch_workspace(void* pending, uint64_t* labels,
                                                   uint32_t* predecessors, uint64_t* state_owners,
                                                   uint64_t* predecessor_owners) {
  if (pending == nullptr) return invariant("workspace readback received a null pending batch");
  auto* p = static_cast<PendingBatch*>(pending);
  if (!p->workspace_mode) {
    return set_error(APGAR_B200_UNSUPPORTED, "this batch ran in compact-path form");
  }
  if (int rc = check_device(p->view->device); rc != APGAR_B200_OK) return rc;
  Workspace& w = p->view->ws;
  const uint64_t total = static_cast<uint64_t>(p->query_count) * p->states;
  if (labels) APGAR_B200_CUDA("cudaMemcpy(labels)", cudaMemcpy(labels, w.labels.get(), total * 8, cudaMemcpyDeviceToHost));
  if (predecessors) APGAR_B200_CUDA("cudaMemcpy(predecessors)", cudaMemcpy(predecessors, w.stage.get(), total * 4, cudaMemcpyDeviceToHost));
  if (state_owners) APGAR_B200_CUDA("cudaMemcpy(owners)", cudaMemcpy(state_owners, w.owners.get(), total * 8, cudaMemcpyDeviceToHost));
  if (predecessor_owners) APGAR_B200_CUDA("cudaMemcpy(pred owners)", cudaMemcpy(predecessor_owners, w.pred_owners.get(), total * 8, cudaMemcpyDeviceToHost));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_release_batch(void* pending) {
  delete static_cast<PendingBatch*>(pending);
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_execute_route(void* view, uint8_t generator, uint32_t start_node,
                                        uint32_t goal_node, uint64_t routing_profile_fingerprint,
                                        uint32_t maximum_rounds, uint64_t maximum_device_bytes,
                                        const volatile uint8_t* cancel, void** out_pending) {
  if (view == nullptr || out_pending == nullptr) return invariant("route received a null argument");
  auto* v = static_cast<ViewObject*>(view);
  const uint64_t n = v->legal.size();
  if (start_node >= n || goal_node >= n || maximum_rounds == 0 || start_node == goal_node ||
      generator > APGAR_B200_GENERATOR_B200_PERSISTENT_WORKSPACE) {
    return invariant("route received invalid endpoint, generator or budget bounds");
  }
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  try {
    auto route = std::make_unique<PendingRoute>();
    route->batch = std::make_unique<PendingBatch>();
    v->lease.acquire();
    route->batch->view = v;
    route->batch->leased = true;
    apgar_b200_batch_request req{};
    req.schema_version = 1;
    req.generator = APGAR_B200_GENERATOR_BUCKETED_FRONTIER;  // full labels + predecessors
    req.batch_id = 1;
    req.maximum_rounds = maximum_rounds;
    req.maximum_workspace_states_per_query = ~0ull;
    req.maximum_frontier_states_per_query = ~0ull;
    req.maximum_device_bytes = maximum_device_bytes;
    req.maximum_host_bytes = ~0ull;
    apgar_b200_batch_query_v1 q{};
    q.schema_version = 1;
    q.batch_id = 1;
    q.query_id = 1;
    q.workspace_owner = 1;
    q.routing_profile_fingerprint = routing_profile_fingerprint;
    q.start_node = start_node;
    q.goal_node = goal_node;
    q.workspace_state_count = 9ull * n;
    q.frontier_state_capacity = 9ull * n;
    q.maximum_rounds = maximum_rounds;
    q.generator = APGAR_B200_GENERATOR_BUCKETED_FRONTIER;
    if (int rc = run_batch(v, req, &q, 1, nullptr, 0, cancel, route->batch.get()); rc != APGAR_B200_OK) {
      return rc;
    }
    apgar_b200_route_result_header_v1& h = route->header;
    h.schema_version = 1;
    h.compiler_version = v->header.compiler_version;
    h.start_node = start_node;
    h.goal_node = goal_node;
    h.source_board_content_hash = v->header.source_board_content_hash;
    h.compiler_profile_fingerprint = v->header.compiler_profile_fingerprint;
    h.routing_profile_fingerprint = routing_profile_fingerprint;
    h.rule_bucket_identity = v->header.rule_bucket_identity;
    h.device_view_fingerprint = v->header.device_view_fingerprint;
    h.generator = generator;
    *out_pending = route.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during route execution");
  }
}

extern "C" int apgar_b200_readback_route(void* pending, apgar_b200_route_result_header_v1* header,
                                         uint8_t* completion, uint32_t* goal_state,
                                         uint64_t* labels, uint32_t* predecessors,
                                         apgar_b200_batch_telemetry* telemetry) {
  if (pending == nullptr) return invariant("route readback received a null argument");
  auto* r = static_cast<PendingRoute*>(pending);
  apgar_b200_batch_result_v1 res{};
  if (int rc = apgar_b200_readback_batch(r->batch.get(), &res, nullptr, nullptr, 0, nullptr, telemetry);
      rc != APGAR_B200_OK) {
    return rc;
  }
  if (int rc = apgar_b200_readback_batch_workspace(r->batch.get(), labels, predecessors, nullptr, nullptr);
      rc != APGAR_B200_OK) {
    return rc;
  }
  if (header != nullptr) *header = r->header;
  if (completion != nullptr) *completion = res.completion;
  if (goal_state != nullptr) *goal_state = res.goal_state;
  if (telemetry != nullptr) {
    telemetry->device_to_host_readback_bytes =
        sizeof(apgar_b200_route_result_header_v1) + r->batch->states * 12u;
  }
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_release_route(void* pending) {
  delete static_cast<PendingRoute*>(pending);
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_validate_compact_paths(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count,
    const apgar_b200_batch_result_v1* results, const apgar_b200_compact_path_v1* compact_paths,
    const uint32_t* path_states, uint64_t path_state_count, apgar_b200_path_verdict* verdicts) {
  if (view == nullptr || verdicts == nullptr ||
      (query_count > 0 && (queries == nullptr || results == nullptr || compact_paths == nullptr)) ||
      (policy_edge_count > 0 && policy_edges == nullptr) ||
      (path_state_count > 0 && path_states == nullptr)) {
    return invariant("path validation received a null argument");
  }
  auto* v = static_cast<ViewObject*>(view);
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  // policy slices must stay inside the supplied edges (a malformed query is
  // an invariant failure of the caller, not a path verdict)
  for (uint32_t i = 0; i < query_count; ++i) {
    if (static_cast<uint64_t>(queries[i].policy_offset) + queries[i].policy_count > policy_edge_count) {
      return invariant("path validation query names policy edges outside the batch");
    }
  }
  try {
    const uint64_t n = v->legal.size();
    const uint64_t words = (9u * n + 63u) / 64u;
    DeviceBuffer<apgar_b200_batch_query_v1> d_q;
    DeviceBuffer<apgar_b200_policy_edge_v1> d_pol;
    DeviceBuffer<apgar_b200_batch_result_v1> d_res;
    DeviceBuffer<apgar_b200_compact_path_v1> d_cp;
    DeviceBuffer<uint32_t> d_states;
    DeviceBuffer<uint64_t> d_visited;
    DeviceBuffer<apgar_b200_path_verdict> d_out;
    const uint64_t Q = std::max<uint64_t>(query_count, 1);
    APGAR_B200_CUDA("cudaMalloc(queries)", d_q.ensure(Q));
    APGAR_B200_CUDA("cudaMalloc(policy)", d_pol.ensure(std::max<uint64_t>(policy_edge_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(results)", d_res.ensure(Q));
    APGAR_B200_CUDA("cudaMalloc(compact)", d_cp.ensure(Q));
    APGAR_B200_CUDA("cudaMalloc(states)", d_states.ensure(std::max<uint64_t>(path_state_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(visited)", d_visited.ensure(Q * words));
    APGAR_B200_CUDA("cudaMalloc(verdicts)", d_out.ensure(Q));
    if (query_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(queries)", cudaMemcpy(d_q.get(), queries, query_count * sizeof(*queries), cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(results)", cudaMemcpy(d_res.get(), results, query_count * sizeof(*results), cudaMemcpyHostToDevice));
      APGAR_B200_CUDA("cudaMemcpy(compact)", cudaMemcpy(d_cp.get(), compact_paths, query_count * sizeof(*compact_paths), cudaMemcpyHostToDevice));
    }
    if (policy_edge_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(policy)", cudaMemcpy(d_pol.get(), policy_edges, policy_edge_count * sizeof(*policy_edges), cudaMemcpyHostToDevice));
    }
    if (path_state_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(states)", cudaMemcpy(d_states.get(), path_states, path_state_count * 4, cudaMemcpyHostToDevice));
    }
    PathCheckLaunch L{};
    L.nodes = v->nodes_dev.get();
    L.node_count = static_cast<uint32_t>(n);
    L.orth = v->header.orthogonal_step;
    L.diag = v->header.diagonal_step;
    L.bend = v->header.bend;
    L.queries = d_q.get();
    L.policy = d_pol.get();
    L.results = d_res.get();
    L.compact = d_cp.get();
    L.states = d_states.get();
    L.state_count = path_state_count;
    L.visited = d_visited.get();
    L.out = d_out.get();
    L.query_count = query_count;
    APGAR_B200_CUDA("path validation launch", launch_validate_paths(L, nullptr));
    if (query_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(verdicts)", cudaMemcpy(verdicts, d_out.get(), query_count * sizeof(*verdicts), cudaMemcpyDeviceToHost));
    }
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during path validation");
  }
}

extern "C" int apgar_b200_validate_predecessors(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count, const uint8_t* partial,
    const uint64_t* labels, const uint32_t* predecessors, apgar_b200_path_verdict* verdicts) {
  if (view == nullptr ||
      (query_count > 0 && (queries == nullptr || labels == nullptr || predecessors == nullptr ||
                           verdicts == nullptr)) ||
      (policy_edge_count > 0 && policy_edges == nullptr)) {
    return invariant("predecessor validation received a null argument");
  }
  auto* v = static_cast<ViewObject*>(view);
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  for (uint32_t i = 0; i < query_count; ++i) {
    if (static_cast<uint64_t>(queries[i].policy_offset) + queries[i].policy_count > policy_edge_count) {
      return invariant("predecessor validation query names policy edges outside the batch");
    }
  }
  if (query_count == 0) {
    clear_error();
    return APGAR_B200_OK;
  }
  const uint64_t n = v->legal.size();
  const uint64_t states = 9u * n * query_count;
  DeviceBuffer<apgar_b200_batch_query_v1> d_q;
  DeviceBuffer<apgar_b200_policy_edge_v1> d_pol;
  DeviceBuffer<uint64_t> d_labels;
  DeviceBuffer<uint32_t> d_preds;
  DeviceBuffer<uint8_t> d_partial;
  DeviceBuffer<unsigned long long> d_first;
  APGAR_B200_CUDA("cudaMalloc(queries)", d_q.ensure(query_count));
  APGAR_B200_CUDA("cudaMalloc(policy)", d_pol.ensure(std::max<uint64_t>(policy_edge_count, 1)));
  APGAR_B200_CUDA("cudaMalloc(labels)", d_labels.ensure(std::max<uint64_t>(states, 1)));
  APGAR_B200_CUDA("cudaMalloc(predecessors)", d_preds.ensure(std::max<uint64_t>(states, 1)));
  APGAR_B200_CUDA("cudaMalloc(partial)", d_partial.ensure(query_count));
  APGAR_B200_CUDA("cudaMalloc(first failures)", d_first.ensure(query_count));
  APGAR_B200_CUDA("cudaMemcpy(queries)", cudaMemcpy(d_q.get(), queries, query_count * sizeof(*queries), cudaMemcpyHostToDevice));
  if (policy_edge_count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(policy)", cudaMemcpy(d_pol.get(), policy_edges, policy_edge_count * sizeof(*policy_edges), cudaMemcpyHostToDevice));
  }
  APGAR_B200_CUDA("cudaMemcpy(labels)", cudaMemcpy(d_labels.get(), labels, states * 8, cudaMemcpyHostToDevice));
  APGAR_B200_CUDA("cudaMemcpy(predecessors)", cudaMemcpy(d_preds.get(), predecessors, states * 4, cudaMemcpyHostToDevice));
  if (partial != nullptr) {
    APGAR_B200_CUDA("cudaMemcpy(partial)", cudaMemcpy(d_partial.get(), partial, query_count, cudaMemcpyHostToDevice));
  }
  APGAR_B200_CUDA("cudaMemset(first failures)", cudaMemset(d_first.get(), 0xFF, query_count * 8));
  PredCheckLaunch L{};
  L.nodes = v->nodes_dev.get();
  L.node_count = static_cast<uint32_t>(n);
  L.orth = v->header.orthogonal_step;
  L.diag = v->header.diagonal_step;
  L.bend = v->header.bend;
  L.queries = d_q.get();
  L.policy = d_pol.get();
  L.labels = d_labels.get();
  L.predecessors = d_preds.get();
  L.partial = partial != nullptr ? d_partial.get() : nullptr;
  L.first = d_first.get();
  L.query_count = query_count;
  APGAR_B200_CUDA("predecessor validation launch", launch_validate_predecessors(L, nullptr));
  std::vector<unsigned long long> first(query_count);
  APGAR_B200_CUDA("cudaMemcpy(first failures)", cudaMemcpy(first.data(), d_first.get(), query_count * 8, cudaMemcpyDeviceToHost));
  for (uint32_t i = 0; i < query_count; ++i) {
    apgar_b200_path_verdict out{};
    if (first[i] != ~0ull) {
      out.code = static_cast<uint32_t>(first[i] & 0xFFFFFFFFull);
      const uint64_t key_state = first[i] >> 32;
      out.failing_index = key_state == 0 ? 9ull * queries[i].start_node + 8u : key_state - 1u;
    }
    verdicts[i] = out;
  }
  clear_error();
  return APGAR_B200_OK;
}

// Device scratch of one reachability chunk (visited bits and two node lists
// per query); larger batches run in several chunks.
constexpr uint64_t kReachScratchBytes = 1ull << 30;

extern "C" int apgar_b200_confirm_disconnected(
    void* view, const apgar_b200_batch_query_v1* queries, uint32_t query_count,
    const apgar_b200_policy_edge_v1* policy_edges, uint64_t policy_edge_count,
    const apgar_b200_batch_result_v1* results, apgar_b200_disconnect_verdict* verdicts) {
  if (view == nullptr || (query_count > 0 && (queries == nullptr || results == nullptr || verdicts == nullptr)) ||
      (policy_edge_count > 0 && policy_edges == nullptr)) {
    return invariant("disconnected confirmation received a null argument");
  }
  auto* v = static_cast<ViewObject*>(view);
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  const uint64_t n = v->legal.size();
  using u128 = unsigned __int128;
  constexpr u128 kMaxFinite = static_cast<u128>(~0ull) - 1u;
  std::vector<uint32_t> selected;
  std::vector<u128> max_transition(query_count, 0);
  for (uint32_t i = 0; i < query_count; ++i) {
    verdicts[i] = apgar_b200_disconnect_verdict{APGAR_B200_DISCONNECT_NOT_CLAIMED, 0u, 0u};
    if (results[i].completion != APGAR_B200_COMPLETION_DISCONNECTED) continue;
    const apgar_b200_batch_query_v1& q = queries[i];
    if (q.start_node >= n || q.goal_node >= n) {
      return invariant("disconnected confirmation query names a node outside the view");
    }
    if (static_cast<uint64_t>(q.policy_offset) + q.policy_count > policy_edge_count) {
      return invariant("disconnected confirmation query names policy edges outside the batch");
    }
    // the largest transition the query's CPU search can take
    // (StepCostUnderPolicy, src/routing/candidate_policy.cc:419-438)
    u128 penalty = 0;
    const apgar_b200_policy_edge_v1* pol = policy_edges + q.policy_offset;
    for (uint32_t e = 0; e < q.policy_count; ++e) {
      if (e > 0 && pol[e].physical_edge_index <= pol[e - 1].physical_edge_index) {
        return invariant("disconnected confirmation policy edges are not strictly sorted");
      }
      if (pol[e].adjustment != kGraphInf && pol[e].adjustment > penalty) penalty = pol[e].adjustment;
    }
    const u128 orth = static_cast<u128>(v->header.orthogonal_step) + q.orthogonal_step_surcharge;
    const u128 diag = static_cast<u128>(v->header.diagonal_step) + q.diagonal_step_surcharge;
    max_transition[i] = (orth > diag ? orth : diag) + v->header.bend + q.bend_surcharge + penalty;
    selected.push_back(i);
  }
  if (selected.empty()) {
    clear_error();
    return APGAR_B200_OK;
  }
  try {
    const uint64_t words = (n + 31u) / 32u;
    const uint64_t per_query = words * 4u + 2u * n * 4u;
    const uint64_t chunk = std::max<uint64_t>(1u, std::min<uint64_t>(selected.size(), kReachScratchBytes / per_query));
    DeviceBuffer<apgar_b200_batch_query_v1> d_q;
    DeviceBuffer<apgar_b200_policy_edge_v1> d_pol;
    DeviceBuffer<uint32_t> d_sel, d_visited, d_queues, d_reached;
    DeviceBuffer<uint64_t> d_nodes;
    APGAR_B200_CUDA("cudaMalloc(queries)", d_q.ensure(query_count));
    APGAR_B200_CUDA("cudaMalloc(policy)", d_pol.ensure(std::max<uint64_t>(policy_edge_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(selected)", d_sel.ensure(selected.size()));
    APGAR_B200_CUDA("cudaMalloc(visited)", d_visited.ensure(chunk * words));
    APGAR_B200_CUDA("cudaMalloc(queues)", d_queues.ensure(chunk * 2u * n));
    APGAR_B200_CUDA("cudaMalloc(reached)", d_reached.ensure(selected.size()));
    APGAR_B200_CUDA("cudaMalloc(reach nodes)", d_nodes.ensure(selected.size()));
    APGAR_B200_CUDA("cudaMemcpy(queries)", cudaMemcpy(d_q.get(), queries, query_count * sizeof(*queries), cudaMemcpyHostToDevice));
    if (policy_edge_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(policy)", cudaMemcpy(d_pol.get(), policy_edges, policy_edge_count * sizeof(*policy_edges), cudaMemcpyHostToDevice));
    }
    APGAR_B200_CUDA("cudaMemcpy(selected)", cudaMemcpy(d_sel.get(), selected.data(), selected.size() * 4, cudaMemcpyHostToDevice));
    for (uint64_t first = 0; first < selected.size(); first += chunk) {
      ReachLaunch L{};
      L.neighbors = v->neighbors.get();
      L.legal = v->legal_dev.get();
      L.node_count = static_cast<uint32_t>(n);
      L.queries = d_q.get();
      L.policy = d_pol.get();
      L.selected = d_sel.get() + first;
      L.count = static_cast<uint32_t>(std::min<uint64_t>(chunk, selected.size() - first));
      L.visited = d_visited.get();
      L.queues = d_queues.get();
      L.reached = d_reached.get() + first;
      L.reach_nodes = d_nodes.get() + first;
      APGAR_B200_CUDA("reachability launch", launch_reach(L, nullptr));
    }
    std::vector<uint32_t> reached(selected.size());
    std::vector<uint64_t> reach_nodes(selected.size());
    APGAR_B200_CUDA("cudaMemcpy(reached)", cudaMemcpy(reached.data(), d_reached.get(), reached.size() * 4, cudaMemcpyDeviceToHost));
    APGAR_B200_CUDA("cudaMemcpy(reach nodes)", cudaMemcpy(reach_nodes.data(), d_nodes.get(), reach_nodes.size() * 8, cudaMemcpyDeviceToHost));
    for (size_t k = 0; k < selected.size(); ++k) {
      const uint32_t i = selected[k];
      apgar_b200_disconnect_verdict& out = verdicts[i];
      out.reachable_nodes = reach_nodes[k];
      if (reached[k] != 0u) {
        out.code = APGAR_B200_DISCONNECT_REACHABLE;
        continue;
      }
      // every reachable state's exact cost is at most (states - 1) transitions,
      // so no checked add of the CPU search can leave the finite range when
      // (8 * nodes + 1) * max transition stays finite
      const u128 states = 8u * static_cast<u128>(reach_nodes[k]) + 1u;
      const u128 t = max_transition[i];
      const bool bounded = t == 0 || states <= kMaxFinite / t;
      out.code = bounded ? APGAR_B200_DISCONNECT_CONFIRMED : APGAR_B200_DISCONNECT_UNBOUNDED;
    }
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during disconnected confirmation");
  }
}

extern "C" int apgar_b200_path_segments(void* view, const apgar_b200_compact_path_v1* paths,
                                        uint32_t path_count, const uint32_t* path_states,
                                        uint64_t path_state_count, apgar_b200_segment* segments,
                                        uint64_t segment_capacity, uint32_t* segment_counts) {
  if (view == nullptr || (path_count > 0 && (paths == nullptr || segment_counts == nullptr)) ||
      (path_state_count > 0 && (path_states == nullptr || segments == nullptr))) {
    return invariant("path segments received a null argument");
  }
  if (segment_capacity < path_state_count) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "segment output is smaller than the path states");
  }
  auto* v = static_cast<ViewObject*>(view);
  if (int rc = check_device(v->device); rc != APGAR_B200_OK) return rc;
  try {
    DeviceBuffer<apgar_b200_compact_path_v1> d_paths;
    DeviceBuffer<uint32_t> d_states, d_counts;
    DeviceBuffer<apgar_b200_segment> d_segs;
    APGAR_B200_CUDA("cudaMalloc(paths)", d_paths.ensure(std::max<uint32_t>(path_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(states)", d_states.ensure(std::max<uint64_t>(path_state_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(counts)", d_counts.ensure(std::max<uint32_t>(path_count, 1)));
    APGAR_B200_CUDA("cudaMalloc(segments)", d_segs.ensure(std::max<uint64_t>(path_state_count, 1)));
    if (path_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(paths)", cudaMemcpy(d_paths.get(), paths, path_count * sizeof(*paths), cudaMemcpyHostToDevice));
    }
    if (path_state_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(states)", cudaMemcpy(d_states.get(), path_states, path_state_count * 4, cudaMemcpyHostToDevice));
    }
    APGAR_B200_CUDA("path segments launch",
                    launch_path_segments(v->nodes_dev.get(), static_cast<uint32_t>(v->legal.size()),
                                         v->header.lattice_origin_x, v->header.lattice_origin_y,
                                         v->header.lattice_step, d_paths.get(), d_states.get(),
                                         path_state_count, path_count, d_segs.get(), d_counts.get(),
                                         nullptr));
    if (path_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(counts)", cudaMemcpy(segment_counts, d_counts.get(), path_count * 4, cudaMemcpyDeviceToHost));
    }
    if (path_state_count > 0) {
      APGAR_B200_CUDA("cudaMemcpy(segments)", cudaMemcpy(segments, d_segs.get(), path_state_count * sizeof(apgar_b200_segment), cudaMemcpyDeviceToHost));
    }
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during path segments");
  }
}
