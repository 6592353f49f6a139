// Drop-in IPlanarRouteBackend over the apgar_b200 C ABI.
//
// This file takes the place of the reference's CUDA translation unit
// (gpu/cuda/planar_router.cu) in a build of the reference: it defines the
// private constructor of the final wrapper CudaPlanarRouteBackend and the
// factory CreateCudaPlanarRouteBackend() (include/apgar/gpu/cuda_backend.h:10;
// the reference defines both at gpu/cuda/planar_router.cu:2861-2863), and
// installs B200PlanarRouteBackend as the wrapper's implementation.  Callers
// keep using the reference's own interface (include/apgar/gpu/planar_router.h
// :543-560); nothing of CUDA crosses it.
//
// The record types cross unchanged: the static_asserts below pin the C ABI's
// V1 records to the reference's, field by field, so vectors are passed as
// plain pointers.  Error codes map 1:1 (apgar_b200_status 1..4 are
// BackendErrorCode's four values in order).
//
// Build: compiled as C++20 against the reference's include/ tree and linked
// with libapgar_b200.so (apgar_b200/adapter/build_adapter.sh).
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstring>
#include <memory>
#include <string>
#include <utility>
#include <variant>
#include <vector>

#include "apgar/gpu/cuda_backend.h"
#include "apgar/gpu/planar_router.h"
#include "apgar_b200.h"

namespace apgar::gpu {
namespace {

// ---- record layouts: the C ABI's V1 structs are the reference's, byte for byte ----
#define APGAR_B200_SAME_FIELD(ours, theirs, a, b) \
  static_assert(offsetof(ours, a) == offsetof(theirs, b), #theirs "::" #b " offset")
static_assert(sizeof(apgar_b200_compiled_header_v1) == sizeof(DeviceCompiledHeaderV1));
APGAR_B200_SAME_FIELD(apgar_b200_compiled_header_v1, DeviceCompiledHeaderV1, represented_nodes,
                      represented_nodes);
APGAR_B200_SAME_FIELD(apgar_b200_compiled_header_v1, DeviceCompiledHeaderV1, lattice_origin_x,
                      lattice_origin);
APGAR_B200_SAME_FIELD(apgar_b200_compiled_header_v1, DeviceCompiledHeaderV1, orthogonal_step, costs);
APGAR_B200_SAME_FIELD(apgar_b200_compiled_header_v1, DeviceCompiledHeaderV1, heading_mask,
                      heading_mask);
static_assert(sizeof(apgar_b200_layer_range_v1) == sizeof(DeviceLayerRangeV1));
APGAR_B200_SAME_FIELD(apgar_b200_layer_range_v1, DeviceLayerRangeV1, node_count, node_count);
APGAR_B200_SAME_FIELD(apgar_b200_layer_range_v1, DeviceLayerRangeV1, minimum_lattice_x,
                      minimum_lattice_x);
static_assert(sizeof(apgar_b200_node_v1) == sizeof(DeviceNodeV1));
APGAR_B200_SAME_FIELD(apgar_b200_node_v1, DeviceNodeV1, layer, layer);
APGAR_B200_SAME_FIELD(apgar_b200_node_v1, DeviceNodeV1, legal_edges, legal_edges);
APGAR_B200_SAME_FIELD(apgar_b200_node_v1, DeviceNodeV1, neighbors, neighbors);
static_assert(sizeof(apgar_b200_run_v1) == sizeof(DeviceRunV1));
APGAR_B200_SAME_FIELD(apgar_b200_run_v1, DeviceRunV1, direction, direction);
static_assert(sizeof(apgar_b200_policy_edge_v1) == sizeof(DeviceCandidatePolicyEdgeV1));
APGAR_B200_SAME_FIELD(apgar_b200_policy_edge_v1, DeviceCandidatePolicyEdgeV1, adjustment, adjustment);
static_assert(sizeof(apgar_b200_batch_query_v1) == sizeof(DeviceCandidateBatchQueryV1));
APGAR_B200_SAME_FIELD(apgar_b200_batch_query_v1, DeviceCandidateBatchQueryV1, start_node, start_node);
APGAR_B200_SAME_FIELD(apgar_b200_batch_query_v1, DeviceCandidateBatchQueryV1, workspace_offset,
                      workspace_offset);
APGAR_B200_SAME_FIELD(apgar_b200_batch_query_v1, DeviceCandidateBatchQueryV1, bend_surcharge,
                      bend_surcharge);
APGAR_B200_SAME_FIELD(apgar_b200_batch_query_v1, DeviceCandidateBatchQueryV1, generator, generator);
static_assert(sizeof(apgar_b200_batch_result_v1) == sizeof(DeviceCandidateBatchResultV1));
APGAR_B200_SAME_FIELD(apgar_b200_batch_result_v1, DeviceCandidateBatchResultV1, goal_state, goal_state);
APGAR_B200_SAME_FIELD(apgar_b200_batch_result_v1, DeviceCandidateBatchResultV1, completion, completion);
APGAR_B200_SAME_FIELD(apgar_b200_batch_result_v1, DeviceCandidateBatchResultV1, examined_work,
                      examined_work);
static_assert(sizeof(apgar_b200_compact_path_v1) == sizeof(DeviceCandidateCompactPathV1));
APGAR_B200_SAME_FIELD(apgar_b200_compact_path_v1, DeviceCandidateCompactPathV1, state_offset,
                      state_offset);
static_assert(sizeof(apgar_b200_route_result_header_v1) == sizeof(DeviceRouteResultHeaderV1));
APGAR_B200_SAME_FIELD(apgar_b200_route_result_header_v1, DeviceRouteResultHeaderV1, generator,
                      generator);
#undef APGAR_B200_SAME_FIELD

// The C ABI samples a cancellation byte; std::atomic_bool is that byte.
static_assert(sizeof(std::atomic_bool) == 1 && std::atomic_bool::is_always_lock_free);

const volatile std::uint8_t* cancel_byte(const std::atomic_bool* flag) {
  return reinterpret_cast<const volatile std::uint8_t*>(flag);
}

BackendError last_error(int status) {
  char buf[1024];
  apgar_b200_last_error(buf, sizeof(buf));
  BackendErrorCode code = BackendErrorCode::kInternalInvariant;
  switch (status) {
    case APGAR_B200_UNSUPPORTED: code = BackendErrorCode::kUnsupported; break;
    case APGAR_B200_RESOURCE_EXHAUSTED: code = BackendErrorCode::kResourceExhausted; break;
    case APGAR_B200_BACKEND_FAILURE: code = BackendErrorCode::kBackendFailure; break;
    default: code = BackendErrorCode::kInternalInvariant; break;
  }
  return BackendError{code, std::string("apgar_b200: ") + buf};
}

BackendError invariant(const char* what) {
  return BackendError{BackendErrorCode::kInternalInvariant, what};
}

CandidateBatchTelemetry telemetry_of(const apgar_b200_batch_telemetry& t,
                                     std::uint64_t batch_host_bytes, std::uint32_t chunk_rounds) {
  CandidateBatchTelemetry out;
  out.persistent_device_bytes = t.persistent_device_bytes;
  out.batch_device_bytes = t.batch_device_bytes;
  out.workspace_capacity_device_bytes = t.workspace_capacity_device_bytes;
  out.peak_device_bytes = t.peak_device_bytes;
  out.batch_host_bytes = batch_host_bytes;
  out.device_to_host_readback_bytes = t.device_to_host_readback_bytes;
  out.kernel_launch_count = t.kernel_launch_count;
  out.blocking_status_readback_count = t.blocking_status_readback_count;
  out.dispatched_rounds = t.dispatched_rounds;
  out.finalization_launch_count = t.finalization_launch_count;
  out.chunk_rounds = chunk_rounds;
  out.kernel_milliseconds = t.kernel_milliseconds;
  return out;
}

// ---- opaque handles (the reference's UploadedCompiledView / Pending* roles) ----
class B200UploadedView final : public UploadedCompiledView {
 public:
  B200UploadedView(void* handle, std::uint64_t represented_states)
      : handle_(handle), represented_states_(represented_states) {}
  ~B200UploadedView() override { apgar_b200_view_release(handle_); }
  void* handle() const { return handle_; }
  std::uint64_t represented_states() const { return represented_states_; }

 private:
  void* handle_;
  std::uint64_t represented_states_;
};

class B200PendingBatch final : public PendingCandidateBatchExecution {
 public:
  B200PendingBatch(void* handle, const BackendCandidateBatchExecutionRequest& request,
                   std::uint64_t represented_states)
      : handle_(handle),
        batch_id_(request.batch_id),
        schema_version_(request.schema_version),
        generator_(request.generator),
        represented_states_(represented_states),
        policy_edges_(request.policy_edges.size()) {
    offsets_.reserve(request.queries.size());
    for (const DeviceCandidateBatchQueryV1& q : request.queries) {
      offsets_.emplace_back(q.workspace_offset, q.workspace_state_count);
    }
  }
  ~B200PendingBatch() override { apgar_b200_release_batch(handle_); }

  void* handle_;
  std::uint64_t batch_id_;
  std::uint32_t schema_version_;
  PlanarGenerator generator_;
  std::uint64_t represented_states_;
  std::uint64_t policy_edges_;
  std::vector<std::pair<std::uint64_t, std::uint64_t>> offsets_;  // workspace slice per query
};

class B200PendingRoute final : public PendingRouteExecution {
 public:
  B200PendingRoute(void* handle, std::uint64_t states) : handle_(handle), states_(states) {}
  ~B200PendingRoute() override { apgar_b200_release_route(handle_); }
  void* handle_;
  std::uint64_t states_;
};

// Readback form by generator value: the stock frontier and the added
// persistent-workspace generator return the full workspace, the others
// compact paths.  Values, not enumerator names, so that the shim builds
// against the stock header as well as the patched one.
bool full_workspace(PlanarGenerator generator) {
  return generator == PlanarGenerator::kBucketedFrontier ||
         static_cast<std::uint8_t>(generator) == APGAR_B200_GENERATOR_B200_PERSISTENT_WORKSPACE;
}

// ---- the backend ----
class B200PlanarRouteBackend final : public IPlanarRouteBackend {
 public:
  BackendMetadataResult QueryMetadata() const override {
    apgar_b200_metadata m{};
    if (int rc = apgar_b200_query_metadata(&m); rc != APGAR_B200_OK) return last_error(rc);
    BackendMetadata out;
    out.backend = "cuda";
    out.device_name = m.device_name;
    out.device_uuid = m.device_uuid;
    out.compute_capability_major = m.compute_capability_major;
    out.compute_capability_minor = m.compute_capability_minor;
    out.runtime_version = m.runtime_version;
    out.driver_version = m.driver_version;
    out.global_memory_bytes = m.global_memory_bytes;
    return out;
  }

  UploadResult UploadCompiledView(const DeviceCompiledBoardV1& board) override {
    void* handle = nullptr;
    const int rc = apgar_b200_view_upload(
        reinterpret_cast<const apgar_b200_compiled_header_v1*>(&board.header),
        reinterpret_cast<const apgar_b200_layer_range_v1*>(board.layers.data()), board.layers.size(),
        reinterpret_cast<const apgar_b200_node_v1*>(board.nodes.data()), board.nodes.size(),
        reinterpret_cast<const apgar_b200_run_v1*>(board.runs.data()), board.runs.size(),
        board.run_nodes.data(), board.run_nodes.size(), &handle);
    if (rc != APGAR_B200_OK) return last_error(rc);
    return std::unique_ptr<UploadedCompiledView>(
        std::make_unique<B200UploadedView>(handle, board.header.represented_states));
  }

  ExecutionResult ExecuteRoute(const UploadedCompiledView& board,
                               const BackendExecutionRequest& request) override {
    const auto* view = dynamic_cast<const B200UploadedView*>(&board);
    if (view == nullptr) return invariant("compiled view was not uploaded by this backend");
    void* handle = nullptr;
    const int rc = apgar_b200_execute_route(
        view->handle(), static_cast<std::uint8_t>(request.generator), request.start_node,
        request.goal_node, request.routing_profile_fingerprint, request.maximum_rounds,
        request.maximum_device_bytes, cancel_byte(request.cancellation), &handle);
    if (rc != APGAR_B200_OK) return last_error(rc);
    return std::unique_ptr<PendingRouteExecution>(
        std::make_unique<B200PendingRoute>(handle, view->represented_states()));
  }

  ReadbackResult ReadbackRoute(const PendingRouteExecution& execution) override {
    const auto* pending = dynamic_cast<const B200PendingRoute*>(&execution);
    if (pending == nullptr) return invariant("route execution does not belong to this backend");
    UntrustedKernelResult out;
    out.labels.resize(pending->states_);
    out.predecessors.resize(pending->states_);
    DeviceRouteResultHeaderV1 header;
    std::uint8_t completion = 0;
    apgar_b200_batch_telemetry t{};
    const int rc = apgar_b200_readback_route(
        pending->handle_, reinterpret_cast<apgar_b200_route_result_header_v1*>(&header), &completion,
        &out.goal_state, out.labels.data(), out.predecessors.data(), &t);
    if (rc != APGAR_B200_OK) return last_error(rc);
    out.schema_version = header.schema_version;
    out.source_board_content_hash = header.source_board_content_hash;
    out.compiler_profile_fingerprint = header.compiler_profile_fingerprint;
    out.routing_profile_fingerprint = header.routing_profile_fingerprint;
    out.compiler_version = header.compiler_version;
    out.rule_bucket_identity = header.rule_bucket_identity;
    out.device_view_fingerprint = header.device_view_fingerprint;
    out.generator = header.generator;
    out.completion = static_cast<KernelCompletion>(completion);
    out.start_node = header.start_node;
    out.goal_node = header.goal_node;
    out.telemetry.persistent_device_bytes = t.persistent_device_bytes;
    out.telemetry.batch_device_bytes = t.batch_device_bytes;
    out.telemetry.peak_device_bytes = t.peak_device_bytes;
    out.telemetry.rounds = t.dispatched_rounds;
    out.telemetry.kernel_milliseconds = t.kernel_milliseconds;
    return out;
  }

  CandidateBatchExecutionResult ExecuteCandidateBatch(
      const UploadedCompiledView& board,
      const BackendCandidateBatchExecutionRequest& request) override {
    const auto* view = dynamic_cast<const B200UploadedView*>(&board);
    if (view == nullptr) return invariant("compiled view was not uploaded by this backend");
    if (request.queries.size() > UINT32_MAX) return invariant("candidate batch is too large");
    apgar_b200_batch_request r{};
    r.schema_version = request.schema_version;
    r.generator = static_cast<std::uint8_t>(request.generator);
    r.batch_id = request.batch_id;
    r.maximum_rounds = request.maximum_rounds;
    r.maximum_workspace_states_per_query = request.maximum_workspace_states_per_query;
    r.maximum_frontier_states_per_query = request.maximum_frontier_states_per_query;
    r.maximum_device_bytes = request.maximum_device_bytes;
    r.maximum_host_bytes = request.maximum_host_bytes;
    void* handle = nullptr;
    const int rc = apgar_b200_execute_batch(
        view->handle(), &r, reinterpret_cast<const apgar_b200_batch_query_v1*>(request.queries.data()),
        static_cast<std::uint32_t>(request.queries.size()),
        reinterpret_cast<const apgar_b200_policy_edge_v1*>(request.policy_edges.data()),
        request.policy_edges.size(), cancel_byte(request.cancellation), &handle);
    if (rc != APGAR_B200_OK) return last_error(rc);
    return std::unique_ptr<PendingCandidateBatchExecution>(
        std::make_unique<B200PendingBatch>(handle, request, view->represented_states()));
  }

  CandidateBatchReadbackResult ReadbackCandidateBatch(
      const PendingCandidateBatchExecution& execution) override {
    const auto* p = dynamic_cast<const B200PendingBatch*>(&execution);
    if (p == nullptr) return invariant("candidate batch does not belong to this backend");
    const std::size_t query_count = p->offsets_.size();
    std::vector<DeviceCandidateBatchResultV1> headers(query_count);
    std::vector<DeviceCandidateCompactPathV1> compact(query_count);
    const bool workspace = full_workspace(p->generator_);
    UntrustedCandidateBatchResult out;
    out.schema_version = p->schema_version_;
    out.batch_id = p->batch_id_;
    out.generator = p->generator_;
    out.readback_kind = workspace ? CandidateBatchReadbackKind::kFullWorkspace
                                  : CandidateBatchReadbackKind::kCompactPaths;
    apgar_b200_batch_telemetry t{};
    std::uint64_t path_states = 0;
    // first pass: headers, compact headers and the packed path length
    int rc = apgar_b200_readback_batch(
        p->handle_, reinterpret_cast<apgar_b200_batch_result_v1*>(headers.data()),
        workspace ? nullptr : reinterpret_cast<apgar_b200_compact_path_v1*>(compact.data()), nullptr,
        0, &path_states, &t);
    if (rc != APGAR_B200_OK) return last_error(rc);
    if (workspace) {
      const std::uint64_t per_query = p->represented_states_;
      std::vector<std::uint64_t> labels(query_count * per_query), owners(query_count * per_query),
          pred_owners(query_count * per_query);
      std::vector<std::uint32_t> preds(query_count * per_query);
      rc = apgar_b200_readback_batch_workspace(p->handle_, labels.data(), preds.data(), owners.data(),
                                               pred_owners.data());
      if (rc != APGAR_B200_OK) return last_error(rc);
      // the workspace arrays just read are part of this readback
      t.device_to_host_readback_bytes +=
          query_count * per_query *
          (sizeof(std::uint64_t) + sizeof(std::uint32_t) + 2 * sizeof(std::uint64_t));
      // place each query's rows at the workspace slice its request named
      std::uint64_t extent = 0;
      for (const auto& [offset, count] : p->offsets_) extent = std::max(extent, offset + count);
      out.labels.assign(extent, kInfiniteRouteCost);
      out.predecessors.assign(extent, kInvalidStateIndex);
      out.state_owners.assign(extent, 0);
      out.predecessor_owners.assign(extent, 0);
      for (std::size_t i = 0; i < query_count; ++i) {
        const auto [offset, count] = p->offsets_[i];
        const std::uint64_t n = std::min(count, per_query);
        std::copy_n(labels.begin() + i * per_query, n, out.labels.begin() + offset);
        std::copy_n(preds.begin() + i * per_query, n, out.predecessors.begin() + offset);
        std::copy_n(owners.begin() + i * per_query, n, out.state_owners.begin() + offset);
        std::copy_n(pred_owners.begin() + i * per_query, n, out.predecessor_owners.begin() + offset);
      }
    } else if (path_states > 0) {
      out.compact_path_states.resize(path_states);
      rc = apgar_b200_readback_batch(
          p->handle_, reinterpret_cast<apgar_b200_batch_result_v1*>(headers.data()),
          reinterpret_cast<apgar_b200_compact_path_v1*>(compact.data()),
          out.compact_path_states.data(), path_states, &path_states, &t);
      if (rc != APGAR_B200_OK) return last_error(rc);
    }
    const std::optional<PlanarGeneratorDescriptor> descriptor =
        DescribePlanarGenerator(p->generator_);
    const std::optional<std::uint64_t> host_bytes = EstimateCandidateBatchHostBytesV1(
        query_count, p->policy_edges_, p->represented_states_, p->generator_);
    out.telemetry = telemetry_of(t, host_bytes.value_or(0),
                                 descriptor ? descriptor->chunk_rounds : t.dispatched_rounds);
    out.queries.reserve(query_count);
    for (std::size_t i = 0; i < query_count; ++i) {
      UntrustedCandidateBatchQueryResult q;
      q.header = headers[i];
      q.workspace_offset = p->offsets_[i].first;
      q.workspace_state_count = p->offsets_[i].second;
      if (!workspace) q.compact_path = compact[i];
      q.telemetry.examined_work = headers[i].examined_work;
      q.telemetry.heading_turn_relaxations = headers[i].heading_turn_relaxations;
      q.telemetry.rounds = headers[i].rounds;
      out.queries.push_back(std::move(q));
    }
    return out;
  }
};

}  // namespace

CudaPlanarRouteBackend::CudaPlanarRouteBackend()
    : implementation_(std::make_unique<B200PlanarRouteBackend>()) {}

std::unique_ptr<IPlanarRouteBackend> CreateCudaPlanarRouteBackend() {
  return std::unique_ptr<IPlanarRouteBackend>(new CudaPlanarRouteBackend());
}

}  // namespace apgar::gpu
