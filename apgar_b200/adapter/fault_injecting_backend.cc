// Host-side fault injection over any IPlanarRouteBackend (the shim included).
//
// TEST INFRASTRUCTURE.  This defines the factories the reference declares in
// include/apgar/gpu/fault_injecting_backend.h:43-57 (its own implementation is
// src/gpu/fault_injecting_backend.cc:83-230).  A decorator forwards every call
// to the wrapped backend and corrupts only the untrusted readback on the host,
// after the device work is done, so no GPU state is ever touched: the point is
// to show that the reference's host validation (planar_router.cc) rejects each
// corruption of this backend's results with the invariant id it names for
// that class.  Each fault corrupts the first query of a batch (or the single
// route), the batch envelope, or the telemetry, as its class describes:
//
//   class                 corruption                                  invariant raised
//   kWorkspaceBounds      query's workspace state count off by one     gpu.batch.workspace.bounds.v1
//   kWorkspaceOwner       one state owner in the query's slice         gpu.batch.workspace.owner.v1
//   kQueryTelemetry       header rounds disagree with telemetry        gpu.batch.query.telemetry.v1
//   kMemoryAccounting     batch host bytes off by one                  gpu.batch.memory.accounting.v1
//   kBatchTelemetry       one extra kernel launch reported             gpu.batch.telemetry.v1
//   kQueryIdentity        query id changed                             gpu.batch.query.identity.v1
//   kFalseDisconnected    a reached query reported disconnected        gpu.disconnected.cpu_reachable.v1
//   kCompactPathBounds    compact-path schema version changed          gpu.batch.compact_path.bounds.v1
//   kCompactPathEndpoint  the path's goal state made invalid           gpu.batch.compact_path.endpoint.v1
//   kCompactPathCycle     one state repeated                           gpu.batch.compact_path.cycle.v1
//   kCompactPathHeading   an interior state given the start heading    gpu.batch.compact_path.heading.v1
//   kCompactPathEdge      an interior state given another heading      gpu.batch.compact_path.edge.v1
//   kGoalPredecessorSelfCycle (route)  goal state its own predecessor  gpu.predecessor.self_reference.v1
#include <algorithm>
#include <cstdint>
#include <limits>
#include <memory>
#include <span>
#include <variant>

#include "apgar/gpu/fault_injecting_backend.h"

namespace apgar::gpu {
namespace {

constexpr std::uint32_t kHeadings = 9;       // incoming headings per node (8 = none)
constexpr std::uint32_t kStartHeading = 8;   // the start state's "no incoming heading"

template <typename T>
T bumped(T v) {
  return v == std::numeric_limits<T>::max() ? v - 1 : v + 1;
}

// The query's rows of a query-major workspace array (empty if out of range).
template <typename T>
std::span<T> slice_of(std::vector<T>& rows, const UntrustedCandidateBatchQueryResult& q) {
  if (q.workspace_offset > rows.size() || q.workspace_state_count > rows.size() - q.workspace_offset) {
    return {};
  }
  return std::span<T>(rows).subspan(static_cast<std::size_t>(q.workspace_offset),
                                    static_cast<std::size_t>(q.workspace_state_count));
}

// The query's reverse compact path (goal first), empty without one.
std::span<std::uint32_t> path_of(UntrustedCandidateBatchResult& r,
                                 const UntrustedCandidateBatchQueryResult& q) {
  if (!q.compact_path.has_value()) return {};
  const std::uint64_t at = q.compact_path->state_offset, n = q.compact_path->state_count;
  if (at > r.compact_path_states.size() || n > r.compact_path_states.size() - at) return {};
  return std::span<std::uint32_t>(r.compact_path_states)
      .subspan(static_cast<std::size_t>(at), static_cast<std::size_t>(n));
}

bool holds(std::span<const std::uint32_t> states, std::uint32_t s) {
  return std::find(states.begin(), states.end(), s) != states.end();
}

void corrupt(UntrustedCandidateBatchResultFault fault, UntrustedCandidateBatchResult& r) {
  if (r.queries.empty()) return;
  UntrustedCandidateBatchQueryResult& q = r.queries.front();
  using F = UntrustedCandidateBatchResultFault;
  switch (fault) {
    case F::kNone:
      return;
    case F::kWorkspaceBounds:
      q.workspace_state_count = q.workspace_state_count > 0 ? q.workspace_state_count - 1 : 1;
      return;
    case F::kWorkspaceOwner: {
      const std::span<std::uint64_t> owners = slice_of(r.state_owners, q);
      if (!owners.empty()) owners[0] = bumped(q.header.workspace_owner);
      return;
    }
    case F::kQueryTelemetry:
      q.header.rounds = bumped(q.telemetry.rounds);
      return;
    case F::kMemoryAccounting:
      r.telemetry.batch_host_bytes = bumped(r.telemetry.batch_host_bytes);
      return;
    case F::kBatchTelemetry:
      r.telemetry.kernel_launch_count = bumped(r.telemetry.kernel_launch_count);
      return;
    case F::kQueryIdentity:
      q.header.query_id = q.header.query_id == std::numeric_limits<std::uint64_t>::max()
                              ? 0
                              : q.header.query_id + 1;
      return;
    case F::kFalseDisconnected: {
      // a consistent-looking DISCONNECTED result: only the start is labelled
      q.header.completion = KernelCompletion::kDisconnected;
      q.header.goal_state = kInvalidStateIndex;
      const std::span<std::uint64_t> labels = slice_of(r.labels, q);
      const std::span<std::uint32_t> preds = slice_of(r.predecessors, q);
      std::fill(labels.begin(), labels.end(), kInfiniteRouteCost);
      std::fill(preds.begin(), preds.end(), kInvalidStateIndex);
      const std::uint64_t start = static_cast<std::uint64_t>(q.header.start_node) * kHeadings + kStartHeading;
      if (start < labels.size()) labels[static_cast<std::size_t>(start)] = 0;
      return;
    }
    case F::kCompactPathBounds:
      if (q.compact_path.has_value()) q.compact_path->schema_version = bumped(q.compact_path->schema_version);
      return;
    case F::kCompactPathEndpoint: {
      const std::span<std::uint32_t> p = path_of(r, q);
      if (!p.empty()) p[0] = kInvalidStateIndex;
      return;
    }
    case F::kCompactPathCycle: {
      const std::span<std::uint32_t> p = path_of(r, q);
      if (p.size() >= 4) p[1] = p[2];
      return;
    }
    case F::kCompactPathHeading: {
      // the first interior state (not on the start node) whose start-heading
      // twin is not on the path already
      const std::span<std::uint32_t> p = path_of(r, q);
      for (std::size_t i = 1; i + 1 < p.size(); ++i) {
        const std::uint32_t node = p[i] / kHeadings;
        const std::uint32_t twin = node * kHeadings + kStartHeading;
        if (node != q.header.start_node && !holds(p, twin)) {
          p[i] = twin;
          return;
        }
      }
      return;
    }
    case F::kCompactPathEdge: {
      // the first interior state that has another planar heading not on the path
      const std::span<std::uint32_t> p = path_of(r, q);
      for (std::size_t i = 1; i + 1 < p.size(); ++i) {
        const std::uint32_t node = p[i] / kHeadings, heading = p[i] % kHeadings;
        for (std::uint32_t h = 0; h < 8; ++h) {
          const std::uint32_t other = node * kHeadings + h;
          if (h != heading && !holds(p, other)) {
            p[i] = other;
            return;
          }
        }
      }
      return;
    }
  }
}

// Forwards every call; corrupts readbacks after the wrapped backend returns.
class FaultDecorator final : public IPlanarRouteBackend {
 public:
  FaultDecorator(IPlanarRouteBackend& inner, std::optional<UntrustedResultFault> route_fault,
                 UntrustedCandidateBatchResultFault batch_fault)
      : inner_(inner), route_fault_(route_fault), batch_fault_(batch_fault) {}

  BackendMetadataResult QueryMetadata() const override { return inner_.QueryMetadata(); }
  UploadResult UploadCompiledView(const DeviceCompiledBoardV1& board) override {
    return inner_.UploadCompiledView(board);
  }
  ExecutionResult ExecuteRoute(const UploadedCompiledView& board,
                               const BackendExecutionRequest& request) override {
    return inner_.ExecuteRoute(board, request);
  }
  ReadbackResult ReadbackRoute(const PendingRouteExecution& execution) override {
    ReadbackResult rb = inner_.ReadbackRoute(execution);
    auto* k = std::get_if<UntrustedKernelResult>(&rb);
    if (k != nullptr && route_fault_ == UntrustedResultFault::kGoalPredecessorSelfCycle &&
        k->completion == KernelCompletion::kReached && k->goal_state < k->predecessors.size()) {
      k->predecessors[k->goal_state] = k->goal_state;
    }
    return rb;
  }
  CandidateBatchExecutionResult ExecuteCandidateBatch(
      const UploadedCompiledView& board, const BackendCandidateBatchExecutionRequest& request) override {
    return inner_.ExecuteCandidateBatch(board, request);
  }
  CandidateBatchReadbackResult ReadbackCandidateBatch(
      const PendingCandidateBatchExecution& execution) override {
    CandidateBatchReadbackResult rb = inner_.ReadbackCandidateBatch(execution);
    if (auto* r = std::get_if<UntrustedCandidateBatchResult>(&rb)) corrupt(batch_fault_, *r);
    return rb;
  }

 private:
  IPlanarRouteBackend& inner_;
  std::optional<UntrustedResultFault> route_fault_;
  UntrustedCandidateBatchResultFault batch_fault_;
};

}  // namespace

std::unique_ptr<IPlanarRouteBackend> CreateFaultInjectingPlanarRouteBackend(
    IPlanarRouteBackend& inner, UntrustedResultFault fault) {
  return std::make_unique<FaultDecorator>(inner, fault, UntrustedCandidateBatchResultFault::kNone);
}

std::unique_ptr<IPlanarRouteBackend> CreateFaultInjectingCandidateBatchBackend(
    IPlanarRouteBackend& inner, UntrustedCandidateBatchResultFault fault) {
  return std::make_unique<FaultDecorator>(inner, std::nullopt, fault);
}

}  // namespace apgar::gpu
