// GPU check of the drop-in shim through the reference's own interface.
//
// TEST INFRASTRUCTURE.  Built by apgar_b200/adapter/build_adapter.sh against
// the reference headers.  For every golden fixture case
// (tests/golden/ref_corpus/*.bin, written by the reference's corpus builders
// and CPU A*) it:
//  1. uploads the reference DeviceCompiledBoardV1 through
//     CreateCudaPlanarRouteBackend() and checks the metadata;
//  2. runs the batch with the frontier generator (full workspace) and checks
//     every query's completion and goal label against the reference CPU A*
//     outcome;
//  3. runs the same batch with the sweep generator (compact paths) and checks
//     each compact path against the path the frontier's canonical
//     predecessors give;
//  4. runs ExecuteRoute / ReadbackRoute for the first query and checks its
//     goal label.
// Prints "adapter ok: ..." and exits 0 when every check holds.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <memory>
#include <optional>
#include <string>
#include <variant>
#include <vector>

#include "apgar/gpu/cuda_backend.h"
#include "apgar/gpu/planar_router.h"

using namespace apgar::gpu;

namespace {

struct FixtureQuery {
  std::uint32_t start = 0, goal = 0;
  std::uint64_t orth = 0, diag = 0, bend = 0, policy_identity = 0;
  std::uint32_t cpu_status = 0;
  std::uint64_t cpu_cost = 0;
  std::vector<DeviceCandidatePolicyEdgeV1> policy;
};

struct Fixture {
  std::string name;
  DeviceCompiledBoardV1 board;
  std::vector<FixtureQuery> queries;
};

class Reader {
 public:
  explicit Reader(std::vector<char> data) : data_(std::move(data)) {}
  template <typename T>
  T get() {
    T v{};
    take(&v, sizeof(T));
    return v;
  }
  void take(void* out, std::size_t n) {
    if (pos_ + n > data_.size()) throw std::runtime_error("truncated fixture");
    std::memcpy(out, data_.data() + pos_, n);
    pos_ += n;
  }
  template <typename T>
  std::vector<T> array() {
    std::vector<T> v(get<std::uint64_t>());
    if (!v.empty()) take(v.data(), v.size() * sizeof(T));
    return v;
  }

 private:
  std::vector<char> data_;
  std::size_t pos_ = 0;
};

Fixture load(const std::filesystem::path& path) {
  std::ifstream in(path, std::ios::binary);
  Reader r(std::vector<char>((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>()));
  if (r.get<std::uint64_t>() != 0x3158495446524741ull) throw std::runtime_error("bad magic");
  Fixture f;
  f.name = path.stem().string();
  r.take(&f.board.header, sizeof(f.board.header));
  f.board.layers = r.array<DeviceLayerRangeV1>();
  f.board.nodes = r.array<DeviceNodeV1>();
  f.board.runs = r.array<DeviceRunV1>();
  f.board.run_nodes = r.array<std::uint32_t>();
  const std::uint64_t count = r.get<std::uint64_t>();
  for (std::uint64_t i = 0; i < count; ++i) {
    FixtureQuery q;
    q.start = r.get<std::uint32_t>();
    q.goal = r.get<std::uint32_t>();
    q.orth = r.get<std::uint64_t>();
    q.diag = r.get<std::uint64_t>();
    q.bend = r.get<std::uint64_t>();
    q.policy_identity = r.get<std::uint64_t>();
    q.cpu_status = r.get<std::uint32_t>();
    r.get<std::uint32_t>();
    q.cpu_cost = r.get<std::uint64_t>();
    q.policy = r.array<DeviceCandidatePolicyEdgeV1>();
    f.queries.push_back(std::move(q));
  }
  return f;
}

BackendCandidateBatchExecutionRequest make_request(const Fixture& f, PlanarGenerator generator) {
  BackendCandidateBatchExecutionRequest req;
  req.batch_id = 7;
  req.generator = generator;
  req.maximum_rounds = 100000;
  const std::uint64_t states = 9ull * f.board.nodes.size();
  std::uint32_t offset = 0;
  for (std::size_t i = 0; i < f.queries.size(); ++i) {
    const FixtureQuery& fq = f.queries[i];
    DeviceCandidateBatchQueryV1 q;
    q.input_ordinal = static_cast<std::uint32_t>(i);
    q.batch_id = req.batch_id;
    q.query_id = i + 1;
    q.workspace_owner = i + 1;
    q.policy_identity = fq.policy_identity;
    q.start_node = fq.start;
    q.goal_node = fq.goal;
    q.policy_offset = offset;
    q.policy_count = static_cast<std::uint32_t>(fq.policy.size());
    q.workspace_offset = i * states;
    q.workspace_state_count = states;
    q.frontier_state_capacity = generator == PlanarGenerator::kBucketedFrontier ? states : 0;
    q.orthogonal_step_surcharge = fq.orth;
    q.diagonal_step_surcharge = fq.diag;
    q.bend_surcharge = fq.bend;
    q.maximum_rounds = req.maximum_rounds;
    q.generator = generator;
    req.queries.push_back(q);
    req.policy_edges.insert(req.policy_edges.end(), fq.policy.begin(), fq.policy.end());
    offset += q.policy_count;
  }
  return req;
}

int failures = 0;
void check(bool ok, const std::string& what) {
  if (!ok) {
    ++failures;
    std::fprintf(stderr, "FAIL: %s\n", what.c_str());
  }
}

template <typename V>
bool is_error(const V& v, const char* stage) {
  if (std::holds_alternative<BackendError>(v)) {
    std::fprintf(stderr, "FAIL: %s: %s\n", stage, std::get<BackendError>(v).detail.c_str());
    ++failures;
    return true;
  }
  return false;
}

// Executes and reads back one batch.  The pending execution holds the view's
// execution lease until it is destroyed (as in the reference), so it must not
// outlive its readback when the same view runs another batch.
std::optional<UntrustedCandidateBatchResult> run_batch(IPlanarRouteBackend& backend,
                                                       const UploadedCompiledView& view,
                                                       const BackendCandidateBatchExecutionRequest& req,
                                                       const char* stage) {
  CandidateBatchExecutionResult ex = backend.ExecuteCandidateBatch(view, req);
  if (is_error(ex, stage)) return std::nullopt;
  CandidateBatchReadbackResult rb =
      backend.ReadbackCandidateBatch(*std::get<std::unique_ptr<PendingCandidateBatchExecution>>(ex));
  if (is_error(rb, stage)) return std::nullopt;
  return std::move(std::get<UntrustedCandidateBatchResult>(rb));
}

}  // namespace

int main(int argc, char** argv) {
  const std::filesystem::path dir = argc > 1 ? argv[1] : "tests/golden/ref_corpus";
  std::unique_ptr<IPlanarRouteBackend> backend = CreateCudaPlanarRouteBackend();
  const BackendMetadataResult meta = backend->QueryMetadata();
  if (is_error(meta, "QueryMetadata")) return 1;
  check(std::get<BackendMetadata>(meta).backend == "cuda", "metadata backend name");
  check(std::get<BackendMetadata>(meta).compute_capability_major >= 10, "compute capability");
  std::vector<std::filesystem::path> files;
  for (const auto& e : std::filesystem::directory_iterator(dir)) {
    // device-view cases only: the directory also holds reference outputs
    // (segments, clearance verdicts, compile inputs) under other magics
    if (e.path().extension() != ".bin") continue;
    std::ifstream probe(e.path(), std::ios::binary);
    std::uint64_t magic = 0;
    probe.read(reinterpret_cast<char*>(&magic), sizeof(magic));
    if (magic == 0x3158495446524741ull) files.push_back(e.path());
  }
  std::sort(files.begin(), files.end());
  std::size_t cases = 0, queries = 0;
  for (const auto& path : files) {
    const Fixture f = load(path);
    UploadResult up = backend->UploadCompiledView(f.board);
    if (is_error(up, "UploadCompiledView")) continue;
    const UploadedCompiledView& view = *std::get<std::unique_ptr<UploadedCompiledView>>(up);
    // frontier generator: full workspace, goal labels against the CPU A*
    const auto full_run = run_batch(*backend, view, make_request(f, PlanarGenerator::kBucketedFrontier),
                                    "candidate batch (frontier)");
    if (!full_run) continue;
    const UntrustedCandidateBatchResult& full = *full_run;
    check(full.readback_kind == CandidateBatchReadbackKind::kFullWorkspace, f.name + " readback kind");
    check(full.queries.size() == f.queries.size(), f.name + " query count");
    // sweep generator: compact paths
    const auto compact_run = run_batch(*backend, view,
                                       make_request(f, PlanarGenerator::kHeadingAwareSweep),
                                       "candidate batch (sweep)");
    if (!compact_run) continue;
    const UntrustedCandidateBatchResult& compact = *compact_run;
    check(compact.readback_kind == CandidateBatchReadbackKind::kCompactPaths, f.name + " compact kind");
    for (std::size_t i = 0; i < f.queries.size() && i < full.queries.size(); ++i) {
      const FixtureQuery& fq = f.queries[i];
      const UntrustedCandidateBatchQueryResult& q = full.queries[i];
      const std::string tag = f.name + " query " + std::to_string(i);
      ++queries;
      if (fq.cpu_status == 1) {
        check(q.header.completion == KernelCompletion::kDisconnected, tag + " disconnected");
        check(compact.queries[i].header.completion == KernelCompletion::kDisconnected,
              tag + " compact disconnected");
        continue;
      }
      check(q.header.completion == KernelCompletion::kReached, tag + " reached");
      if (q.header.completion != KernelCompletion::kReached) continue;
      check(full.labels[q.workspace_offset + q.header.goal_state] == fq.cpu_cost, tag + " goal label");
      // canonical reverse path from the full workspace's predecessors
      std::vector<std::uint32_t> path;
      std::uint32_t s = q.header.goal_state;
      while (s != kInvalidStateIndex && path.size() <= q.workspace_state_count) {
        path.push_back(s);
        s = full.predecessors[q.workspace_offset + s];
      }
      const auto& cq = compact.queries[i];
      check(cq.compact_path.has_value(), tag + " compact path present");
      if (!cq.compact_path) continue;
      const std::vector<std::uint32_t> got(
          compact.compact_path_states.begin() + cq.compact_path->state_offset,
          compact.compact_path_states.begin() + cq.compact_path->state_offset +
              cq.compact_path->state_count);
      check(got == path, tag + " compact path equals the canonical predecessor chain");
    }
    // single route pair on the first query (base policy)
    const FixtureQuery& q0 = f.queries.front();
    if (q0.policy.empty() && q0.orth == 0 && q0.diag == 0 && q0.bend == 0 && q0.start != q0.goal) {
      BackendExecutionRequest rr{PlanarGenerator::kBucketedFrontier, q0.start, q0.goal, 0, 100000,
                                 UINT64_MAX, nullptr};
      ExecutionResult er = backend->ExecuteRoute(view, rr);
      if (!is_error(er, "ExecuteRoute")) {
        ReadbackResult rr2 = backend->ReadbackRoute(*std::get<std::unique_ptr<PendingRouteExecution>>(er));
        er = BackendError{};  // release the execution (and the view's lease) now
        if (!is_error(rr2, "ReadbackRoute")) {
          const UntrustedKernelResult& k = std::get<UntrustedKernelResult>(rr2);
          if (q0.cpu_status == 0) {
            check(k.completion == KernelCompletion::kReached &&
                      k.labels.at(k.goal_state) == q0.cpu_cost,
                  f.name + " route pair goal label");
          } else {
            check(k.completion == KernelCompletion::kDisconnected, f.name + " route pair disconnected");
          }
        }
      }
    }
    ++cases;
  }
  if (failures == 0) {
    std::printf("adapter ok: %zu cases, %zu queries through IPlanarRouteBackend\n", cases, queries);
    return 0;
  }
  std::printf("adapter FAILED: %d checks\n", failures);
  return 1;
}
