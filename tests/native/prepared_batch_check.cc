// GPU check of the drop-in through the reference's own prepared host path.
//
// TEST INFRASTRUCTURE.  Built by apgar_b200/adapter/build_adapter.sh against
// the reference sources with apgar_b200/adapter/reference_generator.patch
// applied (the two B200 persistent generators and their descriptor), and
// linked with the shim (b200_planar_backend.cc), this repository's fault
// decorator (fault_injecting_backend.cc) and libapgar_b200.so.
//
// 1. For every case of the reference's parity corpus (BuildPhase3CandidateCorpus:
//    the generated Phase-2/Phase-3 boards and the KiCad fixture), with the
//    case request forward and reversed under the base policy and the
//    deterministic alternative policies: PrepareCudaPlanarCompiledView over
//    CreateCudaPlanarRouteBackend(), then
//    RouteCandidateBatchWithPreparedPlanarGpuBackend (preflight, telemetry
//    validation, compact-path or full-workspace validation and
//    reconstruction, disconnected confirmation, sealing) with each persistent
//    generator.  Every reached item must be sealed with authenticated CUDA
//    producer evidence at the reference CPU A* cost, and every other item
//    must be the CPU A*'s own outcome.  RouteWithPreparedPlanarGpuBackend
//    (single route) must give the CPU cost too.  Every sealed item is then
//    turned into a route candidate by the reference's candidate adapter
//    (BuildGeneratedCandidateFromGpuBatchItem, one item at a time, and
//    BuildGeneratedCandidatesFromGpuBatchItems over the batch, which must
//    agree), with the CUDA provenance of its generator, and the candidate
//    must pass the reference's admission (AdmitRouteCandidate: exact
//    geometry, resources, metrics and signatures recomputed).
// 2. Each of the reference's fault classes, injected on the host by the
//    decorator over the shim, must fail the first query (or the whole batch,
//    or the route) with the invariant id the reference names for it.
// Prints "prepared ok: ..." and exits 0 when every check holds.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <span>
#include <string>
#include <string_view>
#include <variant>
#include <vector>

#include "apgar/benchmark/planar_corpus.h"
#include "apgar/candidates/gpu_candidate_adapter.h"
#include "apgar/candidates/route_candidate.h"
#include "apgar/gpu/cuda_backend.h"
#include "apgar/gpu/fault_injecting_backend.h"
#include "apgar/gpu/planar_router.h"
#include "apgar/routing/candidate_policy.h"
#include "apgar/routing/cpu_astar.h"

// The KiCad fixture's text, embedded at build time from the reference tree.
extern const char kKicadFixture[];
extern const unsigned long kKicadFixtureSize;

using namespace apgar;
using gpu::PlanarGenerator;

namespace {

int failures = 0;
std::size_t admitted = 0;  // sealed items the candidate adapter and admission accepted
void check(bool ok, const std::string& what) {
  if (!ok) {
    ++failures;
    std::fprintf(stderr, "FAIL: %s\n", what.c_str());
  }
}

struct Expected {
  bool reached = false;
  bool disconnected = false;
  std::uint64_t cost = 0;
};

std::vector<routing::CandidateGenerationPolicy> policies_for(const benchmark::PlanarCorpusCase& c) {
  std::vector<routing::CandidateGenerationPolicy> out{c.request.candidate_policy};
  // alternative resources: the edges of the base CPU route, as the corpus tools do
  std::vector<routing::EdgeResourceKey> alt;
  const auto base = routing::RouteWithCpuAStar(c.board, c.compiled_board, c.request);
  if (const auto* route = std::get_if<routing::CpuRoute>(&base)) {
    const auto& profile = c.compiled_board.profile();
    for (std::size_t i = 1; i < route->lattice_path.size() && alt.size() < 12; ++i) {
      const auto a = geometry_compiler::ExactPointToLatticeIndex(profile, route->lattice_path[i - 1]);
      const auto b = geometry_compiler::ExactPointToLatticeIndex(profile, route->lattice_path[i]);
      if (!a || !b) continue;
      for (auto d : geometry_compiler::kStableDirectionOrder) {
        const auto delta = geometry_compiler::DeltaFor(d);
        if (a->x + delta.x == b->x && a->y + delta.y == b->y) {
          if (auto r = routing::CanonicalPhysicalEdgeResource(c.request.start_layer, *a, d)) {
            alt.push_back(*r);
          }
        }
      }
    }
  }
  std::sort(alt.begin(), alt.end());
  alt.erase(std::unique(alt.begin(), alt.end()), alt.end());
  routing::DeterministicAlternativePolicySchedule schedule;
  schedule.candidate_count = 5;
  schedule.step_surcharge_increment = 3;
  schedule.bend_surcharge_increment = 5;
  schedule.resource_penalty_increment = 7;
  schedule.alternative_resources = alt;
  const auto alts = routing::BuildDeterministicAlternativePolicies(c.compiled_board,
                                                                   c.request.candidate_policy, schedule);
  if (const auto* list = std::get_if<std::vector<routing::NormalizedCandidateGenerationPolicy>>(&alts)) {
    for (std::size_t i = 1; i < list->size(); ++i) out.push_back((*list)[i].policy);
  }
  return out;
}

std::vector<gpu::PlanarCandidateBatchQuery> queries_for(const benchmark::PlanarCorpusCase& c) {
  std::vector<gpu::PlanarCandidateBatchQuery> out;
  std::uint64_t id = 1;
  for (int reverse = 0; reverse < 2; ++reverse) {
    for (const auto& policy : policies_for(c)) {
      routing::CpuRouteRequest req = c.request;
      if (reverse) {
        std::swap(req.start, req.goal);
        std::swap(req.start_layer, req.goal_layer);
      }
      req.candidate_policy = policy;
      out.push_back(gpu::PlanarCandidateBatchQuery{
          .query_id = id, .input_ordinal = static_cast<std::uint32_t>(id - 1), .request = req});
      ++id;
    }
  }
  return out;
}

Expected cpu_outcome(const benchmark::PlanarCorpusCase& c, const routing::CpuRouteRequest& req) {
  Expected e;
  const auto r = routing::RouteWithCpuAStar(c.board, c.compiled_board, req);
  if (const auto* route = std::get_if<routing::CpuRoute>(&r)) {
    e.reached = true;
    e.cost = route->total_cost;
  } else {
    e.disconnected = std::get<routing::RouteFailure>(r).code == routing::RouteFailureCode::kDisconnected;
  }
  return e;
}

gpu::PlanarCandidateBatchPolicy batch_policy(PlanarGenerator generator, std::uint64_t batch_id) {
  gpu::PlanarCandidateBatchPolicy p;
  p.batch_id = batch_id;
  p.generator = generator;
  p.maximum_rounds = 100000;
  return p;
}

const char* name_of(PlanarGenerator g) {
  return g == PlanarGenerator::kB200Persistent ? "persistent" : "persistent-workspace";
}

// The sealed items of one batch through the reference's candidate adapter and
// admission; the candidate generator kind follows the patched mapping
// (compact paths as the sweep's, the full workspace as the frontier's).
void convert_items(const benchmark::PlanarCorpusCase& c,
                   const std::vector<gpu::PlanarCandidateBatchQuery>& queries,
                   const gpu::PlanarCandidateBatch& batch, PlanarGenerator g, const std::string& tag) {
  const candidates::CandidateGeneratorKind kind = g == PlanarGenerator::kB200Persistent
                                                      ? candidates::CandidateGeneratorKind::kCudaSweep
                                                      : candidates::CandidateGeneratorKind::kCudaFrontier;
  std::vector<routing::NormalizedCandidateGenerationPolicy> policies;
  policies.reserve(queries.size());
  for (const auto& q : queries) {
    auto norm = routing::NormalizeCandidateGenerationPolicy(c.compiled_board, q.request.candidate_policy);
    if (auto* np = std::get_if<routing::NormalizedCandidateGenerationPolicy>(&norm)) {
      policies.push_back(*np);
    } else {
      check(false, tag + ": policy normalisation failed");
      return;
    }
  }
  std::vector<candidates::GpuCandidateBatchBuildRequest> requests;
  std::vector<candidates::CandidateDraftBuildResult> singles;
  for (const gpu::PlanarCandidateBatchItem& item : batch.items) {
    if (std::get_if<gpu::PlanarGpuRoute>(&item.result()) == nullptr) continue;
    const std::size_t i = static_cast<std::size_t>(item.query_id() - 1);
    if (i >= queries.size()) continue;  // reported by the caller
    const std::string qtag = tag + " query " + std::to_string(item.query_id());
    requests.push_back(candidates::GpuCandidateBatchBuildRequest{
        .query = queries[i], .normalized_policy = policies[i], .item = item});
    singles.push_back(candidates::BuildGeneratedCandidateFromGpuBatchItem(
        c.board, c.compiled_board, queries[i], policies[i], batch, item));
    const auto* gen = std::get_if<candidates::GeneratedRouteCandidate>(&singles.back());
    if (gen == nullptr) {
      const auto& rej = std::get<candidates::CandidateRejection>(singles.back());
      check(false, qtag + ": candidate rejected: " + rej.invariant_id + " " + rej.detail);
      continue;
    }
    check(gen->provenance.generator == kind, qtag + ": candidate generator kind");
    check(gen->provenance.backend == candidates::CandidateBackendKind::kCuda, qtag + ": CUDA backend");
    check(gen->provenance.query_identity == item.query_id(), qtag + ": query identity");
    const auto admission = candidates::AdmitRouteCandidate(
        candidates::CandidateAdmissionContext{c.board, c.compiled_board, queries[i].request}, *gen);
    if (const auto* rej = std::get_if<candidates::CandidateRejection>(&admission)) {
      check(false, qtag + ": admission rejected: " + rej->invariant_id + " " + rej->detail);
      continue;
    }
    ++admitted;
  }
  const auto batched =
      candidates::BuildGeneratedCandidatesFromGpuBatchItems(c.board, c.compiled_board, batch, requests);
  if (const auto* list = std::get_if<std::vector<candidates::CandidateDraftBuildResult>>(&batched)) {
    check(*list == singles, tag + ": batch conversion equals the per-item conversion");
  } else {
    const auto& f = std::get<candidates::GpuCandidateBatchBuildFailure>(batched);
    check(false, tag + ": batch conversion failed: " + f.invariant_id + " " + f.detail);
  }
}

// Part 1: one case through the prepared batch and single-route paths.
std::size_t run_case(const benchmark::PlanarCorpusCase& c, gpu::IPlanarRouteBackend& backend,
                     std::uint64_t batch_id) {
  auto prepared_result = gpu::PrepareCudaPlanarCompiledView(c.board, c.compiled_board, backend);
  if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&prepared_result)) {
    check(false, c.name + ": prepare: " + f->detail);
    return 0;
  }
  gpu::PreparedPlanarCompiledView& prepared =
      *std::get<std::unique_ptr<gpu::PreparedPlanarCompiledView>>(prepared_result);
  // single route with the full-workspace persistent generator, first on the
  // fresh view: the reference checks a route's peak against persistent +
  // route bytes, and later batches would leave a larger workspace cached
  {
    gpu::PlanarRoutePolicy rp;
    rp.generator = PlanarGenerator::kB200PersistentWorkspace;
    const auto single =
        gpu::RouteWithPreparedPlanarGpuBackend(c.board, c.compiled_board, c.request, rp, prepared);
    const Expected e = cpu_outcome(c, c.request);
    if (const auto* route = std::get_if<gpu::PlanarGpuRoute>(&single)) {
      check(e.reached && route->total_cost == e.cost, c.name + ": single route cost");
    } else {
      const auto& f = std::get<gpu::PlanarGpuFailure>(single);
      check(e.disconnected && f.code == gpu::PlanarGpuFailureCode::kDisconnected,
            c.name + ": single route failure " + f.invariant_id + " " + f.detail);
    }
  }
  const std::vector<gpu::PlanarCandidateBatchQuery> queries = queries_for(c);
  std::vector<Expected> expected;
  for (const auto& q : queries) expected.push_back(cpu_outcome(c, q.request));
  std::size_t sealed = 0;
  for (PlanarGenerator g : {PlanarGenerator::kB200Persistent, PlanarGenerator::kB200PersistentWorkspace}) {
    const std::string tag = c.name + " (" + name_of(g) + ")";
    auto result = gpu::RouteCandidateBatchWithPreparedPlanarGpuBackend(
        c.board, c.compiled_board, queries, batch_policy(g, batch_id++), prepared);
    if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&result)) {
      check(false, tag + ": batch failed: " + f->invariant_id + " " + f->detail);
      continue;
    }
    const gpu::PlanarCandidateBatch& batch = std::get<gpu::PlanarCandidateBatch>(result);
    check(batch.items.size() == queries.size(), tag + ": item count");
    check(batch.telemetry.blocking_status_readback_count == 0, tag + ": no blocking readbacks");
    for (const gpu::PlanarCandidateBatchItem& item : batch.items) {
      const std::size_t i = static_cast<std::size_t>(item.query_id() - 1);
      const std::string qtag = tag + " query " + std::to_string(item.query_id());
      if (i >= expected.size()) {
        check(false, qtag + ": unknown query id");
        continue;
      }
      const Expected& e = expected[i];
      if (const auto* route = std::get_if<gpu::PlanarGpuRoute>(&item.result())) {
        check(e.reached && route->total_cost == e.cost,
              qtag + ": cost " + std::to_string(route->total_cost) + " vs CPU A* " +
                  std::to_string(e.cost));
        check(item.has_validated_route_evidence(), qtag + ": sealed");
        check(item.has_authenticated_cuda_producer_evidence(), qtag + ": authenticated producer");
        sealed += route->total_cost == e.cost ? 1 : 0;
      } else {
        const auto& f = std::get<gpu::PlanarGpuFailure>(item.result());
        check(e.disconnected && f.code == gpu::PlanarGpuFailureCode::kDisconnected,
              qtag + ": failure " + f.invariant_id + " " + f.detail);
      }
    }
    convert_items(c, queries, batch, g, tag);
  }
  return sealed;
}

struct FaultCase {
  gpu::UntrustedCandidateBatchResultFault fault;
  PlanarGenerator generator;
  const char* invariant;
  bool whole_batch;  // a batch-envelope fault fails every item (a changed
                     // query id fails only the two queries it confuses)
};

// Part 2: the reference's fault classes through its own host validation.
void run_faults(const benchmark::PlanarCorpusCase& c, gpu::IPlanarRouteBackend& shim) {
  using F = gpu::UntrustedCandidateBatchResultFault;
  const PlanarGenerator compact = PlanarGenerator::kB200Persistent;
  const PlanarGenerator full = PlanarGenerator::kB200PersistentWorkspace;
  const FaultCase cases[] = {
      {F::kWorkspaceBounds, full, "gpu.batch.workspace.bounds.v1", false},
      {F::kWorkspaceOwner, full, "gpu.batch.workspace.owner.v1", false},
      {F::kQueryTelemetry, full, "gpu.batch.query.telemetry.v1", false},
      {F::kMemoryAccounting, full, "gpu.batch.memory.accounting.v1", true},
      {F::kBatchTelemetry, full, "gpu.batch.telemetry.v1", true},
      {F::kQueryIdentity, full, "gpu.batch.query.identity.v1", false},
      {F::kFalseDisconnected, full, "gpu.disconnected.cpu_reachable.v1", false},
      {F::kCompactPathBounds, compact, "gpu.batch.compact_path.bounds.v1", false},
      {F::kCompactPathEndpoint, compact, "gpu.batch.compact_path.endpoint.v1", false},
      {F::kCompactPathCycle, compact, "gpu.batch.compact_path.cycle.v1", false},
      {F::kCompactPathHeading, compact, "gpu.batch.compact_path.heading.v1", false},
      {F::kCompactPathEdge, compact, "gpu.batch.compact_path.edge.v1", false},
  };
  const std::vector<gpu::PlanarCandidateBatchQuery> queries = queries_for(c);
  std::uint64_t batch_id = 9000;
  // the clean decorator (kNone) first: everything must still validate
  for (PlanarGenerator g : {compact, full}) {
    auto clean = gpu::CreateFaultInjectingCandidateBatchBackend(shim, F::kNone);
    auto pr = gpu::PreparePlanarCompiledView(c.board, c.compiled_board, *clean);
    if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&pr)) {
      check(false, "fault decorator: prepare: " + f->detail);
      return;
    }
    auto result = gpu::RouteCandidateBatchWithPreparedPlanarGpuBackend(
        c.board, c.compiled_board, queries, batch_policy(g, batch_id++),
        *std::get<std::unique_ptr<gpu::PreparedPlanarCompiledView>>(pr));
    const auto* batch = std::get_if<gpu::PlanarCandidateBatch>(&result);
    check(batch != nullptr && std::get_if<gpu::PlanarGpuRoute>(&batch->items.front().result()) != nullptr,
          std::string("no fault (") + name_of(g) + "): first query routed");
  }
  for (const FaultCase& fc : cases) {
    auto decorator = gpu::CreateFaultInjectingCandidateBatchBackend(shim, fc.fault);
    auto pr = gpu::PreparePlanarCompiledView(c.board, c.compiled_board, *decorator);
    if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&pr)) {
      check(false, std::string(fc.invariant) + ": prepare: " + f->detail);
      continue;
    }
    auto result = gpu::RouteCandidateBatchWithPreparedPlanarGpuBackend(
        c.board, c.compiled_board, queries, batch_policy(fc.generator, batch_id++),
        *std::get<std::unique_ptr<gpu::PreparedPlanarCompiledView>>(pr));
    std::string got;
    if (const auto* f = std::get_if<gpu::PlanarGpuFailure>(&result)) {
      got = f->invariant_id;
    } else {
      const auto& items = std::get<gpu::PlanarCandidateBatch>(result).items;
      if (const auto* f = std::get_if<gpu::PlanarGpuFailure>(&items.front().result())) got = f->invariant_id;
      if (fc.whole_batch) {
        for (const auto& item : items) {
          const auto* f = std::get_if<gpu::PlanarGpuFailure>(&item.result());
          check(f != nullptr && f->invariant_id == fc.invariant,
                std::string(fc.invariant) + ": every item fails");
        }
      }
    }
    check(got == fc.invariant, std::string("fault ") + fc.invariant + " raised " + got);
    std::printf("fault %-36s -> %s\n", fc.invariant, got.c_str());
  }
  // the single-route fault: the goal state made its own predecessor
  auto route_decorator =
      gpu::CreateFaultInjectingPlanarRouteBackend(shim, gpu::UntrustedResultFault::kGoalPredecessorSelfCycle);
  auto pr = gpu::PreparePlanarCompiledView(c.board, c.compiled_board, *route_decorator);
  if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&pr)) {
    check(false, "route fault: prepare: " + f->detail);
    return;
  }
  gpu::PlanarRoutePolicy rp;
  rp.generator = full;
  const auto single = gpu::RouteWithPreparedPlanarGpuBackend(
      c.board, c.compiled_board, c.request, rp,
      *std::get<std::unique_ptr<gpu::PreparedPlanarCompiledView>>(pr));
  const auto* f = std::get_if<gpu::PlanarGpuFailure>(&single);
  const std::string got = f != nullptr ? f->invariant_id : std::string("(routed)");
  check(got == "gpu.predecessor.self_reference.v1", "route fault raised " + got);
  std::printf("fault %-36s -> %s\n", "gpu.predecessor.self_reference.v1", got.c_str());
}

}  // namespace

int main() {
  const std::string_view kicad(kKicadFixture, kKicadFixtureSize);
  auto corpus_result = benchmark::BuildPhase3CandidateCorpus(kicad);
  if (auto* e = std::get_if<std::string>(&corpus_result)) {
    std::fprintf(stderr, "corpus: %s\n", e->c_str());
    return 1;
  }
  const auto& corpus = std::get<std::vector<benchmark::PlanarCorpusCase>>(corpus_result);
  std::unique_ptr<gpu::IPlanarRouteBackend> backend = gpu::CreateCudaPlanarRouteBackend();
  std::size_t sealed = 0;
  std::uint64_t batch_id = 100;
  for (const auto& c : corpus) {
    sealed += run_case(c, *backend, batch_id);
    batch_id += 10;
  }
  // faults on the KiCad fixture case (its routes are long enough for every
  // compact-path class), which the corpus lists last
  run_faults(corpus.back(), *backend);
  if (failures == 0) {
    std::printf("prepared ok: %zu cases, %zu items sealed at the CPU A* cost, %zu route candidates "
                "built and admitted by the reference's candidate adapter, 13 fault classes\n",
                corpus.size(), sealed, admitted);
    return 0;
  }
  std::printf("prepared FAILED: %d checks\n", failures);
  return 1;
}
