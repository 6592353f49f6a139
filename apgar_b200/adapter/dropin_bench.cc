// Drop-in benchmark on the reference's own workload.
//
// Built by apgar_b200/adapter/build_adapter.sh against the patched reference
// (reference_generator.patch) and run by `bench.py --workload dropin`.  For
// every case of the reference's parity corpus (BuildPhase3CandidateCorpus:
// the generated Phase-2/Phase-3 boards and the KiCad fixture) it builds up to
// 512 candidate policies with the reference's own schedule
// (BuildDeterministicAlternativePolicies over the base route's edge
// resources, as the reference's Phase-3 tool does), and for each batch size
// k in 4 .. 512 times, as medians over repetitions:
//  * gpu:     RouteCandidateBatchWithPreparedPlanarGpuBackend of the k queries
//             over this backend (generator kB200Persistent): the prepared
//             end-to-end scope of the reference's report, i.e. H2D of the
//             queries and policies, the search, D2H of compact paths and the
//             reference's host validation, reconstruction and sealing (the
//             view upload is prepared once and excluded, as there);
//             gpu_kernel: the batch telemetry's kernel time, the part of gpu spent on the device;
//  * cpu_par: the reference's RouteWithCpuAStar over the k queries on all
//             host threads (one query per task);
//  * cpu_ser: the same on one thread.
// Every sealed GPU cost must equal the CPU A* cost of its query.  Prints one
// JSON object.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <string>
#include <string_view>
#include <thread>
#include <variant>
#include <vector>

#include "apgar/benchmark/planar_corpus.h"
#include "apgar/gpu/cuda_backend.h"
#include "apgar/gpu/planar_router.h"
#include "apgar/routing/candidate_policy.h"
#include "apgar/routing/cpu_astar.h"

extern const char kKicadFixture[];
extern const unsigned long kKicadFixtureSize;

using namespace apgar;

namespace {

constexpr std::uint32_t kBatchSizes[] = {4, 8, 16, 32, 64, 128, 256, 512};
constexpr int kRepetitions = 9;

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

double median(std::vector<double> v) {
  std::sort(v.begin(), v.end());
  return v[v.size() / 2];
}

std::vector<routing::EdgeResourceKey> base_resources(const benchmark::PlanarCorpusCase& c) {
  std::vector<routing::EdgeResourceKey> out;
  const auto base = routing::RouteWithCpuAStar(c.board, c.compiled_board, c.request);
  const auto* route = std::get_if<routing::CpuRoute>(&base);
  if (route == nullptr) return out;
  const auto& profile = c.compiled_board.profile();
  for (std::size_t i = 1; i < route->lattice_path.size(); ++i) {
    const auto a = geometry_compiler::ExactPointToLatticeIndex(profile, route->lattice_path[i - 1]);
    const auto b = geometry_compiler::ExactPointToLatticeIndex(profile, route->lattice_path[i]);
    if (!a || !b) continue;
    for (auto d : geometry_compiler::kStableDirectionOrder) {
      const auto delta = geometry_compiler::DeltaFor(d);
      if (a->x + delta.x == b->x && a->y + delta.y == b->y) {
        if (auto r = routing::CanonicalPhysicalEdgeResource(c.request.start_layer, *a, d)) out.push_back(*r);
      }
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

std::vector<routing::CandidateGenerationPolicy> policies_for(const benchmark::PlanarCorpusCase& c) {
  std::vector<routing::CandidateGenerationPolicy> out;
  routing::DeterministicAlternativePolicySchedule schedule;
  schedule.candidate_count = 512;
  schedule.step_surcharge_increment = 1;
  schedule.bend_surcharge_increment = 1;
  schedule.resource_penalty_increment = 3;
  schedule.alternative_resources = base_resources(c);
  const auto list = routing::BuildDeterministicAlternativePolicies(c.compiled_board,
                                                                   c.request.candidate_policy, schedule);
  if (const auto* v = std::get_if<std::vector<routing::NormalizedCandidateGenerationPolicy>>(&list)) {
    for (const auto& p : *v) out.push_back(p.policy);
  }
  if (out.empty()) out.push_back(c.request.candidate_policy);
  return out;
}

// CPU A* over queries [0, k) on `threads` threads; costs (UINT64_MAX when not reached).
std::vector<std::uint64_t> cpu_batch(const benchmark::PlanarCorpusCase& c,
                                     const std::vector<routing::CandidateGenerationPolicy>& pols,
                                     std::uint32_t k, unsigned threads) {
  std::vector<std::uint64_t> costs(k, UINT64_MAX);
  std::atomic<std::uint32_t> next{0};
  const auto work = [&] {
    for (;;) {
      const std::uint32_t i = next.fetch_add(1);
      if (i >= k) return;
      routing::CpuRouteRequest req = c.request;
      req.candidate_policy = pols[i % pols.size()];
      const auto r = routing::RouteWithCpuAStar(c.board, c.compiled_board, req);
      if (const auto* route = std::get_if<routing::CpuRoute>(&r)) costs[i] = route->total_cost;
    }
  };
  if (threads <= 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < std::min<unsigned>(threads, k); ++t) pool.emplace_back(work);
    for (auto& t : pool) t.join();
  }
  return costs;
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
  const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
  bool costs_match = true;
  std::uint64_t batch_id = 1;
  std::printf("{\"threads\": %u, \"repetitions\": %d, \"cases\": [", threads, kRepetitions);
  for (std::size_t ci = 0; ci < corpus.size(); ++ci) {
    const auto& c = corpus[ci];
    auto prepared_result = gpu::PrepareCudaPlanarCompiledView(c.board, c.compiled_board, *backend);
    if (auto* f = std::get_if<gpu::PlanarGpuFailure>(&prepared_result)) {
      std::fprintf(stderr, "%s: prepare: %s\n", c.name.c_str(), f->detail.c_str());
      return 1;
    }
    auto& prepared = *std::get<std::unique_ptr<gpu::PreparedPlanarCompiledView>>(prepared_result);
    const auto pols = policies_for(c);
    std::printf("%s{\"name\": \"%s\", \"nodes\": %llu, \"policies\": %zu, \"k\": [", ci ? ", " : "",
                c.name.c_str(),
                static_cast<unsigned long long>(c.compiled_board.telemetry().represented_nodes),
                pols.size());
    bool first_k = true;
    for (std::uint32_t k : kBatchSizes) {
      std::vector<gpu::PlanarCandidateBatchQuery> queries;
      for (std::uint32_t i = 0; i < k; ++i) {
        routing::CpuRouteRequest req = c.request;
        req.candidate_policy = pols[i % pols.size()];
        queries.push_back(gpu::PlanarCandidateBatchQuery{.query_id = i + 1, .input_ordinal = i, .request = req});
      }
      const std::vector<std::uint64_t> want = cpu_batch(c, pols, k, threads);
      std::vector<double> g, gk, cp, cs;
      std::uint64_t sealed = 0;
      for (int rep = 0; rep < kRepetitions + 1; ++rep) {
        gpu::PlanarCandidateBatchPolicy policy;
        policy.batch_id = batch_id++;
        policy.generator = gpu::PlanarGenerator::kB200Persistent;
        policy.maximum_rounds = 100000;
        const double t0 = now_ms();
        auto result = gpu::RouteCandidateBatchWithPreparedPlanarGpuBackend(c.board, c.compiled_board,
                                                                           queries, policy, prepared);
        const double t1 = now_ms();
        const double t2 = now_ms();
        const auto par = cpu_batch(c, pols, k, threads);
        const double t3 = now_ms();
        if (rep == 0) {
          // the first repetition warms up (and is checked)
          const auto* batch = std::get_if<gpu::PlanarCandidateBatch>(&result);
          if (batch == nullptr) {
            std::fprintf(stderr, "%s k=%u: batch failed\n", c.name.c_str(), k);
            return 1;
          }
          for (const auto& item : batch->items) {
            const std::size_t i = static_cast<std::size_t>(item.query_id() - 1);
            const auto* route = std::get_if<gpu::PlanarGpuRoute>(&item.result());
            const std::uint64_t got = route != nullptr ? route->total_cost : UINT64_MAX;
            if (got != want[i] || par[i] != want[i]) costs_match = false;
            if (route != nullptr && item.has_validated_route_evidence()) ++sealed;
          }
          continue;
        }
        g.push_back(t1 - t0);
        if (const auto* batch = std::get_if<gpu::PlanarCandidateBatch>(&result)) {
          gk.push_back(batch->telemetry.kernel_milliseconds);
        }
        cp.push_back(t3 - t2);
        if (rep <= 3) {  // the serial CPU form is slow: three repetitions
          const double t4 = now_ms();
          cpu_batch(c, pols, k, 1);
          cs.push_back(now_ms() - t4);
        }
      }
      std::printf("%s{\"k\": %u, \"gpu_ms\": %.4f, \"gpu_kernel_ms\": %.4f, \"cpu_par_ms\": %.4f, "
                  "\"cpu_ser_ms\": %.4f, \"sealed\": %llu}",
                  first_k ? "" : ", ", k, median(g), gk.empty() ? 0.0 : median(gk), median(cp), median(cs),
                  static_cast<unsigned long long>(sealed));
      first_k = false;
    }
    std::printf("]}");
    std::fflush(stdout);
  }
  std::printf("], \"costs_match\": %s}\n", costs_match ? "true" : "false");
  return costs_match ? 0 : 2;
}
