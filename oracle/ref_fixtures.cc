// Golden-fixture generator.  TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own CPU path (compiled from its sources by
// oracle/build_ref.sh) on its own parity corpus and writes, per case, the
// flattened device view (DeviceCompiledBoardV1 arrays, byte-for-byte) and a
// list of queries with the reference CPU A* outcome:
//   * corpus: benchmark::BuildPhase3CandidateCorpus (src/benchmark/planar_corpus.cc),
//     the Phase-2 bakeoff cases plus the Phase-3 candidate cases and the
//     KiCad fixture (tests/fixtures/m1_exactness.kicad_pcb);
//   * device view: gpu::BuildDeviceCompiledBoardV1 (src/gpu/device_board.cc:136-325);
//   * queries: each case's request forward and reversed, under the normalized
//     base policy and the deterministic alternative policies of
//     routing::BuildDeterministicAlternativePolicies (candidate_policy.h) with the
//     base route's edge resources as alternative resources;
//   * policy edges encoded like the reference host dispatch
//     (src/gpu/planar_router.cc:1625-1694): canonical resource -> node*8+dir,
//     bans as UINT64_MAX, sorted by physical edge index;
//   * expected outcome: routing::RouteWithCpuAStar (src/routing/cpu_astar.cc:323-638).
//
// usage: ref_fixtures <kicad_fixture.kicad_pcb> <out_dir>
// Writes <out_dir>/<case>.bin and <out_dir>/manifest.json (format in
// tests/golden/ref_corpus.py).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <variant>
#include <vector>

#include "apgar/benchmark/planar_corpus.h"
#include "apgar/geometry/exact.h"
#include "apgar/gpu/planar_router.h"
#include "apgar/routing/candidate_policy.h"
#include "apgar/routing/cpu_astar.h"

namespace {

using apgar::gpu::DeviceCandidatePolicyEdgeV1;
using apgar::gpu::DeviceCompiledBoardV1;

struct Writer {
  std::vector<unsigned char> bytes;
  template <typename T>
  void pod(const T& v) {
    const auto* p = reinterpret_cast<const unsigned char*>(&v);
    bytes.insert(bytes.end(), p, p + sizeof(T));
  }
  template <typename T>
  void array(const std::vector<T>& v) {
    pod<uint64_t>(v.size());
    const auto* p = reinterpret_cast<const unsigned char*>(v.data());
    bytes.insert(bytes.end(), p, p + v.size() * sizeof(T));
  }
};

struct QueryOut {
  uint32_t start_node, goal_node;
  uint64_t orth_s, diag_s, bend_s;
  std::vector<DeviceCandidatePolicyEdgeV1> edges;
  uint32_t cpu_status;  // 0 reached, 1 disconnected, 2 other failure
  uint64_t cpu_cost;
  uint64_t policy_identity;
  // reached routes: forward device nodes of the lattice path and the
  // reference's coalesced segments (routing::CoalesceSegments)
  std::vector<uint32_t> route_nodes;
  std::vector<apgar::routing::LayerSegment> segments;
};

// Seeded cases for the exact swept-trace clearance predicate: one-step
// lattice segments (8 headings) against boxes placed around them, at small
// and at near-envelope coordinates, with widths and clearances from zero
// clearance to several steps.  Written with the reference's verdicts.
void write_clearance_cases(const std::string& path) {
  uint64_t state = 0x9E3779B97F4A7C15ull;
  const auto next = [&state]() {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return state;
  };
  const auto pick = [&next](int64_t lo, int64_t hi) {
    return lo + static_cast<int64_t>(next() % static_cast<uint64_t>(hi - lo + 1));
  };
  static const int dx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
  static const int dy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  Writer w;
  w.pod<uint64_t>(0x3143524c43524741ull);  // magic "AGRCLRC1"
  const uint64_t count = 12000;
  w.pod<uint64_t>(count);
  for (uint64_t i = 0; i < count; ++i) {
    const bool far = (i % 8) == 7;  // near the 10^12 envelope
    const int64_t step = far ? pick(1, 5) * 100000 : pick(1, 12);
    const int64_t base = far ? 999999000000ll - pick(0, 1000) * step : 0;
    const int64_t sx = base + pick(-20, 20) * step, sy = (far ? -base : 0) + pick(-20, 20) * step;
    const int d = static_cast<int>(next() % 8);
    apgar::board_ir::Segment64 seg{};
    seg.start = {sx, sy};
    seg.end = {sx + dx[d] * step, sy + dy[d] * step};
    const int64_t cx = sx + pick(-3, 3) * step + pick(-step, step);
    const int64_t cy = sy + pick(-3, 3) * step + pick(-step, step);
    const int64_t hw = pick(0, 2 * step), hh = pick(0, 2 * step);
    apgar::board_ir::AxisAlignedBox64 box{};
    box.min = {cx - hw, cy - hh};
    box.max = {cx + hw, cy + hh};
    const int64_t width = pick(1, 2 * step);
    const int64_t clearance = pick(0, 2 * step);
    const auto r = apgar::geometry::SweptTraceClearanceAtLeast(seg, box, width, clearance);
    w.pod<int64_t>(seg.start.x);
    w.pod<int64_t>(seg.start.y);
    w.pod<int64_t>(seg.end.x);
    w.pod<int64_t>(seg.end.y);
    w.pod<int64_t>(box.min.x);
    w.pod<int64_t>(box.min.y);
    w.pod<int64_t>(box.max.x);
    w.pod<int64_t>(box.max.y);
    w.pod<int64_t>(width);
    w.pod<int64_t>(clearance);
    w.pod<uint32_t>(static_cast<uint32_t>(r.error));
    w.pod<uint32_t>(r.clearance_satisfied ? 1u : 0u);
  }
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(w.bytes.data()), static_cast<std::streamsize>(w.bytes.size()));
}

std::vector<apgar::routing::EdgeResourceKey> path_resources(
    const apgar::geometry_compiler::CompiledBoard& compiled, apgar::board_ir::LayerId layer,
    const std::vector<apgar::board_ir::Point64>& path) {
  std::vector<apgar::routing::EdgeResourceKey> out;
  for (size_t i = 1; i < path.size(); ++i) {
    const auto a = apgar::geometry_compiler::ExactPointToLatticeIndex(compiled.profile(), path[i - 1]);
    const auto b = apgar::geometry_compiler::ExactPointToLatticeIndex(compiled.profile(), path[i]);
    if (!a || !b) continue;
    for (auto d : apgar::geometry_compiler::kStableDirectionOrder) {
      const auto delta = apgar::geometry_compiler::DeltaFor(d);
      if (a->x + delta.x == b->x && a->y + delta.y == b->y) {
        if (auto r = apgar::routing::CanonicalPhysicalEdgeResource(layer, *a, d)) out.push_back(*r);
      }
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

bool encode_policy(const DeviceCompiledBoardV1& device,
                   const apgar::routing::CandidateGenerationPolicy& policy,
                   std::vector<DeviceCandidatePolicyEdgeV1>* edges) {
  auto physical = [&](const apgar::routing::EdgeResourceKey& r) -> int64_t {
    const auto dir = static_cast<uint8_t>(r.direction);
    if (dir >= 4) return -1;
    const auto node = apgar::gpu::FindDeviceNodeIndex(
        device, r.layer, apgar::geometry_compiler::LatticeIndex{.x = r.lattice_x, .y = r.lattice_y});
    if (!node || (device.nodes[*node].legal_edges & (1u << dir)) == 0) return -1;
    return static_cast<int64_t>(*node) * 8 + dir;
  };
  for (const auto& r : policy.banned_resources) {
    const int64_t p = physical(r);
    if (p < 0) return false;
    edges->push_back(DeviceCandidatePolicyEdgeV1{.physical_edge_index = static_cast<uint32_t>(p),
                                                 .adjustment = UINT64_MAX});
  }
  for (const auto& pen : policy.resource_penalties) {
    const int64_t p = physical(pen.resource);
    if (p < 0) return false;
    edges->push_back(DeviceCandidatePolicyEdgeV1{.physical_edge_index = static_cast<uint32_t>(p),
                                                 .adjustment = pen.additional_cost});
  }
  std::sort(edges->begin(), edges->end(), [](const auto& a, const auto& b) {
    return a.physical_edge_index < b.physical_edge_index;
  });
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: ref_fixtures <kicad_fixture> <out_dir>\n";
    return 2;
  }
  std::ifstream in(argv[1]);
  std::stringstream buf;
  buf << in.rdbuf();
  const std::string kicad = buf.str();
  const std::string out_dir = argv[2];
  auto corpus_result = apgar::benchmark::BuildPhase3CandidateCorpus(kicad);
  if (std::holds_alternative<std::string>(corpus_result)) {
    std::cerr << "corpus: " << std::get<std::string>(corpus_result) << "\n";
    return 1;
  }
  auto& corpus = std::get<std::vector<apgar::benchmark::PlanarCorpusCase>>(corpus_result);
  std::ostringstream manifest;
  manifest << "{\n  \"cases\": [\n";
  bool first_case = true;
  // segments.bin: per reached route, (case, query, layer, forward nodes,
  // reference segments as layer, x0, y0, x1, y1)
  Writer segw;
  segw.pod<uint64_t>(0x3147455354524741ull);  // magic "AGRTSEG1"
  uint64_t segment_records = 0;
  Writer segbody;
  uint32_t case_index = 0;
  // geometry.bin: per case, the compile inputs of every edge's legality (the
  // routing profile's width, clearance and net, the compiler's heading mask
  // and lattice placement, and every obstacle box with its layer and whether
  // the routed net owns it)
  Writer geow;
  geow.pod<uint64_t>(0x314f454754524741ull);  // magic "AGRTGEO1"
  geow.pod<uint64_t>(corpus.size());
  for (auto& c : corpus) {
    auto dev_result = apgar::gpu::BuildDeviceCompiledBoardV1(c.board, c.compiled_board);
    if (std::holds_alternative<apgar::gpu::PlanarGpuFailure>(dev_result)) {
      std::cerr << c.name << ": device view failed: "
                << std::get<apgar::gpu::PlanarGpuFailure>(dev_result).detail << "\n";
      return 1;
    }
    const DeviceCompiledBoardV1& device = std::get<DeviceCompiledBoardV1>(dev_result);
    const auto& profile = c.compiled_board.profile();

    // base route (forward) to seed the alternative resources
    std::vector<apgar::routing::EdgeResourceKey> alt_resources;
    {
      auto base = apgar::routing::RouteWithCpuAStar(c.board, c.compiled_board, c.request);
      if (auto* route = std::get_if<apgar::routing::CpuRoute>(&base)) {
        alt_resources = path_resources(c.compiled_board, c.request.start_layer, route->lattice_path);
      }
    }
    std::vector<apgar::routing::CandidateGenerationPolicy> policies;
    policies.push_back(c.request.candidate_policy);
    {
      apgar::routing::DeterministicAlternativePolicySchedule schedule;
      schedule.candidate_count = 9;
      schedule.step_surcharge_increment = 3;
      schedule.bend_surcharge_increment = 5;
      schedule.resource_penalty_increment = 7;
      if (alt_resources.size() > 12) alt_resources.resize(12);
      schedule.alternative_resources = alt_resources;
      auto alts = apgar::routing::BuildDeterministicAlternativePolicies(
          c.compiled_board, c.request.candidate_policy, schedule);
      if (auto* list = std::get_if<std::vector<apgar::routing::NormalizedCandidateGenerationPolicy>>(&alts)) {
        for (size_t i = 1; i < list->size(); ++i) policies.push_back((*list)[i].policy);
      } else {
        std::cerr << c.name << ": alternative policies unavailable: "
                  << std::get<apgar::routing::CandidatePolicyError>(alts).detail << "\n";
      }
    }

    std::vector<QueryOut> queries;
    for (int reverse = 0; reverse < 2; ++reverse) {
      for (const auto& policy : policies) {
        apgar::routing::CpuRouteRequest req = c.request;
        if (reverse) {
          std::swap(req.start, req.goal);
          std::swap(req.start_layer, req.goal_layer);
        }
        req.candidate_policy = policy;
        auto normalized = apgar::routing::NormalizeCandidateGenerationPolicy(c.compiled_board, policy);
        if (!std::holds_alternative<apgar::routing::NormalizedCandidateGenerationPolicy>(normalized)) {
          continue;
        }
        const auto& norm = std::get<apgar::routing::NormalizedCandidateGenerationPolicy>(normalized);
        const auto si = apgar::geometry_compiler::ExactPointToLatticeIndex(profile, req.start);
        const auto gi = apgar::geometry_compiler::ExactPointToLatticeIndex(profile, req.goal);
        if (!si || !gi) continue;
        const auto sn = apgar::gpu::FindDeviceNodeIndex(device, req.start_layer, *si);
        const auto gn = apgar::gpu::FindDeviceNodeIndex(device, req.goal_layer, *gi);
        if (!sn || !gn) continue;
        QueryOut q{};
        q.start_node = *sn;
        q.goal_node = *gn;
        q.orth_s = norm.policy.orthogonal_step_surcharge;
        q.diag_s = norm.policy.diagonal_step_surcharge;
        q.bend_s = norm.policy.bend_surcharge;
        q.policy_identity = norm.identity;
        if (!encode_policy(device, norm.policy, &q.edges)) continue;
        auto result = apgar::routing::RouteWithCpuAStar(c.board, c.compiled_board, req);
        if (auto* route = std::get_if<apgar::routing::CpuRoute>(&result)) {
          q.cpu_status = 0;
          q.cpu_cost = route->total_cost;
          bool mapped = true;
          for (const auto& point : route->lattice_path) {
            const auto idx = apgar::geometry_compiler::ExactPointToLatticeIndex(profile, point);
            const auto node = idx ? apgar::gpu::FindDeviceNodeIndex(device, req.start_layer, *idx)
                                  : std::nullopt;
            if (!node) {
              mapped = false;
              break;
            }
            q.route_nodes.push_back(*node);
          }
          if (mapped) q.segments = route->segments;
        } else {
          const auto& f = std::get<apgar::routing::RouteFailure>(result);
          q.cpu_status = f.code == apgar::routing::RouteFailureCode::kDisconnected ? 1u : 2u;
          q.cpu_cost = UINT64_MAX;
        }
        queries.push_back(std::move(q));
      }
    }

    {
      const auto& routing = c.compiled_board.prepared_routing_profile().profile();
      geow.pod<uint32_t>(case_index);
      geow.pod<uint32_t>(profile.heading_mask);
      geow.pod<int64_t>(routing.nominal_width);
      geow.pod<int64_t>(routing.clearance);
      geow.pod<int64_t>(profile.lattice_origin.x);
      geow.pod<int64_t>(profile.lattice_origin.y);
      geow.pod<int64_t>(profile.lattice_step);
      std::vector<const apgar::board_ir::Obstacle*> obstacles;
      for (const auto& layer : c.board.data().layers) {
        for (const auto& o : c.board.ObstaclesOnLayer(layer.routing_id)) obstacles.push_back(&o);
      }
      geow.pod<uint64_t>(obstacles.size());
      for (const auto* o : obstacles) {
        geow.pod<int64_t>(o->bounds.min.x);
        geow.pod<int64_t>(o->bounds.min.y);
        geow.pod<int64_t>(o->bounds.max.x);
        geow.pod<int64_t>(o->bounds.max.y);
        geow.pod<uint32_t>(o->layer);
        geow.pod<uint32_t>(o->owner_net.has_value() && *o->owner_net == routing.net ? 1u : 0u);
      }
    }
    for (size_t qi = 0; qi < queries.size(); ++qi) {
      const QueryOut& q = queries[qi];
      if (q.cpu_status != 0 || q.route_nodes.empty()) continue;
      segbody.pod<uint32_t>(case_index);
      segbody.pod<uint32_t>(static_cast<uint32_t>(qi));
      segbody.array(q.route_nodes);
      segbody.pod<uint64_t>(q.segments.size());
      for (const auto& sgm : q.segments) {
        segbody.pod<uint32_t>(static_cast<uint32_t>(sgm.layer));
        segbody.pod<uint32_t>(0);
        segbody.pod<int64_t>(sgm.centerline.start.x);
        segbody.pod<int64_t>(sgm.centerline.start.y);
        segbody.pod<int64_t>(sgm.centerline.end.x);
        segbody.pod<int64_t>(sgm.centerline.end.y);
      }
      ++segment_records;
    }
    ++case_index;

    Writer w;
    w.pod<uint64_t>(0x3158495446524741ull);  // magic "AGRFTIX1"
    w.pod(device.header);
    w.array(device.layers);
    w.array(device.nodes);
    w.array(device.runs);
    w.array(device.run_nodes);
    w.pod<uint64_t>(queries.size());
    for (const auto& q : queries) {
      w.pod(q.start_node);
      w.pod(q.goal_node);
      w.pod(q.orth_s);
      w.pod(q.diag_s);
      w.pod(q.bend_s);
      w.pod(q.policy_identity);
      w.pod(q.cpu_status);
      w.pod<uint32_t>(0);
      w.pod(q.cpu_cost);
      w.array(q.edges);
    }
    const std::string path = out_dir + "/" + c.name + ".bin";
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(w.bytes.data()), static_cast<std::streamsize>(w.bytes.size()));
    if (!first_case) manifest << ",\n";
    first_case = false;
    manifest << "    {\"name\": \"" << c.name << "\", \"family\": \"" << c.family
             << "\", \"nodes\": " << device.nodes.size() << ", \"runs\": " << device.runs.size()
             << ", \"costs\": {\"orthogonal\": " << device.header.costs.orthogonal_step
             << ", \"diagonal\": " << device.header.costs.diagonal_step
             << ", \"bend\": " << device.header.costs.bend << "}, \"queries\": [";
    for (size_t i = 0; i < queries.size(); ++i) {
      if (i) manifest << ", ";
      if (queries[i].cpu_status == 0) {
        manifest << queries[i].cpu_cost;
      } else {
        manifest << (queries[i].cpu_status == 1 ? "\"disconnected\"" : "\"failed\"");
      }
    }
    manifest << "]}";
    std::cerr << c.name << ": " << device.nodes.size() << " nodes, " << queries.size()
              << " queries\n";
  }
  manifest << "\n  ]\n}\n";
  std::ofstream(out_dir + "/manifest.json") << manifest.str();
  segw.pod<uint64_t>(segment_records);
  segw.bytes.insert(segw.bytes.end(), segbody.bytes.begin(), segbody.bytes.end());
  write_clearance_cases(out_dir + "/clearance.bin");
  {
    std::ofstream out(out_dir + "/geometry.bin", std::ios::binary);
    out.write(reinterpret_cast<const char*>(geow.bytes.data()),
              static_cast<std::streamsize>(geow.bytes.size()));
  }
  {
    std::ofstream out(out_dir + "/segments.bin", std::ios::binary);
    out.write(reinterpret_cast<const char*>(segw.bytes.data()),
              static_cast<std::streamsize>(segw.bytes.size()));
  }
  return 0;
}
