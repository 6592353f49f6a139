// Reference lattice pin.  TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own geometry compiler and CPU A* (compiled from its
// sources by oracle/build_ref.sh) on a planar board whose obstacles are
// axis-aligned boxes, so that the lattice move rule and the A* restatement of
// this repository's oracle can be checked against the reference itself:
//   * board: board_ir::CreateBoardSnapshot with two routable layers (M1 boards
//     need two or four; routes use the first), one
//     two-terminal net per query and one obstacle box per blocked rectangle;
//   * compile: geometry_compiler::CompileBoard
//     (src/geometry_compiler/compiled_board.cc:368-521), whose per-edge
//     legality is geometry::ValidateMovement's swept-trace clearance
//     (src/geometry/exact.cc:364-409);
//   * route: routing::RouteWithCpuAStar (src/routing/cpu_astar.cc:323-638).
//
// Geometry: lattice step 100, node (x, y) at exact point (100x, 100y); a
// blocked rectangle of cells [x0, x1] x [y0, y1] (inclusive) is the box
// [100 x0 - 40, 100 x1 + 40] x [100 y0 - 40, 100 y1 + 40]; trace width 20 and
// clearance 15 (25 units of required distance).  With these numbers a move
// between two free nodes passes 60 units from every box of a non-side cell,
// while a diagonal passes 14 units from a blocked side cell's box, so the
// compiled legality is exactly the lattice rule (orthogonal: both cells free;
// diagonal: both cells and both side cells free).  Costs: 10 / 14 / bend 0.
//
// usage: ref_lattice <input.bin> <output.bin>
// input:  u32 size, u32 rects, rects x (u32 x0, y0, x1, y1),
//         u32 nets, nets x (u32 sx, sy, gx, gy)
// output: u64 magic "AGRTLAT1", u32 size, size*size u8 legal_edges of the
//         first net's compile (node y*size + x, bit d = Direction d), u32 nets,
//         per net: u32 status (0 reached, 1 disconnected, 2 other failure),
//         u64 cost, u64 expanded_states, u64 queue_pops, u32 path length,
//         path x (u32 x, u32 y) in forward order.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <variant>
#include <vector>

#include "apgar/board_ir/board.h"
#include "apgar/geometry_compiler/compiled_board.h"
#include "apgar/routing/cpu_astar.h"
#include "apgar/routing/planar_route.h"

namespace {

using apgar::board_ir::AxisAlignedBox64;
using apgar::board_ir::BoardData;
using apgar::board_ir::BoardSnapshot;
using apgar::board_ir::EntityRef;
using apgar::board_ir::Point64;

constexpr int64_t kStep = 100;
constexpr int64_t kHalfBox = 40;
constexpr EntityRef kNet{.id = 10, .generation = 0};
constexpr EntityRef kFirst{.id = 20, .generation = 0};
constexpr EntityRef kSecond{.id = 21, .generation = 0};

struct Rect {
  uint32_t x0, y0, x1, y1;
};
struct Query {
  uint32_t sx, sy, gx, gy;
};

Point64 node_point(uint32_t x, uint32_t y) {
  return Point64{.x = static_cast<int64_t>(x) * kStep, .y = static_cast<int64_t>(y) * kStep};
}

AxisAlignedBox64 around(Point64 c, int64_t r) {
  return AxisAlignedBox64{.min = Point64{.x = c.x - r, .y = c.y - r},
                          .max = Point64{.x = c.x + r, .y = c.y + r}};
}

BoardData make_board(const std::vector<Rect>& rects, const Query& q) {
  BoardData b{
      .schema_version = apgar::board_ir::kBoardSchemaVersion,
      .dbu_per_millimeter = 1'000'000,
      .revision = 1,
      .adapter_name = "apgar-b200-lattice-pin",
      .adapter_version = "1",
      // M1 boards carry two or four routable signal layers; the search uses
      // the first (the reference is planar).
      .layers = {apgar::board_ir::Layer{.ref = EntityRef{.id = 1, .generation = 0},
                                        .routing_id = 0,
                                        .name = "front",
                                        .physical_order = 0,
                                        .type = apgar::board_ir::LayerType::kSignal,
                                        .routable = true},
                 apgar::board_ir::Layer{.ref = EntityRef{.id = 2, .generation = 0},
                                        .routing_id = 31,
                                        .name = "back",
                                        .physical_order = 1,
                                        .type = apgar::board_ir::LayerType::kSignal,
                                        .routable = true}},
      .nets = {apgar::board_ir::Net{.ref = kNet, .name = "NET", .terminals = {kFirst, kSecond}}},
      .terminals = {apgar::board_ir::Terminal{.ref = kFirst,
                                              .net = kNet,
                                              .component = "S",
                                              .pin = "1",
                                              .center = node_point(q.sx, q.sy),
                                              .connection_region = around(node_point(q.sx, q.sy), 1),
                                              .layers = {0}},
                    apgar::board_ir::Terminal{.ref = kSecond,
                                              .net = kNet,
                                              .component = "G",
                                              .pin = "1",
                                              .center = node_point(q.gx, q.gy),
                                              .connection_region = around(node_point(q.gx, q.gy), 1),
                                              .layers = {0}}},
      .obstacles = {},
      .routing_profile = apgar::board_ir::RoutingProfile{.net = kNet,
                                                         .nominal_width = 20,
                                                         .clearance = 15,
                                                         .allowed_layers = {0},
                                                         .allowed_headings =
                                                             apgar::board_ir::kM1HeadingMask},
  };
  uint64_t id = 1000;
  for (const Rect& r : rects) {
    b.obstacles.push_back(apgar::board_ir::Obstacle{
        .ref = EntityRef{.id = id++, .generation = 0},
        .layer = 0,
        .bounds = AxisAlignedBox64{
            .min = Point64{.x = r.x0 * kStep - kHalfBox, .y = r.y0 * kStep - kHalfBox},
            .max = Point64{.x = r.x1 * kStep + kHalfBox, .y = r.y1 * kStep + kHalfBox}},
        .owner_net = std::nullopt,
        .provenance = "blocked rectangle"});
  }
  return b;
}

apgar::geometry_compiler::CompilerProfile make_profile(uint32_t size) {
  const AxisAlignedBox64 roi{.min = Point64{.x = 0, .y = 0},
                             .max = Point64{.x = (size - 1) * kStep, .y = (size - 1) * kStep}};
  apgar::geometry_compiler::CompilerProfile p{
      .schema_version = apgar::geometry_compiler::kCompilerProfileSchemaVersion,
      .lattice_origin = Point64{.x = 0, .y = 0},
      .lattice_step = kStep,
      .tile_width_nodes = 16,
      .tile_height_nodes = 16,
      .compilation_roi = roi,
      .active_regions = {apgar::geometry_compiler::ActiveRegion{.layer = 0, .bounds = roi}},
      .heading_mask = apgar::board_ir::kM1HeadingMask,
      .costs = apgar::geometry_compiler::DeterministicCosts{
          .orthogonal_step = 10, .diagonal_step = 14, .bend = 0},
  };
  return p;
}

template <typename T>
void put(std::vector<unsigned char>* out, const T& v) {
  const auto* p = reinterpret_cast<const unsigned char*>(&v);
  out->insert(out->end(), p, p + sizeof(T));
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::cerr << "usage: ref_lattice <input.bin> <output.bin>\n";
    return 2;
  }
  std::ifstream in(argv[1], std::ios::binary);
  uint32_t size = 0, nrect = 0, nnet = 0;
  in.read(reinterpret_cast<char*>(&size), 4);
  in.read(reinterpret_cast<char*>(&nrect), 4);
  std::vector<Rect> rects(nrect);
  in.read(reinterpret_cast<char*>(rects.data()), static_cast<std::streamsize>(nrect * sizeof(Rect)));
  in.read(reinterpret_cast<char*>(&nnet), 4);
  std::vector<Query> queries(nnet);
  in.read(reinterpret_cast<char*>(queries.data()),
          static_cast<std::streamsize>(nnet * sizeof(Query)));
  if (!in || size == 0 || nnet == 0) {
    std::cerr << "ref_lattice: malformed input\n";
    return 2;
  }
  std::vector<unsigned char> out;
  put<uint64_t>(&out, 0x3154414c54524741ull);  // "AGRTLAT1"
  put<uint32_t>(&out, size);
  std::vector<unsigned char> routes;
  for (uint32_t qi = 0; qi < nnet; ++qi) {
    const Query& q = queries[qi];
    auto board_result = apgar::board_ir::CreateBoardSnapshot(make_board(rects, q));
    if (!std::holds_alternative<BoardSnapshot>(board_result)) {
      std::cerr << "board: " << std::get<apgar::board_ir::BoardValidationError>(board_result).message
                << "\n";
      return 1;
    }
    const BoardSnapshot& board = std::get<BoardSnapshot>(board_result);
    auto compiled_result = apgar::geometry_compiler::CompileBoard(board, make_profile(size));
    if (!std::holds_alternative<apgar::geometry_compiler::CompiledBoard>(compiled_result)) {
      std::cerr << "compile: "
                << std::get<apgar::geometry_compiler::CompileError>(compiled_result).detail << "\n";
      return 1;
    }
    const auto& compiled = std::get<apgar::geometry_compiler::CompiledBoard>(compiled_result);
    if (qi == 0) {
      for (uint32_t y = 0; y < size; ++y) {
        for (uint32_t x = 0; x < size; ++x) {
          const auto* node = compiled.FindNode(0, x, y);
          put<uint8_t>(&out, node == nullptr ? 0 : node->legal_edges);
        }
      }
    }
    apgar::routing::CpuRouteRequest req{.net = kNet,
                                        .start = node_point(q.sx, q.sy),
                                        .goal = node_point(q.gx, q.gy),
                                        .start_layer = 0,
                                        .goal_layer = 0,
                                        .candidate_policy = {}};
    auto result = apgar::routing::RouteWithCpuAStar(board, compiled, req);
    if (auto* route = std::get_if<apgar::routing::CpuRoute>(&result)) {
      put<uint32_t>(&routes, 0);
      put<uint64_t>(&routes, route->total_cost);
      put<uint64_t>(&routes, route->telemetry.expanded_states);
      put<uint64_t>(&routes, route->telemetry.queue_pops);
      put<uint32_t>(&routes, static_cast<uint32_t>(route->lattice_path.size()));
      for (const Point64& p : route->lattice_path) {
        put<uint32_t>(&routes, static_cast<uint32_t>(p.x / kStep));
        put<uint32_t>(&routes, static_cast<uint32_t>(p.y / kStep));
      }
    } else {
      const auto& f = std::get<apgar::routing::RouteFailure>(result);
      const bool disconnected = f.code == apgar::routing::RouteFailureCode::kDisconnected;
      put<uint32_t>(&routes, disconnected ? 1u : 2u);
      put<uint64_t>(&routes, UINT64_MAX);
      put<uint64_t>(&routes, 0);
      put<uint64_t>(&routes, 0);
      put<uint32_t>(&routes, 0);
      if (!disconnected) std::cerr << "query " << qi << ": " << f.detail << "\n";
    }
  }
  put<uint32_t>(&out, nnet);
  out.insert(out.end(), routes.begin(), routes.end());
  std::ofstream o(argv[2], std::ios::binary);
  o.write(reinterpret_cast<const char*>(out.data()), static_cast<std::streamsize>(out.size()));
  return o ? 0 : 1;
}
