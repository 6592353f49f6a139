// Launch record of the GPU geometry compile (geometry.cu, geometry_host.cu).
#pragma once

#include <cstdint>

namespace apgar_b200 {

struct GeometryLaunch {
  const int64_t* xy;          // lattice x, y per node
  const uint32_t* layer;      // per node
  const uint32_t* neighbor;   // [node][8], UINT32_MAX when not represented
  uint32_t node_count;
  const int64_t* box;         // [k][4] min x, min y, max x, max y (board units)
  const uint32_t* bin_start;  // per node: first index into bin_boxes
  const uint32_t* bin_count;  // per node: number of boxes
  const uint32_t* bin_boxes;  // box indices
  int64_t origin_x, origin_y, step;
  int64_t required;           // w + 2c (doubled distance)
  uint32_t heading_mask;      // bit 0 horizontal, 1 vertical, 2 diagonal
  uint8_t* legal;
};

}  // namespace apgar_b200
