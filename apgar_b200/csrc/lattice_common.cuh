// Shared definitions for the lattice-mode kernels (dense bit-packed layers,
// per-net windows, uint32 labels, bend 0, vias).
//
// Move model (identical to the CPU oracle):
//   orthogonal move legal iff both cells are free;
//   diagonal move legal iff both cells and both side cells are free;
//   via (l,x,y)<->(l+1,x,y) legal iff both cells are free and the via bit of
//   layer pair l is set (no via mask = all set);
//   a cell is free iff it is inside the net window and not blocked.
#pragma once

#include <cstdint>

#include "apgar_b200.h"

namespace apgar_b200 {

// Labels inside the kernels use 0x7FFFFFFF as "unreachable" so that
// label + cost never wraps in 32-bit arithmetic; the host admits a net only
// when (window cells) * (largest move cost) stays below this sentinel.
constexpr uint32_t kLabelInf = 0x7FFFFFFFu;
constexpr int kMaxLayers = 8;

struct LatticeDeviceView {
  const uint32_t* blocked;    // row planes [layers][height][words], as uploaded
  const uint32_t* via_ok;     // row planes [layers-1][height][words] or nullptr
  // Sweep planes: every plane row carries one guard word on each side (data
  // at +1), so a lane's 32-bit span fetch needs no bounds test.  Row-major
  // planes serve frames whose rows are lattice rows; column-major planes
  // (plane row = lattice column, bit = y) serve transposed frames.
  const uint32_t* sweep_rows;      // [layers][height][words + 2]
  const uint32_t* sweep_cols;      // [layers][width][words_t + 2]
  const uint32_t* sweep_via_rows;  // [layers-1][height][words + 2] or nullptr
  const uint32_t* sweep_via_cols;  // [layers-1][width][words_t + 2] or nullptr
  int32_t layers, height, width, words, words_t;
  uint32_t orth, diag, via;
  // Move legality per cell [layers][height][width]: bit d (0-7) = the planar
  // move in heading d is legal (target free, both side cells free for a
  // diagonal, target inside the lattice); bit 8 / 9 = the via to the layer
  // below / above is legal.  Built once at upload (frontier generator).
  const uint16_t* moves;
};

// Per-net workspace record produced by the host planner.  The net is swept
// in a frame whose rows are lattice rows (transposed == 0) or lattice
// columns (transposed == 1, chosen when the window is taller than wide), so
// the sequential sweep dimension is the window's shorter side.
struct NetPlan {
  uint32_t net;          // index into the caller's net array
  uint32_t pitch;        // frame row pitch in cells (multiple of 4)
  uint64_t dist_offset;  // cell offset of this net's label slab in the pool
  uint32_t rows;         // frame rows (swept sequentially)
  uint32_t width;        // frame row width
  uint32_t transposed;
  uint32_t reserved;
};

struct SweepLaunch {
  LatticeDeviceView lat;
  const apgar_b200_lattice_net* nets;
  const NetPlan* plans;
  uint32_t plan_count;
  uint32_t max_sweeps;
  uint32_t* dist_pool;
  apgar_b200_lattice_result* results;
  uint32_t* path_arena;
  uint64_t path_arena_capacity;
  unsigned long long* arena_cursor;
  const volatile uint32_t* cancel;  // host-mapped flag or nullptr
};

// One width class of the frontier form (lattice_frontier.cu).  The kernel
// is persistent: each resident warp group owns one workspace slot and reuses
// it for every net it takes.  Slot s holds `slab_cells` label words
// (label << 32 | ~list stamp, window layout [layer][y][x]) at
// words + s * slab_cells, and three queue lists of `list_cap` entries at
// lists + s * 3 * list_cap.
struct FrontierLaunch {
  LatticeDeviceView lat;
  const apgar_b200_lattice_net* nets;
  const NetPlan* plans;
  uint32_t plan_count;
  uint32_t max_rounds;
  uint32_t bucket_width;
  unsigned long long* words;
  uint32_t* lists;
  uint64_t slab_cells;  // label words per slot (>= the class's largest padded window)
  uint32_t list_cap;    // entries per queue list per slot
  uint32_t slots;       // workspace slots of this class (resident groups)
  // per_net != 0: every net has its own slab at plan.dist_offset (words) and
  // lists at 3 * plan.dist_offset (entries), used when all of them fit; the
  // slots then only bound the number of groups
  uint32_t per_net;
  apgar_b200_lattice_result* results;
  uint32_t* path_arena;
  uint64_t path_arena_capacity;
  unsigned long long* arena_cursor;
  unsigned int* next_plan;            // work-stealing cursor of this class
  const volatile uint32_t* cancel;  // host-mapped flag or nullptr
  // optional per-cell entry price [layers][height][width] (negotiated
  // congestion snapshot); a move into cell c costs its move cost + cell_cost[c]
  const uint32_t* cell_cost;
  // optional partial rip-up: a net with skip[net] != 0 is not searched; its
  // previous result and path (prev_results, packed prev_paths) are carried over
  const uint8_t* skip;
  const apgar_b200_lattice_result* prev_results;
  const uint32_t* prev_paths;
  // optional rip-up pricing (needs cell_cost, prev_results and prev_paths):
  // a move into a cell of the net's own previous path costs cell_cost_own
  // instead of cell_cost.  own_bits is one bit per label word, laid out like
  // `words` (bit i of word k / 32 belongs to label word k); a net clears and
  // fills its slab's bits before its search.
  const uint32_t* cell_cost_own;
  uint32_t* own_bits;
  // optional corridor mode: net n's corridor is the 64 x 64 coarse bitmap at
  // corridor + 128 * n (bit cx of word 2 * cy + cx / 32; a coarse cell covers
  // 2^s x 2^s window cells on every layer, s the least value >= 2 that keeps
  // the window within 63 coarse cells per side); corridor_status[n] receives
  // the net's APGAR_B200_CORRIDOR_* outcome
  const uint32_t* corridor;
  uint8_t* corridor_status;
  // optional: the class's plan count, read on the device (overrides plan_count)
  const uint32_t* plan_count_dev;
  // chained expansions after each queued cell within a round (0 = none)
  uint32_t chain;
};

// Threads of a frontier CTA: one 16-warp group, which splits down to single
// warps as the width classes drain.
constexpr int kFrontierThreads = 512;

// The width classes of one frontier execution, by warps per net 1, 2, 4, 8
// and 16 (a class with no slots or no nets is skipped).
struct FrontierClasses {
  FrontierLaunch c[5];
};

__device__ __forceinline__ uint32_t sat(uint32_t v) { return v < kLabelInf ? v : kLabelInf; }

// 32 bits of a bit-packed row starting at signed bit position `pos`; bits
// outside [0, words*32) read as 1 (blocked).
__device__ __forceinline__ uint32_t fetch_bits32(const uint32_t* row, int words, int pos) {
  const int wi = pos >= 0 ? (pos >> 5) : -(((-pos) + 31) >> 5);
  const int sh = pos - wi * 32;
  const uint32_t lo = (wi >= 0 && wi < words) ? __ldg(row + wi) : 0xFFFFFFFFu;
  const uint32_t hi = (wi + 1 >= 0 && wi + 1 < words) ? __ldg(row + wi + 1) : 0xFFFFFFFFu;
  return __funnelshift_r(lo, hi, sh);
}

}  // namespace apgar_b200
