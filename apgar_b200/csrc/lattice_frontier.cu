// Lattice-mode frontier search: bucketed, label-correcting A* per net window,
// one warp group per net, persistent work stealing over the nets of a width
// class, all classes in one launch of 16-warp CTAs that split into narrower
// groups as the classes drain (lattice_frontier_kernel, at the end).
//
// A cell is keyed by f = g + h, with h the admissible, consistent
// octile-plus-via bound to the goal.  The search works through key levels
// of width delta (the bucket width), with thr the current level's upper bound:
//   * a round expands every cell of the current list.  It relaxes the 8
//     planar moves and the 2 vias, and a lowered cell joins the next round's
//     list if its key is below thr, else the deferred ("far") list;
//   * when a round leaves the current list empty, the level is done: thr
//     grows by delta and the far list becomes the current list.  Every
//     child key lies within twice the largest move cost of its parent's key,
//     and the host keeps delta >= 2 * max move, so the far list holds exactly
//     the next level: a cell that left it keeps a key below thr from then on
//     and never rejoins it, which is why far bits are never cleared.
// The search stops when nothing is queued (disconnected, or every reachable
// cell is final), or when a level is done with thr above the goal label.
//
// Why the labels the canonical walk reads are exact: f is non-decreasing
// along any optimal path under a consistent h, so every cell on an optimal
// start-goal path has true f at most the optimum C*.
//  - Suppose such a cell's label were still above its distance.  Take the
//    first inexact cell on its optimal path; its predecessor p is exact.
//  - When p's label became exact, p was queued.  Had p been expanded since,
//    the next cell would be exact, so p must still be waiting.
//  - A cell waiting in the current list blocks the stop (the list is empty at
//    a stop).  p in the far list means its key was at least the current thr,
//    yet its key f*(p) <= C* <= goal label < thr at the stop, a contradiction.
// The canonical walk accepts a predecessor only when label + move cost equals
// the current label, and an upper-bound label passes that test only when it
// is exact.  So the reverse path equals the one under full-window exact
// labels (reference tie-break, gpu/cuda/planar_router.cu:977-1009 and
// :1084-1165).
//
// The heuristic follows the reference's octile bound (src/routing/
// cpu_astar.cc:176-190), plus |dl| * via for the layer difference.
//
// Each cell's 64-bit word holds its label in the high half and, in the low
// half, ~s for the list it last joined: s = r + 1 for the list of round r,
// s = 2^31 | k for the far list of level k.  One 64-bit atomicMin both lowers
// the label and reports whether the cell already sits in the list it would
// join (a lowered cell joins the current level's next list or the far list,
// never both in one level, because its key only falls).  So no list ever
// holds more entries than the window has cells.
// Every search clears its words first (the whole window, or the corridor's
// blocks).  Measured against an epoch tag in the word (no clearing: a stale
// tag reads as unlabelled) on the medium batch: the clear-first form is 18.1
// ms per batch, the epoch form 22.0 ms with the same rounds and expansions.
// The stores pull the window into L2 before the latency-bound round chain
// starts, and with the label in the high half every label read and atomic
// result is a plain register, where a tag costs a shift, mask and compare
// on every one.
// Queue lists hold at most `list_cap` entries per slot; a net whose list
// would outgrow it is reported REJECTED (never a truncated search).
// Queue entries are packed cells (layer << 28 | y << 14 | x, window-local).
// Appends take one packed warp scan and one shared atomic per warp and list.
//
// Corridor mode (kCorr): a net first searches only the cells of its corridor,
// a bitmap of coarse cells (2^s x 2^s lattice cells, all layers) over its
// window.  Every legal move from a corridor cell u into a window cell v
// outside the corridor is an exit; the search keeps the least key g(u) +
// cost(u, v) + h(v) over all exits it expands.  The corridor result is
// accepted (certified) only when its goal label C is strictly below that
// least exit key:
//  - any start-goal path that leaves the corridor first leaves it by some
//    exit (u, v) with its prefix inside the corridor, so it costs at least
//    that exit's key with the exact corridor distance of u;
//  - every exit whose exact key is at most C is expanded with its exact
//    label before the search stops (the same argument as for the labels
//    above, on the corridor subgraph), and the least key over stale labels
//    is never below the exact one;
//  - so with C below the least key no optimal full-window path leaves the
//    corridor: C is the full-window optimum, every cell on an optimal path
//    has its exact label, and no outside cell passes the walk's equality
//    test, so the canonical path is the full-window one as well.
// Otherwise (goal not reached in the corridor, a terminal outside it, or an
// exit key at or below C) the same group clears the whole window and searches
// it without the corridor.  Cells outside the corridor are never read or
// written in the corridor pass, so only the corridor's blocks are cleared.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "lattice_common.cuh"

namespace apgar_b200 {
namespace {

// The cancel flag lives in host-mapped memory: every read crosses the bus, so
// each group reads it at the start of a net and then every 256 rounds.
constexpr int kCancelPollRounds = 256;

// No chained expansion follows (a packed cell never has all bits set).
constexpr uint32_t kNoLink = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t pack_cell(int l, int x, int y) {
  return (static_cast<uint32_t>(l) << 28) | (static_cast<uint32_t>(y) << 14) |
         static_cast<uint32_t>(x);
}

struct Window {
  int x0, y0, w, h;
  int gl, gx, gy;  // goal, window-local
};

__device__ __forceinline__ uint32_t cell_index(const Window& win, int l, int x, int y) {
  return (static_cast<uint32_t>(l) * static_cast<uint32_t>(win.h) + static_cast<uint32_t>(y)) *
             static_cast<uint32_t>(win.w) +
         static_cast<uint32_t>(x);
}

// Planar heading d (0 E, 1 NE, 2 N, 3 NW, 4 W, 5 SW, 6 S, 7 SE) as a step.
__host__ __device__ constexpr int fdx(int d) {
  return (d == 0 || d == 1 || d == 7) ? 1 : (d == 2 || d == 6) ? 0 : -1;
}
__host__ __device__ constexpr int fdy(int d) {
  return (d >= 1 && d <= 3) ? 1 : (d == 0 || d == 4) ? 0 : -1;
}

// Admissible, consistent bound on the remaining cost: octile in the plane,
// the via cost per layer of difference.
__device__ __forceinline__ uint32_t heuristic(const LatticeDeviceView& lat, const Window& win,
                                              int l, int x, int y) {
  const uint32_t dx = static_cast<uint32_t>(abs(x - win.gx));
  const uint32_t dy = static_cast<uint32_t>(abs(y - win.gy));
  const uint32_t lo = min(dx, dy), hi = max(dx, dy);
  const uint32_t planar = lat.diag >= lat.orth
                              ? lo * min(lat.diag, 2u * lat.orth) + (hi - lo) * lat.orth
                              : hi * lat.diag;
  return planar + static_cast<uint32_t>(abs(l - win.gl)) * lat.via;
}

__device__ __forceinline__ bool cell_free_w(const LatticeDeviceView& lat, const Window& win, int l,
                                            int x, int y) {
  if (l < 0 || l >= lat.layers || x < 0 || y < 0 || x >= win.w || y >= win.h) return false;
  const int gx = win.x0 + x, gy = win.y0 + y;
  const uint32_t word =
      __ldg(lat.blocked + (static_cast<size_t>(l) * lat.height + gy) * lat.words + (gx >> 5));
  return ((word >> (gx & 31)) & 1u) == 0;
}

__device__ __forceinline__ bool via_allowed(const LatticeDeviceView& lat, const Window& win,
                                            int lower, int x, int y) {
  if (lat.via_ok == nullptr) return true;
  const int gx = win.x0 + x, gy = win.y0 + y;
  const uint32_t word =
      __ldg(lat.via_ok + (static_cast<size_t>(lower) * lat.height + gy) * lat.words + (gx >> 5));
  return ((word >> (gx & 31)) & 1u) != 0;
}

__device__ __forceinline__ uint32_t label_of(const unsigned long long* w) {
  return static_cast<uint32_t>(__ldcg(w) >> 32);
}

// Corridor membership of window cell (x, y): bit x >> s of row y >> s of the
// net's 64 x 64 coarse bitmap (two words per coarse row).
__device__ __forceinline__ bool corr_has(const uint32_t* corr, int cshift, int x, int y) {
  const uint32_t cx = static_cast<uint32_t>(x) >> cshift, cy = static_cast<uint32_t>(y) >> cshift;
  return ((corr[cy * 2u + (cx >> 5)] >> (cx & 31u)) & 1u) != 0u;
}

template <int G>
__device__ __forceinline__ void fsync(int barrier_id) {
  if constexpr (G == 1) {
    __syncwarp();
  } else {
    __threadfence_block();
    asm volatile("bar.sync %0, %1;" ::"r"(barrier_id), "r"(G * 32) : "memory");
  }
}

// Expands one queued cell.  The memory operations are issued move-parallel in
// three waves: the cell's label and its precomputed move legality, then the
// labels of the legal neighbours, then their 64-bit atomicMins.  Lowered
// neighbours whose list stamp this call set are flagged in cur_mask (next
// round's list) or far_mask (far list); ne[d] holds the packed cell, and link
// the least-key cell flagged in cur_mask (kNoLink if none).
// kSpeculate: the neighbour labels are loaded together with the legality word
// (one wave less per hop, for the latency-bound wide classes); otherwise only
// the legal neighbours' labels are loaded (fewer requests, for the
// throughput-bound narrow classes).
template <bool kPriced, bool kCorr, bool kSpeculate>
__device__ __forceinline__ void expand_cell(const LatticeDeviceView& lat, const Window& win,
                                            uint32_t e, unsigned long long* words, uint32_t thr,
                                            uint32_t cur_low, uint32_t far_low,
                                            const uint32_t* cell_cost, const uint32_t* cost_own,
                                            const uint32_t* own, const uint32_t* corr, int cshift,
                                            uint32_t& exit_min, uint32_t (&ne)[10],
                                            uint32_t& cur_mask, uint32_t& far_mask, bool& overflow,
                                            uint32_t& link) {
  const int l = static_cast<int>(e >> 28), y = static_cast<int>((e >> 14) & 0x3FFFu),
            x = static_cast<int>(e & 0x3FFFu);
  const uint32_t w = static_cast<uint32_t>(win.w);
  const uint32_t plane = w * static_cast<uint32_t>(win.h);
  const uint32_t here = (static_cast<uint32_t>(l) * static_cast<uint32_t>(win.h) +
                         static_cast<uint32_t>(y)) * w + static_cast<uint32_t>(x);
  const bool xl = x > 0, xr = x + 1 < win.w, yd = y > 0, yu = y + 1 < win.h;
  const bool ld = l > 0, lu = l + 1 < lat.layers;
  const uint32_t inside = (xr ? 1u : 0u) | ((xr && yu) ? 2u : 0u) | (yu ? 4u : 0u) |
                          ((xl && yu) ? 8u : 0u) | (xl ? 16u : 0u) | ((xl && yd) ? 32u : 0u) |
                          (yd ? 64u : 0u) | ((xr && yd) ? 128u : 0u) | (ld ? 256u : 0u) |
                          (lu ? 512u : 0u);
  const int X = win.x0 + x, Y = win.y0 + y;
  // wave 1: own label and the cell's move legality (one precomputed word)
  const uint32_t gv = static_cast<uint32_t>(__ldcg(words + here) >> 32);
  const uint16_t* mv_at = lat.moves + (static_cast<size_t>(l) * lat.height + Y) * lat.width + X;
  // neighbours inside the corridor (a via keeps the cell's column); only
  // these are read, lowered or priced
  uint32_t corr_in = 0x3FFu;
  if constexpr (kCorr) {
    corr_in = 0x300u;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
      if ((inside & (1u << d)) && corr_has(corr, cshift, x + fdx(d), y + fdy(d))) corr_in |= 1u << d;
    }
  }
  uint32_t seen[10];
  uint32_t legal, reach;
  if constexpr (kSpeculate) {
    // wave 1 also loads every in-window neighbour label
#pragma unroll
    for (int d = 0; d < 10; ++d) {
      const uint32_t ni = d < 8 ? here + static_cast<uint32_t>(fdy(d)) * w + static_cast<uint32_t>(fdx(d))
                                : (d == 8 ? here - plane : here + plane);
      seen[d] = ((inside & corr_in) & (1u << d)) ? static_cast<uint32_t>(__ldcg(words + ni) >> 32) : 0u;
    }
    legal = static_cast<uint32_t>(__ldg(mv_at)) & inside;
    reach = legal & corr_in;
  } else {
    legal = static_cast<uint32_t>(__ldg(mv_at)) & inside;
    reach = legal & corr_in;
    // wave 2: the labels of the legal neighbours only
#pragma unroll
    for (int d = 0; d < 10; ++d) {
      const uint32_t ni = d < 8 ? here + static_cast<uint32_t>(fdy(d)) * w + static_cast<uint32_t>(fdx(d))
                                : (d == 8 ? here - plane : here + plane);
      seen[d] = (reach & (1u << d)) ? static_cast<uint32_t>(__ldcg(words + ni) >> 32) : 0u;
    }
  }
  // entry prices of the neighbours (0 without a price snapshot); a cell of
  // the net's own previous path is priced without the net's own use
  uint32_t price[10];
#pragma unroll
  for (int d = 0; d < 10; ++d) {
    price[d] = 0u;
    if (kPriced && (reach & (1u << d))) {
      const int nl = d == 8 ? l - 1 : (d == 9 ? l + 1 : l);
      const int px = d < 8 ? X + fdx(d) : X, py = d < 8 ? Y + fdy(d) : Y;
      const uint32_t* src = cell_cost;
      if (own != nullptr) {
        const uint32_t ni = d < 8 ? here + static_cast<uint32_t>(fdy(d)) * w + static_cast<uint32_t>(fdx(d))
                                  : (d == 8 ? here - plane : here + plane);
        if ((__ldcg(own + (ni >> 5)) >> (ni & 31u)) & 1u) src = cost_own;
      }
      price[d] = __ldg(src + (static_cast<size_t>(nl) * lat.height + py) * lat.width + px);
    }
  }
  // heuristic parts: |column - goal| and |row - goal| for the 3x3 neighbourhood
  const int ax[3] = {abs(x - 1 - win.gx), abs(x - win.gx), abs(x + 1 - win.gx)};
  const int ay[3] = {abs(y - 1 - win.gy), abs(y - win.gy), abs(y + 1 - win.gy)};
  const uint32_t dstep = lat.diag >= lat.orth ? min(lat.diag, 2u * lat.orth) : lat.diag;
  // wave 3: lower the labels (all atomics issued before any result is used);
  // the low half records the list the cell joins
  uint32_t cand[10], low[10];
  unsigned long long old[10];
  // key of the neighbour reached by move m at label c
  const auto key_of = [&](int m, uint32_t c) {
    const int mx = m < 8 ? fdx(m) : 0, my = m < 8 ? fdy(m) : 0;
    const int nl = m == 8 ? l - 1 : (m == 9 ? l + 1 : l);
    const uint32_t a = static_cast<uint32_t>(ax[1 + mx]), b = static_cast<uint32_t>(ay[1 + my]);
    const uint32_t lo = min(a, b), hi = max(a, b);
    const uint32_t planar = lat.diag >= lat.orth ? lo * dstep + (hi - lo) * lat.orth : hi * dstep;
    return c + planar + static_cast<uint32_t>(abs(nl - win.gl)) * lat.via;
  };
#pragma unroll
  for (int d = 0; d < 10; ++d) {
    const uint32_t cost = d >= 8 ? lat.via : ((d & 1) ? lat.diag : lat.orth);
    // gv < 2^31 and price < 2^31: the sum cannot wrap; at or above the
    // sentinel it leaves the 32-bit cost domain and the net is rejected
    cand[d] = gv + cost + price[d];
    low[d] = 0u;
    old[d] = 0ull;
    if (kPriced && (legal & (1u << d)) && cand[d] >= kLabelInf) {
      overflow = true;
      continue;
    }
    if constexpr (kCorr) {
      if (legal & ~corr_in & (1u << d)) exit_min = min(exit_min, key_of(d, cand[d]));  // a corridor exit
    }
    if ((legal & (1u << d)) && cand[d] < seen[d]) {
      const int dx = d < 8 ? fdx(d) : 0, dy = d < 8 ? fdy(d) : 0;
      const uint32_t key = key_of(d, cand[d]);
      low[d] = key < thr ? cur_low : far_low;
      const uint32_t ni = d < 8 ? here + static_cast<uint32_t>(dy) * w + static_cast<uint32_t>(dx)
                                : (d == 8 ? here - plane : here + plane);
      old[d] = atomicMin(words + ni, (static_cast<unsigned long long>(cand[d]) << 32) | low[d]);
    }
  }
  cur_mask = 0;
  far_mask = 0;
  link = kNoLink;
  uint32_t link_key = 0xFFFFFFFFu;
#pragma unroll
  for (int d = 0; d < 10; ++d) {
    // old == 0 marks a move that was not attempted (label 0 is never lowered)
    if (cand[d] < static_cast<uint32_t>(old[d] >> 32) && static_cast<uint32_t>(old[d]) != low[d]) {
      const int dx = d < 8 ? fdx(d) : 0, dy = d < 8 ? fdy(d) : 0;
      const int nl = d == 8 ? l - 1 : (d == 9 ? l + 1 : l);
      ne[d] = pack_cell(nl, x + dx, y + dy);
      if (low[d] == cur_low) {
        cur_mask |= 1u << d;
        // the least-key cell this expansion queued for the next round: the
        // one a chained expansion follows
        const uint32_t k = key_of(d, cand[d]);
        if (k < link_key) {
          link_key = k;
          link = ne[d];
        }
        // (no L2 prefetch of the queued cell's neighbourhood: measured on the
        // medium batch, the prefetches cost 4% of the batch and 8% of the
        // largest window's round chain)
      } else {
        far_mask |= 1u << d;
      }
    }
  }
}

struct GroupShared {
  uint32_t count[3];  // next-round list being built, rotated per round
  uint32_t far_count;
  uint32_t plan;
  uint32_t cancel[2];
  uint32_t overflow;
  uint32_t bound;  // corridor pass: least expanded exit key
  uint32_t corr_any;  // the net's corridor bitmap has a bit set
  uint32_t sums[16];
};

// One warp group of G warps works through the nets of one width class until
// the class's work-stealing cursor runs past its last net, then returns.
// g: the warp's index within the group; barrier_id: the group's named
// barrier (unused for G = 1); sh and corr: the group's own shared state.
// kPriced: the plan carries per-cell entry prices (p.cell_cost != nullptr);
// the unpriced instantiation has no price loads or overflow tests at all.
// kCorr: corridor mode (p.corridor != nullptr), priced or not: entry prices
// are non-negative, so the octile-plus-via bound stays admissible and every
// exit key (which leaves out the exit cell's own price) stays a lower bound
// on any path through that exit.
template <int G, bool kPriced, bool kCorr>
__device__ __forceinline__ void frontier_group(const FrontierLaunch& p, uint32_t slot, int g,
                                               int barrier_id, GroupShared& sh,
                                               uint32_t* const corr) {
  constexpr int T = G * 32;
  const int lane = threadIdx.x & 31;
  const int tid = g * 32 + lane;
  const LatticeDeviceView& lat = p.lat;
  const uint32_t orth = lat.orth, diag = lat.diag, via = lat.via;
  if (slot >= p.slots) return;  // whole group: no workspace slot of its own in this class
  unsigned long long* const slot_words = p.words + static_cast<uint64_t>(slot) * p.slab_cells;
  uint32_t* const slot_lists = p.lists + static_cast<uint64_t>(slot) * 3u * p.list_cap;
  const uint32_t cap = p.list_cap;

  for (;;) {
    if (tid == 0) {
      sh.plan = atomicAdd(p.next_plan, 1u);
      sh.corr_any = 0u;
    }
    fsync<G>(barrier_id);
    const uint32_t plan_index = sh.plan;
    if (plan_index >= (p.plan_count_dev != nullptr ? *p.plan_count_dev : p.plan_count)) {
      return;  // uniform within the group
    }
    const NetPlan plan = p.plans[plan_index];
    if (p.skip != nullptr && p.skip[plan.net] != 0u) {  // uniform within the group
      // kept route: carry the previous result and path into this execution
      if (g == 0) {
        apgar_b200_lattice_result res = p.prev_results[plan.net];
        res.arena_offset = 0;
        if (res.completion == APGAR_B200_COMPLETION_REACHED && res.path_len > 0) {
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(p.arena_cursor, static_cast<unsigned long long>(res.path_len));
          base = __shfl_sync(0xFFFFFFFFu, base, 0);
          if (base + res.path_len > p.path_arena_capacity) {
            res.completion = APGAR_B200_COMPLETION_REJECTED;
            res.cost = APGAR_B200_UNREACHABLE;
            res.path_len = 0;
          } else {
            for (uint32_t j = lane; j < res.path_len; j += 32) {
              p.path_arena[base + j] = p.prev_paths[res.path_offset + j];
            }
            res.arena_offset = base;
          }
        }
        if (lane == 0) p.results[plan.net] = res;
      }
      fsync<G>(barrier_id);
      continue;
    }
    const apgar_b200_lattice_net net = p.nets[plan.net];
    Window win;
    win.x0 = static_cast<int>(net.win_x0);
    win.y0 = static_cast<int>(net.win_y0);
    win.w = static_cast<int>(net.win_w);
    win.h = static_cast<int>(net.win_h);
    win.gl = static_cast<int>(net.goal_layer);
    win.gx = static_cast<int>(net.goal_x) - win.x0;
    win.gy = static_cast<int>(net.goal_y) - win.y0;
    const int sl = static_cast<int>(net.start_layer);
    const int sx = static_cast<int>(net.start_x) - win.x0, sy = static_cast<int>(net.start_y) - win.y0;
    const uint32_t cells = static_cast<uint32_t>(lat.layers) * win.w * win.h;
    const uint32_t padded = (cells + 127u) & ~127u;
    // a list never holds more entries than the net has cells, so the three
    // lists sit that far apart (inside a slot the cap binds above it)
    const uint32_t span = p.per_net ? cells : (cells < cap ? cells : cap);
    unsigned long long* words = p.per_net ? p.words + plan.dist_offset : slot_words;
    // own-path bits of this slab (rip-up pricing from the second round on)
    uint32_t* const own =
        (kPriced && p.cell_cost_own != nullptr)
            ? p.own_bits + (p.per_net ? plan.dist_offset : static_cast<uint64_t>(slot) * p.slab_cells) / 32u
            : nullptr;
    uint32_t* list_a = p.per_net ? p.lists + 3ull * plan.dist_offset : slot_lists;
    uint32_t* list_b = list_a + span;
    uint32_t* list_c = list_b + span;

    // corridor: the coarse scale keeps the window within 63 x 63 coarse cells
    int cshift = 2;
    bool use_corr = false;
    uint32_t cstatus = 0;  // corridor outcome of this net (APGAR_B200_CORRIDOR_*)
    if constexpr (kCorr) {
      const int span_max = win.w > win.h ? win.w : win.h;
      while (((span_max - 1) >> cshift) >= 63) ++cshift;  // at most 63 coarse cells a side
      const uint32_t* src = p.corridor + static_cast<size_t>(plan.net) * 128u;
      for (int i = tid; i < 128; i += T) {
        const uint32_t word = __ldg(src + i);
        corr[i] = word;
        if (word != 0u) sh.corr_any = 1u;
      }
      fsync<G>(barrier_id);
      use_corr = corr_has(corr, cshift, sx, sy) && corr_has(corr, cshift, win.gx, win.gy);
      // an empty bitmap proposes no corridor: the window is searched at once
      cstatus = use_corr ? APGAR_B200_CORRIDOR_CERTIFIED
                         : (sh.corr_any != 0u ? APGAR_B200_CORRIDOR_FALLBACK_UNREACHED
                                              : APGAR_B200_CORRIDOR_NONE);
    }
    const bool endpoints_free = cell_free_w(lat, win, sl, sx, sy) &&
                                cell_free_w(lat, win, win.gl, win.gx, win.gy);
    uint32_t completion = APGAR_B200_COMPLETION_DISCONNECTED;
    uint32_t rounds = 0, levels = 0, total_rounds = 0, total_levels = 0;
    uint32_t expanded = 0;  // this thread's expansions
    bool first_pass = true;  // the own-route bits are set once per net
    // corridor pass first (corridor mode), then the whole window if the
    // corridor result is not certified
    for (;;) {
    if (kCorr && use_corr) {
      // only the corridor's blocks are ever touched: clear them, row by row
      const uint32_t bs = 1u << cshift;
      const uint32_t rows_all = static_cast<uint32_t>(lat.layers) * static_cast<uint32_t>(win.h);
      for (uint32_t rr = tid; rr < rows_all; rr += T) {
        const uint32_t yy = rr % static_cast<uint32_t>(win.h);
        const uint32_t cy = yy >> cshift;
        unsigned long long* row = words + static_cast<size_t>(rr) * static_cast<uint32_t>(win.w);
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
          uint32_t bits = corr[cy * 2u + half];
          while (bits != 0u) {
            const uint32_t cx = static_cast<uint32_t>(half * 32 + __ffs(bits) - 1);
            bits &= bits - 1u;
            const uint32_t x0 = cx << cshift;
            const uint32_t x1 = min(x0 + bs, static_cast<uint32_t>(win.w));
            for (uint32_t x = x0; x < x1; ++x) row[x] = 0x7FFFFFFFFFFFFFFFull;
          }
        }
      }
    } else {
      // clear the net's label words (16-byte stores over the padded slab)
      uint4* w4 = reinterpret_cast<uint4*>(words);
      const uint4 inf2 = make_uint4(0xFFFFFFFFu, kLabelInf, 0xFFFFFFFFu, kLabelInf);
      for (uint32_t i = tid; i < padded / 2; i += T) w4[i] = inf2;
    }
    if (own != nullptr && first_pass) {
      for (uint32_t i = tid; i < padded / 32u; i += T) own[i] = 0u;
    }
    // every clearing store of the group lands before the start is seeded
    fsync<G>(barrier_id);
    if (own != nullptr && first_pass) {
      // mark the cells of the net's previous route (packed reverse path of
      // global cell ids); cells outside the window cannot be entered anyway
      const apgar_b200_lattice_result prev = p.prev_results[plan.net];
      if (prev.completion == APGAR_B200_COMPLETION_REACHED) {
        const uint32_t lw = static_cast<uint32_t>(lat.width), lh = static_cast<uint32_t>(lat.height);
        for (uint32_t j = tid; j < prev.path_len; j += T) {
          const uint32_t c = p.prev_paths[prev.path_offset + j];
          const int cx = static_cast<int>(c % lw) - win.x0;
          const int cy = static_cast<int>((c / lw) % lh) - win.y0;
          const uint32_t cl = c / lw / lh;
          if (cl < static_cast<uint32_t>(lat.layers) && cx >= 0 && cx < win.w && cy >= 0 && cy < win.h) {
            const uint32_t i = cell_index(win, static_cast<int>(cl), cx, cy);
            atomicOr(own + (i >> 5), 1u << (i & 31u));
          }
        }
      }
    }
    if (tid == 0) {
      sh.count[0] = sh.count[1] = sh.count[2] = 0;
      sh.far_count = 0;
      sh.cancel[0] = sh.cancel[1] = 0;
      sh.overflow = 0;
      sh.bound = 0xFFFFFFFFu;
      if (endpoints_free) {
        // label 0, in the list of round 0 (stamp 1)
        words[cell_index(win, sl, sx, sy)] = 0xFFFFFFFFull - 1ull;
        list_a[0] = pack_cell(sl, sx, sy);
      }
    }
    fsync<G>(barrier_id);

    completion = APGAR_B200_COMPLETION_DISCONNECTED;
    rounds = 0;
    levels = 0;
    uint32_t exit_min = 0xFFFFFFFFu;  // this thread's least corridor exit key
    if (endpoints_free) {
      const uint32_t goal_index = cell_index(win, win.gl, win.gx, win.gy);
      const uint32_t delta = p.bucket_width;
      const uint32_t h0 = heuristic(lat, win, sl, sx, sy);
      uint32_t thr = h0 + min(delta, 0xFFFFFFFFu - h0);
      uint32_t n = 1;
      uint32_t* cur = list_a;
      uint32_t* nxt = list_b;
      uint32_t* far = list_c;
      completion = APGAR_B200_COMPLETION_REACHED;  // refined from the goal label below
      for (uint32_t r = 0;; ++r) {
        // written during round r - 1, before its closing barrier
        if (r > 0 && sh.cancel[(r + 1) & 1] != 0u) {
          completion = APGAR_B200_COMPLETION_CANCELLED;
          break;
        }
        if (n == 0u) {
          // ---- the level is done: open the next one from the far list ----
          const uint32_t nf = sh.far_count;
          const uint32_t goal_label = label_of(words + goal_index);
          if (nf == 0u) break;           // every reachable cell is final
          if (thr > goal_label) break;   // every cell with key <= C* is final
          ++levels;
          thr += min(delta, 0xFFFFFFFFu - thr);
          uint32_t* t = cur;
          cur = far;
          far = t;
          n = nf;
          fsync<G>(barrier_id);  // everyone has read the far count
          if (tid == 0) sh.far_count = 0;
          fsync<G>(barrier_id);
        }
        if (r == p.max_rounds) {
          completion = APGAR_B200_COMPLETION_BUDGET_EXHAUSTED;
          break;
        }
        rounds = r + 1;
        if (tid == 0) {
          sh.count[(r + 1) % 3] = 0;  // last read after round r - 2
          if (p.cancel != nullptr && (r % kCancelPollRounds) == 0u) {
            sh.cancel[r & 1] = *p.cancel != 0u ? 1u : 0u;
          } else {
            sh.cancel[r & 1] = sh.cancel[(r + 1) & 1];
          }
        }
        uint32_t* count = &sh.count[r % 3];
        const uint32_t cur_low = 0xFFFFFFFFu - (r + 2);              // list of round r + 1
        const uint32_t far_low = 0xFFFFFFFFu - (0x80000000u | levels);  // far list of this level
        for (uint32_t base = static_cast<uint32_t>(g) * 32u; base < n; base += T) {
          const uint32_t i = base + static_cast<uint32_t>(lane);
          bool valid = i < n;
          uint32_t cell = valid ? cur[i] : 0u;
          // the queued cell, then up to p.chain chained expansions: each
          // follows the least-key cell the previous one queued for the next
          // round (it stays queued, so the lists and the stop rule are
          // unchanged; the chain only moves labels ahead within the round)
#pragma unroll 1
          for (uint32_t step = 0;; ++step) {
          uint32_t cur_mask = 0, far_mask = 0;
          uint32_t ne[10];
          uint32_t link = kNoLink;
          if (valid) {
            ++expanded;
            bool overflow = false;
            if (kCorr && use_corr) {
              expand_cell<kPriced, kCorr, (G >= 4)>(lat, win, cell, words, thr, cur_low, far_low,
                                          p.cell_cost, p.cell_cost_own, own, corr, cshift,
                                          exit_min, ne, cur_mask, far_mask, overflow, link);
            } else {
              expand_cell<kPriced, false, (G >= 4)>(lat, win, cell, words, thr, cur_low, far_low,
                                          p.cell_cost, p.cell_cost_own, own, corr, cshift,
                                          exit_min, ne, cur_mask, far_mask, overflow, link);
            }
            if (overflow) sh.overflow = 1u;
          }
          // one packed warp scan places both lists' entries
          const uint32_t nc = __popc(cur_mask), nfar = __popc(far_mask);
          uint32_t packed = nc | (nfar << 16);
#pragma unroll
          for (int sft = 1; sft < 32; sft <<= 1) {
            const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, packed, sft);
            if (lane >= sft) packed += o;
          }
          const uint32_t totals = __shfl_sync(0xFFFFFFFFu, packed, 31);
          uint32_t at_cur = 0, at_far = 0;
          if (lane == 0) {
            if ((totals & 0xFFFFu) != 0u) at_cur = atomicAdd(count, totals & 0xFFFFu);
            if ((totals >> 16) != 0u) at_far = atomicAdd(&sh.far_count, totals >> 16);
          }
          at_cur = __shfl_sync(0xFFFFFFFFu, at_cur, 0) + (packed & 0xFFFFu) - nc;
          at_far = __shfl_sync(0xFFFFFFFFu, at_far, 0) + (packed >> 16) - nfar;
          if (p.per_net) {
            // a per-net list spans the net's cells: it cannot overflow
#pragma unroll
            for (int d = 0; d < 10; ++d) {
              if (cur_mask & (1u << d)) nxt[at_cur++] = ne[d];
              if (far_mask & (1u << d)) far[at_far++] = ne[d];
            }
          } else {
            bool lost = false;
#pragma unroll
            for (int d = 0; d < 10; ++d) {
              if (cur_mask & (1u << d)) {
                if (at_cur < span) nxt[at_cur] = ne[d]; else lost = true;
                ++at_cur;
              }
              if (far_mask & (1u << d)) {
                if (at_far < span) far[at_far] = ne[d]; else lost = true;
                ++at_far;
              }
            }
            if (lost) sh.overflow = 1u;  // a queue list is full: the net is rejected
          }
          if (step >= p.chain) break;  // uniform
          valid = valid && link != kNoLink;
          if (!__any_sync(0xFFFFFFFFu, valid)) break;
          cell = link;
          }  // chain
        }
        fsync<G>(barrier_id);
        n = *count;
        if (sh.overflow != 0u) break;  // uniform: read after the barrier
        uint32_t* t = cur;
        cur = nxt;
        nxt = t;
      }
    }
    total_rounds += rounds;
    total_levels += levels;
    if constexpr (kCorr) {
      if (use_corr) {
        // the certificate: goal label strictly below every expanded exit key
        exit_min = __reduce_min_sync(0xFFFFFFFFu, exit_min);
        if (lane == 0 && exit_min != 0xFFFFFFFFu) atomicMin(&sh.bound, exit_min);
        fsync<G>(barrier_id);
        const uint32_t goal_label = label_of(words + cell_index(win, win.gl, win.gx, win.gy));
        const bool reached = completion == APGAR_B200_COMPLETION_REACHED && goal_label < kLabelInf;
        const bool certified = !endpoints_free || (reached && goal_label < sh.bound);
        if (certified || completion == APGAR_B200_COMPLETION_CANCELLED) break;
        cstatus = reached ? APGAR_B200_CORRIDOR_FALLBACK_EXIT : APGAR_B200_CORRIDOR_FALLBACK_UNREACHED;
        use_corr = false;
        first_pass = false;
        fsync<G>(barrier_id);  // the bound and goal label are read before the next clear
        continue;
      }
    }
    break;
    }  // corridor retry
    rounds = total_rounds;
    levels = total_levels;
    // expansions summed over the group (reported in the row_steps field)
    expanded = __reduce_add_sync(0xFFFFFFFFu, expanded);
    if constexpr (G > 1) {
      fsync<G>(barrier_id);
      if (lane == 0) sh.sums[g] = expanded;
      fsync<G>(barrier_id);
      expanded = __reduce_add_sync(0xFFFFFFFFu, lane < G ? sh.sums[lane] : 0u);
    }

    // ------------------------- result + canonical walk -------------------------
    if (g == 0) {
      apgar_b200_lattice_result res{};
      res.cost = APGAR_B200_UNREACHABLE;
      res.completion = completion;
      res.sweeps = rounds;
      res.row_steps = expanded;
      res.row_stores = levels;
      if (sh.overflow != 0u) {
        // a path cost reached the 32-bit sentinel: no exact result exists here
        res.completion = APGAR_B200_COMPLETION_REJECTED;
      } else if (completion == APGAR_B200_COMPLETION_REACHED) {
        const uint32_t goal = label_of(words + cell_index(win, win.gl, win.gx, win.gy));
        if (goal >= kLabelInf) {
          res.completion = APGAR_B200_COMPLETION_DISCONNECTED;
        } else {
          res.cost = goal;
          const uint32_t min_move = min(orth, min(diag, via));
          const unsigned long long bound = goal / min_move + 1ull;
          unsigned long long base = 0;
          if (lane == 0) base = atomicAdd(p.arena_cursor, bound);
          base = __shfl_sync(0xFFFFFFFFu, base, 0);
          if (base + bound > p.path_arena_capacity) {
            res.completion = APGAR_B200_COMPLETION_REJECTED;
            res.cost = APGAR_B200_UNREACHABLE;
          } else {
            int cl = win.gl, cx = win.gx, cy = win.gy;
            uint32_t here = goal;
            uint32_t len = 0;
            bool ok = false;
            while (len < bound) {
              if (lane == 0) {
                p.path_arena[base + len] = static_cast<uint32_t>(
                    (static_cast<size_t>(cl) * lat.height + (win.y0 + cy)) * lat.width +
                    (win.x0 + cx));
              }
              ++len;
              if (cl == sl && cx == sx && cy == sy) {
                ok = true;
                break;
              }
              // the move into the current cell paid its entry price
              uint32_t here_price = 0u;
              if (kPriced) {
                const uint32_t hi = cell_index(win, cl, cx, cy);
                const bool mine = own != nullptr && ((__ldcg(own + (hi >> 5)) >> (hi & 31u)) & 1u);
                here_price = __ldg((mine ? p.cell_cost_own : p.cell_cost) +
                                   (static_cast<size_t>(cl) * lat.height + (win.y0 + cy)) *
                                       lat.width + (win.x0 + cx));
              }
              // lanes 0..7: planar predecessors by incoming heading; 8, 9: vias
              bool cand = false;
              int pl = cl, px = cx, py = cy;
              uint32_t pd = kLabelInf;
              if (lane < 8) {
                px = cx - fdx(lane);
                py = cy - fdy(lane);
                bool legal = cell_free_w(lat, win, cl, px, py);
                if (legal && (lane & 1)) {
                  legal = cell_free_w(lat, win, cl, cx, py) && cell_free_w(lat, win, cl, px, cy);
                }
                if (kCorr && use_corr && legal) legal = corr_has(corr, cshift, px, py);
                if (legal) {
                  pd = label_of(words + cell_index(win, cl, px, py));
                  cand = pd < kLabelInf && pd + ((lane & 1) ? diag : orth) + here_price == here;
                }
              } else if (lane == 8 || lane == 9) {
                pl = (lane == 8) ? cl - 1 : cl + 1;
                const int lower = (lane == 8) ? cl - 1 : cl;
                if (pl >= 0 && pl < lat.layers && cell_free_w(lat, win, pl, cx, cy) &&
                    via_allowed(lat, win, lower, cx, cy)) {
                  pd = label_of(words + cell_index(win, pl, cx, cy));
                  cand = pd < kLabelInf && pd + via + here_price == here;
                }
              }
              const unsigned ballot = __ballot_sync(0xFFFFFFFFu, cand);
              if (ballot == 0u) break;
              const int hsel = __ffs(ballot) - 1;
              cl = __shfl_sync(0xFFFFFFFFu, pl, hsel);
              cx = __shfl_sync(0xFFFFFFFFu, px, hsel);
              cy = __shfl_sync(0xFFFFFFFFu, py, hsel);
              here = __shfl_sync(0xFFFFFFFFu, pd, hsel);
            }
            if (ok) {
              res.path_len = len;
              res.arena_offset = base;
            } else {
              res.completion = APGAR_B200_COMPLETION_REJECTED;
              res.cost = APGAR_B200_UNREACHABLE;
            }
          }
        }
      }
      if (lane == 0) p.results[plan.net] = res;
      if (kCorr && lane == 0) p.corridor_status[plan.net] = static_cast<uint8_t>(cstatus);
    }
    // the group's shared slots are reused by its next net
    fsync<G>(barrier_id);
  }
}

// Group state of every (width, first warp) pair a CTA can hold: the 16-warp
// group, two 8-warp groups, four 4-warp, eight 2-warp and sixteen 1-warp
// groups (31 in all).  A group that splits hands over to its halves while
// they may still read its state, so no two of them share an entry.
__host__ __device__ constexpr int group_entry(int G, int w0) {
  return (G == 16 ? 0 : G == 8 ? 1 : G == 4 ? 3 : G == 2 ? 7 : 15) + w0 / G;
}

// The whole frontier of a plan in one persistent launch of 16-warp CTAs.
// Each CTA first serves the widest class as one 16-warp group; when that
// class's cursor is past its last net, the group splits into two 8-warp
// groups that serve the next class, and so on down to single warps.  So the
// widest nets (the batch's critical path) always start first, and a finished
// group's warps move on to narrower nets without waiting for the rest of the
// CTA.  Named barriers: 1 for the 16-warp group, 2-3, 4-7 and 8-15 for the
// 8-, 4- and 2-warp groups (single warps use __syncwarp).
template <bool kPriced, bool kCorr>
__global__ void __launch_bounds__(kFrontierThreads, 1)
    lattice_frontier_kernel(const __grid_constant__ FrontierClasses pc) {
  __shared__ GroupShared shared_groups[31];
  __shared__ uint32_t corridor_bits[kCorr ? 31 * 128 : 1];
  const int warp = threadIdx.x >> 5;
  const auto entry = [&](int G, int w0) { return group_entry(G, w0); };
  const auto corr_of = [&](int e) { return corridor_bits + (kCorr ? e * 128 : 0); };
  {
    const int e = entry(16, 0);
    frontier_group<16, kPriced, kCorr>(pc.c[4], blockIdx.x, warp, 1, shared_groups[e], corr_of(e));
  }
  {
    const int w0 = warp & ~7, e = entry(8, w0);
    frontier_group<8, kPriced, kCorr>(pc.c[3], blockIdx.x * 2u + w0 / 8, warp - w0, 2 + w0 / 8,
                                      shared_groups[e], corr_of(e));
  }
  {
    const int w0 = warp & ~3, e = entry(4, w0);
    frontier_group<4, kPriced, kCorr>(pc.c[2], blockIdx.x * 4u + w0 / 4, warp - w0, 4 + w0 / 4,
                                      shared_groups[e], corr_of(e));
  }
  {
    const int w0 = warp & ~1, e = entry(2, w0);
    frontier_group<2, kPriced, kCorr>(pc.c[1], blockIdx.x * 8u + w0 / 2, warp - w0, 8 + w0 / 2,
                                      shared_groups[e], corr_of(e));
  }
  {
    const int e = entry(1, warp);
    frontier_group<1, kPriced, kCorr>(pc.c[0], blockIdx.x * 16u + warp, 0, 0, shared_groups[e],
                                      corr_of(e));
  }
}

// Resident 16-warp CTAs per SM of the fullest instantiation (the others then
// keep their extra CTAs waiting: they start as others finish, and find the
// cursors past the end).
// Per device ordinal: resident CTAs per SM, 0 until first queried.
std::atomic<int> g_frontier_blocks[64];

cudaError_t frontier_blocks_per_sm(int* out) {
  int device = 0;
  if (cudaError_t e = cudaGetDevice(&device); e != cudaSuccess) return e;
  const bool cacheable = device >= 0 && device < 64;
  if (cacheable) {
    const int cached = g_frontier_blocks[device].load(std::memory_order_acquire);
    if (cached > 0) {
      *out = cached;
      return cudaSuccess;
    }
  }
  int plain = 0, priced = 0, corridor = 0, priced_corridor = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &plain, lattice_frontier_kernel<false, false>, kFrontierThreads, 0);
  if (e == cudaSuccess) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &priced, lattice_frontier_kernel<true, false>, kFrontierThreads, 0);
  }
  if (e == cudaSuccess) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &corridor, lattice_frontier_kernel<false, true>, kFrontierThreads, 0);
  }
  if (e == cudaSuccess) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &priced_corridor, lattice_frontier_kernel<true, true>, kFrontierThreads, 0);
  }
  if (e != cudaSuccess) return e;
  *out = max(1, max(max(plain, priced_corridor), max(priced, corridor)));
  if (cacheable) g_frontier_blocks[device].store(*out, std::memory_order_release);
  return cudaSuccess;
}

}  // namespace

namespace {

__device__ __forceinline__ bool lattice_free(const LatticeDeviceView& lat, int l, int x, int y) {
  if (l < 0 || l >= lat.layers || x < 0 || y < 0 || x >= lat.width || y >= lat.height) return false;
  const uint32_t word = lat.blocked[(static_cast<size_t>(l) * lat.height + y) * lat.words + (x >> 5)];
  return ((word >> (x & 31)) & 1u) == 0u;
}

// One thread per cell: the move rule of expand_cell, evaluated once.
__global__ void build_moves_kernel(LatticeDeviceView lat, uint16_t* __restrict__ moves) {
  const size_t cells = static_cast<size_t>(lat.layers) * lat.height * lat.width;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % lat.width);
    const int y = static_cast<int>((i / lat.width) % lat.height);
    const int l = static_cast<int>(i / (static_cast<size_t>(lat.width) * lat.height));
    uint32_t m = 0;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
      const int dx = fdx(d), dy = fdy(d);
      bool ok = lattice_free(lat, l, x + dx, y + dy);
      if (ok && (d & 1)) ok = lattice_free(lat, l, x + dx, y) && lattice_free(lat, l, x, y + dy);
      if (ok) m |= 1u << d;
    }
    const size_t col = static_cast<size_t>(y) * lat.words + (x >> 5);
    const size_t via_layer = static_cast<size_t>(lat.height) * lat.words;
    if (l > 0 && lattice_free(lat, l - 1, x, y) &&
        (lat.via_ok == nullptr || ((lat.via_ok[(l - 1) * via_layer + col] >> (x & 31)) & 1u))) {
      m |= 256u;
    }
    if (l + 1 < lat.layers && lattice_free(lat, l + 1, x, y) &&
        (lat.via_ok == nullptr || ((lat.via_ok[l * via_layer + col] >> (x & 31)) & 1u))) {
      m |= 512u;
    }
    moves[i] = static_cast<uint16_t>(m);
  }
}

}  // namespace

cudaError_t launch_build_moves(const LatticeDeviceView& lat, uint16_t* moves, cudaStream_t stream) {
  const size_t cells = static_cast<size_t>(lat.layers) * lat.height * lat.width;
  if (cells == 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>(std::min<size_t>((cells + 255) / 256, 148 * 32));
  build_moves_kernel<<<blocks, 256, 0, stream>>>(lat, moves);
  return cudaGetLastError();
}

cudaError_t lattice_frontier_resident_groups(int warps_per_net, int sm_count, uint32_t* out) {
  if (warps_per_net < 1 || warps_per_net > 16 || (warps_per_net & (warps_per_net - 1)) != 0) {
    return cudaErrorInvalidValue;
  }
  int blocks = 0;
  if (cudaError_t e = frontier_blocks_per_sm(&blocks); e != cudaSuccess) return e;
  *out = static_cast<uint32_t>(blocks) * static_cast<uint32_t>(max(1, sm_count)) *
         static_cast<uint32_t>(16 / warps_per_net);
  return cudaSuccess;
}

cudaError_t launch_lattice_frontier(const FrontierClasses& classes, int sm_count,
                                    cudaStream_t stream) {
  bool any = false, priced = false, corridor = false;
  for (const FrontierLaunch& c : classes.c) {
    if (c.plan_count == 0 && c.plan_count_dev == nullptr) continue;
    any = any || c.slots > 0;
    priced = priced || c.cell_cost != nullptr;
    corridor = corridor || c.corridor != nullptr;
  }
  if (!any) return cudaSuccess;
  int blocks = 0;
  if (cudaError_t e = frontier_blocks_per_sm(&blocks); e != cudaSuccess) return e;
  // every CTA that can be resident at once; the class slots were sized to it
  const unsigned grid = static_cast<unsigned>(blocks * max(1, sm_count));
  if (priced && corridor) {
    lattice_frontier_kernel<true, true><<<grid, kFrontierThreads, 0, stream>>>(classes);
  } else if (priced) {
    lattice_frontier_kernel<true, false><<<grid, kFrontierThreads, 0, stream>>>(classes);
  } else if (corridor) {
    lattice_frontier_kernel<false, true><<<grid, kFrontierThreads, 0, stream>>>(classes);
  } else {
    lattice_frontier_kernel<false, false><<<grid, kFrontierThreads, 0, stream>>>(classes);
  }
  return cudaGetLastError();
}

}  // namespace apgar_b200
