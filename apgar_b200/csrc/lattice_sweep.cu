// Lattice-mode batched search: exact single-source labels over each net's
// window by alternating forward/backward row sweeps, then the canonical
// reverse path.
//
// Frame: a net is swept along its window's shorter side.  Frame rows are
// lattice rows, or lattice columns when the window is taller than wide (the
// column-major bit planes uploaded with the lattice serve that case); the
// move model is symmetric under the swap.
//
// Work split: a net is owned by a group of G warps; each lane owns C
// consecutive cells of the frame row on every layer (L*C labels in
// registers), so a group covers rows of up to 32*C*G cells.  Small nets use
// one warp (no block barrier at all) and several nets share a CTA; wide nets
// use G warps that meet at named barriers once per row-local pass.
//
// A row step:
//   1. relaxes the row from the previous row in sweep order (straight plus
//      both diagonals; the previous row stays in registers between steps);
//   2. runs, for every layer, a two-sided row scan: the east and west
//      one-sided scans of the same input combined by min (equal to an east
//      scan followed by a west scan on every connected segment).  Each is a
//      lane-serial add-min chain, a 5-step warp shuffle scan of
//      (value, crossing cost) lane summaries and a fold over the group's
//      preceding warps;
//   3. applies the via cascade across layers inside each lane (registers
//      only) and repeats 2-3 until no via lowers a label;
//   4. writes back only the layers whose labels changed.
// Blocked cells hold INF and every update is clamped back to INF there, so
// orthogonal moves need no legality test; diagonal moves test their two side
// cells.  The next row's labels and mask bits are prefetched while the
// current row is processed whenever the schedule guarantees it will run.
//
// Schedule (restated on the CPU by the oracle, lo_sweep_schedule): a row is
// skipped when neither it nor its predecessor row changed since the previous
// sweep in the same direction (first sweep per direction: when both are still
// all-INF); a sweep that changes nothing, after one sweep in each direction,
// proves the labels are the exact shortest-path fixed point.  Rows that never
// held a finite label are never read or written.
//
// Canonical path (reference gpu/cuda/planar_router.cu :977-1009 goal state,
// :1084-1165 reverse walk) on exact labels: from the goal, step to the
// predecessor through the smallest legal incoming heading whose label plus
// move cost equals the current label.  Headings 0..7 are the planar
// directions (geometry_compiler::Direction order), 8 = via from the layer
// below, 9 = via from the layer above.
#include <cuda_runtime.h>

#include <cstdint>

#include "lattice_common.cuh"

namespace apgar_b200 {
namespace {

constexpr int16_t kNever = -32000;
constexpr int kMaxRowPasses = 4096;

// Geometry of one net in its frame.
struct Frame {
  int transposed;
  int R, K, pitch;
  int x0, y0;
};

// Per-lane view of the guard-padded sweep planes for one net: the two words
// holding the lane's span (frame positions xs-1 .. xs+C) of frame row r on
// layer l sit at base + l*layer_stride + r*row_stride.
struct BitSpan {
  const uint32_t* blocked;
  const uint32_t* via;  // nullptr without a via mask
  size_t layer_stride;
  int row_stride;
  int shift;
  uint32_t valid;  // span positions inside the frame (bit j <-> position xs-1+j)
};

template <int C>
__device__ __forceinline__ BitSpan make_span(const LatticeDeviceView& lat, const Frame& f, int xs) {
  static_assert(C + 2 <= 32, "a lane's span must fit one word");
  BitSpan s;
  const int origin = f.transposed ? f.y0 : f.x0;
  const int limit = (f.transposed ? lat.height : lat.width) - 1;
  const int first_row = f.transposed ? f.x0 : f.y0;
  const int rows_in_plane = f.transposed ? lat.width : lat.height;
  s.row_stride = (f.transposed ? lat.words_t : lat.words) + 2;
  s.layer_stride = static_cast<size_t>(rows_in_plane) * s.row_stride;
  // a lane wholly outside the frame clamps its position; its valid mask is 0
  const int pos = min(origin + xs - 1, limit);
  const int wi = pos >> 5;  // -1 for pos == -1: the leading guard word
  s.shift = pos & 31;
  const size_t base = static_cast<size_t>(first_row) * s.row_stride + 1 + wi;
  s.blocked = (f.transposed ? lat.sweep_cols : lat.sweep_rows) + base;
  const uint32_t* via_plane = f.transposed ? lat.sweep_via_cols : lat.sweep_via_rows;
  s.via = via_plane == nullptr ? nullptr : via_plane + base;
  const int lo = 1 - xs;        // j >= lo  <=> p >= 0
  const int hi = f.K - xs + 1;  // j <  hi  <=> p <  K
  uint32_t valid = 0;
  if (hi > lo) {
    const uint32_t hi_mask = hi >= 32 ? 0xFFFFFFFFu : ((1u << (hi > 0 ? hi : 0)) - 1u);
    const uint32_t lo_mask = lo <= 0 ? 0u : ((1u << lo) - 1u);
    valid = hi_mask & ~lo_mask;
  }
  s.valid = valid & ((1u << (C + 2)) - 1u);
  return s;
}

// Free bits of the lane's span (bit j+1 is the lane's cell j).
__device__ __forceinline__ uint32_t span_free(const BitSpan& s, int l, int r) {
  const uint32_t* w = s.blocked + l * s.layer_stride + static_cast<size_t>(r) * s.row_stride;
  return ~__funnelshift_r(__ldg(w), __ldg(w + 1), s.shift) & s.valid;
}

// Via bits of layer pair (l, l+1) for the span; all ones without a via mask.
__device__ __forceinline__ uint32_t span_via(const BitSpan& s, int l, int r) {
  if (s.via == nullptr) return 0xFFFFFFFFu;
  const uint32_t* w = s.via + l * s.layer_stride + static_cast<size_t>(r) * s.row_stride;
  return __funnelshift_r(__ldg(w), __ldg(w + 1), s.shift);
}

template <int C>
__device__ __forceinline__ void load_cells(const uint32_t* src, int pitch, int xs,
                                           uint32_t (&v)[C]) {
  static_assert(C % 2 == 0, "C must be even");
  if constexpr (C % 4 == 0) {
#pragma unroll
    for (int q = 0; q < C / 4; ++q) {
      const int x = xs + 4 * q;
      if (x < pitch) {
        const uint4 t = *reinterpret_cast<const uint4*>(src + x);
        v[4 * q + 0] = t.x;
        v[4 * q + 1] = t.y;
        v[4 * q + 2] = t.z;
        v[4 * q + 3] = t.w;
      } else {
        v[4 * q + 0] = v[4 * q + 1] = v[4 * q + 2] = v[4 * q + 3] = kLabelInf;
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < C / 2; ++q) {
      const int x = xs + 2 * q;
      if (x < pitch) {
        const uint2 t = *reinterpret_cast<const uint2*>(src + x);
        v[2 * q + 0] = t.x;
        v[2 * q + 1] = t.y;
      } else {
        v[2 * q + 0] = v[2 * q + 1] = kLabelInf;
      }
    }
  }
}

template <int C>
__device__ __forceinline__ void store_cells(uint32_t* dst, int pitch, int xs,
                                            const uint32_t (&v)[C]) {
  if constexpr (C % 4 == 0) {
#pragma unroll
    for (int q = 0; q < C / 4; ++q) {
      const int x = xs + 4 * q;
      if (x < pitch) {
        *reinterpret_cast<uint4*>(dst + x) =
            make_uint4(v[4 * q + 0], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < C / 2; ++q) {
      const int x = xs + 2 * q;
      if (x < pitch) *reinterpret_cast<uint2*>(dst + x) = make_uint2(v[2 * q + 0], v[2 * q + 1]);
    }
  }
}

__device__ __forceinline__ bool cell_free(const LatticeDeviceView& lat,
                                          const apgar_b200_lattice_net& n, int l, int x, int y) {
  if (l < 0 || l >= lat.layers || x < 0 || y < 0 || x >= static_cast<int>(n.win_w) ||
      y >= static_cast<int>(n.win_h)) {
    return false;
  }
  const int gx = static_cast<int>(n.win_x0) + x, gy = static_cast<int>(n.win_y0) + y;
  const uint32_t word =
      __ldg(lat.blocked + (static_cast<size_t>(l) * lat.height + gy) * lat.words + (gx >> 5));
  return ((word >> (gx & 31)) & 1u) == 0;
}

__device__ __forceinline__ bool via_bit_at(const LatticeDeviceView& lat,
                                           const apgar_b200_lattice_net& n, int lower, int x,
                                           int y) {
  if (lat.via_ok == nullptr) return true;
  const int gx = static_cast<int>(n.win_x0) + x, gy = static_cast<int>(n.win_y0) + y;
  const uint32_t word =
      __ldg(lat.via_ok + (static_cast<size_t>(lower) * lat.height + gy) * lat.words + (gx >> 5));
  return ((word >> (gx & 31)) & 1u) != 0;
}

__constant__ int kDxc[8] = {1, 1, 0, -1, -1, -1, 0, 1};
__constant__ int kDyc[8] = {0, 1, 1, 1, 0, -1, -1, -1};

// Nets (warp groups) per CTA: small groups share a CTA to keep blocks at 128+
// threads.
__host__ __device__ constexpr int groups_per_block(int G) { return G >= 4 ? 1 : 4 / G; }

// Per-group shared memory carve-up (shared by the kernel and the host).
struct GroupSmem {
  size_t modified, edges, sums, flags, total;
};

__host__ __device__ inline GroupSmem group_smem(int L, int G, int max_rows) {
  GroupSmem s{};
  size_t off = 0;
  s.modified = off;
  off += (static_cast<size_t>(max_rows) * sizeof(int16_t) + 15) & ~size_t(15);
  s.edges = off;  // [2 buffers][G][L][first, last] of the previous row
  off += 2 * static_cast<size_t>(G) * L * 2 * sizeof(uint32_t);
  s.sums = off;  // [G][L][aE, bE, aW, bW]
  off += static_cast<size_t>(G) * L * 4 * sizeof(uint32_t);
  s.flags = off;  // [2 parities][G]: bit 0 via improved, bit 1 changed, bit 8+l layer l changed
  off += 2 * static_cast<size_t>(G) * sizeof(uint32_t);
  s.total = (off + 15) & ~size_t(15);
  return s;
}

template <int G>
__device__ __forceinline__ void group_sync(int barrier_id) {
  if constexpr (G == 1) {
    __syncwarp();
  } else {
    __threadfence_block();
    asm volatile("bar.sync %0, %1;" ::"r"(barrier_id), "r"(G * 32) : "memory");
  }
}

template <int L, int C, int G>
__global__ void __launch_bounds__(groups_per_block(G) * G * 32)
    lattice_sweep_kernel(SweepLaunch p, int max_rows) {
  constexpr int kGroups = groups_per_block(G);
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int gi = warp / G;      // group (net) within the CTA
  const int g = warp - gi * G;  // warp within the group
  const uint32_t plan_index = blockIdx.x * kGroups + gi;
  if (plan_index >= p.plan_count) return;  // whole group leaves together
  const int barrier_id = gi + 1;
  const NetPlan plan = p.plans[plan_index];
  const apgar_b200_lattice_net net = p.nets[plan.net];
  const LatticeDeviceView& lat = p.lat;
  const int xs = (g * 32 + lane) * C;  // frame position of this lane's first cell
  Frame f;
  f.transposed = static_cast<int>(plan.transposed);
  f.R = static_cast<int>(plan.rows);
  f.K = static_cast<int>(plan.width);
  f.pitch = static_cast<int>(plan.pitch);
  f.x0 = static_cast<int>(net.win_x0);
  f.y0 = static_cast<int>(net.win_y0);
  uint32_t* slab = p.dist_pool + plan.dist_offset;
  const size_t layer_stride = static_cast<size_t>(f.R) * f.pitch;
  const BitSpan span = make_span<C>(lat, f, xs);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const GroupSmem gs = group_smem(L, G, max_rows);
  unsigned char* my_smem = smem_raw + gs.total * gi;
  int16_t* modified = reinterpret_cast<int16_t*>(my_smem + gs.modified);
  uint32_t* const sh_edges = reinterpret_cast<uint32_t*>(my_smem + gs.edges);
  constexpr int kEdgeBuf = G * L * 2;  // entries of one edge buffer
  uint32_t* sh_sum = reinterpret_cast<uint32_t*>(my_smem + gs.sums);
  uint32_t* sh_flags = reinterpret_cast<uint32_t*>(my_smem + gs.flags);

  const uint32_t orth = p.lat.orth, diag = p.lat.diag, via = p.lat.via;
  const int lsx = static_cast<int>(net.start_x) - f.x0, lsy = static_cast<int>(net.start_y) - f.y0;
  const int lgx = static_cast<int>(net.goal_x) - f.x0, lgy = static_cast<int>(net.goal_y) - f.y0;
  const int s_layer = static_cast<int>(net.start_layer), g_layer = static_cast<int>(net.goal_layer);
  const int sr = f.transposed ? lsx : lsy, sp = f.transposed ? lsy : lsx;

  for (int y = g * 32 + lane; y < f.R; y += G * 32) modified[y] = kNever;
  const bool endpoints_free =
      cell_free(lat, net, s_layer, lsx, lsy) && cell_free(lat, net, g_layer, lgx, lgy);
  // counters live in registers (every warp of a group follows the same
  // control flow; warp 0's copy is reported)
  uint32_t stat_rows = 0, stat_stores = 0, stat_loads = 0;
  bool fault = false;
  group_sync<G>(barrier_id);

  uint32_t completion = APGAR_B200_COMPLETION_DISCONNECTED;
  uint32_t sweeps_done = 0;
  if (endpoints_free) {
    {  // initial row: INF except the start cell
#pragma unroll
      for (int l = 0; l < L; ++l) {
        uint32_t v0[C];
#pragma unroll
        for (int j = 0; j < C; ++j) v0[j] = (l == s_layer && xs + j == sp) ? 0u : kLabelInf;
        store_cells<C>(slab + l * layer_stride + static_cast<size_t>(sr) * f.pitch, f.pitch, xs, v0);
      }
      modified[sr] = 0;  // same value from every thread
      stat_stores += L;
    }
    group_sync<G>(barrier_id);

    bool converged = false, cancelled = false;
    int parity = 0;
    // The row step reads its predecessor row's warp-edge labels from buffer
    // eb and publishes its own into the other buffer before its last group
    // vote, which therefore also ends the step (no barrier of its own).
    int eb = 0;
    uint32_t prv[L][C], nxt[L][C];
    uint32_t pf[L], nf[L], nvb[L];
    for (uint32_t k = 1; k <= p.max_sweeps; ++k) {
      // The host-mapped flag is read by one thread and broadcast, so every
      // thread of the group takes the same branch.
      uint32_t cancel_now = 0;
      if (g == 0 && lane == 0) cancel_now = (p.cancel != nullptr && *p.cancel != 0u) ? 1u : 0u;
      if constexpr (G == 1) {
        cancel_now = __shfl_sync(0xFFFFFFFFu, cancel_now, 0);
      } else {
        if (g == 0 && lane == 0) sh_flags[parity * G] = cancel_now;
        group_sync<G>(barrier_id);
        cancel_now = sh_flags[parity * G];
        group_sync<G>(barrier_id);
      }
      if (cancel_now != 0u) {
        cancelled = true;
        break;
      }
      sweeps_done = k;
      const bool fwd = (k & 1u) != 0;
      const int dr = fwd ? 1 : -1;
      const int ki = static_cast<int>(k);
      bool any_change = false;
      bool have_prev = false;
      bool have_next = false;  // nxt/nf/nvb hold this step's row
      bool next_loaded = false;
      for (int step = 0; step < f.R; ++step) {
        const int r = fwd ? step : f.R - 1 - step;
        const int pr = r - dr;
        const int16_t mp = (pr >= 0 && pr < f.R) ? modified[pr] : kNever;
        const int16_t my = modified[r];
        const bool skip = (ki <= 2) ? (mp == kNever && my == kNever)
                                    : (mp <= ki - 2 && my <= ki - 2);
        if (skip) {
          have_prev = false;
          have_next = false;
          continue;
        }
        // ---- previous row (registers, or reloaded after a skipped row) ----
        if (!have_prev) {
#pragma unroll
          for (int l = 0; l < L; ++l) {
            if (mp != kNever) {
              load_cells<C>(slab + l * layer_stride + static_cast<size_t>(pr) * f.pitch, f.pitch,
                            xs, prv[l]);
              pf[l] = span_free(span, l, pr);
            } else {
#pragma unroll
              for (int j = 0; j < C; ++j) prv[l][j] = kLabelInf;
              pf[l] = 0;
            }
          }
          if (mp != kNever) stat_loads += L;
          if constexpr (G > 1) {
            if (lane == 0 || lane == 31) {
#pragma unroll
              for (int l = 0; l < L; ++l) {
                sh_edges[eb * kEdgeBuf + (g * L + l) * 2 + (lane == 0 ? 0 : 1)] =
                    lane == 0 ? prv[l][0] : prv[l][C - 1];
              }
            }
            group_sync<G>(barrier_id);
          }
        }
        // ---- current row ----
        uint32_t v[L][C];
        uint32_t cf[L], vb[L];
        if (have_next) {
#pragma unroll
          for (int l = 0; l < L; ++l) {
#pragma unroll
            for (int j = 0; j < C; ++j) v[l][j] = next_loaded ? nxt[l][j] : kLabelInf;
            cf[l] = nf[l];
            vb[l] = nvb[l];
          }
          if (next_loaded) stat_loads += L;
        } else {
#pragma unroll
          for (int l = 0; l < L; ++l) {
            if (my != kNever) {
              load_cells<C>(slab + l * layer_stride + static_cast<size_t>(r) * f.pitch, f.pitch, xs,
                            v[l]);
            } else {
#pragma unroll
              for (int j = 0; j < C; ++j) v[l][j] = kLabelInf;
            }
            cf[l] = span_free(span, l, r);
            vb[l] = (l + 1 < L) ? span_via(span, l, r) : 0u;
          }
          if (my != kNever) stat_loads += L;
        }
        // ---- prefetch the next row when the schedule guarantees it runs ----
        {
          const int nr = r + dr;
          have_next = false;
          next_loaded = false;
          if (nr >= 0 && nr < f.R) {
            const int16_t mn = modified[nr];
            const bool sure = (ki <= 2) ? (my != kNever || mn != kNever)
                                        : (my >= ki - 1 || mn >= ki - 1);
            if (sure) {
              have_next = true;
              next_loaded = mn != kNever;
#pragma unroll
              for (int l = 0; l < L; ++l) {
                if (next_loaded) {
                  load_cells<C>(slab + l * layer_stride + static_cast<size_t>(nr) * f.pitch,
                                f.pitch, xs, nxt[l]);
                }
                nf[l] = span_free(span, l, nr);
                nvb[l] = (l + 1 < L) ? span_via(span, l, nr) : 0u;
              }
            }
          }
        }
        uint32_t orig[L][C];
        uint32_t blk[L][C];  // 0 where free, INF where blocked
#pragma unroll
        for (int l = 0; l < L; ++l) {
#pragma unroll
          for (int j = 0; j < C; ++j) {
            orig[l][j] = v[l][j];
            blk[l][j] = ((cf[l] >> (j + 1)) & 1u) ? 0u : kLabelInf;
          }
        }
        // ---- 1. relax from the previous row ----
#pragma unroll
        for (int l = 0; l < L; ++l) {
          // diagonal side cells: (p in the previous row, p-1 / p+1 in this row)
          const uint32_t side_l = (pf[l] >> 1) & cf[l];
          const uint32_t side_r = (pf[l] >> 1) & (cf[l] >> 2);
          uint32_t left = __shfl_up_sync(0xFFFFFFFFu, prv[l][C - 1], 1);
          uint32_t right = __shfl_down_sync(0xFFFFFFFFu, prv[l][0], 1);
          if constexpr (G > 1) {
            const uint32_t* const sh_edge = sh_edges + eb * kEdgeBuf;
            if (lane == 0) left = (g > 0) ? sh_edge[((g - 1) * L + l) * 2 + 1] : kLabelInf;
            if (lane == 31) right = (g + 1 < G) ? sh_edge[((g + 1) * L + l) * 2 + 0] : kLabelInf;
          } else {
            if (lane == 0) left = kLabelInf;
            if (lane == 31) right = kLabelInf;
          }
#pragma unroll
          for (int j = 0; j < C; ++j) {
            const uint32_t pl = (j == 0) ? left : prv[l][j - 1];
            const uint32_t prr = (j == C - 1) ? right : prv[l][j + 1];
            const uint32_t cl = ((side_l >> j) & 1u) ? diag : kLabelInf;
            const uint32_t cr = ((side_r >> j) & 1u) ? diag : kLabelInf;
            uint32_t t = __viaddmin_u32(prv[l][j], orth, v[l][j]);
            t = __viaddmin_u32(pl, cl, t);
            t = __viaddmin_u32(prr, cr, t);
            v[l][j] = max(t, blk[l][j]);
          }
        }
        // Lanes whose whole chunk is free pass a carry straight through; the
        // nearest non-free lane at or below (east scan) / at or above (west
        // scan) bounds the segment a lane's scan value can come from.
        const uint32_t stepC = orth * C;
        const uint32_t below_me = (lane == 31) ? 0xFFFFFFFFu : ((2u << lane) - 1u);
        const uint32_t above_me = ~((1u << lane) - 1u);
        int segE[L], segW[L];
        bool through_below[L], through_above[L];
        uint32_t warp_free[L];
#pragma unroll
        for (int l = 0; l < L; ++l) {
          const uint32_t m = (1u << C) - 1u;
          const uint32_t free_lanes = __ballot_sync(0xFFFFFFFFu, ((cf[l] >> 1) & m) == m);
          const uint32_t blocked_lanes = ~free_lanes;
          const uint32_t lo = blocked_lanes & below_me;
          const uint32_t hi = blocked_lanes & above_me;
          segE[l] = lo ? 31 - __clz(lo) : 0;
          segW[l] = hi ? __ffs(hi) - 1 : 31;
          through_below[l] = (blocked_lanes & ((1u << lane) - 1u)) == 0u;   // lanes < me all free
          through_above[l] = (blocked_lanes & ~below_me) == 0u;             // lanes > me all free
          warp_free[l] = free_lanes;
        }
        // via hop costs of the row (INF where the via bit forbids the hop)
        uint32_t hopc[L > 1 ? L - 1 : 1][C];
#pragma unroll
        for (int l = 0; l + 1 < L; ++l) {
#pragma unroll
          for (int j = 0; j < C; ++j) hopc[l][j] = ((vb[l] >> (j + 1)) & 1u) ? via : kLabelInf;
        }
        // via cascade inside the lane: upwards then downwards through
        // consecutive legal vias (blocked cells clamp the cascade); returns
        // whether any label changed
        auto via_cascade = [&]() -> uint32_t {
          uint32_t diff = 0;
          if constexpr (L > 1) {
#pragma unroll
            for (int j = 0; j < C; ++j) {
              uint32_t d = v[0][j];
#pragma unroll
              for (int l = 1; l < L; ++l) {
                const uint32_t t = max(__viaddmin_u32(d, hopc[l - 1][j], v[l][j]), blk[l][j]);
                diff |= t ^ v[l][j];
                v[l][j] = t;
                d = t;
              }
#pragma unroll
              for (int l = L - 2; l >= 0; --l) {
                const uint32_t t = max(__viaddmin_u32(d, hopc[l][j], v[l][j]), blk[l][j]);
                diff |= t ^ v[l][j];
                v[l][j] = t;
                d = t;
              }
            }
          }
          return diff;
        };
        // a path that switches layer as it arrives needs no second pass
        via_cascade();
        // ---- 2./3. row-local fixed point ----
        // Each pass lowers at least one label, so the loop is finite; the cap
        // only guards against a broken invariant (reported, never silent).
        uint32_t row_flags = 0;  // group-wide: bit 1 changed, bit 8+l layer l changed
        for (int pass = 0;; ++pass) {
          if (pass == kMaxRowPasses) {
            fault = true;
            break;
          }
          uint32_t inclE[L], inclW[L];
#pragma unroll
          for (int l = 0; l < L; ++l) {
            // lane-local one-sided scans: value at the far cell with no carry
            uint32_t ce = v[l][0];
#pragma unroll
            for (int j = 1; j < C; ++j) ce = max(__viaddmin_u32(ce, orth, v[l][j]), blk[l][j]);
            uint32_t cw = v[l][C - 1];
#pragma unroll
            for (int j = C - 2; j >= 0; --j) cw = max(__viaddmin_u32(cw, orth, v[l][j]), blk[l][j]);
            // segmented min scans over lanes of lane-offset values: a chunk's
            // far-cell value reaches lane i through free chunks at C*orth each
            inclE[l] = ce + static_cast<uint32_t>(31 - lane) * stepC;
            inclW[l] = cw + static_cast<uint32_t>(lane) * stepC;
          }
#pragma unroll
          for (int sft = 1; sft < 32; sft <<= 1) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
              const uint32_t oE = __shfl_up_sync(0xFFFFFFFFu, inclE[l], sft);
              const uint32_t oW = __shfl_down_sync(0xFFFFFFFFu, inclW[l], sft);
              if (lane - sft >= segE[l]) inclE[l] = min(inclE[l], oE);
              if (lane + sft <= segW[l]) inclW[l] = min(inclW[l], oW);
            }
          }
#pragma unroll
          for (int l = 0; l < L; ++l) {
            inclE[l] = min(inclE[l] - static_cast<uint32_t>(31 - lane) * stepC, kLabelInf);
            inclW[l] = min(inclW[l] - static_cast<uint32_t>(lane) * stepC, kLabelInf);
          }
          uint32_t warp_cE[L], warp_cW[L];
#pragma unroll
          for (int l = 0; l < L; ++l) warp_cE[l] = warp_cW[l] = kLabelInf;
          if constexpr (G > 1) {
            // warp summaries: far-cell value without outside carry, and the
            // cost to cross the whole warp (INF unless every chunk is free)
            if (lane == 31) {
#pragma unroll
              for (int l = 0; l < L; ++l) sh_sum[(g * L + l) * 4 + 0] = inclE[l];
            }
            if (lane == 0) {
#pragma unroll
              for (int l = 0; l < L; ++l) {
                sh_sum[(g * L + l) * 4 + 1] = warp_free[l] == 0xFFFFFFFFu ? 32u * stepC : kLabelInf;
                sh_sum[(g * L + l) * 4 + 2] = inclW[l];
              }
            }
            group_sync<G>(barrier_id);
#pragma unroll
            for (int l = 0; l < L; ++l) {
              for (int q = 0; q < g; ++q) {
                warp_cE[l] = __viaddmin_u32(warp_cE[l], sh_sum[(q * L + l) * 4 + 1],
                                            sh_sum[(q * L + l) * 4 + 0]);
              }
              for (int q = G - 1; q > g; --q) {
                warp_cW[l] = __viaddmin_u32(warp_cW[l], sh_sum[(q * L + l) * 4 + 1],
                                            sh_sum[(q * L + l) * 4 + 2]);
              }
            }
          }
#pragma unroll
          for (int l = 0; l < L; ++l) {
            // carry into the lane: the neighbour lane's far-cell value, or the
            // warp carry when every chunk between is free
            uint32_t carryE = __shfl_up_sync(0xFFFFFFFFu, inclE[l], 1);
            uint32_t carryW = __shfl_down_sync(0xFFFFFFFFu, inclW[l], 1);
            if (lane == 0) carryE = kLabelInf;
            if (lane == 31) carryW = kLabelInf;
            if (through_below[l]) carryE = __viaddmin_u32(warp_cE[l], static_cast<uint32_t>(lane) * stepC, carryE);
            if (through_above[l]) carryW = __viaddmin_u32(warp_cW[l], static_cast<uint32_t>(31 - lane) * stepC, carryW);
            uint32_t e[C];
#pragma unroll
            for (int j = 0; j < C; ++j) {
              carryE = max(__viaddmin_u32(carryE, orth, v[l][j]), blk[l][j]);
              e[j] = carryE;
            }
#pragma unroll
            for (int j = C - 1; j >= 0; --j) {
              carryW = max(__viaddmin_u32(carryW, orth, v[l][j]), blk[l][j]);
              v[l][j] = min(e[j], carryW);
            }
          }
          const uint32_t via_diff = via_cascade();
          // group vote: did a via lower a label (another pass needed), and
          // which layers changed since the row was loaded
          uint32_t lane_flags = via_diff != 0u ? 1u : 0u;
#pragma unroll
          for (int l = 0; l < L; ++l) {
            uint32_t diff = 0;
#pragma unroll
            for (int j = 0; j < C; ++j) diff |= v[l][j] ^ orig[l][j];
            if (diff != 0u) lane_flags |= 2u | (1u << (8 + l));
          }
          uint32_t warp_flags = __reduce_or_sync(0xFFFFFFFFu, lane_flags);
          if constexpr (G > 1) {
            // this pass's row edges for the next step (final if the vote ends
            // the row): buffer eb ^ 1 is read by no warp until the next step,
            // and every read of it by the previous step came before this
            // step's first barrier
            if (lane == 0 || lane == 31) {
#pragma unroll
              for (int l = 0; l < L; ++l) {
                sh_edges[(eb ^ 1) * kEdgeBuf + (g * L + l) * 2 + (lane == 0 ? 0 : 1)] =
                    lane == 0 ? v[l][0] : v[l][C - 1];
              }
            }
            if (lane == 0) sh_flags[parity * G + g] = warp_flags;
            group_sync<G>(barrier_id);
            warp_flags = 0;
            for (int q = 0; q < G; ++q) warp_flags |= sh_flags[parity * G + q];
            parity ^= 1;
          }
          row_flags = warp_flags;
          if ((warp_flags & 1u) == 0u || L == 1) break;
        }
        // ---- 4. write-back ----
        if (row_flags & 2u) {
          const bool materialise = (my == kNever);
#pragma unroll
          for (int l = 0; l < L; ++l) {
            if (materialise || (row_flags & (1u << (8 + l)))) {
              store_cells<C>(slab + l * layer_stride + static_cast<size_t>(r) * f.pitch, f.pitch,
                             xs, v[l]);
              ++stat_stores;
            }
          }
          modified[r] = static_cast<int16_t>(k);  // same value from every thread
          any_change = true;
        }
        ++stat_rows;
#pragma unroll
        for (int l = 0; l < L; ++l) {
#pragma unroll
          for (int j = 0; j < C; ++j) prv[l][j] = v[l][j];
          pf[l] = cf[l];
        }
        have_prev = true;
        eb ^= 1;
        // The step's last vote barrier published the edges; every thread
        // wrote modified[r] itself (the same value) and reads only its own
        // lane's cells of the slab.  A faulted row left the pass loop before
        // its vote, so it ends with a barrier of its own.
        if (fault) group_sync<G>(barrier_id);
      }
      if (!any_change && k >= 2) {
        converged = true;
        break;
      }
    }
    group_sync<G>(barrier_id);
    if (fault) {
      completion = APGAR_B200_COMPLETION_REJECTED;
    } else if (cancelled) {
      completion = APGAR_B200_COMPLETION_CANCELLED;
    } else if (!converged) {
      completion = APGAR_B200_COMPLETION_BUDGET_EXHAUSTED;
    } else {
      completion = APGAR_B200_COMPLETION_REACHED;  // refined below from the goal label
    }
  }

  // ----------------------------- result + walk -----------------------------
  if (g != 0) return;
  apgar_b200_lattice_result res{};
  res.cost = APGAR_B200_UNREACHABLE;
  res.completion = completion;
  res.sweeps = sweeps_done;
  res.row_steps = stat_rows;
  res.row_stores = stat_stores;
  res.row_loads = stat_loads;
  auto label_at = [&](int l, int x, int y) -> uint32_t {
    const int r = f.transposed ? x : y, q = f.transposed ? y : x;
    if (modified[r] == kNever) return kLabelInf;
    return slab[static_cast<size_t>(l) * layer_stride + static_cast<size_t>(r) * f.pitch + q];
  };
  if (completion == APGAR_B200_COMPLETION_REACHED) {
    const uint32_t goal = label_at(g_layer, lgx, lgy);
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
        const int Ln = lat.layers;
        int cl = g_layer, cx = lgx, cy = lgy;
        uint32_t here = goal;
        uint32_t n = 0;
        bool ok = false;
        while (n < bound) {
          if (lane == 0) {
            p.path_arena[base + n] = static_cast<uint32_t>(
                (static_cast<size_t>(cl) * lat.height + (f.y0 + cy)) * lat.width + (f.x0 + cx));
          }
          ++n;
          if (cl == s_layer && cx == lsx && cy == lsy) {
            ok = true;
            break;
          }
          bool cand = false;
          int pl = cl, px = cx, py = cy;
          uint32_t pd = kLabelInf;
          if (lane < 8) {
            px = cx - kDxc[lane];
            py = cy - kDyc[lane];
            bool legal = cell_free(lat, net, cl, px, py);
            if (legal && (lane & 1)) {
              legal = cell_free(lat, net, cl, cx, py) && cell_free(lat, net, cl, px, cy);
            }
            if (legal) {
              pd = label_at(cl, px, py);
              cand = pd < kLabelInf && pd + ((lane & 1) ? diag : orth) == here;
            }
          } else if (lane == 8 || lane == 9) {
            pl = (lane == 8) ? cl - 1 : cl + 1;
            const int lower = (lane == 8) ? cl - 1 : cl;
            if (pl >= 0 && pl < Ln && cell_free(lat, net, pl, cx, cy) &&
                via_bit_at(lat, net, lower, cx, cy)) {
              pd = label_at(pl, cx, cy);
              cand = pd < kLabelInf && pd + via == here;
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
          res.path_len = n;
          res.arena_offset = base;
        } else {
          res.completion = APGAR_B200_COMPLETION_REJECTED;
          res.cost = APGAR_B200_UNREACHABLE;
        }
      }
    }
  }
  if (lane == 0) p.results[plan.net] = res;
}

// Deterministic packing of the reverse paths in caller net order: one block
// computes exclusive offsets, then every block copies its nets' paths.
__global__ void pack_offsets_kernel(apgar_b200_lattice_result* results, uint32_t count,
                                    unsigned long long* total) {
  __shared__ unsigned long long warp_sums[32];
  __shared__ unsigned long long base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t chunk = 0; chunk < count; chunk += blockDim.x) {
    const uint32_t i = chunk + threadIdx.x;
    const unsigned long long len = i < count ? results[i].path_len : 0ull;
    unsigned long long x = len;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, k);
      if (lane >= k) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long s = lane < static_cast<int>(blockDim.x >> 5) ? warp_sums[lane] : 0ull;
#pragma unroll
      for (int k = 1; k < 32; k <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, s, k);
        if (lane >= k) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const unsigned long long warp_base = warp == 0 ? 0ull : warp_sums[warp - 1];
    if (i < count) results[i].path_offset = base + warp_base + x - len;
    __syncthreads();
    if (threadIdx.x == 0) base += warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = base;
}

__global__ void pack_copy_kernel(apgar_b200_lattice_result* results, uint32_t count,
                                 const uint32_t* arena, uint32_t* paths) {
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const apgar_b200_lattice_result r = results[i];
    for (uint32_t j = threadIdx.x; j < r.path_len; j += blockDim.x) {
      paths[r.path_offset + j] = arena[r.arena_offset + j];
    }
    // the staging offset depends on the order nets finished; clear it so the
    // returned records are deterministic
    __syncthreads();
    if (threadIdx.x == 0) results[i].arena_offset = 0;
  }
}

template <int L, int C, int G>
cudaError_t launch_one(const SweepLaunch& launch, int max_rows, cudaStream_t stream) {
  constexpr int kGroups = groups_per_block(G);
  const size_t smem = group_smem(L, G, max_rows).total * kGroups;
  cudaError_t e = cudaFuncSetAttribute(lattice_sweep_kernel<L, C, G>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  const unsigned grid = (launch.plan_count + kGroups - 1) / kGroups;
  lattice_sweep_kernel<L, C, G><<<grid, kGroups * G * 32, smem, stream>>>(launch, max_rows);
  return cudaGetLastError();
}

template <int L, int C>
cudaError_t launch_layers(int G, const SweepLaunch& launch, int max_rows, cudaStream_t stream) {
  // every group size 1..16: the host gives a net the fewest warps that
  // cover its frame row
  switch (G) {
    case 1: return launch_one<L, C, 1>(launch, max_rows, stream);
    case 2: return launch_one<L, C, 2>(launch, max_rows, stream);
    case 3: return launch_one<L, C, 3>(launch, max_rows, stream);
    case 4: return launch_one<L, C, 4>(launch, max_rows, stream);
    case 5: return launch_one<L, C, 5>(launch, max_rows, stream);
    case 6: return launch_one<L, C, 6>(launch, max_rows, stream);
    case 7: return launch_one<L, C, 7>(launch, max_rows, stream);
    case 8: return launch_one<L, C, 8>(launch, max_rows, stream);
    case 9: return launch_one<L, C, 9>(launch, max_rows, stream);
    case 10: return launch_one<L, C, 10>(launch, max_rows, stream);
    case 11: return launch_one<L, C, 11>(launch, max_rows, stream);
    case 12: return launch_one<L, C, 12>(launch, max_rows, stream);
    case 13: return launch_one<L, C, 13>(launch, max_rows, stream);
    case 14: return launch_one<L, C, 14>(launch, max_rows, stream);
    case 15: return launch_one<L, C, 15>(launch, max_rows, stream);
    case 16: return launch_one<L, C, 16>(launch, max_rows, stream);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

// Cells per lane per layer for a layer count (L*C labels per lane).
int lattice_cells_per_lane(int layers) {
  switch (layers) {
    case 1: return 16;
    case 2: return 8;
    case 3:
    case 4: return 4;
    default: return 2;
  }
}

size_t lattice_sweep_smem_bytes(int layers, int warps_per_net, int max_rows) {
  return group_smem(layers, warps_per_net, max_rows).total * groups_per_block(warps_per_net);
}

cudaError_t launch_lattice_sweep(int layers, int warps_per_net, const SweepLaunch& launch,
                                 int max_rows, cudaStream_t stream) {
  if (launch.plan_count == 0) return cudaSuccess;
  switch (layers) {
    case 1: return launch_layers<1, 16>(warps_per_net, launch, max_rows, stream);
    case 2: return launch_layers<2, 8>(warps_per_net, launch, max_rows, stream);
    case 3: return launch_layers<3, 4>(warps_per_net, launch, max_rows, stream);
    case 4: return launch_layers<4, 4>(warps_per_net, launch, max_rows, stream);
    case 6: return launch_layers<6, 2>(warps_per_net, launch, max_rows, stream);
    case 8: return launch_layers<8, 2>(warps_per_net, launch, max_rows, stream);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_lattice_pack(apgar_b200_lattice_result* results, uint32_t count,
                                unsigned long long* total, const uint32_t* arena, uint32_t* paths,
                                int sm_count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  pack_offsets_kernel<<<1, 1024, 0, stream>>>(results, count, total);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const uint32_t cap = static_cast<uint32_t>(sm_count > 0 ? sm_count * 8 : 1024);
  const unsigned grid = count < cap ? count : cap;
  pack_copy_kernel<<<grid, 128, 0, stream>>>(results, count, arena, paths);
  return cudaGetLastError();
}

}  // namespace apgar_b200
