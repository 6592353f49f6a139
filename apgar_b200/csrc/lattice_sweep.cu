// Lattice-mode batched search: exact single-source labels over each net's
// window by alternating up/down row sweeps, then the canonical reverse path.
//
// One CTA owns one net; warp l owns layer l of the current window row and each
// lane owns C consecutive cells of it (C = 4..64 chooses the width class).
// A row step relaxes the row from the previous row in sweep order (straight
// plus both diagonals), then iterates {east scan, west scan, via cascade}
// to the row-local fixed point.  Scans are lane-serial over the C cells plus
// a 5-step warp shuffle scan of (value, connected) lane summaries.  Labels
// live in one slab per net in HBM (uint32, row pitch rounded to 4 cells so
// every lane moves 16-byte vectors); rows that have never held a finite label
// are never read or written ("materialised" rows, tracked in shared memory).
//
// A row is skipped when neither it nor its predecessor row changed since the
// previous sweep in the same direction; a sweep that changes nothing (after
// at least one sweep in each direction) proves the labels are the exact
// shortest-path fixed point.  This is the schedule restated on the CPU by the
// oracle (lo_sweep_schedule); the per-net counters returned here must match it.
//
// The canonical path follows the reference rule (gpu/cuda/planar_router.cu
// :977-1009 goal state, :1084-1165 reverse walk) on exact labels: from the
// goal, step to the predecessor through the smallest legal incoming heading
// whose label + move cost equals the current label.  Headings 0..7 are the
// planar directions (geometry_compiler::Direction order), 8 = via from the
// layer below, 9 = via from the layer above.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "lattice_common.cuh"

namespace apgar_b200 {
namespace {

constexpr int16_t kNever = -32000;
constexpr int kMaxRowPasses = 4096;

template <int C>
using BitsT = typename std::conditional<(C + 2 <= 64), unsigned long long, unsigned __int128>::type;

template <typename B>
__device__ __forceinline__ B low_mask(int n) {
  constexpr int kBits = sizeof(B) * 8;
  if (n <= 0) return B(0);
  if (n >= kBits) return ~B(0);
  return (B(1) << n) - B(1);
}

// Free bits for window-local cells x = xs - 1 + j, j in [0, C+2).
template <int C>
__device__ __forceinline__ BitsT<C> row_free_bits(const LatticeDeviceView& lat, int layer, int gy,
                                                  int x0, int xs, int w) {
  using B = BitsT<C>;
  constexpr int kWords = (C + 2 + 31) / 32;
  const uint32_t* row = lat.blocked + (static_cast<size_t>(layer) * lat.height + gy) * lat.words;
  const int pos = x0 + xs - 1;
  B blocked = 0;
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    blocked |= B(fetch_bits32(row, lat.words, pos + 32 * k)) << (32 * k);
  }
  const int lo = 1 - xs;      // j >= lo  <=> x >= 0
  const int hi = w - xs + 1;  // j <  hi  <=> x <  w
  const B valid = (hi > lo) ? (low_mask<B>(hi) & ~low_mask<B>(lo)) : B(0);
  return ~blocked & valid & low_mask<B>(C + 2);
}

// Via bits (pair lower/lower+1) for the same span; all ones without a mask.
template <int C>
__device__ __forceinline__ BitsT<C> row_via_bits(const LatticeDeviceView& lat, int lower, int gy,
                                                 int x0, int xs) {
  using B = BitsT<C>;
  if (lat.via_ok == nullptr) return ~B(0);
  constexpr int kWords = (C + 2 + 31) / 32;
  const uint32_t* row = lat.via_ok + (static_cast<size_t>(lower) * lat.height + gy) * lat.words;
  const int pos = x0 + xs - 1;
  B bits = 0;
#pragma unroll
  for (int k = 0; k < kWords; ++k) {
    // out-of-range words read as 1; they only matter where a cell is free,
    // which the free bits already exclude.
    bits |= B(fetch_bits32(row, lat.words, pos + 32 * k)) << (32 * k);
  }
  return bits;
}

template <typename B>
__device__ __forceinline__ bool bit(B v, int j) {
  return static_cast<bool>((v >> j) & B(1));
}

template <int C>
__device__ __forceinline__ void load_row(const uint32_t* src, int pitch, int xs, uint32_t (&v)[C]) {
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
}

template <int C>
__device__ __forceinline__ void store_row(uint32_t* dst, int pitch, int xs, const uint32_t (&v)[C]) {
#pragma unroll
  for (int q = 0; q < C / 4; ++q) {
    const int x = xs + 4 * q;
    if (x < pitch) {
      *reinterpret_cast<uint4*>(dst + x) =
          make_uint4(v[4 * q + 0], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
  }
}

// East scan: v[x] = min(v[x], v[x-1] + orth) along legal east edges.
// e_in bit j  <=> edge (xs+j-1) -> (xs+j) is legal.
template <int C, typename B>
__device__ __forceinline__ void east_scan(uint32_t (&v)[C], B e_in, uint32_t orth, int lane) {
#pragma unroll
  for (int j = 1; j < C; ++j) {
    if (bit(e_in, j)) v[j] = min(v[j], v[j - 1] + orth);
  }
  uint32_t a = v[C - 1];
  uint32_t b = ((e_in & low_mask<B>(C)) == low_mask<B>(C)) ? orth * C : kLabelInf;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const uint32_t ap = __shfl_up_sync(0xFFFFFFFFu, a, k);
    const uint32_t bp = __shfl_up_sync(0xFFFFFFFFu, b, k);
    if (lane >= k) {
      a = min(a, ap + b);
      b = sat(bp + b);
    }
  }
  uint32_t carry = __shfl_up_sync(0xFFFFFFFFu, a, 1);
  if (lane == 0) carry = kLabelInf;
#pragma unroll
  for (int j = 0; j < C; ++j) {
    if (bit(e_in, j)) v[j] = min(v[j], carry + orth);
    carry = v[j];
  }
}

// West scan: v[x] = min(v[x], v[x+1] + orth) along legal west edges.
// w_in bit j <=> edge (xs+j+1) -> (xs+j) is legal.
template <int C, typename B>
__device__ __forceinline__ void west_scan(uint32_t (&v)[C], B w_in, uint32_t orth, int lane) {
#pragma unroll
  for (int j = C - 2; j >= 0; --j) {
    if (bit(w_in, j)) v[j] = min(v[j], v[j + 1] + orth);
  }
  uint32_t a = v[0];
  uint32_t b = ((w_in & low_mask<B>(C)) == low_mask<B>(C)) ? orth * C : kLabelInf;
#pragma unroll
  for (int k = 1; k < 32; k <<= 1) {
    const uint32_t an = __shfl_down_sync(0xFFFFFFFFu, a, k);
    const uint32_t bn = __shfl_down_sync(0xFFFFFFFFu, b, k);
    if (lane + k < 32) {
      a = min(a, an + b);
      b = sat(bn + b);
    }
  }
  uint32_t carry = __shfl_down_sync(0xFFFFFFFFu, a, 1);
  if (lane == 31) carry = kLabelInf;
#pragma unroll
  for (int j = C - 1; j >= 0; --j) {
    if (bit(w_in, j)) v[j] = min(v[j], carry + orth);
    carry = v[j];
  }
}

template <int C>
__device__ __forceinline__ unsigned long long row_sum(const uint32_t (&v)[C]) {
  unsigned long long s = 0;
#pragma unroll
  for (int j = 0; j < C; ++j) s += v[j];
  return s;
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

template <int C>
__global__ void __launch_bounds__(kMaxLayers * 32)
    lattice_sweep_kernel(SweepLaunch p) {
  using B = BitsT<C>;
  const uint32_t plan_index = blockIdx.x;
  if (plan_index >= p.plan_count) return;
  const NetPlan plan = p.plans[plan_index];
  const apgar_b200_lattice_net net = p.nets[plan.net];
  const LatticeDeviceView& lat = p.lat;
  const int L = lat.layers;
  const int layer = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int w = static_cast<int>(net.win_w), h = static_cast<int>(net.win_h);
  const int pitch = static_cast<int>(plan.pitch);
  const int x0 = static_cast<int>(net.win_x0), y0 = static_cast<int>(net.win_y0);
  const int xs = lane * C;
  uint32_t* slab = p.dist_pool + plan.dist_offset;
  const size_t layer_stride = static_cast<size_t>(h) * pitch;
  uint32_t* my_layer = slab + static_cast<size_t>(layer) * layer_stride;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  // [modified rows: int16 h][free bits: B L*32][via bits: B L*32][row values: u32 L*32*C]
  int16_t* modified = reinterpret_cast<int16_t*>(smem_raw);
  size_t off = (static_cast<size_t>(h) * sizeof(int16_t) + 15) & ~size_t(15);
  B* sh_free = reinterpret_cast<B*>(smem_raw + off);
  off += sizeof(B) * L * 32;
  B* sh_via = reinterpret_cast<B*>(smem_raw + off);
  off += sizeof(B) * L * 32;
  uint32_t* sh_row = reinterpret_cast<uint32_t*>(smem_raw + off);
  __shared__ unsigned long long stat_rows, stat_stores, stat_loads;
  __shared__ int sh_cancel;
  __shared__ int sh_fault;

  const uint32_t orth = lat.orth, diag = lat.diag, via = lat.via;
  const int sl = static_cast<int>(net.start_layer), sx = static_cast<int>(net.start_x) - x0,
            sy = static_cast<int>(net.start_y) - y0;
  const int gl = static_cast<int>(net.goal_layer), gx = static_cast<int>(net.goal_x) - x0,
            gyy = static_cast<int>(net.goal_y) - y0;

  for (int y = threadIdx.x; y < h; y += blockDim.x) modified[y] = kNever;
  if (threadIdx.x == 0) {
    stat_rows = 0;
    stat_stores = 0;
    stat_loads = 0;
    sh_cancel = 0;
    sh_fault = 0;
  }
  const bool endpoints_free = cell_free(lat, net, sl, sx, sy) && cell_free(lat, net, gl, gx, gyy);
  __syncthreads();

  uint32_t completion = APGAR_B200_COMPLETION_DISCONNECTED;
  uint32_t sweeps_done = 0;
  if (endpoints_free) {
    // initial row: INF except the start cell
    {
      uint32_t v[C];
#pragma unroll
      for (int j = 0; j < C; ++j) v[j] = (layer == sl && xs + j == sx) ? 0u : kLabelInf;
      store_row<C>(my_layer + static_cast<size_t>(sy) * pitch, pitch, xs, v);
      if (threadIdx.x == 0) {
        modified[sy] = 0;
        stat_stores += L;
      }
    }
    __syncthreads();

    bool converged = false;
    bool cancelled = false;
    uint32_t prv[C];
    B pf = 0;
    for (uint32_t k = 1; k <= p.max_sweeps; ++k) {
      // One thread samples the host-mapped flag; the block follows its copy so
      // every thread takes the same branch.
      if (threadIdx.x == 0) sh_cancel = (p.cancel != nullptr && *p.cancel != 0u) ? 1 : 0;
      __syncthreads();
      if (sh_cancel != 0) {
        cancelled = true;
        break;
      }
      sweeps_done = k;
      const bool up = (k & 1u) != 0;
      const int dy = up ? 1 : -1;
      bool any_change = false;
      bool have_prev = false;
      for (int step = 0; step < h; ++step) {
        const int y = up ? step : h - 1 - step;
        const int py = y - dy;
        const int16_t mp = (py >= 0 && py < h) ? modified[py] : kNever;
        const int16_t my = modified[y];
        bool skip;
        if (k <= 2) {
          skip = (mp == kNever && my == kNever);
        } else {
          skip = (mp <= static_cast<int>(k) - 2 && my <= static_cast<int>(k) - 2);
        }
        if (skip) {
          have_prev = false;
          continue;
        }
        // previous row (values + free bits)
        if (!have_prev) {
          if (mp != kNever) {
            load_row<C>(my_layer + static_cast<size_t>(py) * pitch, pitch, xs, prv);
            pf = row_free_bits<C>(lat, layer, y0 + py, x0, xs, w);
            if (lane == 0) atomicAdd(&stat_loads, 1ull);
          } else {
#pragma unroll
            for (int j = 0; j < C; ++j) prv[j] = kLabelInf;
            pf = 0;
          }
        }
        uint32_t v[C];
        if (my != kNever) {
          load_row<C>(my_layer + static_cast<size_t>(y) * pitch, pitch, xs, v);
          if (lane == 0) atomicAdd(&stat_loads, 1ull);
        } else {
#pragma unroll
          for (int j = 0; j < C; ++j) v[j] = kLabelInf;
        }
        const B cf = row_free_bits<C>(lat, layer, y0 + y, x0, xs, w);
        const B vb = (layer + 1 < L) ? row_via_bits<C>(lat, layer, y0 + y, x0, xs) : B(0);
        const unsigned long long before = row_sum<C>(v);

        // relax from the previous row: straight, and the two diagonals
        {
          const B n_in = (pf >> 1) & (cf >> 1);
          const B dl_in = pf & (cf >> 1) & (pf >> 1) & cf;                 // from x-1
          const B dr_in = (pf >> 2) & (cf >> 1) & (pf >> 1) & (cf >> 2);   // from x+1
          uint32_t left = __shfl_up_sync(0xFFFFFFFFu, prv[C - 1], 1);
          uint32_t right = __shfl_down_sync(0xFFFFFFFFu, prv[0], 1);
          if (lane == 0) left = kLabelInf;
          if (lane == 31) right = kLabelInf;
#pragma unroll
          for (int j = 0; j < C; ++j) {
            const uint32_t pl = (j == 0) ? left : prv[j - 1];
            const uint32_t pr = (j == C - 1) ? right : prv[j + 1];
            if (bit(n_in, j)) v[j] = min(v[j], prv[j] + orth);
            if (bit(dl_in, j)) v[j] = min(v[j], pl + diag);
            if (bit(dr_in, j)) v[j] = min(v[j], pr + diag);
          }
        }
        const B e_in = cf & (cf >> 1);
        const B w_in = (cf >> 1) & (cf >> 2);
        if (L > 1) {
          sh_free[layer * 32 + lane] = cf;
          sh_via[layer * 32 + lane] = vb;
        }
        // Each pass lowers at least one label, so the loop is finite; the cap
        // only guards against a broken invariant (reported, never silent).
        for (int pass = 0;; ++pass) {
          if (pass == kMaxRowPasses) {
            if (threadIdx.x == 0) sh_fault = 1;
            break;
          }
          east_scan<C, B>(v, e_in, orth, lane);
          west_scan<C, B>(v, w_in, orth, lane);
          if (L == 1) break;
#pragma unroll
          for (int j = 0; j < C; ++j) sh_row[(layer * 32 + lane) * C + j] = v[j];
          __syncthreads();
          bool improved = false;
          // via chains downwards (k < layer) and upwards (k > layer)
          {
            B chain = sh_free[layer * 32 + lane];
            for (int kk = layer - 1; kk >= 0; --kk) {
              chain &= sh_free[kk * 32 + lane] & sh_via[kk * 32 + lane];
              if (chain == B(0)) break;
              const uint32_t add = via * static_cast<uint32_t>(layer - kk);
#pragma unroll
              for (int j = 0; j < C; ++j) {
                if (bit(chain, j + 1)) {
                  const uint32_t cand = sh_row[(kk * 32 + lane) * C + j] + add;
                  if (cand < v[j]) {
                    v[j] = cand;
                    improved = true;
                  }
                }
              }
            }
            chain = sh_free[layer * 32 + lane];
            for (int kk = layer + 1; kk < L; ++kk) {
              chain &= sh_free[kk * 32 + lane] & sh_via[(kk - 1) * 32 + lane];
              if (chain == B(0)) break;
              const uint32_t add = via * static_cast<uint32_t>(kk - layer);
#pragma unroll
              for (int j = 0; j < C; ++j) {
                if (bit(chain, j + 1)) {
                  const uint32_t cand = sh_row[(kk * 32 + lane) * C + j] + add;
                  if (cand < v[j]) {
                    v[j] = cand;
                    improved = true;
                  }
                }
              }
            }
          }
          if (!__syncthreads_or(improved)) break;
        }
        const bool lane_changed = row_sum<C>(v) != before;
        const bool row_changed = __syncthreads_or(lane_changed) != 0;
        const bool warp_changed = __any_sync(0xFFFFFFFFu, lane_changed);
        if (row_changed) {
          const bool materialise = (my == kNever);
          if (warp_changed || materialise) {
            store_row<C>(my_layer + static_cast<size_t>(y) * pitch, pitch, xs, v);
            if (lane == 0) atomicAdd(&stat_stores, 1ull);
          }
          modified[y] = static_cast<int16_t>(k);  // same value from every thread
          any_change = true;
        }
        if (threadIdx.x == 0) stat_rows += 1;
#pragma unroll
        for (int j = 0; j < C; ++j) prv[j] = v[j];
        pf = cf;
        have_prev = true;
      }
      if (!any_change && k >= 2) {
        converged = true;
        break;
      }
      // Make this sweep's stores visible to the next sweep's loads.
      __syncthreads();
    }
    __syncthreads();
    if (sh_fault != 0) {
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
  if (layer != 0) return;
  __threadfence_block();
  apgar_b200_lattice_result res{};
  res.cost = APGAR_B200_UNREACHABLE;
  res.completion = completion;
  res.sweeps = sweeps_done;
  res.path_len = 0;
  res.path_offset = 0;
  res.arena_offset = 0;
  res.row_steps = static_cast<uint32_t>(stat_rows);
  res.row_stores = static_cast<uint32_t>(stat_stores);
  res.row_loads = static_cast<uint32_t>(stat_loads);
  res.reserved = 0;
  auto label_at = [&](int l, int x, int y) -> uint32_t {
    if (modified[y] == kNever) return kLabelInf;
    return slab[static_cast<size_t>(l) * layer_stride + static_cast<size_t>(y) * pitch + x];
  };
  if (completion == APGAR_B200_COMPLETION_REACHED) {
    const uint32_t goal = label_at(gl, gx, gyy);
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
        int cl = gl, cx = gx, cy = gyy;
        uint32_t here = goal;
        uint32_t n = 0;
        bool ok = false;
        while (n < bound) {
          if (lane == 0) {
            p.path_arena[base + n] = static_cast<uint32_t>(
                (static_cast<size_t>(cl) * lat.height + (y0 + cy)) * lat.width + (x0 + cx));
          }
          ++n;
          if (cl == sl && cx == sx && cy == sy) {
            ok = true;
            break;
          }
          bool cand = false;
          int pl = cl, px = cx, py = cy;
          uint32_t pd = kLabelInf;
          if (lane < 8) {
            const int dxh = kDxc[lane], dyh = kDyc[lane];
            px = cx - dxh;
            py = cy - dyh;
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
            if (pl >= 0 && pl < L && cell_free(lat, net, pl, cx, cy) &&
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

__global__ void pack_copy_kernel(const apgar_b200_lattice_result* results, uint32_t count,
                                 const uint32_t* arena, uint32_t* paths) {
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const apgar_b200_lattice_result r = results[i];
    for (uint32_t j = threadIdx.x; j < r.path_len; j += blockDim.x) {
      paths[r.path_offset + j] = arena[r.arena_offset + j];
    }
  }
}

}  // namespace

size_t lattice_sweep_smem_bytes(int cells_per_lane, int layers, int max_rows) {
  const size_t bits_bytes = (cells_per_lane + 2 <= 64) ? 8 : 16;
  size_t off = (static_cast<size_t>(max_rows) * sizeof(int16_t) + 15) & ~size_t(15);
  off += bits_bytes * layers * 32 * 2;
  off += static_cast<size_t>(layers) * 32 * cells_per_lane * sizeof(uint32_t);
  return off;
}

cudaError_t launch_lattice_sweep(int cells_per_lane, const SweepLaunch& launch, int layers,
                                 int max_rows, cudaStream_t stream) {
  if (launch.plan_count == 0) return cudaSuccess;
  const size_t smem = lattice_sweep_smem_bytes(cells_per_lane, layers, max_rows);
  const dim3 grid(launch.plan_count), block(layers * 32);
  switch (cells_per_lane) {
#define APGAR_B200_CASE(CC)                                                                   \
  case CC: {                                                                                  \
    cudaError_t e = cudaFuncSetAttribute(lattice_sweep_kernel<CC>,                            \
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                         static_cast<int>(smem));                             \
    if (e != cudaSuccess) return e;                                                           \
    lattice_sweep_kernel<CC><<<grid, block, smem, stream>>>(launch);                          \
    return cudaGetLastError();                                                                \
  }
    APGAR_B200_CASE(4)
    APGAR_B200_CASE(8)
    APGAR_B200_CASE(16)
    APGAR_B200_CASE(32)
    APGAR_B200_CASE(64)
#undef APGAR_B200_CASE
    default:
      return cudaErrorInvalidValue;
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
