// Drop-in engine: batched single-source search over the reference device
// view (DeviceCompiledBoardV1 node graph), heading states, uint64 checked
// costs, bends and per-query surcharges and edge policies.
//
// One CTA owns one query for the whole search (no host round trips):
//   * labels live in the query's slab of the query-major workspace
//     (9 states per node), read at L2 (ld.global.cg) because other threads of
//     the CTA lower them with 64-bit atomicMin while a round runs;
//   * the frontier is a queue of nodes whose labels dropped, processed in
//     buckets of width delta = the cheapest move: each round takes the
//     smallest node label m in the queue and expands every queued node whose
//     best label is below m + delta (8 lanes per node, one direction each);
//     nodes above the bucket are carried to the next round.  Enqueueing is
//     deduplicated by per-node round stamps and warp-aggregated (ballot +
//     popc + one shared atomic per warp);
//   * a node's departure in direction d is min over its 9 heading labels of
//     label + (bend + bend surcharge if the heading changes from a real
//     heading), and the move adds step + surcharge + the edge's policy
//     adjustment (UINT64_MAX = banned), all checked against the sentinel
//     (reference planar_router.cu:557-583 and :847-875);
//   * the search ends when the queue empties (exact fixed point) or, when
//     only the goal path is wanted, as soon as the smallest queued label
//     exceeds the best goal label (every label not above it is then final).
// Afterwards the CTA emits either the canonical reverse compact path or, for
// the full-workspace form, the canonical predecessor of every state, using
// the reference tie-break (planar_router.cu:977-1009 goal state, :486-524 and
// :1084-1165 predecessor rule: smallest predecessor state index).
#include <cuda_runtime.h>

#include <cstdint>

#include "graph_common.cuh"

namespace apgar_b200 {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ bool checked_add(uint64_t a, uint64_t b, uint64_t* out) {
  constexpr uint64_t kMaxFinite = kGraphInf - 1u;
  if (a > kMaxFinite || b > kMaxFinite - a) return false;
  *out = a + b;
  return true;
}

// A label read while other threads of the CTA may lower it: at L2 for the
// global slab, volatile for the shared-memory copy of a small graph.
template <bool kShared>
__device__ __forceinline__ uint64_t load_label(const uint64_t* p) {
  if constexpr (kShared) {
    return *reinterpret_cast<const volatile uint64_t*>(p);
  } else {
    return __ldcg(p);
  }
}

__device__ __forceinline__ uint32_t nbr(const GraphDeviceView& g, uint32_t node, uint32_t d) {
  return g.neighbors[static_cast<size_t>(d) * g.node_count + node];  // global or staged
}

__device__ __forceinline__ uint64_t policy_adjustment(const apgar_b200_policy_edge_v1* pol,
                                                      uint32_t count, uint32_t edge) {
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2u;
    if (pol[mid].physical_edge_index < edge) {
      lo = mid + 1u;
    } else {
      hi = mid;
    }
  }
  if (lo < count && pol[lo].physical_edge_index == edge) return pol[lo].adjustment;
  return 0;
}

// Cost of the move source --d--> for incoming heading h_in; false when the
// edge is banned, missing, or the sum would reach the sentinel.
__device__ __forceinline__ bool transition_cost(const GraphDeviceView& g,
                                                const apgar_b200_batch_query_v1& q,
                                                const apgar_b200_policy_edge_v1* pol,
                                                uint32_t source, uint32_t d, uint32_t h_in,
                                                uint64_t* cost) {
  uint32_t edge;
  if (d < 4u) {
    edge = source * 8u + d;
  } else {
    const uint32_t canon = nbr(g, source, d);
    if (canon == kInvalid32) return false;
    edge = canon * 8u + d - 4u;
  }
  const uint64_t adj = policy_adjustment(pol, q.policy_count, edge);
  if (adj == kGraphInf) return false;
  uint64_t value = (d & 1u) ? static_cast<uint64_t>(g.diag) + q.diagonal_step_surcharge
                            : static_cast<uint64_t>(g.orth) + q.orthogonal_step_surcharge;
  if (h_in != 8u && h_in != d) {
    if (!checked_add(value, static_cast<uint64_t>(g.bend) + q.bend_surcharge, &value)) return false;
  }
  return checked_add(value, adj, cost);
}

// Canonical predecessor of state `s` (reference rule): the smallest
// predecessor state index whose label plus the move cost equals label[s].
template <bool kShared>
__device__ uint32_t canonical_predecessor(const GraphDeviceView& g,
                                          const apgar_b200_batch_query_v1& q,
                                          const apgar_b200_policy_edge_v1* pol,
                                          const uint64_t* lab, uint32_t s) {
  const uint32_t node = s / 9u, h = s % 9u;
  const uint64_t here = load_label<kShared>(lab + s);
  if (h == 8u || here == kGraphInf) return kInvalid32;
  const uint32_t pred = nbr(g, node, (h + 4u) & 7u);
  if (pred == kInvalid32) return kInvalid32;
  for (uint32_t ph = 0; ph < 9u; ++ph) {
    if (ph == 8u && pred != q.start_node) continue;
    uint64_t t, c;
    if (!transition_cost(g, q, pol, pred, h, ph, &t)) continue;
    if (checked_add(load_label<kShared>(lab + pred * 9u + ph), t, &c) && c == here) return pred * 9u + ph;
  }
  return kInvalid32;
}

__device__ __forceinline__ void set_completion(apgar_b200_batch_result_v1& r, uint32_t c) {
  r.completion = static_cast<uint8_t>(c);
}

// kShared: the query's labels, queues and stamps, and the neighbour table,
// live in shared memory (a graph small enough for them to fit: the drop-in
// corpus has 10-697 nodes), so each round's label reads, atomics and
// neighbour lookups stay on the SM; the labels are copied to the query's
// global slab at the end where the host reads them.  Either form stages the
// query's policy edges in shared memory when they fit.
template <bool kShared>
__global__ void __launch_bounds__(kThreads) graph_search_kernel(GraphLaunch p) {
  const uint32_t qi = blockIdx.x;
  if (qi >= p.query_count) return;
  GraphDeviceView g = p.g;
  const apgar_b200_batch_query_v1 q = p.queries[qi];
  const uint32_t N = g.node_count;
  const uint64_t S = 9ull * N;
  uint64_t* lab = p.labels + static_cast<uint64_t>(qi) * S;
  uint32_t* queue0 = p.queues + static_cast<uint64_t>(qi) * 2u * N;
  uint32_t* queue1 = queue0 + N;
  uint32_t* stamp = p.stamps + static_cast<uint64_t>(qi) * N;
  extern __shared__ __align__(16) uint8_t graph_smem[];
  if constexpr (kShared) {
    lab = reinterpret_cast<uint64_t*>(graph_smem);
    queue0 = reinterpret_cast<uint32_t*>(graph_smem + S * 8u);
    queue1 = queue0 + N;
    stamp = queue1 + N;
  }
  const apgar_b200_policy_edge_v1* pol = p.policy + q.policy_offset;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (p.policy_smem_offset != kInvalid32) {
    // the query's policy edges, searched on every move, staged on the SM
    auto* staged = reinterpret_cast<apgar_b200_policy_edge_v1*>(graph_smem + p.policy_smem_offset);
    for (uint32_t i = tid; i < q.policy_count; i += kThreads) staged[i] = pol[i];
    pol = staged;
  }
  if (p.nbr_smem_offset != kInvalid32) {
    // the neighbour table [8][N], read on every move and path step
    auto* staged = reinterpret_cast<uint32_t*>(graph_smem + p.nbr_smem_offset);
    for (uint32_t i = tid; i < 8u * N; i += kThreads) staged[i] = __ldg(p.g.neighbors + i);
    g.neighbors = staged;
  }

  __shared__ uint32_t sh_count[2];
  __shared__ uint64_t sh_wmin[kThreads / 32];
  __shared__ uint64_t sh_min, sh_goal;
  __shared__ int sh_stop;
  __shared__ unsigned long long sh_examined, sh_turns;

  for (uint64_t s = tid; s < S; s += kThreads) lab[s] = kGraphInf;
  for (uint32_t n = tid; n < N; n += kThreads) stamp[n] = 0u;
  if (tid == 0) {
    sh_count[0] = 1u;
    sh_count[1] = 0u;
    sh_goal = kGraphInf;
    sh_examined = 0;
    sh_turns = 0;
  }
  __syncthreads();
  if (tid == 0) {
    lab[static_cast<uint64_t>(q.start_node) * 9u + 8u] = 0;
    queue0[0] = q.start_node;
    stamp[q.start_node] = 1u;
  }
  __threadfence_block();
  __syncthreads();

  // cheapest single move: the bucket width
  const uint64_t delta_orth = static_cast<uint64_t>(g.orth) + q.orthogonal_step_surcharge;
  const uint64_t delta_diag = static_cast<uint64_t>(g.diag) + q.diagonal_step_surcharge;
  const uint64_t delta = delta_orth < delta_diag ? delta_orth : delta_diag;
  const uint64_t bend_cost = static_cast<uint64_t>(g.bend) + q.bend_surcharge;

  uint32_t completion = APGAR_B200_COMPLETION_BUDGET_EXHAUSTED;
  uint32_t rounds = 0;
  unsigned long long examined = 0, turns = 0;
  for (;;) {
    const int cur = static_cast<int>(rounds & 1u);
    uint32_t* qcur = cur ? queue1 : queue0;
    uint32_t* qnxt = cur ? queue0 : queue1;
    const uint32_t count = sh_count[cur];
    if (count == 0u) {
      completion = APGAR_B200_COMPLETION_REACHED;  // converged; refined below
      break;
    }
    if (rounds >= p.maximum_rounds) break;
    // the cancel flag is host-mapped memory (every read crosses the bus):
    // read it on the first round and every 64 rounds after
    if (tid == 0 && (rounds % 64u) == 0u) {
      sh_stop = (p.cancel != nullptr && *p.cancel != 0u) ? 1 : 0;
    }
    // ---- phase A: smallest queued label ----
    uint64_t local_min = kGraphInf;
    for (uint32_t i = tid; i < count; i += kThreads) {
      const uint32_t n = qcur[i];
      for (uint32_t h = 0; h < 9u; ++h) {
        const uint64_t v = load_label<kShared>(lab + n * 9u + h);
        local_min = v < local_min ? v : local_min;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, local_min, o);
      local_min = other < local_min ? other : local_min;
    }
    if (lane == 0) sh_wmin[warp] = local_min;
    __syncthreads();
    if (tid == 0) {
      uint64_t m = kGraphInf;
      for (int w = 0; w < kThreads / 32; ++w) m = sh_wmin[w] < m ? sh_wmin[w] : m;
      sh_min = m;
      sh_count[cur ^ 1] = 0u;
    }
    __syncthreads();
    if (sh_stop != 0) {
      completion = APGAR_B200_COMPLETION_CANCELLED;
      break;
    }
    const uint64_t m = sh_min;
    if (!p.workspace_mode && sh_goal != kGraphInf && m > sh_goal) {
      // every label not above the best goal label is final
      completion = APGAR_B200_COMPLETION_REACHED;
      break;
    }
    const uint64_t threshold = (m > kGraphInf - delta) ? kGraphInf : m + delta;
    const uint32_t next_stamp = rounds + 2u;
    // ---- phase B: expand the bucket, carry the rest ----
    const uint32_t pairs = count * 8u;
    for (uint32_t base = 0; base < pairs; base += kThreads) {
      const uint32_t pr = base + tid;
      bool enqueue = false;
      uint32_t target = 0;
      if (pr < pairs) {
        const uint32_t n = qcur[pr >> 3];
        const uint32_t d = pr & 7u;
        uint64_t labs[9];
        uint64_t node_min = kGraphInf;
#pragma unroll
        for (uint32_t h = 0; h < 9u; ++h) {
          labs[h] = load_label<kShared>(lab + n * 9u + h);
          node_min = labs[h] < node_min ? labs[h] : node_min;
        }
        if (node_min >= threshold) {
          if (d == 0u) {  // carried to the next round
            enqueue = atomicExch(&stamp[n], next_stamp) != next_stamp;
            target = n;
          }
        } else if ((__ldg(g.legal + n) >> d) & 1u) {
          ++examined;
          // departure in direction d
          // heading 8 (no incoming heading) is finite only at the start node;
          // labs[d] is selected with an unrolled compare so labs stays in
          // registers
          uint64_t dep = kGraphInf;
#pragma unroll
          for (uint32_t h = 0; h < 8u; ++h) dep = (h == d) ? labs[h] : dep;
          bool turned = false;
#pragma unroll
          for (uint32_t h = 0; h < 9u; ++h) {
            if (h == d || labs[h] == kGraphInf) continue;
            uint64_t c = labs[h];
            if (h != 8u && !checked_add(c, bend_cost, &c)) continue;
            if (c < dep) {
              dep = c;
              turned = h != 8u;
            }
          }
          if (turned) ++turns;
          uint64_t t, cand;
          const uint32_t nb = nbr(g, n, d);
          // the departure already carries any bend, so the move is priced
          // with the outgoing direction as its incoming heading
          if (dep != kGraphInf && nb != kInvalid32 && transition_cost(g, q, pol, n, d, d, &t) &&
              checked_add(dep, t, &cand)) {
            const unsigned long long old = atomicMin(
                reinterpret_cast<unsigned long long*>(lab + nb * 9u + d),
                static_cast<unsigned long long>(cand));
            if (cand < old) {
              enqueue = atomicExch(&stamp[nb], next_stamp) != next_stamp;
              target = nb;
            }
          }
        }
      }
      // warp-aggregated enqueue
      const unsigned mask = __ballot_sync(0xFFFFFFFFu, enqueue);
      if (mask != 0u) {
        uint32_t wbase = 0;
        if (lane == __ffs(mask) - 1) wbase = atomicAdd(&sh_count[cur ^ 1], __popc(mask));
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, __ffs(mask) - 1);
        if (enqueue) qnxt[wbase + __popc(mask & ((1u << lane) - 1u))] = target;
      }
    }
    __threadfence_block();
    __syncthreads();
    // best goal label after this round
    if (warp == 0) {
      uint64_t gv = lane < 8 ? load_label<kShared>(lab + static_cast<uint64_t>(q.goal_node) * 9u + lane) : kGraphInf;
      for (int o = 4; o > 0; o >>= 1) {
        const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, gv, o);
        gv = other < gv ? other : gv;
      }
      if (lane == 0) sh_goal = gv;
    }
    ++rounds;
    __syncthreads();
  }
  atomicAdd(&sh_examined, examined);
  atomicAdd(&sh_turns, turns);
  __syncthreads();

  // ---- goal state (smallest label, then smallest state) ----
  __shared__ uint32_t sh_goal_state;
  if (warp == 0) {
    const uint32_t s = q.goal_node * 9u + static_cast<uint32_t>(lane);
    uint64_t v = lane < 8 ? load_label<kShared>(lab + s) : kGraphInf;
    uint32_t st = lane < 8 ? s : kInvalid32;
    for (int o = 4; o > 0; o >>= 1) {
      const uint64_t ov = __shfl_xor_sync(0xFFFFFFFFu, v, o);
      const uint32_t os = __shfl_xor_sync(0xFFFFFFFFu, st, o);
      if (ov < v || (ov == v && os < st)) {
        v = ov;
        st = os;
      }
    }
    if (lane == 0) sh_goal_state = (v == kGraphInf) ? kInvalid32 : st;
  }
  __syncthreads();
  const uint32_t goal_state = sh_goal_state;
  if (completion == APGAR_B200_COMPLETION_REACHED && goal_state == kInvalid32) {
    completion = APGAR_B200_COMPLETION_DISCONNECTED;
  }

  if (p.workspace_mode) {
    if constexpr (kShared) {
      uint64_t* out = p.labels + static_cast<uint64_t>(qi) * S;
      for (uint64_t s = tid; s < S; s += kThreads) out[s] = lab[s];
    }
    uint32_t* pred = p.predecessors + static_cast<uint64_t>(qi) * S;
    uint64_t* own = p.state_owners + static_cast<uint64_t>(qi) * S;
    uint64_t* pown = p.predecessor_owners + static_cast<uint64_t>(qi) * S;
    for (uint64_t s = tid; s < S; s += kThreads) {
      pred[s] = (static_cast<uint32_t>(s) == q.start_node * 9u + 8u)
                    ? kInvalid32
                    : canonical_predecessor<kShared>(g, q, pol, lab, static_cast<uint32_t>(s));
      own[s] = q.workspace_owner;
      pown[s] = q.workspace_owner;
    }
  } else if (warp == 0) {
    // canonical reverse walk: lanes 0..8 test the predecessor headings
    apgar_b200_compact_path_v1 cp{};
    cp.schema_version = 1;
    cp.query_id = q.query_id;
    cp.workspace_owner = q.workspace_owner;
    uint32_t* stage = p.path_stage + static_cast<uint64_t>(qi) * S;
    uint32_t n = 0;
    bool complete = false;
    if (completion == APGAR_B200_COMPLETION_REACHED) {
      const uint32_t start_state = q.start_node * 9u + 8u;
      uint32_t cursor = goal_state;
      while (n < S) {
        if (lane == 0) stage[n] = cursor;
        ++n;
        if (cursor == start_state) {
          complete = true;
          break;
        }
        const uint32_t node = cursor / 9u, h = cursor % 9u;
        if (h == 8u) break;
        const uint32_t pred = nbr(g, node, (h + 4u) & 7u);
        if (pred == kInvalid32) break;
        const uint64_t here = load_label<kShared>(lab + cursor);
        bool ok = false;
        if (lane < 9 && !(lane == 8 && pred != q.start_node)) {
          uint64_t t, c;
          ok = transition_cost(g, q, pol, pred, h, static_cast<uint32_t>(lane), &t) &&
               checked_add(load_label<kShared>(lab + pred * 9u + lane), t, &c) && c == here;
        }
        const unsigned ballot = __ballot_sync(0xFFFFFFFFu, ok);
        if (ballot == 0u) break;
        cursor = pred * 9u + static_cast<uint32_t>(__ffs(ballot) - 1);
      }
    }
    cp.state_count = complete ? n : 0u;
    if (completion == APGAR_B200_COMPLETION_REACHED && !complete) {
      completion = APGAR_B200_COMPLETION_DISCONNECTED;  // unreachable with exact labels
    }
    if (lane == 0) p.compact[qi] = cp;
  }

  if (tid == 0) {
    apgar_b200_batch_result_v1 r{};
    r.schema_version = 1;
    r.compiler_version = g.compiler_version;
    r.input_ordinal = q.input_ordinal;
    r.start_node = q.start_node;
    r.goal_node = q.goal_node;
    r.goal_state = completion == APGAR_B200_COMPLETION_REACHED ? goal_state : kInvalid32;
    r.rounds = rounds;
    r.generator = p.generator;
    set_completion(r, completion);
    r.batch_id = q.batch_id;
    r.query_id = q.query_id;
    r.workspace_owner = q.workspace_owner;
    r.policy_identity = q.policy_identity;
    r.routing_profile_fingerprint = q.routing_profile_fingerprint;
    r.source_board_content_hash = g.source_board_content_hash;
    r.compiler_profile_fingerprint = g.compiler_profile_fingerprint;
    r.rule_bucket_identity = g.rule_bucket_identity;
    r.device_view_fingerprint = g.device_view_fingerprint;
    r.examined_work = sh_examined;
    r.heading_turn_relaxations = sh_turns;
    p.results[qi] = r;
  }
}

// Deterministic packing of the compact paths in query order.
__global__ void graph_pack_offsets(apgar_b200_compact_path_v1* compact, uint32_t count,
                                   unsigned long long* total) {
  __shared__ unsigned long long warp_sums[32];
  __shared__ unsigned long long base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint32_t chunk = 0; chunk < count; chunk += blockDim.x) {
    const uint32_t i = chunk + threadIdx.x;
    const unsigned long long len = i < count ? compact[i].state_count : 0ull;
    unsigned long long x = len;
    for (int k = 1; k < 32; k <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, k);
      if (lane >= k) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned long long s = lane < static_cast<int>(blockDim.x >> 5) ? warp_sums[lane] : 0ull;
      for (int k = 1; k < 32; k <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, s, k);
        if (lane >= k) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const unsigned long long warp_base = warp == 0 ? 0ull : warp_sums[warp - 1];
    if (i < count) compact[i].state_offset = base + warp_base + x - len;
    __syncthreads();
    if (threadIdx.x == 0) base += warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = base;
}

__global__ void graph_pack_copy(const apgar_b200_compact_path_v1* compact, uint32_t count,
                                uint64_t states_per_query, const uint32_t* stage,
                                uint32_t* packed) {
  for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
    const apgar_b200_compact_path_v1 c = compact[i];
    for (uint32_t j = threadIdx.x; j < c.state_count; j += blockDim.x) {
      packed[c.state_offset + j] = stage[static_cast<uint64_t>(i) * states_per_query + j];
    }
  }
}

}  // namespace

// Shared-memory search for graphs whose labels, queues and stamps fit in
// this many bytes (two CTAs per SM).
constexpr size_t kSharedSearchBytes = 100 * 1024;
// Policy edges staged in shared memory up to this many bytes (2048 edges).
constexpr size_t kStagedPolicyBytes = 32 * 1024;

cudaError_t launch_graph_search(const GraphLaunch& launch, cudaStream_t stream) {
  if (launch.query_count == 0) return cudaSuccess;
  const size_t n = launch.g.node_count;
  // shared layout: labels, queues and stamps; the neighbour table; the policy edges
  const size_t state_bytes = (n * 9u * 8u + n * 12u + 15u) & ~static_cast<size_t>(15);
  const size_t nbr_bytes = n * 8u * 4u;
  const size_t policy_bytes = static_cast<size_t>(launch.max_policy_edges) * sizeof(apgar_b200_policy_edge_v1);
  const size_t staged_policy = policy_bytes <= kStagedPolicyBytes ? policy_bytes : 0;
  GraphLaunch l = launch;
  l.policy_smem_offset = kInvalid32;
  l.nbr_smem_offset = kInvalid32;
  if (state_bytes + nbr_bytes + staged_policy <= kSharedSearchBytes) {
    l.nbr_smem_offset = static_cast<uint32_t>(state_bytes);
    if (staged_policy > 0) l.policy_smem_offset = static_cast<uint32_t>(state_bytes + nbr_bytes);
    const cudaError_t e = cudaFuncSetAttribute(graph_search_kernel<true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(kSharedSearchBytes));
    if (e != cudaSuccess) return e;
    graph_search_kernel<true><<<l.query_count, kThreads, state_bytes + nbr_bytes + staged_policy, stream>>>(l);
  } else {
    if (staged_policy > 0) l.policy_smem_offset = 0u;
    graph_search_kernel<false><<<l.query_count, kThreads, staged_policy, stream>>>(l);
  }
  return cudaGetLastError();
}

cudaError_t launch_graph_pack(apgar_b200_compact_path_v1* compact, uint32_t count,
                              uint64_t states_per_query, const uint32_t* stage, uint32_t* packed,
                              unsigned long long* total, int sm_count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  graph_pack_offsets<<<1, 1024, 0, stream>>>(compact, count, total);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const uint32_t cap = static_cast<uint32_t>(sm_count > 0 ? sm_count * 8 : 1024);
  graph_pack_copy<<<count < cap ? count : cap, 128, 0, stream>>>(compact, count, states_per_query,
                                                                 stage, packed);
  return cudaGetLastError();
}

}  // namespace apgar_b200
