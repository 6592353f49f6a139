// Host side of lattice mode: lattice upload (the prepared view), the batch
// planner (admission, width classes, label-slab layout, LPT order) and the
// C-ABI entry points.  No CPU search fallback exists: every admitted net is
// searched by the CUDA kernels in lattice_sweep.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "host_common.h"
#include "lattice_common.cuh"

namespace apgar_b200 {

int lattice_cells_per_lane(int layers);
size_t lattice_sweep_smem_bytes(int layers, int warps_per_net, int max_rows);
cudaError_t launch_lattice_sweep(int layers, int warps_per_net, const SweepLaunch& launch,
                                 int max_rows, cudaStream_t stream);
cudaError_t launch_accumulate_cells(const apgar_b200_lattice_result* results, uint32_t count,
                                    const uint32_t* paths, uint32_t* usage, uint64_t cell_count,
                                    int sm_count, cudaStream_t stream);
cudaError_t launch_lattice_frontier(const FrontierClasses& classes, int sm_count,
                                    cudaStream_t stream);
cudaError_t launch_lattice_validate(const LatticeDeviceView& lat, const apgar_b200_lattice_net* nets,
                                    const apgar_b200_lattice_result* results, const uint32_t* paths,
                                    uint64_t path_count, uint32_t count,
                                    apgar_b200_path_verdict* out, cudaStream_t stream);
cudaError_t lattice_frontier_resident_groups(int warps_per_net, int sm_count, uint32_t* out);
cudaError_t launch_build_moves(const LatticeDeviceView& lat, uint16_t* moves, cudaStream_t stream);
cudaError_t launch_price_update(uint32_t count, const uint32_t* usage, uint64_t factor,
                                uint64_t next_factor, uint64_t hist_inc, uint64_t capacity,
                                uint64_t max_value, uint64_t* present, uint64_t* history,
                                uint64_t* total, uint64_t* next_cost, uint32_t* next_cost32,
                                uint32_t* next_cost_own32, uint32_t* status,
                                unsigned long long* stats, cudaStream_t stream);
cudaError_t launch_mark_dirty(const apgar_b200_lattice_result* results, uint32_t count,
                              const uint32_t* paths, const uint32_t* usage, uint64_t cell_count,
                              uint32_t capacity, uint8_t* skip, int sm_count, cudaStream_t stream);
cudaError_t launch_lattice_pack(apgar_b200_lattice_result* results, uint32_t count,
                                unsigned long long* total, const uint32_t* arena, uint32_t* paths,
                                int sm_count, cudaStream_t stream);
cudaError_t launch_rasters(const LatticeDeviceView& lat, const apgar_b200_lattice_net* nets,
                           uint32_t count, const uint32_t* cell_cost, void* rasters, uint32_t* dims,
                           cudaStream_t stream);
cudaError_t launch_labels(const apgar_b200_lattice_net* nets, uint32_t count, const uint32_t* dims,
                          int lat_w, int lat_h, const apgar_b200_lattice_result* results,
                          const uint32_t* paths, uint8_t* labels, cudaStream_t stream);
cudaError_t launch_lattice_segments(const apgar_b200_lattice_result* results, const uint32_t* paths,
                                    uint32_t count, uint32_t width, uint32_t height, int64_t ox,
                                    int64_t oy, int64_t step, apgar_b200_segment* segments,
                                    uint32_t* segment_counts, cudaStream_t stream);
cudaError_t launch_corridors(const float* logits, const uint32_t* dims,
                             const apgar_b200_lattice_net* nets, uint32_t count, float threshold,
                             int dilate, uint64_t max_cells, int layers, uint32_t* bits,
                             cudaStream_t stream);

namespace {

// Width classes: warps per net.  A sweep net takes the fewest warps whose
// lanes cover its frame row (each lane holds lattice_cells_per_lane(L) cells
// of every layer, so G warps cover 32 * C * G cells): the widest class is
// issue-bound, and warps past the row's end would run every instruction on
// padding.  The frontier uses the power-of-two sizes (kFrontierClasses).
constexpr int kGroupSizes[] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};
constexpr int kClassCount = 16;
// Frontier width classes 0..4 (1, 2, 4, 8 and 16 warps) as kGroupSizes indices.
constexpr int kFrontierClasses[] = {0, 1, 3, 7, 15};
constexpr size_t kMaxSmemPerBlock = 227 * 1024;

struct LatticeObject;

struct ClassRange {
  int warps_per_net = 0;
  uint32_t begin = 0;  // into plans
  uint32_t count = 0;
  int max_rows = 0;
  // frontier workspace: `slots` persistent slots of `slab_cells` label words
  // and 3 x `list_cap` queue entries, starting at these pool offsets
  uint64_t slab_cells = 0;
  uint32_t list_cap = 0;
  uint32_t slots = 0;
  uint64_t words_offset = 0;
  uint64_t lists_offset = 0;
};

// Chained expansions per queued cell by width class (the default when the
// plan's options leave it to the class).
// Measured on the medium batch: the batch is bound by expansion throughput,
// so the extra expansions of a chain cost more than the rounds it saves.
uint32_t default_chain(int) { return 0u; }

// Default frontier width-class limits (log2 window cells of the 1-, 2-, 4-
// and 8-warp classes), the autotuner's choice on the medium batch.
constexpr uint32_t kDefaultClassBounds = 12u | (15u << 8) | (17u << 16) | (19u << 24);

// Queue entries per list per frontier slot (a net needing more is rejected).
constexpr uint64_t kMaxListEntries = 1ull << 25;
// Frontier workspace above which nets share persistent slot slabs instead of
// owning one slab each.
constexpr uint64_t kPerNetFrontierBytes = 24ull << 30;
// Budget of the persistent slot workspace (label words and queue lists).
constexpr uint64_t kSlotFrontierBytes = 64ull << 30;

// A workspace budget, overridable from the environment (bytes, decimal), for
// callers with less device memory to give the frontier.
uint64_t budget_from_env(const char* name, uint64_t fallback) {
  const char* v = std::getenv(name);
  if (v == nullptr || *v == '\0') return fallback;
  char* end = nullptr;
  const unsigned long long b = std::strtoull(v, &end, 10);
  return (end != nullptr && *end == '\0' && b > 0) ? static_cast<uint64_t>(b) : fallback;
}

struct PlanObject {
  LatticeObject* lattice = nullptr;
  int device = -1;
  int sm_count = 0;
  uint32_t count = 0;
  uint32_t max_sweeps = 0;  // sweeps (SWEEP) or rounds (FRONTIER)
  uint32_t generator = APGAR_B200_LATTICE_SWEEP;
  uint32_t bucket_width = 0;
  uint32_t wide_bucket_width = 0;  // FRONTIER: level width of the 16-warp class
  uint32_t chain = 0;    // FRONTIER: apgar_b200_lattice_options::chain
  uint32_t wide_chain = 0;  // FRONTIER: apgar_b200_lattice_options::wide_chain
  uint32_t class_bounds = kDefaultClassBounds;  // FRONTIER: log2 class limits, byte per class
  bool per_net = false;  // FRONTIER: one slab per net (else persistent slots)
  const uint32_t* cell_cost = nullptr;  // caller-owned device prices (frontier only)
  // partial rip-up (set by a negotiation): kept nets and their previous routes
  const uint8_t* skip = nullptr;
  const apgar_b200_lattice_result* prev_results = nullptr;
  const uint32_t* prev_paths = nullptr;
  // rip-up pricing (set by a negotiation): prices of a net's own previous
  // cells, and one bit per label word to mark them
  const uint32_t* cell_cost_own = nullptr;
  uint32_t* own_bits = nullptr;
  // corridor mode: caller-owned device bitmaps and the per-net outcomes
  const uint32_t* corridor = nullptr;
  DeviceBuffer<uint8_t> corridor_status;
  uint32_t* cancel_host = nullptr;  // pinned, mapped; polled by the kernels
  uint32_t* cancel_dev = nullptr;
  std::vector<ClassRange> classes;
  std::vector<apgar_b200_lattice_result> rejected_template;
  DeviceBuffer<apgar_b200_lattice_net> nets;
  DeviceBuffer<NetPlan> plans;
  DeviceBuffer<uint32_t> dist_pool;
  DeviceBuffer<apgar_b200_lattice_result> results;
  DeviceBuffer<uint32_t> arena;
  DeviceBuffer<uint32_t> paths;
  DeviceBuffer<unsigned long long> words;  // FRONTIER: label | ~round stamp per cell
  DeviceBuffer<uint32_t> lists;            // FRONTIER: three queue lists per net
  // [0] arena cursor, [1] packed total, [2 + class] work-stealing cursors
  DeviceBuffer<unsigned long long> counters;
  uint64_t label_cells = 0;
  uint64_t arena_capacity = 0;
  cudaStream_t class_streams[kClassCount] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t joins[kClassCount] = {};

  ~PlanObject() {
    for (cudaStream_t& s : class_streams) {
      if (s != nullptr) cudaStreamDestroy(s);
    }
    for (cudaEvent_t& e : joins) {
      if (e != nullptr) cudaEventDestroy(e);
    }
    if (fork != nullptr) cudaEventDestroy(fork);
    if (cancel_host != nullptr) cudaFreeHost(cancel_host);
  }

  uint64_t workspace_bytes() const {
    return nets.bytes() + plans.bytes() + dist_pool.bytes() + results.bytes() + arena.bytes() +
           paths.bytes() + counters.bytes() + words.bytes() + lists.bytes();
  }
};

struct LatticeObject {
  int device = -1;
  LatticeDeviceView view{};
  DeviceBuffer<uint32_t> blocked;
  DeviceBuffer<uint32_t> via_ok;
  DeviceBuffer<uint32_t> sweep_rows, sweep_cols, sweep_via_rows, sweep_via_cols;
  DeviceBuffer<uint16_t> moves;  // LatticeDeviceView::moves
  std::mutex route_mutex;
  std::unique_ptr<PlanObject> route_plan;  // reusable workspace for route()
  // reusable workspace for validate() (grown as needed, kept for later calls)
  std::mutex validate_mutex;
  DeviceBuffer<apgar_b200_lattice_net> val_nets;
  DeviceBuffer<apgar_b200_lattice_result> val_results;
  DeviceBuffer<uint32_t> val_paths;
  DeviceBuffer<apgar_b200_path_verdict> val_out;
};

int check_device(int expected) {
  int current = -1;
  APGAR_B200_CUDA("cudaGetDevice", cudaGetDevice(&current));
  if (current != expected) {
    return set_error(APGAR_B200_BACKEND_FAILURE,
                     "current CUDA device differs from the device the lattice was uploaded on");
  }
  return APGAR_B200_OK;
}

// Smallest width class whose row coverage holds `width` cells; -1 if none.
int class_for_width(uint32_t width, int layers) {
  const uint32_t per_warp = 32u * static_cast<uint32_t>(lattice_cells_per_lane(layers));
  for (int i = 0; i < kClassCount; ++i) {
    if (per_warp * static_cast<uint32_t>(kGroupSizes[i]) >= width) return i;
  }
  return -1;
}

// Frontier width class (index into kGroupSizes) from the window's cell count.
// A frontier round is a chain of dependent memory waves, so its latency falls
// when more warps share a round's cells; the thresholds (measured on the
// medium batch: 4-layer windows of 10^4 to 10^7 cells) give every window
// above 256k cells 16 warps.
// `bounds` holds log2 of each class's largest window, one byte per class
// (apgar_b200_lattice_options::class_bounds).
int frontier_class(uint64_t cells, uint32_t bounds) {
  for (int k = 0; k < 4; ++k) {
    if (cells <= (1ull << ((bounds >> (8 * k)) & 0xFFu))) return k;
  }
  return 4;
}

bool class_bounds_valid(uint32_t bounds) {
  uint32_t prev = 0;
  for (int k = 0; k < 4; ++k) {
    const uint32_t b = (bounds >> (8 * k)) & 0xFFu;
    if (b < 1 || b > 31 || b <= prev) return false;
    prev = b;
  }
  return true;
}

// Guard-padded sweep planes from row-major bit planes `in`
// ([planes][height][width/32], bit x%32 of word x/32).  Row form: each plane
// row is [guard][words][guard]; column form: plane row x holds bit y of
// column x.  Guards and the bits past `height` in the column form read as
// `pad`.
std::vector<uint32_t> sweep_planes(const uint32_t* in, int planes, int height, int width,
                                   bool columns, uint32_t pad) {
  const int words = width / 32;
  const int words_t = (height + 31) / 32;
  if (!columns) {
    const size_t stride = static_cast<size_t>(words) + 2;
    std::vector<uint32_t> out(static_cast<size_t>(planes) * height * stride, pad);
    for (int l = 0; l < planes; ++l) {
      for (int y = 0; y < height; ++y) {
        const uint32_t* src = in + (static_cast<size_t>(l) * height + y) * words;
        uint32_t* dst = out.data() + (static_cast<size_t>(l) * height + y) * stride + 1;
        std::memcpy(dst, src, static_cast<size_t>(words) * sizeof(uint32_t));
      }
    }
    return out;
  }
  const size_t stride = static_cast<size_t>(words_t) + 2;
  std::vector<uint32_t> out(static_cast<size_t>(planes) * width * stride, 0u);
  for (int l = 0; l < planes; ++l) {
    uint32_t* plane = out.data() + static_cast<size_t>(l) * width * stride;
    for (int x = 0; x < width; ++x) {
      plane[static_cast<size_t>(x) * stride] = pad;
      plane[static_cast<size_t>(x) * stride + stride - 1] = pad;
    }
    for (int y = 0; y < height; ++y) {
      const uint32_t* row = in + (static_cast<size_t>(l) * height + y) * words;
      for (int wi = 0; wi < words; ++wi) {
        uint32_t bits = row[wi];
        while (bits != 0u) {
          const int b = __builtin_ctz(bits);
          bits &= bits - 1u;
          const int x = wi * 32 + b;
          plane[static_cast<size_t>(x) * stride + 1 + (y >> 5)] |= 1u << (y & 31);
        }
      }
    }
    if (pad != 0u && (height & 31) != 0) {
      const uint32_t tail = ~((1u << (height & 31)) - 1u);
      for (int x = 0; x < width; ++x) plane[static_cast<size_t>(x) * stride + words_t] |= tail;
    }
  }
  return out;
}

// Builds (or rebuilds into existing buffers) a plan for `nets`.
int build_plan(LatticeObject* lat, const apgar_b200_lattice_net* host_nets, uint32_t count,
               uint32_t max_sweeps, PlanObject* plan,
               uint32_t generator = APGAR_B200_LATTICE_SWEEP, uint32_t bucket_width = 0,
               uint32_t chain = 0, uint32_t class_bounds = 0, uint32_t wide_bucket_width = 0,
               uint32_t wide_chain = 0) {
  const LatticeDeviceView& v = lat->view;
  const bool frontier = generator == APGAR_B200_LATTICE_FRONTIER;
  plan->lattice = lat;
  plan->device = lat->device;
  plan->count = count;
  plan->max_sweeps = max_sweeps;
  plan->generator = generator;
  // Level width: at least twice the largest move, so that every deferred cell
  // falls in the next level (the frontier kernel relies on it: a cell that
  // left the far list never returns to it, so its far bit needs no clearing).
  plan->bucket_width = std::max(bucket_width, 2u * std::max(v.orth, std::max(v.diag, v.via)));
  plan->wide_bucket_width =
      wide_bucket_width != 0
          ? std::max(wide_bucket_width, 2u * std::max(v.orth, std::max(v.diag, v.via)))
          : plan->bucket_width;
  plan->chain = chain;
  plan->wide_chain = wide_chain != 0 ? wide_chain : chain;
  plan->class_bounds = class_bounds != 0 ? class_bounds : kDefaultClassBounds;
  APGAR_B200_CUDA("cudaDeviceGetAttribute",
                  cudaDeviceGetAttribute(&plan->sm_count, cudaDevAttrMultiProcessorCount,
                                         lat->device));
  const uint64_t max_move = std::max(v.orth, std::max(v.diag, v.via));

  std::vector<std::vector<uint32_t>> members(kClassCount);
  std::vector<apgar_b200_lattice_result> init(count);
  std::memset(init.data(), 0, init.size() * sizeof(apgar_b200_lattice_result));
  for (uint32_t i = 0; i < count; ++i) {
    const apgar_b200_lattice_net& n = host_nets[i];
    apgar_b200_lattice_result& r = init[i];
    r.cost = APGAR_B200_UNREACHABLE;
    r.completion = APGAR_B200_COMPLETION_REJECTED;
    const bool in_lattice =
        n.start_layer < static_cast<uint32_t>(v.layers) &&
        n.goal_layer < static_cast<uint32_t>(v.layers) && n.win_w > 0 && n.win_h > 0 &&
        static_cast<uint64_t>(n.win_x0) + n.win_w <= static_cast<uint64_t>(v.width) &&
        static_cast<uint64_t>(n.win_y0) + n.win_h <= static_cast<uint64_t>(v.height) &&
        n.start_x >= n.win_x0 && n.start_x < n.win_x0 + n.win_w && n.start_y >= n.win_y0 &&
        n.start_y < n.win_y0 + n.win_h && n.goal_x >= n.win_x0 && n.goal_x < n.win_x0 + n.win_w &&
        n.goal_y >= n.win_y0 && n.goal_y < n.win_y0 + n.win_h;
    if (!in_lattice) continue;
    const uint64_t cells = static_cast<uint64_t>(v.layers) * n.win_w * n.win_h;
    if (cells * max_move >= kLabelInf) continue;  // uint32 cost domain not provable
    if (frontier) {
      // packed queue entries hold x and y in 14 bits each
      if (n.win_w > 16384u || n.win_h > 16384u) continue;
      members[kFrontierClasses[frontier_class(cells, plan->class_bounds)]].push_back(i);
      continue;
    }
    const uint32_t frame_width = std::max(n.win_w, n.win_h);
    const uint32_t frame_rows = std::min(n.win_w, n.win_h);
    const int ci = class_for_width(frame_width, v.layers);
    if (ci < 0 || frame_rows > 32000u) continue;
    members[ci].push_back(i);
  }
  plan->rejected_template = init;

  std::vector<NetPlan> plans;
  plans.reserve(count);
  plan->classes.clear();
  uint64_t dist_cells = 0;
  uint64_t arena_cells = 0;
  uint64_t arena_lists = 0;    // frontier queue entries over all slots
  uint64_t per_net_cells = 0;  // frontier: padded window cells over all nets
  for (int ci = 0; ci < kClassCount; ++ci) {
    std::vector<uint32_t>& m = members[ci];
    if (m.empty()) continue;
    // longest-processing-time first: larger windows launch first
    std::stable_sort(m.begin(), m.end(), [&](uint32_t a, uint32_t b) {
      const uint64_t ca = static_cast<uint64_t>(host_nets[a].win_w) * host_nets[a].win_h;
      const uint64_t cb = static_cast<uint64_t>(host_nets[b].win_w) * host_nets[b].win_h;
      return ca > cb;
    });
    ClassRange range;
    range.warps_per_net = kGroupSizes[ci];
    range.begin = static_cast<uint32_t>(plans.size());
    range.count = static_cast<uint32_t>(m.size());
    for (uint32_t i : m) {
      const apgar_b200_lattice_net& n = host_nets[i];
      NetPlan np{};
      np.net = i;
      if (frontier) {
        // window layout [layer][y][x] in the slot's slab, padded to 128 cells
        np.transposed = 0;
        np.rows = n.win_h;
        np.width = n.win_w;
        np.pitch = n.win_w;
        const uint64_t padded = (static_cast<uint64_t>(v.layers) * n.win_w * n.win_h + 127ull) & ~127ull;
        np.dist_offset = per_net_cells;  // used when every net gets its own slab
        per_net_cells += padded;
        range.slab_cells = std::max<uint64_t>(range.slab_cells, padded);
      } else {
        np.transposed = n.win_h > n.win_w ? 1u : 0u;
        np.rows = np.transposed ? n.win_w : n.win_h;
        np.width = np.transposed ? n.win_h : n.win_w;
        np.pitch = (np.width + 3u) & ~3u;
        np.dist_offset = dist_cells;
        dist_cells += static_cast<uint64_t>(v.layers) * np.rows * np.pitch;
      }
      arena_cells += 8ull * (n.win_w + n.win_h) + 64ull * v.layers;
      range.max_rows = std::max(range.max_rows, static_cast<int>(np.rows));
      plans.push_back(np);
    }
    if (!frontier && lattice_sweep_smem_bytes(v.layers, range.warps_per_net, range.max_rows) >
                         kMaxSmemPerBlock) {
      return set_error(APGAR_B200_UNSUPPORTED, "window too tall for the shared-memory row map");
    }
    if (frontier) {
      uint32_t resident = 0;
      APGAR_B200_CUDA("cudaOccupancyMaxActiveBlocksPerMultiprocessor",
                      lattice_frontier_resident_groups(range.warps_per_net, plan->sm_count, &resident));
      range.slots = std::min<uint32_t>(resident, range.count);
      range.list_cap = static_cast<uint32_t>(std::min<uint64_t>(range.slab_cells, kMaxListEntries));
      // slot slabs are spaced by the largest window plus a 4 KB skew, so that
      // equal offsets of different slots do not alias in the L2
      range.slab_cells += 512;
    }
    plan->classes.push_back(range);
  }
  const uint64_t per_net_budget = budget_from_env("APGAR_B200_FRONTIER_PER_NET_BYTES", kPerNetFrontierBytes);
  const uint64_t slot_budget = budget_from_env("APGAR_B200_FRONTIER_SLOT_BYTES", kSlotFrontierBytes);
  if (frontier && per_net_cells * 20ull > per_net_budget) {
    // Slot workspace within its budget: the class with the largest slot
    // gives up an eighth of its slots until the total fits (every class keeps
    // at least one; fewer slots only means fewer of its nets in flight).
    const auto slot_bytes = [](const ClassRange& c) { return c.slab_cells * 8ull + 12ull * c.list_cap; };
    const auto total = [&]() {
      uint64_t t = 0;
      for (const ClassRange& c : plan->classes) t += c.slots * slot_bytes(c);
      return t;
    };
    while (total() > slot_budget) {
      ClassRange* widest = nullptr;
      for (ClassRange& c : plan->classes) {
        if (c.slots > 1 && (widest == nullptr || slot_bytes(c) > slot_bytes(*widest))) widest = &c;
      }
      if (widest == nullptr) break;
      widest->slots -= std::max<uint32_t>(1u, widest->slots / 8u);
    }
  }
  if (frontier) {
    for (ClassRange& range : plan->classes) {
      range.words_offset = dist_cells;
      dist_cells += static_cast<uint64_t>(range.slots) * range.slab_cells;
      range.lists_offset = arena_lists;
      arena_lists += static_cast<uint64_t>(range.slots) * 3ull * range.list_cap;
    }
  }
  plan->label_cells = dist_cells;
  plan->arena_capacity = std::max<uint64_t>(arena_cells, 64);

  APGAR_B200_CUDA("cudaMalloc(nets)", plan->nets.ensure(std::max<uint32_t>(count, 1)));
  APGAR_B200_CUDA("cudaMalloc(plans)", plan->plans.ensure(std::max<size_t>(plans.size(), 1)));
  if (frontier) {
    // Every net gets its own slab (8 B words + 3 x 4 B list entries per
    // cell) when that fits the per-net budget; otherwise the persistent
    // groups reuse their slot slabs net after net.
    plan->per_net = per_net_cells * 20ull <= per_net_budget;
    if (plan->per_net) {
      dist_cells = per_net_cells;
      arena_lists = 3ull * per_net_cells;
    }
    APGAR_B200_CUDA("cudaMalloc(label words)", plan->words.ensure(std::max<uint64_t>(dist_cells, 128)));
    APGAR_B200_CUDA("cudaMalloc(queue lists)", plan->lists.ensure(std::max<uint64_t>(arena_lists, 3)));
  } else {
    APGAR_B200_CUDA("cudaMalloc(label slabs)", plan->dist_pool.ensure(std::max<uint64_t>(dist_cells, 4)));
  }
  APGAR_B200_CUDA("cudaMalloc(results)", plan->results.ensure(std::max<uint32_t>(count, 1)));
  APGAR_B200_CUDA("cudaMalloc(path arena)", plan->arena.ensure(plan->arena_capacity));
  APGAR_B200_CUDA("cudaMalloc(paths)", plan->paths.ensure(plan->arena_capacity));
  APGAR_B200_CUDA("cudaMalloc(counters)", plan->counters.ensure(2 + kClassCount));
  if (count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(nets)",
                    cudaMemcpy(plan->nets.get(), host_nets, count * sizeof(apgar_b200_lattice_net),
                               cudaMemcpyHostToDevice));
    APGAR_B200_CUDA("cudaMemcpy(results init)",
                    cudaMemcpy(plan->results.get(), init.data(),
                               count * sizeof(apgar_b200_lattice_result), cudaMemcpyHostToDevice));
  }
  if (!plans.empty()) {
    APGAR_B200_CUDA("cudaMemcpy(plans)",
                    cudaMemcpy(plan->plans.get(), plans.data(), plans.size() * sizeof(NetPlan),
                               cudaMemcpyHostToDevice));
  }
  int least_priority = 0, greatest_priority = 0;
  APGAR_B200_CUDA("cudaDeviceGetStreamPriorityRange",
                  cudaDeviceGetStreamPriorityRange(&least_priority, &greatest_priority));
  for (int ci = 0; ci < kClassCount; ++ci) {
    if (plan->class_streams[ci] == nullptr) {
      // wider classes (higher positions) get higher priority: their blocks
      // need most of an SM and hold the nets with the most rounds, so they
      // must not wait behind the narrow classes' persistent grids
      const int priority = std::max(greatest_priority, least_priority - ci);
      APGAR_B200_CUDA("cudaStreamCreate",
                      cudaStreamCreateWithPriority(&plan->class_streams[ci], cudaStreamNonBlocking,
                                                   priority));
      APGAR_B200_CUDA("cudaEventCreate",
                      cudaEventCreateWithFlags(&plan->joins[ci], cudaEventDisableTiming));
    }
  }
  if (plan->fork == nullptr) {
    APGAR_B200_CUDA("cudaEventCreate", cudaEventCreateWithFlags(&plan->fork, cudaEventDisableTiming));
  }
  if (plan->cancel_host == nullptr) {
    void* h = nullptr;
    APGAR_B200_CUDA("cudaHostAlloc(cancel flag)",
                    cudaHostAlloc(&h, sizeof(uint32_t), cudaHostAllocMapped));
    plan->cancel_host = static_cast<uint32_t*>(h);
    void* d = nullptr;
    APGAR_B200_CUDA("cudaHostGetDevicePointer(cancel flag)",
                    cudaHostGetDevicePointer(&d, h, 0));
    plan->cancel_dev = static_cast<uint32_t*>(d);
  }
  *reinterpret_cast<volatile uint32_t*>(plan->cancel_host) = 0u;
  return APGAR_B200_OK;
}

int execute_plan(PlanObject* plan, cudaStream_t stream) {
  if (int rc = check_device(plan->device); rc != APGAR_B200_OK) return rc;
  APGAR_B200_CUDA("cudaMemsetAsync(counters)",
                  cudaMemsetAsync(plan->counters.get(), 0,
                                  (2 + kClassCount) * sizeof(unsigned long long), stream));
  const LatticeDeviceView& v = plan->lattice->view;
  FrontierLaunch fbase{};
  fbase.lat = v;
  fbase.nets = plan->nets.get();
  fbase.max_rounds = plan->max_sweeps;
  fbase.bucket_width = plan->bucket_width;
  fbase.words = plan->words.get();
  fbase.lists = plan->lists.get();
  fbase.results = plan->results.get();
  fbase.path_arena = plan->arena.get();
  fbase.path_arena_capacity = plan->arena_capacity;
  fbase.arena_cursor = plan->counters.get();
  fbase.cancel = plan->cancel_dev;
  fbase.cell_cost = plan->cell_cost;
  fbase.skip = plan->skip;
  fbase.prev_results = plan->prev_results;
  fbase.prev_paths = plan->prev_paths;
  fbase.cell_cost_own = plan->cell_cost_own;
  if (plan->corridor != nullptr) {
    fbase.corridor = plan->corridor;
    fbase.corridor_status = plan->corridor_status.get();
  }
  SweepLaunch base{};
  base.lat = v;
  base.nets = plan->nets.get();
  base.max_sweeps = plan->max_sweeps;
  base.dist_pool = plan->dist_pool.get();
  base.results = plan->results.get();
  base.path_arena = plan->arena.get();
  base.path_arena_capacity = plan->arena_capacity;
  base.arena_cursor = plan->counters.get();
  base.cancel = plan->cancel_dev;
  if (plan->generator == APGAR_B200_LATTICE_FRONTIER) {
    // every width class in one persistent launch (the kernel serves the
    // widest class first and splits its groups as the classes drain)
    FrontierClasses fc{};
    for (size_t k = 0; k < plan->classes.size(); ++k) {
      const ClassRange& c = plan->classes[k];
      int pos = 0;
      while ((1 << pos) < c.warps_per_net) ++pos;
      FrontierLaunch& fl = fc.c[pos];
      fl = fbase;
      fl.plans = plan->plans.get() + c.begin;
      fl.plan_count = c.count;
      fl.words = plan->words.get() + c.words_offset;
      fl.lists = plan->lists.get() + c.lists_offset;
      fl.slab_cells = c.slab_cells;
      fl.list_cap = c.list_cap;
      fl.slots = c.slots;
      fl.per_net = plan->per_net ? 1u : 0u;
      fl.own_bits = plan->own_bits == nullptr ? nullptr : plan->own_bits + c.words_offset / 32u;
      if (plan->per_net) {
        fl.words = plan->words.get();
        fl.lists = plan->lists.get();
        fl.own_bits = plan->own_bits;
      }
      fl.next_plan = reinterpret_cast<unsigned int*>(plan->counters.get() + 2 + k);
      // the 16-warp class (the longest searches) may take its own schedule
      const bool wide = c.warps_per_net == 16;
      const uint32_t chain = wide ? plan->wide_chain : plan->chain;
      fl.chain = chain != 0 ? chain - 1 : default_chain(c.warps_per_net);
      if (wide) fl.bucket_width = plan->wide_bucket_width;

    }
    APGAR_B200_CUDA("lattice frontier launch", launch_lattice_frontier(fc, plan->sm_count, stream));
    APGAR_B200_CUDA("lattice pack launch",
                    launch_lattice_pack(plan->results.get(), plan->count, plan->counters.get() + 1,
                                        plan->arena.get(), plan->paths.get(), plan->sm_count, stream));
    return APGAR_B200_OK;
  }
  const bool fan_out = plan->classes.size() > 1;
  if (fan_out) APGAR_B200_CUDA("cudaEventRecord(fork)", cudaEventRecord(plan->fork, stream));
  // widest class first (see the stream priorities above)
  for (size_t kk = plan->classes.size(); kk-- > 0;) {
    const size_t k = kk;
    const ClassRange& c = plan->classes[k];
    SweepLaunch launch = base;
    launch.plans = plan->plans.get() + c.begin;
    launch.plan_count = c.count;
    cudaStream_t s = stream;
    if (fan_out) {
      s = plan->class_streams[k];
      APGAR_B200_CUDA("cudaStreamWaitEvent", cudaStreamWaitEvent(s, plan->fork, 0));
    }
    APGAR_B200_CUDA("lattice sweep launch",
                    launch_lattice_sweep(v.layers, c.warps_per_net, launch, c.max_rows, s));
    if (fan_out) {
      APGAR_B200_CUDA("cudaEventRecord(join)", cudaEventRecord(plan->joins[k], s));
      APGAR_B200_CUDA("cudaStreamWaitEvent", cudaStreamWaitEvent(stream, plan->joins[k], 0));
    }
  }
  APGAR_B200_CUDA("lattice pack launch",
                  launch_lattice_pack(plan->results.get(), plan->count, plan->counters.get() + 1,
                                      plan->arena.get(), plan->paths.get(), plan->sm_count, stream));
  return APGAR_B200_OK;
}

int readback_plan(PlanObject* plan, apgar_b200_lattice_result* results, uint32_t* paths,
                  uint64_t path_capacity, uint64_t* path_total) {
  if (int rc = check_device(plan->device); rc != APGAR_B200_OK) return rc;
  unsigned long long total = 0;
  APGAR_B200_CUDA("cudaMemcpy(path total)",
                  cudaMemcpy(&total, plan->counters.get() + 1, sizeof(total), cudaMemcpyDeviceToHost));
  if (results != nullptr && plan->count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(results)",
                    cudaMemcpy(results, plan->results.get(),
                               plan->count * sizeof(apgar_b200_lattice_result),
                               cudaMemcpyDeviceToHost));
  }
  if (path_total != nullptr) *path_total = total;
  if (paths != nullptr && total > 0) {
    if (total > path_capacity) {
      return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "path output buffer is too small");
    }
    APGAR_B200_CUDA("cudaMemcpy(paths)", cudaMemcpy(paths, plan->paths.get(),
                                                    total * sizeof(uint32_t),
                                                    cudaMemcpyDeviceToHost));
  }
  return APGAR_B200_OK;
}

}  // namespace
}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" int apgar_b200_lattice_upload(const apgar_b200_lattice_desc* d, void** out) {
  if (d == nullptr || out == nullptr || d->blocked == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice upload received a null argument");
  }
  if (d->layers < 1 || d->layers > kMaxLayers || d->layers == 5 || d->layers == 7 ||
      d->height < 1 || d->width < 32 ||
      d->width % 32 != 0 || d->orth == 0 || d->diag == 0 || d->via == 0 ||
      d->orth > 0xFFFFu || d->diag > 0xFFFFu || d->via > 0xFFFFu) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT,
                     "lattice upload rejected layer count, dimensions or move costs");
  }
  try {
    auto lat = std::make_unique<LatticeObject>();
    APGAR_B200_CUDA("cudaGetDevice", cudaGetDevice(&lat->device));
    const size_t words = static_cast<size_t>(d->width / 32);
    const size_t plane = static_cast<size_t>(d->height) * words;
    const size_t blocked_words = plane * d->layers;
    APGAR_B200_CUDA("cudaMalloc(blocked)", lat->blocked.ensure(blocked_words));
    APGAR_B200_CUDA("cudaMemcpy(blocked)",
                    cudaMemcpy(lat->blocked.get(), d->blocked, blocked_words * sizeof(uint32_t),
                               cudaMemcpyHostToDevice));
    if (d->via_ok != nullptr && d->layers > 1) {
      const size_t via_words = plane * (d->layers - 1);
      APGAR_B200_CUDA("cudaMalloc(via)", lat->via_ok.ensure(via_words));
      APGAR_B200_CUDA("cudaMemcpy(via)",
                      cudaMemcpy(lat->via_ok.get(), d->via_ok, via_words * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice));
    }
    // guard-padded sweep planes in both orientations
    const size_t words_t = static_cast<size_t>((d->height + 31) / 32);
    auto upload = [&](DeviceBuffer<uint32_t>& dst, const std::vector<uint32_t>& src,
                      const char* what) -> int {
      APGAR_B200_CUDA(what, dst.ensure(src.size()));
      APGAR_B200_CUDA(what, cudaMemcpy(dst.get(), src.data(), src.size() * sizeof(uint32_t),
                                       cudaMemcpyHostToDevice));
      return APGAR_B200_OK;
    };
    if (int rc = upload(lat->sweep_rows,
                        sweep_planes(d->blocked, d->layers, d->height, d->width, false, ~0u),
                        "upload(sweep rows)");
        rc != APGAR_B200_OK) {
      return rc;
    }
    if (int rc = upload(lat->sweep_cols,
                        sweep_planes(d->blocked, d->layers, d->height, d->width, true, ~0u),
                        "upload(sweep columns)");
        rc != APGAR_B200_OK) {
      return rc;
    }
    if (d->via_ok != nullptr && d->layers > 1) {
      if (int rc = upload(lat->sweep_via_rows,
                          sweep_planes(d->via_ok, d->layers - 1, d->height, d->width, false, 0u),
                          "upload(sweep via rows)");
          rc != APGAR_B200_OK) {
        return rc;
      }
      if (int rc = upload(lat->sweep_via_cols,
                          sweep_planes(d->via_ok, d->layers - 1, d->height, d->width, true, 0u),
                          "upload(sweep via columns)");
          rc != APGAR_B200_OK) {
        return rc;
      }
    }
    lat->view.blocked = lat->blocked.get();
    lat->view.via_ok = lat->via_ok.get();
    lat->view.sweep_rows = lat->sweep_rows.get();
    lat->view.sweep_cols = lat->sweep_cols.get();
    lat->view.sweep_via_rows = lat->sweep_via_rows.get();
    lat->view.sweep_via_cols = lat->sweep_via_cols.get();
    lat->view.words_t = static_cast<int32_t>(words_t);
    lat->view.layers = d->layers;
    lat->view.height = d->height;
    lat->view.width = d->width;
    lat->view.words = static_cast<int32_t>(words);
    lat->view.orth = d->orth;
    lat->view.diag = d->diag;
    lat->view.via = d->via;
    // per-cell move legality for the frontier generator
    const size_t cells = static_cast<size_t>(d->layers) * d->height * d->width;
    APGAR_B200_CUDA("cudaMalloc(move legality)", lat->moves.ensure(std::max<size_t>(cells, 1)));
    APGAR_B200_CUDA("move legality launch", launch_build_moves(lat->view, lat->moves.get(), nullptr));
    APGAR_B200_CUDA("cudaStreamSynchronize(move legality)", cudaStreamSynchronize(nullptr));
    lat->view.moves = lat->moves.get();
    *out = lat.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during upload");
  }
}

extern "C" int apgar_b200_lattice_release(void* lattice) {
  delete static_cast<LatticeObject*>(lattice);
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan(void* lattice, const apgar_b200_lattice_net* nets,
                                       uint32_t count, uint32_t max_sweeps, void** out_plan) {
  if (lattice == nullptr || out_plan == nullptr || (count > 0 && nets == nullptr) ||
      max_sweeps == 0 || max_sweeps > 30000) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice plan received invalid arguments");
  }
  auto* lat = static_cast<LatticeObject*>(lattice);
  if (int rc = check_device(lat->device); rc != APGAR_B200_OK) return rc;
  try {
    auto plan = std::make_unique<PlanObject>();
    if (int rc = build_plan(lat, nets, count, max_sweeps, plan.get()); rc != APGAR_B200_OK) {
      return rc;
    }
    *out_plan = plan.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during planning");
  }
}

extern "C" int apgar_b200_lattice_execute(void* plan, void* stream) {
  if (plan == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan");
  const int rc = execute_plan(static_cast<PlanObject*>(plan), static_cast<cudaStream_t>(stream));
  if (rc == APGAR_B200_OK) clear_error();
  return rc;
}

extern "C" int apgar_b200_lattice_readback(void* plan, apgar_b200_lattice_result* results,
                                           uint32_t* paths, uint64_t path_capacity,
                                           uint64_t* path_total) {
  if (plan == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan");
  const int rc = readback_plan(static_cast<PlanObject*>(plan), results, paths, path_capacity,
                               path_total);
  if (rc == APGAR_B200_OK) clear_error();
  return rc;
}

extern "C" int apgar_b200_lattice_device_results(void* plan,
                                                 const apgar_b200_lattice_result** results,
                                                 const uint32_t** paths) {
  if (plan == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan");
  auto* p = static_cast<PlanObject*>(plan);
  if (results != nullptr) *results = p->results.get();
  if (paths != nullptr) *paths = p->paths.get();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan_set_cell_costs(void* plan, const uint32_t* cell_costs) {
  if (plan == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan");
  auto* p = static_cast<PlanObject*>(plan);
  if (cell_costs != nullptr && p->generator != APGAR_B200_LATTICE_FRONTIER) {
    return set_error(APGAR_B200_UNSUPPORTED, "per-cell prices need the frontier generator");
  }
  p->cell_cost = cell_costs;
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan_set_corridors(void* plan, const uint32_t* corridor_bits) {
  if (plan == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan");
  auto* p = static_cast<PlanObject*>(plan);
  if (corridor_bits != nullptr) {
    if (p->generator != APGAR_B200_LATTICE_FRONTIER) {
      return set_error(APGAR_B200_UNSUPPORTED, "corridors need the frontier generator");
    }
    if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
    APGAR_B200_CUDA("cudaMalloc(corridor status)",
                    p->corridor_status.ensure(std::max<uint32_t>(p->count, 1)));
  }
  p->corridor = corridor_bits;
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan_corridor_status(void* plan, uint8_t* out) {
  if (plan == nullptr || out == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan or output");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (p->corridor_status.get() == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "the plan never had corridors");
  }
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  if (p->count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(corridor status)",
                    cudaMemcpy(out, p->corridor_status.get(), p->count, cudaMemcpyDeviceToHost));
  }
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_corridor_rasters(void* plan, const uint32_t* cell_costs, void* rasters,
                                           uint32_t* dims, void* stream) {
  if (plan == nullptr || rasters == nullptr || dims == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "corridor rasters received a null argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  APGAR_B200_CUDA("raster launch", launch_rasters(p->lattice->view, p->nets.get(), p->count, cell_costs,
                                                  rasters, dims, static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_corridor_labels(void* plan, const uint32_t* dims, uint8_t* labels,
                                          void* stream) {
  if (plan == nullptr || dims == nullptr || labels == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "corridor labels received a null argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  const LatticeDeviceView& v = p->lattice->view;
  APGAR_B200_CUDA("label launch", launch_labels(p->nets.get(), p->count, dims, v.width, v.height,
                                                p->results.get(), p->paths.get(), labels,
                                                static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_corridor_from_logits(void* plan, const float* logits, const uint32_t* dims,
                                               float threshold, int32_t dilate,
                                               uint64_t max_window_cells, uint32_t* bits,
                                               void* stream) {
  if (plan == nullptr || logits == nullptr || dims == nullptr || bits == nullptr || dilate < 0 ||
      dilate > 64) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "corridor extraction received a bad argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  APGAR_B200_CUDA("corridor launch",
                  launch_corridors(logits, dims, p->nets.get(), p->count, threshold, dilate,
                                   max_window_cells, p->lattice->view.layers, bits,
                                   static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_segments(void* plan, int64_t origin_x, int64_t origin_y, int64_t step,
                                           apgar_b200_segment* segments, uint32_t* segment_counts,
                                           void* stream) {
  if (plan == nullptr || segments == nullptr || segment_counts == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice segments received a null argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  const LatticeDeviceView& v = p->lattice->view;
  APGAR_B200_CUDA("lattice segments launch",
                  launch_lattice_segments(p->results.get(), p->paths.get(), p->count,
                                          static_cast<uint32_t>(v.width), static_cast<uint32_t>(v.height),
                                          origin_x, origin_y, step, segments, segment_counts,
                                          static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan_info(void* plan, apgar_b200_plan_info* out) {
  if (plan == nullptr || out == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "null plan or output");
  }
  auto* p = static_cast<PlanObject*>(plan);
  std::memset(out, 0, sizeof(*out));
  out->net_count = p->count;
  out->class_count = static_cast<uint32_t>(p->classes.size());
  // the frontier runs all its classes in one launch; the sweep one per class
  const uint32_t search_launches =
      p->generator == APGAR_B200_LATTICE_FRONTIER ? (out->class_count > 0 ? 1u : 0u) : out->class_count;
  out->kernel_launches = search_launches + (p->count > 0 ? 2u : 0u);
  out->workspace_bytes = p->workspace_bytes();
  out->label_cells = p->label_cells;
  out->path_arena_capacity = p->arena_capacity;
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_plan_release(void* plan) {
  delete static_cast<PlanObject*>(plan);
  return APGAR_B200_OK;
}

namespace apgar_b200 {
namespace {

int check_options(const apgar_b200_lattice_options& o) {
  if (o.generator == APGAR_B200_LATTICE_SWEEP) {
    if (o.max_iterations == 0 || o.max_iterations > 30000) {
      return set_error(APGAR_B200_INTERNAL_INVARIANT, "sweep budget must be 1..30000 sweeps");
    }
    return APGAR_B200_OK;
  }
  if (o.generator == APGAR_B200_LATTICE_FRONTIER) {
    if (o.max_iterations == 0 || o.max_iterations > (1u << 30)) {
      return set_error(APGAR_B200_INTERNAL_INVARIANT, "frontier budget must be 1..2^30 rounds");
    }
    if (o.chain > 16 || o.wide_chain > 16) {
      return set_error(APGAR_B200_INTERNAL_INVARIANT, "frontier chain must be 0..16");
    }
    if (o.class_bounds != 0 && !class_bounds_valid(o.class_bounds)) {
      return set_error(APGAR_B200_INTERNAL_INVARIANT,
                       "frontier class bounds must be strictly increasing log2 sizes in 1..31");
    }
    return APGAR_B200_OK;
  }
  return set_error(APGAR_B200_UNSUPPORTED, "unknown lattice generator");
}

int route_impl(void* lattice, const apgar_b200_lattice_net* nets, uint32_t count,
               const apgar_b200_lattice_options& o, const volatile uint32_t* cancel,
               apgar_b200_lattice_result* results, uint32_t* paths, uint64_t path_capacity,
               uint64_t* path_total) {
  if (lattice == nullptr || (count > 0 && nets == nullptr) || results == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice route received invalid arguments");
  }
  if (int rc = check_options(o); rc != APGAR_B200_OK) return rc;
  auto* lat = static_cast<LatticeObject*>(lattice);
  if (int rc = check_device(lat->device); rc != APGAR_B200_OK) return rc;
  try {
    std::scoped_lock lock(lat->route_mutex);
    if (lat->route_plan == nullptr) lat->route_plan = std::make_unique<PlanObject>();
    PlanObject* plan = lat->route_plan.get();
    if (int rc = build_plan(lat, nets, count, o.max_iterations, plan, o.generator, o.bucket_width,
                            o.chain, o.class_bounds, o.wide_bucket_width, o.wide_chain);
        rc != APGAR_B200_OK) {
      return rc;
    }
    *reinterpret_cast<volatile uint32_t*>(plan->cancel_host) = 0u;
    if (int rc = execute_plan(plan, nullptr); rc != APGAR_B200_OK) return rc;
    // The caller's flag is sampled on the host while the batch runs and is
    // forwarded through the plan's own mapped flag, which the kernels poll
    // (the kernels never dereference caller memory).
    for (;;) {
      const cudaError_t q = cudaStreamQuery(nullptr);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_failure("cudaStreamQuery(route)", q);
      if (cancel != nullptr && *cancel != 0u) {
        *reinterpret_cast<volatile uint32_t*>(plan->cancel_host) = 1u;
      }
      std::this_thread::yield();
    }
    const int rc = readback_plan(plan, results, paths, path_capacity, path_total);
    if (rc == APGAR_B200_OK) clear_error();
    return rc;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during routing");
  }
}

}  // namespace
}  // namespace apgar_b200

extern "C" int apgar_b200_lattice_route(void* lattice, const apgar_b200_lattice_net* nets,
                                        uint32_t count, uint32_t max_sweeps,
                                        const volatile uint32_t* cancel,
                                        apgar_b200_lattice_result* results, uint32_t* paths,
                                        uint64_t path_capacity, uint64_t* path_total) {
  const apgar_b200_lattice_options o{APGAR_B200_LATTICE_SWEEP, max_sweeps, 0, 0, 0, 0, 0};
  return route_impl(lattice, nets, count, o, cancel, results, paths, path_capacity, path_total);
}

extern "C" int apgar_b200_lattice_route_ex(void* lattice, const apgar_b200_lattice_net* nets,
                                           uint32_t count, const apgar_b200_lattice_options* options,
                                           const volatile uint32_t* cancel,
                                           apgar_b200_lattice_result* results, uint32_t* paths,
                                           uint64_t path_capacity, uint64_t* path_total) {
  if (options == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null lattice options");
  return route_impl(lattice, nets, count, *options, cancel, results, paths, path_capacity,
                    path_total);
}

extern "C" int apgar_b200_lattice_plan_ex(void* lattice, const apgar_b200_lattice_net* nets,
                                          uint32_t count, const apgar_b200_lattice_options* options,
                                          void** out_plan) {
  if (lattice == nullptr || out_plan == nullptr || options == nullptr ||
      (count > 0 && nets == nullptr)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice plan received invalid arguments");
  }
  if (int rc = check_options(*options); rc != APGAR_B200_OK) return rc;
  auto* lat = static_cast<LatticeObject*>(lattice);
  if (int rc = check_device(lat->device); rc != APGAR_B200_OK) return rc;
  try {
    auto plan = std::make_unique<PlanObject>();
    if (int rc = build_plan(lat, nets, count, options->max_iterations, plan.get(),
                            options->generator, options->bucket_width, options->chain,
                            options->class_bounds, options->wide_bucket_width,
                            options->wide_chain);
        rc != APGAR_B200_OK) {
      return rc;
    }
    *out_plan = plan.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed during planning");
  }
}

extern "C" int apgar_b200_lattice_validate(void* lattice, const apgar_b200_lattice_net* nets,
                                           uint32_t count, const apgar_b200_lattice_result* results,
                                           const uint32_t* paths, uint64_t path_count,
                                           apgar_b200_path_verdict* verdicts) {
  if (lattice == nullptr || (count > 0 && (nets == nullptr || results == nullptr || verdicts == nullptr)) ||
      (path_count > 0 && paths == nullptr)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "lattice validation received a null argument");
  }
  auto* lat = static_cast<LatticeObject*>(lattice);
  if (int rc = check_device(lat->device); rc != APGAR_B200_OK) return rc;
  if (count == 0) {
    clear_error();
    return APGAR_B200_OK;
  }
  std::scoped_lock lock(lat->validate_mutex);
  auto& d_nets = lat->val_nets;
  auto& d_res = lat->val_results;
  auto& d_paths = lat->val_paths;
  auto& d_out = lat->val_out;
  APGAR_B200_CUDA("cudaMalloc(nets)", d_nets.ensure(count));
  APGAR_B200_CUDA("cudaMalloc(results)", d_res.ensure(count));
  APGAR_B200_CUDA("cudaMalloc(paths)", d_paths.ensure(std::max<uint64_t>(path_count, 1)));
  APGAR_B200_CUDA("cudaMalloc(verdicts)", d_out.ensure(count));
  APGAR_B200_CUDA("cudaMemcpy(nets)", cudaMemcpy(d_nets.get(), nets, count * sizeof(*nets), cudaMemcpyHostToDevice));
  APGAR_B200_CUDA("cudaMemcpy(results)", cudaMemcpy(d_res.get(), results, count * sizeof(*results), cudaMemcpyHostToDevice));
  if (path_count > 0) {
    APGAR_B200_CUDA("cudaMemcpy(paths)", cudaMemcpy(d_paths.get(), paths, path_count * 4, cudaMemcpyHostToDevice));
  }
  APGAR_B200_CUDA("lattice validation launch",
                  launch_lattice_validate(lat->view, d_nets.get(), d_res.get(), d_paths.get(), path_count,
                                          count, d_out.get(), nullptr));
  APGAR_B200_CUDA("cudaMemcpy(verdicts)", cudaMemcpy(verdicts, d_out.get(), count * sizeof(*verdicts), cudaMemcpyDeviceToHost));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_lattice_accumulate_usage(void* plan, uint32_t* usage, uint64_t cell_count,
                                                   void* stream) {
  if (plan == nullptr || usage == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "usage accumulation received a null argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  APGAR_B200_CUDA("usage accumulation launch",
                  launch_accumulate_cells(p->results.get(), p->count, p->paths.get(), usage,
                                          cell_count, p->sm_count, static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free routing (apgar_b200_lattice_route_noalloc).
//
// Some callers must not allocate device memory while they route: a process
// whose device memory is already held by another allocator (a caching
// allocator, a fixed serving budget) gets out-of-memory from cudaMalloc, and a
// router that shares the GPU with work on other streams cannot take the
// device-wide synchronisation that cudaMalloc and cudaFree imply.  This entry
// point serves them from one file-scope device array per device and per
// process, carved into the same buffers a plan owns, and stages its host-side
// plan in fixed file-scope host arrays.  It creates no stream, event or pinned
// buffer; every copy and launch goes to the caller's stream.
//
// The scratch is shared by every call on a device, and the host staging
// arrays by every call of the process.  One process-wide mutex is held from
// the admission pass to the final stream synchronisation, so calls from
// several host threads (on one device or on several) run one after another.
// Without it, overlapping calls would race: one call's plan records could be
// uploaded beside another call's nets, and the sweep would then index label
// slabs laid out for the other batch, which can write out of bounds and fault
// the GPU rather than only corrupt results.  Work that another process or
// a caller's own kernels put on the same scratch cannot exist: the array is
// private to this library and this process.

static __device__ __align__(256) unsigned char g_noalloc_scratch[APGAR_B200_NOALLOC_SCRATCH_BYTES];

namespace apgar_b200 {
namespace {

constexpr uint64_t kNoallocAlign = 256;

// Serialises allocation-free calls (host staging, uploads, launches and the
// final synchronisation).  A std::mutex allocates nothing.
std::mutex g_noalloc_mutex;

struct NoallocStaging {
  NetPlan plans[APGAR_B200_NOALLOC_MAX_NETS];
  apgar_b200_lattice_result init[APGAR_B200_NOALLOC_MAX_NETS];
  uint32_t order[APGAR_B200_NOALLOC_MAX_NETS];
  int8_t width_class[APGAR_B200_NOALLOC_MAX_NETS];
};
NoallocStaging g_noalloc_host;

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a host-side stand-in, so every call looks the
// address up again (with the lattice's device current, which the entry point
// has checked): the lookup allocates nothing, and a module reloaded after a
// device reset may sit at another address.
int noalloc_scratch(unsigned char** out) {
  void* ptr = nullptr;
  APGAR_B200_CUDA("cudaGetSymbolAddress(allocation-free scratch)",
                  cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
  *out = static_cast<unsigned char*>(ptr);
  return APGAR_B200_OK;
}

uint64_t noalloc_take(uint64_t* cursor, uint64_t bytes) {
  const uint64_t at = *cursor;
  *cursor = (at + bytes + kNoallocAlign - 1) & ~(kNoallocAlign - 1);
  return at;
}

int route_noalloc(LatticeObject* lat, const apgar_b200_lattice_net* host_nets, uint32_t count,
                  uint32_t max_sweeps, cudaStream_t stream, apgar_b200_lattice_result* results,
                  uint32_t* paths, uint64_t path_capacity, uint64_t* path_total) {
  if (count > APGAR_B200_NOALLOC_MAX_NETS) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED,
                     "allocation-free route takes at most " +
                         std::to_string(APGAR_B200_NOALLOC_MAX_NETS) +
                         " nets per call; split the batch or use apgar_b200_lattice_route");
  }
  const LatticeDeviceView& v = lat->view;
  const uint64_t max_move = std::max(v.orth, std::max(v.diag, v.via));
  NoallocStaging& h = g_noalloc_host;

  // Admission and width classes: the same rules as a plan.
  for (uint32_t i = 0; i < count; ++i) {
    const apgar_b200_lattice_net& n = host_nets[i];
    apgar_b200_lattice_result& r = h.init[i];
    std::memset(&r, 0, sizeof(r));
    r.cost = APGAR_B200_UNREACHABLE;
    r.completion = APGAR_B200_COMPLETION_REJECTED;
    h.width_class[i] = -1;
    const bool in_lattice =
        n.start_layer < static_cast<uint32_t>(v.layers) &&
        n.goal_layer < static_cast<uint32_t>(v.layers) && n.win_w > 0 && n.win_h > 0 &&
        static_cast<uint64_t>(n.win_x0) + n.win_w <= static_cast<uint64_t>(v.width) &&
        static_cast<uint64_t>(n.win_y0) + n.win_h <= static_cast<uint64_t>(v.height) &&
        n.start_x >= n.win_x0 && n.start_x < n.win_x0 + n.win_w && n.start_y >= n.win_y0 &&
        n.start_y < n.win_y0 + n.win_h && n.goal_x >= n.win_x0 && n.goal_x < n.win_x0 + n.win_w &&
        n.goal_y >= n.win_y0 && n.goal_y < n.win_y0 + n.win_h;
    if (!in_lattice) continue;
    const uint64_t cells = static_cast<uint64_t>(v.layers) * n.win_w * n.win_h;
    if (cells * max_move >= kLabelInf) continue;
    const uint32_t frame_width = std::max(n.win_w, n.win_h);
    const uint32_t frame_rows = std::min(n.win_w, n.win_h);
    const int ci = class_for_width(frame_width, v.layers);
    if (ci < 0 || frame_rows > 32000u) continue;
    h.width_class[i] = static_cast<int8_t>(ci);
  }

  // Plan records, class by class, larger windows first (ties by net index).
  ClassRange ranges[kClassCount];
  int range_count = 0;
  uint32_t planned = 0;
  uint64_t dist_cells = 0, arena_cells = 0;
  for (int ci = 0; ci < kClassCount; ++ci) {
    uint32_t members = 0;
    for (uint32_t i = 0; i < count; ++i) {
      if (h.width_class[i] == ci) h.order[members++] = i;
    }
    if (members == 0) continue;
    std::sort(h.order, h.order + members, [&](uint32_t a, uint32_t b) {
      const uint64_t ca = static_cast<uint64_t>(host_nets[a].win_w) * host_nets[a].win_h;
      const uint64_t cb = static_cast<uint64_t>(host_nets[b].win_w) * host_nets[b].win_h;
      return ca != cb ? ca > cb : a < b;
    });
    ClassRange& range = ranges[range_count++];
    range = ClassRange{};
    range.warps_per_net = kGroupSizes[ci];
    range.begin = planned;
    range.count = members;
    for (uint32_t k = 0; k < members; ++k) {
      const uint32_t i = h.order[k];
      const apgar_b200_lattice_net& n = host_nets[i];
      NetPlan& np = h.plans[planned++];
      np = NetPlan{};
      np.net = i;
      np.transposed = n.win_h > n.win_w ? 1u : 0u;
      np.rows = np.transposed ? n.win_w : n.win_h;
      np.width = np.transposed ? n.win_h : n.win_w;
      np.pitch = (np.width + 3u) & ~3u;
      np.dist_offset = dist_cells;
      dist_cells += static_cast<uint64_t>(v.layers) * np.rows * np.pitch;
      arena_cells += 8ull * (n.win_w + n.win_h) + 64ull * v.layers;
      range.max_rows = std::max(range.max_rows, static_cast<int>(np.rows));
    }
    if (lattice_sweep_smem_bytes(v.layers, range.warps_per_net, range.max_rows) >
        kMaxSmemPerBlock) {
      return set_error(APGAR_B200_UNSUPPORTED, "window too tall for the shared-memory row map");
    }
  }
  const uint64_t arena_capacity = std::max<uint64_t>(arena_cells, 64);

  // Carve the scratch: the same buffers, in the same roles, as a plan's.
  uint64_t cursor = 0;
  const uint64_t nets_at = noalloc_take(&cursor, count * sizeof(apgar_b200_lattice_net));
  const uint64_t plans_at = noalloc_take(&cursor, planned * sizeof(NetPlan));
  const uint64_t results_at = noalloc_take(&cursor, count * sizeof(apgar_b200_lattice_result));
  const uint64_t counters_at = noalloc_take(&cursor, 2 * sizeof(unsigned long long));
  const uint64_t labels_at = noalloc_take(&cursor, dist_cells * sizeof(uint32_t));
  const uint64_t arena_at = noalloc_take(&cursor, arena_capacity * sizeof(uint32_t));
  const uint64_t paths_at = noalloc_take(&cursor, arena_capacity * sizeof(uint32_t));
  if (cursor > APGAR_B200_NOALLOC_SCRATCH_BYTES) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED,
                     "allocation-free route needs " + std::to_string(cursor) +
                         " bytes of scratch for this batch; the fixed scratch holds " +
                         std::to_string(static_cast<uint64_t>(APGAR_B200_NOALLOC_SCRATCH_BYTES)) +
                         " bytes; split the batch or use apgar_b200_lattice_route");
  }
  unsigned char* base = nullptr;
  if (int rc = noalloc_scratch(&base); rc != APGAR_B200_OK) return rc;
  auto* d_nets = reinterpret_cast<apgar_b200_lattice_net*>(base + nets_at);
  auto* d_plans = reinterpret_cast<NetPlan*>(base + plans_at);
  auto* d_results = reinterpret_cast<apgar_b200_lattice_result*>(base + results_at);
  auto* d_counters = reinterpret_cast<unsigned long long*>(base + counters_at);
  auto* d_labels = reinterpret_cast<uint32_t*>(base + labels_at);
  auto* d_arena = reinterpret_cast<uint32_t*>(base + arena_at);
  auto* d_paths = reinterpret_cast<uint32_t*>(base + paths_at);

  int sm_count = 0;
  APGAR_B200_CUDA("cudaDeviceGetAttribute",
                  cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, lat->device));
  // The pageable source copies return once the bytes are staged, so the host
  // staging arrays may be reused by the next call.
  if (count > 0) {
    APGAR_B200_CUDA("cudaMemcpyAsync(nets)",
                    cudaMemcpyAsync(d_nets, host_nets, count * sizeof(apgar_b200_lattice_net),
                                    cudaMemcpyHostToDevice, stream));
    APGAR_B200_CUDA("cudaMemcpyAsync(results init)",
                    cudaMemcpyAsync(d_results, h.init, count * sizeof(apgar_b200_lattice_result),
                                    cudaMemcpyHostToDevice, stream));
  }
  if (planned > 0) {
    APGAR_B200_CUDA("cudaMemcpyAsync(plans)",
                    cudaMemcpyAsync(d_plans, h.plans, planned * sizeof(NetPlan),
                                    cudaMemcpyHostToDevice, stream));
  }
  // Arena cursor and packed total start at zero; label slabs are written by
  // the kernels before they are read.
  APGAR_B200_CUDA("cudaMemsetAsync(counters)",
                  cudaMemsetAsync(d_counters, 0, 2 * sizeof(unsigned long long), stream));
  SweepLaunch launch{};
  launch.lat = v;
  launch.nets = d_nets;
  launch.max_sweeps = max_sweeps;
  launch.dist_pool = d_labels;
  launch.results = d_results;
  launch.path_arena = d_arena;
  launch.path_arena_capacity = arena_capacity;
  launch.arena_cursor = d_counters;
  launch.cancel = nullptr;
  for (int k = 0; k < range_count; ++k) {
    launch.plans = d_plans + ranges[k].begin;
    launch.plan_count = ranges[k].count;
    APGAR_B200_CUDA("lattice sweep launch",
                    launch_lattice_sweep(v.layers, ranges[k].warps_per_net, launch,
                                         ranges[k].max_rows, stream));
  }
  APGAR_B200_CUDA("lattice pack launch",
                  launch_lattice_pack(d_results, count, d_counters + 1, d_arena, d_paths, sm_count,
                                      stream));

  // Device-to-pageable copies return when the bytes have arrived.
  unsigned long long total = 0;
  APGAR_B200_CUDA("cudaMemcpyAsync(path total)",
                  cudaMemcpyAsync(&total, d_counters + 1, sizeof(total), cudaMemcpyDeviceToHost,
                                  stream));
  if (count > 0) {
    APGAR_B200_CUDA("cudaMemcpyAsync(results)",
                    cudaMemcpyAsync(results, d_results, count * sizeof(apgar_b200_lattice_result),
                                    cudaMemcpyDeviceToHost, stream));
  }
  if (path_total != nullptr) *path_total = total;
  if (paths != nullptr && total > 0) {
    if (total > path_capacity) {
      // A pinned results buffer makes the copy above asynchronous: finish it
      // before returning, so the stream is synchronised on every return.
      APGAR_B200_CUDA("cudaStreamSynchronize(route)", cudaStreamSynchronize(stream));
      return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "path output buffer is too small");
    }
    APGAR_B200_CUDA("cudaMemcpyAsync(paths)",
                    cudaMemcpyAsync(paths, d_paths, total * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, stream));
  }
  APGAR_B200_CUDA("cudaStreamSynchronize(route)", cudaStreamSynchronize(stream));
  return APGAR_B200_OK;
}

}  // namespace
}  // namespace apgar_b200

extern "C" int apgar_b200_lattice_route_noalloc(void* lattice, const apgar_b200_lattice_net* nets,
                                                uint32_t count, uint32_t max_sweeps, void* stream,
                                                apgar_b200_lattice_result* results,
                                                uint32_t* paths, uint64_t path_capacity,
                                                uint64_t* path_total) {
  if (lattice == nullptr || (count > 0 && (nets == nullptr || results == nullptr)) ||
      max_sweeps == 0 || max_sweeps > 30000) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT,
                     "allocation-free lattice route received invalid arguments");
  }
  auto* lat = static_cast<LatticeObject*>(lattice);
  if (int rc = check_device(lat->device); rc != APGAR_B200_OK) return rc;
  std::lock_guard<std::mutex> hold(g_noalloc_mutex);
  const int rc = route_noalloc(lat, nets, count, max_sweeps, static_cast<cudaStream_t>(stream),
                               results, paths, path_capacity, path_total);
  if (rc == APGAR_B200_OK) clear_error();
  return rc;
}

// ---------------------------------------------------------------------------
// Negotiated-congestion rounds on a FRONTIER plan.
//
// Round p (Jacobi rip-up and reroute: every net is rerouted against the same
// frozen snapshot):
//   1. search every net of the plan with per-cell entry prices `cell_cost`;
//      from the second round on, a cell of the net's own previous route is
//      priced from the usage of the other nets only (`cell_cost_own`), as
//      the reference rips a net's incumbent route up before pricing its
//      query (cpu_sequential_negotiated_routing.cc:1023-1034);
//   2. usage = number of reached paths through each cell (integer atomics, so
//      order independent);
//   3. one fused price pass at epoch p (src/allocator/negotiated_regeneration_plan.cc
//      :430-442 factor schedule; cpu_sequential_negotiated_routing.cc:1300-1330
//      history update): history += increment * overuse, and the next snapshot
//      cell_cost = history + factor(p + 1) * max(0, usage + 1 - capacity)
//      (cpu_sequential_negotiated_routing.cc:299-505), saturated to 2^31 - 1,
//      and cell_cost_own = the same with usage - 1 in place of usage; the
//      same pass counts overused cells and total overuse for the round.
// The reference's sequential negotiated router reroutes nets one at a time
// (Gauss-Seidel); batched rounds are Jacobi by design, so only each round's
// per-net results under its frozen snapshot are comparable with a CPU run.
// A run starts from zero history and zero prices, so it can be captured once
// as a CUDA graph of all its rounds and replayed.
namespace apgar_b200 {
namespace {

struct NegotiationObject {
  PlanObject* plan = nullptr;
  apgar_b200_price_policy policy{};
  uint64_t cells = 0;
  DeviceBuffer<uint32_t> usage, cell_cost, status;
  uint32_t* usage_ext = nullptr;  // caller's usage buffer (multi-rank steps), or null
  DeviceBuffer<uint32_t> cell_cost_own;  // the snapshot seen from a net's own previous cells
  DeviceBuffer<uint32_t> own_bits;       // one bit per label word of the plan
  DeviceBuffer<uint64_t> history;
  DeviceBuffer<unsigned long long> stats;  // [round][overused cells, total overuse]
  uint32_t rounds_capacity = 0;
  // partial rip-up: previous round's routes and the per-net keep flags
  DeviceBuffer<apgar_b200_lattice_result> prev_results;
  DeviceBuffer<uint32_t> prev_paths;
  DeviceBuffer<uint8_t> skip;
  uint32_t graph_flags = 0;
  cudaStream_t work = nullptr;
  cudaEvent_t entry = nullptr, exit = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_rounds = 0;
  // split-round steps: the next (round, phase) a step may run
  uint32_t step_round = 0, step_phase = 0;

  uint32_t* usage_ptr() { return usage_ext != nullptr ? usage_ext : usage.get(); }

  ~NegotiationObject() {
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    if (entry != nullptr) cudaEventDestroy(entry);
    if (exit != nullptr) cudaEventDestroy(exit);
    if (work != nullptr) cudaStreamDestroy(work);
    if (plan != nullptr) {
      plan->cell_cost = nullptr;
      plan->skip = nullptr;
      plan->prev_results = nullptr;
      plan->prev_paths = nullptr;
      plan->cell_cost_own = nullptr;
      plan->own_bits = nullptr;
    }
  }
};

bool checked_factor(const apgar_b200_price_policy& p, uint64_t epoch, uint64_t* out) {
  const unsigned __int128 f =
      static_cast<unsigned __int128>(epoch) * p.present_factor_increment + p.initial_present_factor;
  if (f > static_cast<unsigned __int128>(~0ull)) return false;
  *out = static_cast<uint64_t>(f);
  return true;
}

// Zero history and zero snapshot prices: the state before round 0.
int enqueue_reset(NegotiationObject* n, cudaStream_t s) {
  APGAR_B200_CUDA("cudaMemsetAsync(history)",
                  cudaMemsetAsync(n->history.get(), 0, n->cells * sizeof(uint64_t), s));
  APGAR_B200_CUDA("cudaMemsetAsync(cell costs)",
                  cudaMemsetAsync(n->cell_cost.get(), 0, n->cells * sizeof(uint32_t), s));
  n->plan->cell_cost = n->cell_cost.get();
  return APGAR_B200_OK;
}

// Steps 1-2 of round r: reroute the plan's nets against the current
// snapshot, then count their per-cell usage.  With `partial`, round r >= 1
// reroutes only the nets whose previous route did not reach its goal or
// crosses a cell overused after round r - 1 (the usage buffer still holds
// round r - 1's usage); the others keep their routes.
int enqueue_route(NegotiationObject* n, uint32_t r, bool partial, cudaStream_t s) {
  PlanObject* plan = n->plan;
  if (r > 0) {
    // the plan still holds round r - 1's routes: they drive rip-up pricing
    APGAR_B200_CUDA("cudaMemcpyAsync(previous results)",
                    cudaMemcpyAsync(n->prev_results.get(), plan->results.get(),
                                    plan->count * sizeof(apgar_b200_lattice_result),
                                    cudaMemcpyDeviceToDevice, s));
    APGAR_B200_CUDA("cudaMemcpyAsync(previous paths)",
                    cudaMemcpyAsync(n->prev_paths.get(), plan->paths.get(),
                                    plan->arena_capacity * sizeof(uint32_t),
                                    cudaMemcpyDeviceToDevice, s));
  }
  plan->cell_cost = n->cell_cost.get();
  plan->prev_results = r > 0 ? n->prev_results.get() : nullptr;
  plan->prev_paths = r > 0 ? n->prev_paths.get() : nullptr;
  plan->cell_cost_own = r > 0 ? n->cell_cost_own.get() : nullptr;
  plan->own_bits = r > 0 ? n->own_bits.get() : nullptr;
  if (partial && r > 0) {
    APGAR_B200_CUDA("mark dirty launch",
                    launch_mark_dirty(n->prev_results.get(), plan->count, n->prev_paths.get(),
                                      n->usage_ptr(), n->cells,
                                      static_cast<uint32_t>(n->policy.capacity), n->skip.get(),
                                      plan->sm_count, s));
    plan->skip = n->skip.get();
  } else {
    plan->skip = nullptr;
  }
  const int exec_rc = execute_plan(plan, s);
  plan->skip = nullptr;
  plan->prev_results = nullptr;
  plan->prev_paths = nullptr;
  plan->cell_cost_own = nullptr;
  plan->own_bits = nullptr;
  if (exec_rc != APGAR_B200_OK) return exec_rc;
  APGAR_B200_CUDA("cudaMemsetAsync(usage)",
                  cudaMemsetAsync(n->usage_ptr(), 0, n->cells * sizeof(uint32_t), s));
  APGAR_B200_CUDA("usage accumulation launch",
                  launch_accumulate_cells(plan->results.get(), plan->count, plan->paths.get(),
                                          n->usage_ptr(), n->cells, plan->sm_count, s));
  return APGAR_B200_OK;
}

// Step 3 of round r: the fused price pass over the usage buffer.
int enqueue_price(NegotiationObject* n, uint32_t r, cudaStream_t s) {
  uint64_t factor = 0, next_factor = 0;
  if (!checked_factor(n->policy, r, &factor) || !checked_factor(n->policy, r + 1ull, &next_factor)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "present-price schedule overflowed uint64");
  }
  APGAR_B200_CUDA("price update launch",
                  launch_price_update(static_cast<uint32_t>(n->cells), n->usage_ptr(), factor,
                                      next_factor, n->policy.historical_price_increment,
                                      n->policy.capacity, n->policy.maximum_value, nullptr,
                                      n->history.get(), nullptr, nullptr, n->cell_cost.get(),
                                      n->cell_cost_own.get(), n->status.get() + r,
                                      n->stats.get() + 2ull * r, s));
  return APGAR_B200_OK;
}

// Enqueues a whole negotiation (reset + `rounds` rounds) on n->work.
int enqueue_negotiation(NegotiationObject* n, uint32_t rounds, bool partial) {
  cudaStream_t s = n->work;
  if (int rc = enqueue_reset(n, s); rc != APGAR_B200_OK) return rc;
  for (uint32_t r = 0; r < rounds; ++r) {
    if (int rc = enqueue_route(n, r, partial, s); rc != APGAR_B200_OK) return rc;
    if (int rc = enqueue_price(n, r, s); rc != APGAR_B200_OK) return rc;
  }
  return APGAR_B200_OK;
}

}  // namespace
}  // namespace apgar_b200

extern "C" int apgar_b200_negotiation_create(void* plan, const apgar_b200_price_policy* policy,
                                             void** out) {
  if (plan == nullptr || policy == nullptr || out == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation received a null argument");
  }
  auto* p = static_cast<PlanObject*>(plan);
  if (p->generator != APGAR_B200_LATTICE_FRONTIER) {
    return set_error(APGAR_B200_UNSUPPORTED, "negotiated rounds need a FRONTIER plan");
  }
  if (int rc = check_device(p->device); rc != APGAR_B200_OK) return rc;
  const LatticeDeviceView& v = p->lattice->view;
  const uint64_t cells = static_cast<uint64_t>(v.layers) * v.height * v.width;
  if (cells > 0xFFFFFFFFull) {
    return set_error(APGAR_B200_UNSUPPORTED, "lattice has more cells than a price pass indexes");
  }
  try {
    auto n = std::make_unique<NegotiationObject>();
    n->plan = p;
    n->policy = *policy;
    n->cells = cells;
    APGAR_B200_CUDA("cudaMalloc(usage)", n->usage.ensure(cells));
    APGAR_B200_CUDA("cudaMalloc(cell costs)", n->cell_cost.ensure(cells));
    APGAR_B200_CUDA("cudaMalloc(own-route cell costs)", n->cell_cost_own.ensure(cells));
    APGAR_B200_CUDA("cudaMalloc(own-route bits)", n->own_bits.ensure(p->words.count() / 32 + 1));
    APGAR_B200_CUDA("cudaMalloc(history)", n->history.ensure(cells));
    APGAR_B200_CUDA("cudaMalloc(previous results)", n->prev_results.ensure(std::max<uint32_t>(p->count, 1)));
    APGAR_B200_CUDA("cudaMalloc(previous paths)", n->prev_paths.ensure(std::max<uint64_t>(p->arena_capacity, 1)));
    APGAR_B200_CUDA("cudaMalloc(keep flags)", n->skip.ensure(std::max<uint32_t>(p->count, 1)));
    APGAR_B200_CUDA("cudaStreamCreate", cudaStreamCreateWithFlags(&n->work, cudaStreamNonBlocking));
    APGAR_B200_CUDA("cudaEventCreate", cudaEventCreateWithFlags(&n->entry, cudaEventDisableTiming));
    APGAR_B200_CUDA("cudaEventCreate", cudaEventCreateWithFlags(&n->exit, cudaEventDisableTiming));
    *out = n.release();
    clear_error();
    return APGAR_B200_OK;
  } catch (const std::bad_alloc&) {
    return set_error(APGAR_B200_RESOURCE_EXHAUSTED, "host allocation failed creating a negotiation");
  }
}

extern "C" int apgar_b200_negotiation_run_ex(void* negotiation, uint32_t rounds, uint32_t flags,
                                             void* stream) {
  if (negotiation == nullptr || rounds == 0 || rounds > 1000 ||
      (flags & ~(APGAR_B200_NEGOTIATE_GRAPH | APGAR_B200_NEGOTIATE_PARTIAL)) != 0u) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation needs 1..1000 rounds and known flags");
  }
  const bool use_graph = (flags & APGAR_B200_NEGOTIATE_GRAPH) != 0u;
  const bool partial = (flags & APGAR_B200_NEGOTIATE_PARTIAL) != 0u;
  auto* n = static_cast<NegotiationObject*>(negotiation);
  if (int rc = check_device(n->plan->device); rc != APGAR_B200_OK) return rc;
  const auto caller = static_cast<cudaStream_t>(stream);
  if (rounds > n->rounds_capacity) {
    APGAR_B200_CUDA("cudaMalloc(round status)", n->status.ensure(rounds));
    APGAR_B200_CUDA("cudaMalloc(round stats)", n->stats.ensure(2ull * rounds));
    n->rounds_capacity = rounds;
  }
  // work runs on the negotiation's own stream, ordered after the caller's
  APGAR_B200_CUDA("cudaEventRecord(entry)", cudaEventRecord(n->entry, caller));
  APGAR_B200_CUDA("cudaStreamWaitEvent", cudaStreamWaitEvent(n->work, n->entry, 0));
  if (!use_graph) {
    if (int rc = enqueue_negotiation(n, rounds, partial); rc != APGAR_B200_OK) return rc;
  } else {
    if (n->exec == nullptr || n->graph_rounds != rounds || n->graph_flags != flags) {
      if (n->exec != nullptr) cudaGraphExecDestroy(n->exec);
      if (n->graph != nullptr) cudaGraphDestroy(n->graph);
      n->exec = nullptr;
      n->graph = nullptr;
      APGAR_B200_CUDA("cudaStreamBeginCapture",
                      cudaStreamBeginCapture(n->work, cudaStreamCaptureModeRelaxed));
      const int rc = enqueue_negotiation(n, rounds, partial);
      cudaGraph_t graph = nullptr;
      const cudaError_t end = cudaStreamEndCapture(n->work, &graph);
      if (rc != APGAR_B200_OK) {
        if (graph != nullptr) cudaGraphDestroy(graph);
        return rc;
      }
      APGAR_B200_CUDA("cudaStreamEndCapture", end);
      n->graph = graph;
      APGAR_B200_CUDA("cudaGraphInstantiate", cudaGraphInstantiate(&n->exec, graph, 0));
      n->graph_rounds = rounds;
      n->graph_flags = flags;
    }
    APGAR_B200_CUDA("cudaGraphLaunch", cudaGraphLaunch(n->exec, n->work));
  }
  APGAR_B200_CUDA("cudaEventRecord(exit)", cudaEventRecord(n->exit, n->work));
  APGAR_B200_CUDA("cudaStreamWaitEvent", cudaStreamWaitEvent(caller, n->exit, 0));
  clear_error();
  return APGAR_B200_OK;
}

// Split-round steps cover up to this many rounds (the per-round stats are
// sized once, at round 0).
constexpr uint32_t kMaxStepRounds = 1000;

extern "C" int apgar_b200_negotiation_set_usage_buffer(void* negotiation, uint32_t* usage_device) {
  if (negotiation == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null negotiation");
  auto* n = static_cast<NegotiationObject*>(negotiation);
  if (int rc = check_device(n->plan->device); rc != APGAR_B200_OK) return rc;
  if (usage_device != nullptr) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, usage_device) != cudaSuccess ||
        attr.type != cudaMemoryTypeDevice || attr.device != n->plan->device) {
      cudaGetLastError();
      return set_error(APGAR_B200_INTERNAL_INVARIANT, "usage buffer is not device memory of the plan's device");
    }
  }
  APGAR_B200_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(n->work));
  n->usage_ext = usage_device;
  if (n->exec != nullptr) {  // a captured run baked in the old buffer
    cudaGraphExecDestroy(n->exec);
    cudaGraphDestroy(n->graph);
    n->exec = nullptr;
    n->graph = nullptr;
  }
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_negotiation_step(void* negotiation, uint32_t round, uint32_t phase,
                                           uint32_t flags, void* stream) {
  if (negotiation == nullptr || phase > APGAR_B200_NEGOTIATE_PRICE ||
      (flags & ~APGAR_B200_NEGOTIATE_PARTIAL) != 0u) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation step needs a known phase and flags");
  }
  auto* n = static_cast<NegotiationObject*>(negotiation);
  if (int rc = check_device(n->plan->device); rc != APGAR_B200_OK) return rc;
  if (round >= kMaxStepRounds) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation steps cover rounds 0..999");
  }
  // round 0's route phase starts a new negotiation; otherwise phases alternate
  const bool restart = round == 0 && phase == APGAR_B200_NEGOTIATE_ROUTE;
  if (!restart && (round != n->step_round || phase != n->step_phase)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation steps must alternate route and price in round order");
  }
  if (restart && n->rounds_capacity < kMaxStepRounds) {
    APGAR_B200_CUDA("cudaMalloc(round status)", n->status.ensure(kMaxStepRounds));
    APGAR_B200_CUDA("cudaMalloc(round stats)", n->stats.ensure(2ull * kMaxStepRounds));
    n->rounds_capacity = kMaxStepRounds;
  }
  const auto caller = static_cast<cudaStream_t>(stream);
  APGAR_B200_CUDA("cudaEventRecord(entry)", cudaEventRecord(n->entry, caller));
  APGAR_B200_CUDA("cudaStreamWaitEvent", cudaStreamWaitEvent(n->work, n->entry, 0));
  int rc = APGAR_B200_OK;
  if (phase == APGAR_B200_NEGOTIATE_ROUTE) {
    if (restart) rc = enqueue_reset(n, n->work);
    if (rc == APGAR_B200_OK) {
      rc = enqueue_route(n, round, (flags & APGAR_B200_NEGOTIATE_PARTIAL) != 0u, n->work);
    }
  } else {
    rc = enqueue_price(n, round, n->work);
  }
  // the exit event is recorded even after a failed enqueue, so the caller's
  // stream never runs ahead of work that was queued
  const cudaError_t rec = cudaEventRecord(n->exit, n->work);
  const cudaError_t wait = rec == cudaSuccess ? cudaStreamWaitEvent(caller, n->exit, 0) : rec;
  if (rc != APGAR_B200_OK) return rc;
  APGAR_B200_CUDA("cudaEventRecord(exit)", wait);
  n->step_round = phase == APGAR_B200_NEGOTIATE_ROUTE ? round : round + 1;
  n->step_phase = phase == APGAR_B200_NEGOTIATE_ROUTE ? APGAR_B200_NEGOTIATE_PRICE : APGAR_B200_NEGOTIATE_ROUTE;
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_negotiation_run(void* negotiation, uint32_t rounds, uint32_t use_graph,
                                          void* stream) {
  return apgar_b200_negotiation_run_ex(negotiation, rounds,
                                       use_graph != 0u ? APGAR_B200_NEGOTIATE_GRAPH : 0u, stream);
}

extern "C" int apgar_b200_negotiation_readback(void* negotiation, uint32_t* usage, uint64_t* history,
                                               uint32_t* cell_costs,
                                               apgar_b200_negotiation_round* rounds,
                                               uint32_t round_count) {
  if (negotiation == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null negotiation");
  auto* n = static_cast<NegotiationObject*>(negotiation);
  if (int rc = check_device(n->plan->device); rc != APGAR_B200_OK) return rc;
  if (round_count > n->rounds_capacity) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "more rounds requested than were run");
  }
  APGAR_B200_CUDA("cudaStreamSynchronize", cudaStreamSynchronize(n->work));
  if (usage) APGAR_B200_CUDA("cudaMemcpy(usage)", cudaMemcpy(usage, n->usage_ptr(), n->cells * 4, cudaMemcpyDeviceToHost));
  if (history) APGAR_B200_CUDA("cudaMemcpy(history)", cudaMemcpy(history, n->history.get(), n->cells * 8, cudaMemcpyDeviceToHost));
  if (cell_costs) APGAR_B200_CUDA("cudaMemcpy(cell costs)", cudaMemcpy(cell_costs, n->cell_cost.get(), n->cells * 4, cudaMemcpyDeviceToHost));
  if (rounds != nullptr && round_count > 0) {
    std::vector<unsigned long long> st(2ull * round_count);
    std::vector<uint32_t> fl(round_count);
    APGAR_B200_CUDA("cudaMemcpy(round stats)", cudaMemcpy(st.data(), n->stats.get(), st.size() * 8, cudaMemcpyDeviceToHost));
    APGAR_B200_CUDA("cudaMemcpy(round status)", cudaMemcpy(fl.data(), n->status.get(), fl.size() * 4, cudaMemcpyDeviceToHost));
    for (uint32_t r = 0; r < round_count; ++r) {
      rounds[r].overused_cells = st[2ull * r];
      rounds[r].total_overuse = st[2ull * r + 1];
      rounds[r].price_status = fl[r];
      rounds[r].reserved = 0;
    }
  }
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_negotiation_device_prices(void* negotiation, const uint32_t** cell_costs) {
  if (negotiation == nullptr || cell_costs == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "negotiation prices received a null argument");
  }
  *cell_costs = static_cast<NegotiationObject*>(negotiation)->cell_cost.get();
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_negotiation_release(void* negotiation) {
  delete static_cast<NegotiationObject*>(negotiation);
  return APGAR_B200_OK;
}
