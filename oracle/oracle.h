/*
 * CPU oracle for the apgar_b200 search path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load this library; the product (apgar_b200/) never links or calls it.
 *
 * Two restatements live here:
 *
 *  1. Lattice mode (dense bit-packed layers with vias, per-net windows, uint32
 *     costs, bend 0).  lo_dijkstra gives exact labels and the canonical path
 *     under the reference tie-break (smallest optimal incoming heading, see
 *     gpu/cuda/planar_router.cu:486-524 and :1084-1165 in the reference);
 *     lo_astar restates RouteWithCpuAStar (src/routing/cpu_astar.cc:323-638)
 *     with its pop key (f, h, g, y, x, heading, sequence) extended by a layer
 *     coordinate and the via move; lo_sweep_schedule restates the GPU row-sweep
 *     pass schedule to count sweeps and row visits for the roofline figure.
 *
 *  2. Graph mode (DeviceCompiledBoardV1 node arrays, heading states, uint64
 *     checked costs, bends, per-query surcharges and per-edge penalty/ban
 *     policies).  go_search computes exact heading-state labels by Dijkstra
 *     and the canonical compact path (reverse state list) exactly as the
 *     reference's batched sweep defines it (planar_router.cu:977-1009 goal
 *     selection, :1084-1165 reverse walk, :557-583 transition cost).
 *
 * Parity pinning: graph mode is checked against golden fixtures produced by
 * the reference's own CPU A* and corpus builders (tests/golden/, generated by
 * oracle/ref_fixtures.cc compiled from the reference sources).  Lattice mode
 * is pinned through graph mode: on single-layer lattices expressed as node
 * records with the lattice move rule, lo_dijkstra and go_search give the same
 * costs and the same canonical reverse paths; vias, which the reference's
 * planar search does not model, are covered by the agreement of the three
 * lattice restatements.
 */
#ifndef APGAR_B200_ORACLE_H_
#define APGAR_B200_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LO_INF 0xFFFFFFFFu

typedef struct lo_lattice {
  int32_t layers, height, width; /* width is a multiple of 32 */
  const uint32_t* blocked;       /* [layers][height][width/32], bit x%32 of word x/32 */
  const uint32_t* via_ok;        /* [layers-1][height][width/32]; NULL = no via restriction */
  uint32_t orth, diag, via;      /* move costs */
  /* Optional per-cell entry cost [layers][height][width] (NULL = none): a
   * move into cell c costs its move cost plus cell_cost[c].  Only lo_dijkstra
   * (and its batch form) reads it; it models a negotiated-congestion price
   * snapshot. */
  const uint32_t* cell_cost;
} lo_lattice;

typedef struct lo_net {
  uint32_t start_layer, start_x, start_y;
  uint32_t goal_layer, goal_x, goal_y;
  uint32_t win_x0, win_y0, win_w, win_h;
} lo_net;

/* Exact window labels by Dijkstra.  dist (optional) receives layers*win_h*win_w
 * labels (window-local, row-major, LO_INF = unreachable).  When full==0 the
 * search stops once every label <= the goal label is settled (the canonical
 * path needs no more).  path (optional, capacity path_cap) receives the reverse
 * canonical path as global cell ids (l*H + y)*W + x, goal first.  Returns the
 * goal cost (LO_INF if disconnected) and writes *path_len (0 if disconnected,
 * or UINT32_MAX if path_cap was too small). */
uint32_t lo_dijkstra(const lo_lattice* lat, const lo_net* net, int full, uint32_t* dist,
                     uint32_t* path, uint32_t path_cap, uint32_t* path_len);

/* A* restatement with the reference pop key.  Returns the goal cost;
 * *expanded receives the count of expanded (popped, current, non-goal)
 * states, the reference's CpuRouteTelemetry::expanded_states. */
uint32_t lo_astar(const lo_lattice* lat, const lo_net* net, uint64_t* expanded);

/* lo_astar that also returns the A* path forward (start first) as global cell
 * ids, from the predecessor recorded by each accepted relaxation (the
 * reference's reconstruction, cpu_astar.cc:518-545).  *path_len is 0 when
 * disconnected and UINT32_MAX when path_cap is too small. */
uint32_t lo_astar_path(const lo_lattice* lat, const lo_net* net, uint64_t* expanded,
                       uint32_t* path, uint32_t path_cap, uint32_t* path_len);

typedef struct lo_sweep_stats {
  uint32_t sweeps;         /* sweeps executed including the final quiet one */
  uint64_t row_visits;     /* row steps processed (one per window row, all layers) */
  uint64_t row_stores;     /* layer rows written back (including the start row) */
  uint64_t cells_loaded;   /* cells read by the row steps */
  uint64_t cells_stored;   /* cells written by the row steps */
  uint64_t row_loads;      /* layer rows read (current rows and predecessor re-reads) */
} lo_sweep_stats;

/* CPU restatement of the GPU row-sweep schedule (same skip rules).  Fills dist
 * (layers*win_h*win_w, required) and returns the goal cost. */
uint32_t lo_sweep_schedule(const lo_lattice* lat, const lo_net* net, uint32_t max_sweeps,
                           uint32_t* dist, lo_sweep_stats* stats);

/* Same schedule with the frame orientation forced (transposed = 0 sweeps along
 * lattice y, 1 along lattice x, -1 picks the window's shorter side). */
uint32_t lo_sweep_schedule_oriented(const lo_lattice* lat, const lo_net* net, uint32_t max_sweeps,
                                    int transposed, uint32_t* dist, lo_sweep_stats* stats);

/* Batch helpers, parallel over nets with up to `threads` POSIX threads. */
void lo_dijkstra_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                       uint32_t* costs, uint32_t* path_lens, uint64_t* path_offsets,
                       uint32_t* paths, uint64_t path_capacity);

/* lo_dijkstra_batch with rip-up pricing (lat->cell_cost required): cells of
 * net i's previous route, own_cells[own_offsets[i] .. own_offsets[i + 1])
 * (global cell ids; own_offsets has count + 1 entries), enter at
 * cell_cost_own[c] instead of cell_cost[c]. */
void lo_dijkstra_batch_own(const lo_lattice* lat, const lo_net* nets, uint32_t count,
                           int threads, const uint32_t* cell_cost_own,
                           const uint64_t* own_offsets, const uint32_t* own_cells,
                           uint32_t* costs, uint32_t* path_lens, uint64_t* path_offsets,
                           uint32_t* paths, uint64_t path_capacity);
void lo_astar_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                    uint32_t* costs);

/* lo_astar_batch that also reports, per net, the expanded states (the
 * reference's expanded_states) and the distinct cells with an expanded state
 * (the cell expansions an exact cell-level A* needs: the frontier's unit of
 * algorithmic work).  Either output may be NULL. */
void lo_astar_batch_ex(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                       uint32_t* costs, uint64_t* expanded_states, uint64_t* expanded_cells);
void lo_sweep_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                    uint32_t max_sweeps, uint32_t* costs, lo_sweep_stats* stats);

/* ---------------- graph mode (DeviceCompiledBoardV1 arrays) ---------------- */

typedef struct go_node { /* bit-identical to DeviceNodeV1 (56 bytes) */
  int64_t lattice_x, lattice_y;
  uint32_t layer;
  uint8_t legal_edges;
  uint8_t reserved[3];
  uint32_t neighbors[8];
} go_node;

typedef struct go_policy_edge { /* bit-identical to DeviceCandidatePolicyEdgeV1 */
  uint32_t physical_edge_index;
  uint32_t reserved;
  uint64_t adjustment;
} go_policy_edge;

typedef struct go_query {
  uint32_t start_node, goal_node;
  uint64_t orthogonal_step_surcharge, diagonal_step_surcharge, bend_surcharge;
  const go_policy_edge* policy; /* sorted by physical_edge_index */
  uint32_t policy_count;
} go_query;

typedef struct go_costs {
  uint32_t orthogonal_step, diagonal_step, bend;
} go_costs;

/* Exact heading-state labels (9 per node, uint64, UINT64_MAX unreachable) by
 * Dijkstra.  Writes labels (optional, 9*node_count), and the canonical reverse
 * state path (optional) exactly as the reference batch sweep reconstructs it.
 * Returns 1 reached, 0 disconnected. */
int go_search(const go_node* nodes, uint32_t node_count, go_costs costs, const go_query* query,
              uint64_t* labels, uint64_t* goal_cost, uint32_t* goal_state, uint32_t* path,
              uint32_t path_cap, uint32_t* path_len);

/* Canonical predecessor of every state from exact labels. */
void go_predecessors(const go_node* nodes, uint32_t node_count, go_costs costs,
                     const go_query* query, const uint64_t* labels, uint32_t* preds);

/* Structural validation of one untrusted compact reverse path (goal state
 * first), restating the device-view checks of the reference's
 * ValidateAndReconstructCompactGpuPath (src/gpu/planar_router.cc:969-1067)
 * in its order; the exact-geometry stage after them is not restated.
 * Returns a GO_PATH_* code; *total_cost receives the path cost when OK and
 * *failing_index the forward index of the first failing state otherwise. */
enum {
  GO_PATH_OK = 0,
  GO_PATH_BOUNDS = 1,    /* gpu.batch.compact_path.bounds.v1 */
  GO_PATH_ENDPOINT = 2,  /* gpu.batch.compact_path.endpoint.v1 */
  GO_PATH_CYCLE = 3,     /* gpu.batch.compact_path.cycle.v1 */
  GO_PATH_HEADING = 4,   /* gpu.batch.compact_path.heading.v1 */
  GO_PATH_EDGE = 5,      /* gpu.batch.compact_path.edge.v1 */
  GO_PATH_BANNED = 6,    /* gpu.policy.banned_predecessor.v1 */
  GO_PATH_NOT_REACHED = 7
};
int go_validate_compact(const go_node* nodes, uint32_t node_count, go_costs costs,
                        const go_query* query, uint8_t completion, uint32_t goal_state,
                        const uint32_t* reverse_states, uint64_t length, uint64_t* total_cost,
                        uint64_t* failing_index);

/* ---------------- congestion prices (integer, checked) ---------------- */

/* Allocator epoch update (negotiated_regeneration_plan.cc:676-760):
 * factor = init + epoch*inc; for overuse>0: present = factor*overuse,
 * history += hinc*overuse, total = present + history; entries with zero
 * overuse keep history, present=0, total=history.  Returns 0 on success,
 * 1 on uint64 overflow. */
int po_epoch_update(uint32_t count, const uint64_t* usage, uint64_t capacity, uint64_t epoch,
                    uint64_t init_factor, uint64_t factor_inc, uint64_t hist_inc,
                    uint64_t* present, uint64_t* history, uint64_t* total);

/* CS-RR-v1 query snapshot cost (cpu_sequential_negotiated_routing.cc:299-505):
 * cost = history + (init + pass*inc) * max(0, usage + 1 - capacity).  Returns 0
 * on success, 1 on overflow, 2 when a cost exceeds max_value. */
int po_snapshot_costs(uint32_t count, const uint64_t* usage, const uint64_t* history,
                      uint64_t capacity, uint32_t pass_index, uint64_t init_present,
                      uint64_t present_inc, uint64_t max_value, uint64_t* cost);

/* CS-RR-v1 history update after a non-terminal pass (:1300-1330). */
int po_history_update(uint32_t count, const uint64_t* usage, uint64_t capacity,
                      uint64_t hist_inc, uint64_t max_value, uint64_t* history);

/* Usage accumulation over paths (resource_accounting.cc:180-230 for cell
 * resources): usage[cell] += 1 for each cell id in each path. */
void po_accumulate_cells(uint32_t path_count, const uint64_t* offsets, const uint32_t* lengths,
                         const uint32_t* cells, uint32_t cell_count, uint32_t* usage);

#ifdef __cplusplus
}
#endif

#endif /* APGAR_B200_ORACLE_H_ */
