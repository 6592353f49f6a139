/*
 * Graph-mode CPU oracle over DeviceCompiledBoardV1 node arrays.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Heading states are node*9 + incoming heading (planar_router.h:261-272).
 * The transition cost follows gpu/cuda/planar_router.cu:557-583 (step plus
 * objective surcharge, bend plus bend surcharge when the heading changes from
 * a real heading, plus the per-edge policy adjustment; UINT64_MAX adjustment
 * bans the edge; every sum is checked against the UINT64_MAX sentinel as in
 * :332-340).  The physical edge index follows :526-534.  Labels are the exact
 * fixed point (computed here by Dijkstra); the goal state and reverse path
 * follow :977-1009 and :1084-1165.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define GO_INF UINT64_MAX
#define GO_INVALID 0xFFFFFFFFu

static int checked_add(uint64_t a, uint64_t b, uint64_t* out) {
  const uint64_t max_finite = GO_INF - 1u;
  if (a > max_finite || b > max_finite - a) return 0;
  *out = a + b;
  return 1;
}

static uint32_t physical_edge(const go_node* nodes, uint32_t source, uint32_t d) {
  if (d < 4) return source * 8u + d;
  const uint32_t canon = nodes[source].neighbors[d];
  return canon == GO_INVALID ? GO_INVALID : canon * 8u + d - 4u;
}

static uint64_t policy_adjustment(const go_query* q, uint32_t edge) {
  uint32_t lo = 0, hi = q->policy_count;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (q->policy[mid].physical_edge_index < edge) {
      lo = mid + 1;
    } else {
      hi = mid;
    }
  }
  if (lo < q->policy_count && q->policy[lo].physical_edge_index == edge) {
    return q->policy[lo].adjustment;
  }
  return 0;
}

/* Returns 1 and the cost when the move source --d--> is traversable. */
static int transition(const go_node* nodes, go_costs costs, const go_query* q, uint32_t source,
                      uint32_t d, uint32_t incoming, uint64_t* cost) {
  const uint32_t edge = physical_edge(nodes, source, d);
  if (edge == GO_INVALID) return 0;
  const uint64_t adj = policy_adjustment(q, edge);
  if (adj == GO_INF) return 0;
  uint64_t value = (d & 1u) ? (uint64_t)costs.diagonal_step + q->diagonal_step_surcharge
                            : (uint64_t)costs.orthogonal_step + q->orthogonal_step_surcharge;
  if (incoming != 8u && incoming != d) {
    const uint64_t bend = (uint64_t)costs.bend + q->bend_surcharge;
    if (!checked_add(value, bend, &value)) return 0;
  }
  return checked_add(value, adj, cost);
}

typedef struct gheap_item {
  uint64_t key;
  uint32_t state;
} gheap_item;

typedef struct gheap {
  gheap_item* items;
  size_t size, cap;
} gheap;

static int gless(const gheap_item* a, const gheap_item* b) {
  return a->key < b->key || (a->key == b->key && a->state < b->state);
}

static void gpush(gheap* hp, uint64_t key, uint32_t state) {
  if (hp->size == hp->cap) {
    hp->cap = hp->cap ? hp->cap * 2 : 1024;
    hp->items = (gheap_item*)realloc(hp->items, hp->cap * sizeof(gheap_item));
  }
  gheap_item it = {key, state};
  size_t i = hp->size++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (!gless(&it, &hp->items[p])) break;
    hp->items[i] = hp->items[p];
    i = p;
  }
  hp->items[i] = it;
}

static gheap_item gpop(gheap* hp) {
  gheap_item top = hp->items[0];
  gheap_item last = hp->items[--hp->size];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1;
    if (l >= hp->size) break;
    size_t r = l + 1;
    size_t m = (r < hp->size && gless(&hp->items[r], &hp->items[l])) ? r : l;
    if (!gless(&hp->items[m], &last)) break;
    hp->items[i] = hp->items[m];
    i = m;
  }
  if (hp->size > 0) hp->items[i] = last;
  return top;
}

int go_search(const go_node* nodes, uint32_t node_count, go_costs costs, const go_query* q,
              uint64_t* labels_out, uint64_t* goal_cost, uint32_t* goal_state_out, uint32_t* path,
              uint32_t path_cap, uint32_t* path_len) {
  const size_t states = (size_t)node_count * 9u;
  uint64_t* labels = labels_out ? labels_out : (uint64_t*)malloc(states * sizeof(uint64_t));
  for (size_t i = 0; i < states; ++i) labels[i] = GO_INF;
  if (path_len) *path_len = 0;
  if (goal_cost) *goal_cost = GO_INF;
  if (goal_state_out) *goal_state_out = GO_INVALID;
  const uint32_t start_state = q->start_node * 9u + 8u;
  labels[start_state] = 0;
  gheap hp = {0};
  gpush(&hp, 0, start_state);
  while (hp.size) {
    const gheap_item it = gpop(&hp);
    if (it.key != labels[it.state]) continue;
    const uint32_t node = it.state / 9u, incoming = it.state % 9u;
    const go_node* nd = &nodes[node];
    for (uint32_t d = 0; d < 8; ++d) {
      if ((nd->legal_edges & (1u << d)) == 0) continue;
      const uint32_t nb = nd->neighbors[d];
      if (nb == GO_INVALID) continue;
      uint64_t tcost, cand;
      if (!transition(nodes, costs, q, node, d, incoming, &tcost)) continue;
      if (!checked_add(it.key, tcost, &cand)) continue;
      const uint32_t target = nb * 9u + d;
      if (cand < labels[target]) {
        labels[target] = cand;
        gpush(&hp, cand, target);
      }
    }
  }
  free(hp.items);

  uint64_t best = GO_INF;
  uint32_t best_state = GO_INVALID;
  for (uint32_t h = 0; h < 8; ++h) {
    const uint32_t s = q->goal_node * 9u + h;
    if (labels[s] < best || (labels[s] == best && s < best_state)) {
      best = labels[s];
      best_state = s;
    }
  }
  int reached = best != GO_INF;
  if (goal_cost) *goal_cost = best;
  if (reached && goal_state_out) *goal_state_out = best_state;
  if (reached && path && path_len) {
    uint32_t cursor = best_state, n = 0;
    int complete = 0;
    while (n < path_cap && n < states) {
      path[n++] = cursor;
      if (cursor == start_state) {
        complete = 1;
        break;
      }
      const uint32_t node = cursor / 9u, incoming = cursor % 9u;
      if (incoming >= 8u) break;
      const uint32_t pred = nodes[node].neighbors[(incoming + 4u) % 8u];
      if (pred == GO_INVALID) break;
      uint32_t chosen = GO_INVALID;
      for (uint32_t ph = 0; ph < 9u; ++ph) {
        if (ph == 8u && pred != q->start_node) continue;
        const uint32_t ps = pred * 9u + ph;
        uint64_t tcost, cand;
        if (!transition(nodes, costs, q, pred, incoming, ph, &tcost)) continue;
        if (checked_add(labels[ps], tcost, &cand) && cand == labels[cursor] && ps < chosen) {
          chosen = ps;
        }
      }
      if (chosen == GO_INVALID) break;
      cursor = chosen;
    }
    *path_len = complete ? n : 0;
  }
  if (!labels_out) free(labels);
  return reached;
}

/* Canonical predecessor of every state from exact labels (the reference's
 * SelectCandidateBatchPredecessors rule, planar_router.cu:1021-1079): the
 * smallest predecessor state whose label plus the move cost equals the
 * state's label; UINT32_MAX for the start state, unreachable states and
 * heading-8 states. */
void go_predecessors(const go_node* nodes, uint32_t node_count, go_costs costs, const go_query* q,
                     const uint64_t* labels, uint32_t* preds) {
  const uint32_t states = node_count * 9u;
  for (uint32_t s = 0; s < states; ++s) {
    preds[s] = GO_INVALID;
    const uint32_t node = s / 9u, h = s % 9u;
    if (h == 8u || labels[s] == GO_INF) continue;
    const uint32_t pred = nodes[node].neighbors[(h + 4u) % 8u];
    if (pred == GO_INVALID) continue;
    for (uint32_t ph = 0; ph < 9u; ++ph) {
      if (ph == 8u && pred != q->start_node) continue;
      uint64_t t, c;
      if (!transition(nodes, costs, q, pred, h, ph, &t)) continue;
      if (checked_add(labels[pred * 9u + ph], t, &c) && c == labels[s]) {
        preds[s] = pred * 9u + ph;
        break;
      }
    }
  }
}

/* Forward walk of a reverse compact path, check by check in the reference's
 * order (planar_router.cc:969-1067): bounds of a reached path, endpoint
 * binding, state bounds, then per state in forward order a repeated state,
 * the start-only heading sentinel, one adjacent compiled legal edge (same
 * layer, lattice delta of the heading, neighbour and legal bit), a banned
 * resource, and the checked finite cost sum. */
int go_validate_compact(const go_node* nodes, uint32_t node_count, go_costs costs,
                        const go_query* q, uint8_t completion, uint32_t goal_state,
                        const uint32_t* rev, uint64_t len, uint64_t* total_cost,
                        uint64_t* failing_index) {
  static const int dx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
  static const int dy[8] = {0, 1, 1, 1, 0, -1, -1, -1};
  const uint64_t states = (uint64_t)node_count * 9u;
  *total_cost = 0;
  *failing_index = 0;
  if (completion != 0) return GO_PATH_NOT_REACHED;
  if (len == 0 || len > states) return GO_PATH_BOUNDS;
  const uint32_t start_state = q->start_node * 9u + 8u;
  if (rev[0] != goal_state || rev[len - 1] != start_state || goal_state / 9u != q->goal_node ||
      goal_state % 9u >= 8u) {
    return GO_PATH_ENDPOINT;
  }
  for (uint64_t i = 0; i < len; ++i) {
    if (rev[i] >= states) return GO_PATH_BOUNDS;
  }
  uint64_t* visited = (uint64_t*)calloc((states + 63u) / 64u, sizeof(uint64_t));
  uint64_t total = 0;
  int code = GO_PATH_OK;
  for (uint64_t index = 0; index < len && code == GO_PATH_OK; ++index) {
    const uint64_t r = len - 1u - index;
    const uint32_t state = rev[r];
    *failing_index = index;
    const uint64_t bit = 1ull << (state % 64u);
    if (visited[state / 64u] & bit) {
      code = GO_PATH_CYCLE;
      break;
    }
    visited[state / 64u] |= bit;
    const uint32_t node = state / 9u;
    if (node >= node_count) {
      code = GO_PATH_BOUNDS;
      break;
    }
    if (index == 0) {
      if (state != start_state) code = GO_PATH_ENDPOINT;
      continue;
    }
    const uint32_t pred_state = rev[r + 1u];
    const uint32_t pred = pred_state / 9u;
    const uint32_t incoming = state % 9u, pred_heading = pred_state % 9u;
    if (incoming >= 8u || (pred_heading == 8u && pred_state != start_state)) {
      code = GO_PATH_HEADING;
      break;
    }
    const go_node* a = &nodes[pred];
    const go_node* b = &nodes[node];
    if (a->layer != b->layer || b->lattice_x - a->lattice_x != dx[incoming] ||
        b->lattice_y - a->lattice_y != dy[incoming] || a->neighbors[incoming] != node ||
        (a->legal_edges & (1u << incoming)) == 0) {
      code = GO_PATH_EDGE;
      break;
    }
    const uint32_t edge = physical_edge(nodes, pred, incoming);
    const uint64_t adj = policy_adjustment(q, edge);
    if (adj == GO_INF) {
      code = GO_PATH_BANNED;
      break;
    }
    /* transition in 128-bit arithmetic, rejected at the sentinel */
    unsigned __int128 t = (incoming & 1u)
                              ? (unsigned __int128)costs.diagonal_step + q->diagonal_step_surcharge
                              : (unsigned __int128)costs.orthogonal_step + q->orthogonal_step_surcharge;
    if (pred_heading != 8u && pred_heading != incoming) t += (unsigned __int128)costs.bend + q->bend_surcharge;
    t += adj;
    uint64_t next;
    if (t >= GO_INF || !checked_add(total, (uint64_t)t, &next)) {
      code = GO_PATH_EDGE;
      break;
    }
    total = next;
  }
  free(visited);
  if (code == GO_PATH_OK) *total_cost = total;
  return code;
}
