/*
 * Lattice-mode CPU oracle.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Move model shared with the GPU kernels (apgar_b200/csrc/lattice_sweep.cu):
 *   orthogonal move legal iff both cells are free;
 *   diagonal move legal iff both cells and both side cells are free;
 *   via (l, x, y) <-> (l+1, x, y) legal iff both cells are free and the via
 *   bit of layer pair l is set (no via mask = every via bit set);
 *   a cell is free iff it lies inside the net window and is not blocked.
 * Costs: orthogonal, diagonal, via (no bend term: the lattice configs use
 * bend 0, which is what makes node-level labels sufficient).
 *
 * Canonical path (reference planar_router.cu:1084-1165 reverse walk, applied
 * to exact labels): from the goal, repeatedly step to the predecessor through
 * the smallest incoming heading h whose move is legal and satisfies
 * label[pred] + cost(h) == label[cur].  Headings 0..7 are the planar
 * directions E, NE, N, NW, W, SW, S, SE (geometry_compiler::Direction order);
 * 8 = via arriving from the layer below, 9 = via arriving from the layer above.
 */
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static const int kDx[8] = {1, 1, 0, -1, -1, -1, 0, 1};
static const int kDy[8] = {0, 1, 1, 1, 0, -1, -1, -1};

typedef struct win_ctx {
  const lo_lattice* lat;
  const lo_net* net;
  int L, w, h, x0, y0, words;
  /* Optional rip-up pricing: cells whose bit is set in `own` (window-local
   * cell index) enter at cost_own[c] instead of cell_cost[c]. */
  const uint8_t* own;
  const uint32_t* cost_own;
} win_ctx;

static inline int lat_blocked(const lo_lattice* lat, int l, int gx, int gy) {
  const uint32_t word = lat->blocked[((size_t)l * lat->height + gy) * (lat->width / 32) + gx / 32];
  return (word >> (gx & 31)) & 1u;
}

static inline int cell_free(const win_ctx* c, int l, int x, int y) {
  if (x < 0 || y < 0 || x >= c->w || y >= c->h || l < 0 || l >= c->L) return 0;
  return !lat_blocked(c->lat, l, c->x0 + x, c->y0 + y);
}

static inline int via_bit(const win_ctx* c, int lower, int x, int y) {
  if (c->lat->via_ok == NULL) return 1;
  const int gx = c->x0 + x, gy = c->y0 + y;
  const uint32_t word =
      c->lat->via_ok[((size_t)lower * c->lat->height + gy) * (c->lat->width / 32) + gx / 32];
  return (word >> (gx & 31)) & 1u;
}

/* Planar move from (x,y) in direction d on layer l. */
static inline int planar_legal(const win_ctx* c, int l, int x, int y, int d) {
  const int nx = x + kDx[d], ny = y + kDy[d];
  if (!cell_free(c, l, x, y) || !cell_free(c, l, nx, ny)) return 0;
  if ((d & 1) == 0) return 1;
  return cell_free(c, l, nx, y) && cell_free(c, l, x, ny);
}

static inline int via_legal(const win_ctx* c, int lower, int x, int y) {
  return cell_free(c, lower, x, y) && cell_free(c, lower + 1, x, y) && via_bit(c, lower, x, y);
}

static void ctx_init(win_ctx* c, const lo_lattice* lat, const lo_net* net) {
  c->lat = lat;
  c->net = net;
  c->L = lat->layers;
  c->w = (int)net->win_w;
  c->h = (int)net->win_h;
  c->x0 = (int)net->win_x0;
  c->y0 = (int)net->win_y0;
  c->words = lat->width / 32;
  c->own = NULL;
  c->cost_own = NULL;
}

static inline size_t cell_index(const win_ctx* c, int l, int x, int y) {
  return ((size_t)l * c->h + y) * c->w + x;
}

/* ---------------------------- binary heap ---------------------------- */

typedef struct heap_item {
  uint64_t key; /* label << 32 | tiebreak */
  uint32_t cell;
} heap_item;

typedef struct heap {
  heap_item* items;
  size_t size, cap;
} heap;

static void heap_push(heap* hp, uint64_t key, uint32_t cell) {
  if (hp->size == hp->cap) {
    hp->cap = hp->cap ? hp->cap * 2 : 1024;
    hp->items = (heap_item*)realloc(hp->items, hp->cap * sizeof(heap_item));
  }
  size_t i = hp->size++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (hp->items[p].key <= key) break;
    hp->items[i] = hp->items[p];
    i = p;
  }
  hp->items[i].key = key;
  hp->items[i].cell = cell;
}

static heap_item heap_pop(heap* hp) {
  heap_item top = hp->items[0];
  heap_item last = hp->items[--hp->size];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1;
    if (l >= hp->size) break;
    size_t r = l + 1;
    size_t m = (r < hp->size && hp->items[r].key < hp->items[l].key) ? r : l;
    if (hp->items[m].key >= last.key) break;
    hp->items[i] = hp->items[m];
    i = m;
  }
  if (hp->size > 0) hp->items[i] = last;
  return top;
}

/* --------------------------- canonical walk --------------------------- */

static inline uint32_t move_cost(const lo_lattice* lat, int h) {
  if (h >= 8) return lat->via;
  return (h & 1) ? lat->diag : lat->orth;
}

/* Entry cost of window cell (l, x, y): its negotiated price, 0 without one. */
static inline uint64_t entry_cost(const win_ctx* c, int l, int x, int y) {
  const lo_lattice* lat = c->lat;
  if (lat->cell_cost == NULL) return 0;
  const size_t g = ((size_t)l * lat->height + (c->y0 + y)) * lat->width + (c->x0 + x);
  if (c->own != NULL) {
    const size_t wi = cell_index(c, l, x, y);
    if ((c->own[wi >> 3] >> (wi & 7)) & 1u) return c->cost_own[g];
  }
  return lat->cell_cost[g];
}

/* Reverse canonical path from exact labels.  Returns path length, or
 * UINT32_MAX when the capacity is exceeded or the labels are inconsistent. */
static uint32_t canonical_walk(const win_ctx* c, const uint32_t* dist, int gl, int gx, int gy,
                               int sl, int sx, int sy, uint32_t* path, uint32_t cap) {
  const lo_lattice* lat = c->lat;
  int l = gl, x = gx, y = gy;
  uint32_t n = 0;
  for (;;) {
    if (n >= cap) return UINT32_MAX;
    path[n++] = (uint32_t)((((size_t)l * lat->height) + (c->y0 + y)) * lat->width + (c->x0 + x));
    if (l == sl && x == sx && y == sy) return n;
    const uint32_t here = dist[cell_index(c, l, x, y)];
    int chosen = -1;
    for (int h = 0; h < 10 && chosen < 0; ++h) {
      int pl = l, px = x, py = y;
      int legal;
      if (h < 8) {
        px = x - kDx[h];
        py = y - kDy[h];
        legal = planar_legal(c, l, px, py, h);
      } else if (h == 8) {
        pl = l - 1;
        legal = pl >= 0 && via_legal(c, pl, x, y);
      } else {
        pl = l + 1;
        legal = pl < c->L && via_legal(c, l, x, y);
      }
      if (!legal) continue;
      const uint32_t pd = dist[cell_index(c, pl, px, py)];
      if (pd == LO_INF) continue;
      if ((uint64_t)pd + move_cost(lat, h) + entry_cost(c, l, x, y) == here) {
        chosen = h;
        l = pl;
        x = px;
        y = py;
      }
    }
    if (chosen < 0) return UINT32_MAX;
  }
}

/* ------------------------------ Dijkstra ------------------------------ */

static uint32_t dijkstra_run(const lo_lattice* lat, const lo_net* net, int full,
                             uint32_t* dist_out, uint32_t* path, uint32_t path_cap,
                             uint32_t* path_len, const uint8_t* own, const uint32_t* cost_own);

uint32_t lo_dijkstra(const lo_lattice* lat, const lo_net* net, int full, uint32_t* dist_out,
                     uint32_t* path, uint32_t path_cap, uint32_t* path_len) {
  return dijkstra_run(lat, net, full, dist_out, path, path_cap, path_len, NULL, NULL);
}

static uint32_t dijkstra_run(const lo_lattice* lat, const lo_net* net, int full,
                             uint32_t* dist_out, uint32_t* path, uint32_t path_cap,
                             uint32_t* path_len, const uint8_t* own, const uint32_t* cost_own) {
  win_ctx c;
  ctx_init(&c, lat, net);
  c.own = own;
  c.cost_own = cost_own;
  const size_t cells = (size_t)c.L * c.w * c.h;
  uint32_t* dist = dist_out ? dist_out : (uint32_t*)malloc(cells * sizeof(uint32_t));
  for (size_t i = 0; i < cells; ++i) dist[i] = LO_INF;
  const int sl = (int)net->start_layer, sx = (int)(net->start_x - net->win_x0),
            sy = (int)(net->start_y - net->win_y0);
  const int gl = (int)net->goal_layer, gx = (int)(net->goal_x - net->win_x0),
            gy = (int)(net->goal_y - net->win_y0);
  if (path_len) *path_len = 0;
  if (!cell_free(&c, sl, sx, sy) || !cell_free(&c, gl, gx, gy)) {
    if (!dist_out) free(dist);
    return LO_INF;
  }
  heap hp = {0};
  dist[cell_index(&c, sl, sx, sy)] = 0;
  heap_push(&hp, 0, (uint32_t)cell_index(&c, sl, sx, sy));
  const size_t goal_index = cell_index(&c, gl, gx, gy);
  while (hp.size) {
    heap_item it = heap_pop(&hp);
    const uint32_t d = (uint32_t)(it.key >> 32);
    if (d != dist[it.cell]) continue;
    if (!full && dist[goal_index] != LO_INF && d > dist[goal_index]) break;
    const int l = (int)(it.cell / ((size_t)c.w * c.h));
    const int rem = (int)(it.cell % ((size_t)c.w * c.h));
    const int y = rem / c.w, x = rem % c.w;
    for (int h = 0; h < 10; ++h) {
      int nl = l, nx = x, ny = y, legal;
      if (h < 8) {
        nx = x + kDx[h];
        ny = y + kDy[h];
        legal = planar_legal(&c, l, x, y, h);
      } else if (h == 8) {
        nl = l + 1;
        legal = nl < c.L && via_legal(&c, l, x, y);
      } else {
        nl = l - 1;
        legal = nl >= 0 && via_legal(&c, nl, x, y);
      }
      if (!legal) continue;
      const uint64_t cand = (uint64_t)d + move_cost(lat, h) + entry_cost(&c, nl, nx, ny);
      const size_t ni = cell_index(&c, nl, nx, ny);
      if (cand >= LO_INF) continue; /* beyond the 32-bit cost domain */
      if (cand < dist[ni]) {
        dist[ni] = (uint32_t)cand;
        heap_push(&hp, (cand << 32) | (uint32_t)ni, (uint32_t)ni);
      }
    }
  }
  free(hp.items);
  const uint32_t cost = dist[goal_index];
  if (cost != LO_INF && path && path_len) {
    *path_len = canonical_walk(&c, dist, gl, gx, gy, sl, sx, sy, path, path_cap);
  }
  if (!dist_out) free(dist);
  return cost;
}

/* -------------------------------- A* -------------------------------- */

/* Pop key of RouteWithCpuAStar (cpu_astar.cc:67-74): (f, h, g, y, x, heading,
 * sequence), extended with the layer between g and y.  The heuristic is the
 * reference octile bound for diag >= orth (cpu_astar.cc:176-190) plus one via
 * cost per layer of separation, which keeps it admissible and consistent. */
typedef struct astar_item {
  uint64_t f, h, g;
  int32_t l, y, x, heading;
  uint64_t seq;
} astar_item;

static int astar_less(const astar_item* a, const astar_item* b) {
  if (a->f != b->f) return a->f < b->f;
  if (a->h != b->h) return a->h < b->h;
  if (a->g != b->g) return a->g < b->g;
  if (a->l != b->l) return a->l < b->l;
  if (a->y != b->y) return a->y < b->y;
  if (a->x != b->x) return a->x < b->x;
  if (a->heading != b->heading) return a->heading < b->heading;
  return a->seq < b->seq;
}

typedef struct aheap {
  astar_item* items;
  size_t size, cap;
} aheap;

static void aheap_push(aheap* hp, astar_item it) {
  if (hp->size == hp->cap) {
    hp->cap = hp->cap ? hp->cap * 2 : 1024;
    hp->items = (astar_item*)realloc(hp->items, hp->cap * sizeof(astar_item));
  }
  size_t i = hp->size++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (!astar_less(&it, &hp->items[p])) break;
    hp->items[i] = hp->items[p];
    i = p;
  }
  hp->items[i] = it;
}

static astar_item aheap_pop(aheap* hp) {
  astar_item top = hp->items[0];
  astar_item last = hp->items[--hp->size];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1;
    if (l >= hp->size) break;
    size_t r = l + 1;
    size_t m = (r < hp->size && astar_less(&hp->items[r], &hp->items[l])) ? r : l;
    if (!astar_less(&hp->items[m], &last)) break;
    hp->items[i] = hp->items[m];
    i = m;
  }
  if (hp->size > 0) hp->items[i] = last;
  return top;
}

static uint64_t octile(const lo_lattice* lat, int dx, int dy, int dl) {
  const uint64_t ax = (uint64_t)(dx < 0 ? -dx : dx), ay = (uint64_t)(dy < 0 ? -dy : dy);
  const uint64_t al = (uint64_t)(dl < 0 ? -dl : dl);
  uint64_t planar;
  if (lat->diag < lat->orth) {
    planar = (ax > ay ? ax : ay) * lat->diag;
  } else {
    const uint64_t dmin = ax < ay ? ax : ay, dmax = ax < ay ? ay : ax;
    const uint64_t eff = lat->diag < 2ull * lat->orth ? lat->diag : 2ull * lat->orth;
    planar = dmin * eff + (dmax - dmin) * lat->orth;
  }
  return planar + al * lat->via;
}

/* Shared body of lo_astar and lo_astar_path.  With `path` non-NULL every
 * accepted relaxation records its predecessor state, as the reference's
 * SearchRecord does (cpu_astar.cc:495-497), and the goal state's chain is
 * written forward (start first) as global cell ids. */
static uint32_t astar_run(const lo_lattice* lat, const lo_net* net, uint64_t* expanded_out,
                          uint32_t* path, uint32_t path_cap, uint32_t* path_len,
                          uint64_t* cells_out) {
  win_ctx c;
  ctx_init(&c, lat, net);
  const size_t cells = (size_t)c.L * c.w * c.h;
  /* Record per (cell, heading): heading 0..7 planar, 8 start / none, 9 via up,
   * 10 via down. */
  const size_t states = cells * 11;
  uint32_t* g = (uint32_t*)malloc(states * sizeof(uint32_t));
  for (size_t i = 0; i < states; ++i) g[i] = LO_INF;
  uint64_t* pred = path ? (uint64_t*)malloc(states * sizeof(uint64_t)) : NULL;
  /* distinct cells with an expanded state (cells_out) */
  uint8_t* seen = cells_out ? (uint8_t*)calloc((cells + 7) / 8, 1) : NULL;
  uint64_t distinct = 0;
  size_t goal_state = (size_t)-1;
  if (path_len) *path_len = 0;
  const int sl = (int)net->start_layer, sx = (int)(net->start_x - net->win_x0),
            sy = (int)(net->start_y - net->win_y0);
  const int gl = (int)net->goal_layer, gx = (int)(net->goal_x - net->win_x0),
            gy = (int)(net->goal_y - net->win_y0);
  uint64_t expanded = 0;
  uint32_t result = LO_INF;
  if (cell_free(&c, sl, sx, sy) && cell_free(&c, gl, gx, gy)) {
    aheap hp = {0};
    uint64_t seq = 0;
    const uint64_t h0 = octile(lat, gx - sx, gy - sy, gl - sl);
    g[cell_index(&c, sl, sx, sy) * 11 + 8] = 0;
    astar_item s = {h0, h0, 0, sl, sy, sx, 8, seq++};
    aheap_push(&hp, s);
    while (hp.size) {
      astar_item cur = aheap_pop(&hp);
      const size_t ci = cell_index(&c, cur.l, cur.x, cur.y);
      if (g[ci * 11 + (size_t)cur.heading] != cur.g) continue;
      if (cur.l == gl && cur.x == gx && cur.y == gy) {
        result = (uint32_t)cur.g;
        goal_state = ci * 11 + (size_t)cur.heading;
        break;
      }
      ++expanded;
      if (seen && !((seen[ci >> 3] >> (ci & 7)) & 1u)) {
        seen[ci >> 3] |= (uint8_t)(1u << (ci & 7));
        ++distinct;
      }
      for (int mv = 0; mv < 10; ++mv) {
        int nl = cur.l, nx = cur.x, ny = cur.y, legal, heading;
        if (mv < 8) {
          nx = cur.x + kDx[mv];
          ny = cur.y + kDy[mv];
          legal = planar_legal(&c, cur.l, cur.x, cur.y, mv);
          heading = mv;
        } else if (mv == 8) {
          nl = cur.l + 1;
          legal = nl < c.L && via_legal(&c, cur.l, cur.x, cur.y);
          heading = 9;
        } else {
          nl = cur.l - 1;
          legal = nl >= 0 && via_legal(&c, nl, cur.x, cur.y);
          heading = 10;
        }
        if (!legal) continue;
        const uint64_t ng = cur.g + move_cost(lat, mv);
        const size_t ni = cell_index(&c, nl, nx, ny) * 11 + (size_t)heading;
        if (g[ni] != LO_INF && g[ni] <= ng) continue;
        g[ni] = (uint32_t)ng;
        if (pred) pred[ni] = ci * 11 + (size_t)cur.heading;
        const uint64_t hh = octile(lat, gx - nx, gy - ny, gl - nl);
        astar_item it = {ng + hh, hh, ng, nl, ny, nx, heading, seq++};
        aheap_push(&hp, it);
      }
    }
    free(hp.items);
  }
  if (path && goal_state != (size_t)-1) {
    /* walk back to the start state (heading 8 at the start cell) */
    const size_t start_state = cell_index(&c, sl, sx, sy) * 11 + 8;
    uint32_t n = 0;
    size_t st = goal_state;
    for (;;) {
      ++n;
      if (st == start_state) break;
      st = (size_t)pred[st];
    }
    if (n > path_cap) {
      if (path_len) *path_len = UINT32_MAX;
    } else {
      st = goal_state;
      for (uint32_t k = n; k-- > 0;) {
        const size_t cell = st / 11;
        const int l = (int)(cell / ((size_t)c.w * c.h));
        const size_t rem = cell % ((size_t)c.w * c.h);
        const int y = (int)(rem / (size_t)c.w), x = (int)(rem % (size_t)c.w);
        path[k] = (uint32_t)(((size_t)l * lat->height + (size_t)(c.y0 + y)) * lat->width +
                             (size_t)(c.x0 + x));
        if (k) st = (size_t)pred[st];
      }
      if (path_len) *path_len = n;
    }
  }
  free(pred);
  free(seen);
  free(g);
  if (expanded_out) *expanded_out = expanded;
  if (cells_out) *cells_out = distinct;
  return result;
}

uint32_t lo_astar(const lo_lattice* lat, const lo_net* net, uint64_t* expanded_out) {
  return astar_run(lat, net, expanded_out, NULL, 0, NULL, NULL);
}

uint32_t lo_astar_path(const lo_lattice* lat, const lo_net* net, uint64_t* expanded_out,
                       uint32_t* path, uint32_t path_cap, uint32_t* path_len) {
  return astar_run(lat, net, expanded_out, path, path_cap, path_len, NULL);
}

/* --------------------------- sweep schedule --------------------------- */

/* The GPU sweeps a window along its shorter side: when the window is taller
 * than wide it works in a transposed frame whose rows are lattice columns.
 * Frame cell (r, p) is lattice (x = p, y = r) normally and (x = r, y = p) when
 * transposed; the move model is symmetric under that swap. */
typedef struct frame {
  const win_ctx* c;
  int transposed;
  int R, K; /* rows (swept sequentially) and row width */
} frame;

static inline int ffree(const frame* f, int l, int r, int p) {
  if (r < 0 || p < 0 || r >= f->R || p >= f->K) return 0;
  return f->transposed ? cell_free(f->c, l, r, p) : cell_free(f->c, l, p, r);
}

static inline int fvia(const frame* f, int lower, int r, int p) {
  return f->transposed ? via_legal(f->c, lower, r, p) : via_legal(f->c, lower, p, r);
}

/* planar move (r0,p0) -> (r1,p1) with |dr|,|dp| <= 1 */
static inline int fmove(const frame* f, int l, int r0, int p0, int r1, int p1) {
  if (!ffree(f, l, r0, p0) || !ffree(f, l, r1, p1)) return 0;
  if (r0 == r1 || p0 == p1) return 1;
  return ffree(f, l, r0, p1) && ffree(f, l, r1, p0);
}

/* Row step semantics (one frame row, all layers together), identical to the
 * GPU kernel: relax from the previous row in sweep order (straight plus the
 * two diagonals), then repeat {two-sided row scan, via cascade up then down}
 * until the via cascade changes nothing.  A row is skipped when neither it
 * nor its predecessor row changed since the last sweep in the same direction
 * (or, for the first sweep in each direction, when both rows are all-INF). */
uint32_t lo_sweep_schedule(const lo_lattice* lat, const lo_net* net, uint32_t max_sweeps,
                           uint32_t* dist, lo_sweep_stats* stats) {
  return lo_sweep_schedule_oriented(lat, net, max_sweeps, -1, dist, stats);
}

uint32_t lo_sweep_schedule_oriented(const lo_lattice* lat, const lo_net* net, uint32_t max_sweeps,
                                    int transposed, uint32_t* dist, lo_sweep_stats* stats) {
  win_ctx c;
  ctx_init(&c, lat, net);
  const int L = c.L, w = c.w, h = c.h;
  const int tr = transposed < 0 ? (h > w) : transposed;
  frame f = {&c, tr, tr ? w : h, tr ? h : w};
  const int R = f.R, K = f.K;
  const size_t cells = (size_t)L * w * h;
  for (size_t i = 0; i < cells; ++i) dist[i] = LO_INF;
  lo_sweep_stats st = {0};
  const int sl = (int)net->start_layer, sx = (int)(net->start_x - net->win_x0),
            sy = (int)(net->start_y - net->win_y0);
  const int gl = (int)net->goal_layer, gx = (int)(net->goal_x - net->win_x0),
            gy = (int)(net->goal_y - net->win_y0);
  if (!cell_free(&c, sl, sx, sy) || !cell_free(&c, gl, gx, gy)) {
    if (stats) *stats = st;
    return LO_INF;
  }
  const int sr = f.transposed ? sx : sy, sp = f.transposed ? sy : sx;
  uint32_t* fd = (uint32_t*)malloc(cells * sizeof(uint32_t)); /* frame labels */
  for (size_t i = 0; i < cells; ++i) fd[i] = LO_INF;
#define FD(l, r, p) fd[((size_t)(l) * R + (r)) * K + (p)]
  const int32_t kNever = -1000000;
  int32_t* modified = (int32_t*)malloc((size_t)R * sizeof(int32_t));
  for (int r = 0; r < R; ++r) modified[r] = kNever;
  FD(sl, sr, sp) = 0;
  modified[sr] = 0; /* initialisation writes the start row on every layer */
  st.row_stores += (uint64_t)L;
  st.cells_stored += (uint64_t)L * K;
  uint32_t* row = (uint32_t*)malloc((size_t)L * K * sizeof(uint32_t));
  uint32_t* orig = (uint32_t*)malloc((size_t)L * K * sizeof(uint32_t));
  uint32_t* east = (uint32_t*)malloc((size_t)K * sizeof(uint32_t));
  uint32_t sweeps = 0;
  for (uint32_t k = 1; k <= max_sweeps; ++k) {
    sweeps = k;
    const int up = (k & 1) != 0;
    const int dr = up ? 1 : -1;
    int any_change = 0;
    int prev_in_regs = 0;
    for (int step = 0; step < R; ++step) {
      const int r = up ? step : R - 1 - step;
      const int pr = r - dr; /* previous row in sweep order */
      const int32_t mp = (pr >= 0 && pr < R) ? modified[pr] : kNever;
      const int32_t my = modified[r];
      int skip;
      if (k <= 2) {
        skip = (mp == kNever && my == kNever);
      } else {
        skip = (mp <= (int32_t)k - 2 && my <= (int32_t)k - 2);
      }
      if (skip) {
        prev_in_regs = 0;
        continue;
      }
      if (mp != kNever && !prev_in_regs) {
        st.cells_loaded += (uint64_t)L * K; /* predecessor row reload */
        st.row_loads += (uint64_t)L;
      }
      if (my != kNever) {
        st.cells_loaded += (uint64_t)L * K;
        st.row_loads += (uint64_t)L;
      }
      st.row_visits += 1;
      for (int l = 0; l < L; ++l) {
        for (int p = 0; p < K; ++p) row[l * K + p] = FD(l, r, p);
      }
      memcpy(orig, row, (size_t)L * K * sizeof(uint32_t));
      if (pr >= 0 && pr < R && mp != kNever) {
        for (int l = 0; l < L; ++l) {
          for (int p = 0; p < K; ++p) {
            uint64_t best = row[l * K + p];
            for (int q = p - 1; q <= p + 1; ++q) {
              if (q < 0 || q >= K) continue;
              const uint32_t pd = FD(l, pr, q);
              if (pd == LO_INF || !fmove(&f, l, pr, q, r, p)) continue;
              const uint64_t cand = (uint64_t)pd + (q == p ? lat->orth : lat->diag);
              if (cand < best) best = cand;
            }
            row[l * K + p] = (uint32_t)best;
          }
        }
      }
      for (;;) {
        for (int l = 0; l < L; ++l) {
          uint32_t* v = row + (size_t)l * K;
          /* two-sided scan: min(east scan, west scan) of the same input,
           * which equals an east scan followed by a west scan */
          uint64_t carry = LO_INF;
          for (int p = 0; p < K; ++p) {
            uint64_t e = v[p];
            if (p > 0 && carry != LO_INF && fmove(&f, l, r, p - 1, r, p) &&
                carry + lat->orth < e) {
              e = carry + lat->orth;
            }
            east[p] = (uint32_t)e;
            carry = e;
          }
          carry = LO_INF;
          for (int p = K - 1; p >= 0; --p) {
            uint64_t wv = v[p];
            if (p + 1 < K && carry != LO_INF && fmove(&f, l, r, p + 1, r, p) &&
                carry + lat->orth < wv) {
              wv = carry + lat->orth;
            }
            carry = wv;
            v[p] = east[p] < wv ? east[p] : (uint32_t)wv;
          }
        }
        int via_change = 0;
        for (int l = 1; l < L; ++l) {
          for (int p = 0; p < K; ++p) {
            const uint32_t a = row[(l - 1) * K + p];
            if (a != LO_INF && fvia(&f, l - 1, r, p) && (uint64_t)a + lat->via < row[l * K + p]) {
              row[l * K + p] = a + lat->via;
              via_change = 1;
            }
          }
        }
        for (int l = L - 2; l >= 0; --l) {
          for (int p = 0; p < K; ++p) {
            const uint32_t a = row[(l + 1) * K + p];
            if (a != LO_INF && fvia(&f, l, r, p) && (uint64_t)a + lat->via < row[l * K + p]) {
              row[l * K + p] = a + lat->via;
              via_change = 1;
            }
          }
        }
        if (!via_change) break;
      }
      int changed = memcmp(orig, row, (size_t)L * K * sizeof(uint32_t)) != 0;
      if (changed) {
        /* a newly materialised row stores every layer; afterwards only the
         * layers whose labels changed are written back */
        const int materialise = (my == kNever);
        for (int l = 0; l < L; ++l) {
          const int layer_changed =
              memcmp(orig + (size_t)l * K, row + (size_t)l * K, (size_t)K * sizeof(uint32_t)) != 0;
          if (!layer_changed && !materialise) continue;
          for (int p = 0; p < K; ++p) FD(l, r, p) = row[l * K + p];
          st.row_stores += 1;
          st.cells_stored += (uint64_t)K;
        }
        modified[r] = (int32_t)k;
        any_change = 1;
      }
      prev_in_regs = 1;
    }
    if (!any_change && k >= 2) break;
  }
  st.sweeps = sweeps;
  for (int l = 0; l < L; ++l) {
    for (int y = 0; y < h; ++y) {
      for (int x = 0; x < w; ++x) {
        dist[cell_index(&c, l, x, y)] = f.transposed ? FD(l, x, y) : FD(l, y, x);
      }
    }
  }
#undef FD
  free(east);
  free(row);
  free(orig);
  free(modified);
  free(fd);
  if (stats) *stats = st;
  return dist[cell_index(&c, gl, gx, gy)];
}

/* ----------------------------- batches ----------------------------- */

typedef struct batch_job {
  const lo_lattice* lat;
  const lo_net* nets;
  uint32_t count;
  /* rip-up pricing (kind 0 only): net i's own cells are
   * own_cells[own_offsets[i] .. own_offsets[i + 1]) (global ids) */
  const uint32_t* cost_own;
  const uint64_t* own_offsets;
  const uint32_t* own_cells;
  int kind; /* 0 dijkstra, 1 astar, 2 sweep */
  uint32_t max_sweeps;
  uint32_t* costs;
  uint32_t* path_lens;
  const uint64_t* path_offsets;
  uint32_t* paths;
  uint64_t path_capacity;
  lo_sweep_stats* stats;
  uint64_t* expanded_states; /* kind 1, optional */
  uint64_t* expanded_cells;  /* kind 1, optional */
  uint32_t next;
  pthread_mutex_t lock;
} batch_job;

static void* batch_worker(void* arg) {
  batch_job* job = (batch_job*)arg;
  for (;;) {
    pthread_mutex_lock(&job->lock);
    const uint32_t i = job->next++;
    pthread_mutex_unlock(&job->lock);
    if (i >= job->count) break;
    const lo_net* net = &job->nets[i];
    if (job->kind == 0) {
      uint32_t len = 0;
      uint32_t* path = NULL;
      uint32_t cap = 0;
      if (job->paths) {
        path = job->paths + job->path_offsets[i];
        const uint64_t end = (i + 1 < job->count) ? job->path_offsets[i + 1] : job->path_capacity;
        cap = (uint32_t)(end - job->path_offsets[i]);
      }
      uint8_t* own = NULL;
      if (job->own_offsets != NULL && job->own_offsets[i + 1] > job->own_offsets[i]) {
        const lo_lattice* lat = job->lat;
        const size_t wcells = (size_t)lat->layers * net->win_w * net->win_h;
        own = (uint8_t*)calloc((wcells + 7) / 8, 1);
        for (uint64_t k = job->own_offsets[i]; k < job->own_offsets[i + 1]; ++k) {
          const size_t gcell = job->own_cells[k];
          const size_t plane = (size_t)lat->height * lat->width;
          const int l = (int)(gcell / plane);
          const int gy = (int)((gcell % plane) / (size_t)lat->width);
          const int gx = (int)(gcell % (size_t)lat->width);
          const int x = gx - (int)net->win_x0, y = gy - (int)net->win_y0;
          if (x < 0 || y < 0 || x >= (int)net->win_w || y >= (int)net->win_h) continue;
          const size_t wi = ((size_t)l * net->win_h + (size_t)y) * net->win_w + (size_t)x;
          own[wi >> 3] |= (uint8_t)(1u << (wi & 7));
        }
      }
      job->costs[i] = dijkstra_run(job->lat, net, 0, NULL, path, cap, path ? &len : NULL, own,
                                   job->cost_own);
      free(own);
      if (job->path_lens) job->path_lens[i] = len;
    } else if (job->kind == 1) {
      uint64_t states = 0, cells = 0;
      job->costs[i] = astar_run(job->lat, net, &states, NULL, 0, NULL,
                                job->expanded_cells ? &cells : NULL);
      if (job->expanded_states) job->expanded_states[i] = states;
      if (job->expanded_cells) job->expanded_cells[i] = cells;
    } else {
      const size_t cells = (size_t)job->lat->layers * net->win_w * net->win_h;
      uint32_t* dist = (uint32_t*)malloc(cells * sizeof(uint32_t));
      job->costs[i] =
          lo_sweep_schedule(job->lat, net, job->max_sweeps, dist, job->stats ? &job->stats[i] : NULL);
      free(dist);
    }
  }
  return NULL;
}

static void run_batch(batch_job* job, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_mutex_init(&job->lock, NULL);
  job->next = 0;
  pthread_t tids[256];
  for (int t = 0; t < threads; ++t) pthread_create(&tids[t], NULL, batch_worker, job);
  for (int t = 0; t < threads; ++t) pthread_join(tids[t], NULL);
  pthread_mutex_destroy(&job->lock);
}

void lo_dijkstra_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                       uint32_t* costs, uint32_t* path_lens, uint64_t* path_offsets,
                       uint32_t* paths, uint64_t path_capacity) {
  batch_job job = {0};
  job.lat = lat;
  job.nets = nets;
  job.count = count;
  job.kind = 0;
  job.costs = costs;
  job.path_lens = path_lens;
  job.path_offsets = path_offsets;
  job.paths = paths;
  job.path_capacity = path_capacity;
  run_batch(&job, threads);
}

void lo_dijkstra_batch_own(const lo_lattice* lat, const lo_net* nets, uint32_t count,
                           int threads, const uint32_t* cell_cost_own,
                           const uint64_t* own_offsets, const uint32_t* own_cells,
                           uint32_t* costs, uint32_t* path_lens, uint64_t* path_offsets,
                           uint32_t* paths, uint64_t path_capacity) {
  batch_job job = {0};
  job.lat = lat;
  job.nets = nets;
  job.count = count;
  job.kind = 0;
  job.cost_own = cell_cost_own;
  job.own_offsets = own_offsets;
  job.own_cells = own_cells;
  job.costs = costs;
  job.path_lens = path_lens;
  job.path_offsets = path_offsets;
  job.paths = paths;
  job.path_capacity = path_capacity;
  run_batch(&job, threads);
}

void lo_astar_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                    uint32_t* costs) {
  lo_astar_batch_ex(lat, nets, count, threads, costs, NULL, NULL);
}

void lo_astar_batch_ex(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                       uint32_t* costs, uint64_t* expanded_states, uint64_t* expanded_cells) {
  batch_job job = {0};
  job.lat = lat;
  job.nets = nets;
  job.count = count;
  job.kind = 1;
  job.costs = costs;
  job.expanded_states = expanded_states;
  job.expanded_cells = expanded_cells;
  run_batch(&job, threads);
}

void lo_sweep_batch(const lo_lattice* lat, const lo_net* nets, uint32_t count, int threads,
                    uint32_t max_sweeps, uint32_t* costs, lo_sweep_stats* stats) {
  batch_job job = {0};
  job.lat = lat;
  job.nets = nets;
  job.count = count;
  job.kind = 2;
  job.max_sweeps = max_sweeps;
  job.costs = costs;
  job.stats = stats;
  run_batch(&job, threads);
}
