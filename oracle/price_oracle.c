/*
 * Congestion-price CPU oracle.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates, with checked uint64 arithmetic:
 *  - allocator epoch prices, NextPresentFactor and the per-resource update of
 *    src/allocator/negotiated_regeneration_plan.cc:430-442 and :676-760;
 *  - CS-RR-v1 snapshot costs, src/allocator/cpu_sequential_negotiated_routing.cc:299-505;
 *  - CS-RR-v1 history update, same file :1300-1330;
 *  - usage / overuse accumulation, src/allocator/resource_accounting.cc:180-230
 *    (here over cell resources: one usage unit per path cell).
 */
#include "oracle.h"

static int mul_checked(uint64_t a, uint64_t b, uint64_t* out) {
  if (a != 0 && b > UINT64_MAX / a) return 0;
  *out = a * b;
  return 1;
}

static int add_checked(uint64_t a, uint64_t* acc) {
  if (*acc > UINT64_MAX - a) return 0;
  *acc += a;
  return 1;
}

int po_epoch_update(uint32_t count, const uint64_t* usage, uint64_t capacity, uint64_t epoch,
                    uint64_t init_factor, uint64_t factor_inc, uint64_t hist_inc,
                    uint64_t* present, uint64_t* history, uint64_t* total) {
  uint64_t steps, factor = init_factor;
  if (!mul_checked(epoch, factor_inc, &steps) || !add_checked(steps, &factor)) return 1;
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t overuse = usage[i] > capacity ? usage[i] - capacity : 0;
    if (overuse == 0) {
      present[i] = 0;
      total[i] = history[i];
      continue;
    }
    uint64_t p, hi;
    if (!mul_checked(factor, overuse, &p) || !mul_checked(hist_inc, overuse, &hi)) return 1;
    uint64_t h = history[i];
    if (!add_checked(hi, &h)) return 1;
    uint64_t t = p;
    if (!add_checked(h, &t)) return 1;
    present[i] = p;
    history[i] = h;
    total[i] = t;
  }
  return 0;
}

int po_snapshot_costs(uint32_t count, const uint64_t* usage, const uint64_t* history,
                      uint64_t capacity, uint32_t pass_index, uint64_t init_present,
                      uint64_t present_inc, uint64_t max_value, uint64_t* cost) {
  uint64_t inc, factor = init_present;
  if (!mul_checked(pass_index, present_inc, &inc) || !add_checked(inc, &factor)) return 1;
  for (uint32_t i = 0; i < count; ++i) {
    if (usage[i] == UINT64_MAX) return 1;
    const uint64_t predicted = usage[i] + 1;
    const uint64_t over = predicted > capacity ? predicted - capacity : 0;
    uint64_t p;
    if (!mul_checked(factor, over, &p)) return 1;
    uint64_t c = history[i];
    if (!add_checked(p, &c)) return 1;
    if (c > max_value) return 2;
    cost[i] = c;
  }
  return 0;
}

int po_history_update(uint32_t count, const uint64_t* usage, uint64_t capacity,
                      uint64_t hist_inc, uint64_t max_value, uint64_t* history) {
  for (uint32_t i = 0; i < count; ++i) {
    const uint64_t over = usage[i] > capacity ? usage[i] - capacity : 0;
    if (over == 0) continue;
    uint64_t inc;
    if (!mul_checked(over, hist_inc, &inc)) return 1;
    uint64_t h = history[i];
    if (!add_checked(inc, &h)) return 1;
    if (h > max_value) return 2;
    history[i] = h;
  }
  return 0;
}

void po_accumulate_cells(uint32_t path_count, const uint64_t* offsets, const uint32_t* lengths,
                         const uint32_t* cells, uint32_t cell_count, uint32_t* usage) {
  for (uint32_t p = 0; p < path_count; ++p) {
    for (uint32_t i = 0; i < lengths[p]; ++i) {
      const uint32_t c = cells[offsets[p] + i];
      if (c < cell_count) usage[c] += 1;
    }
  }
}
