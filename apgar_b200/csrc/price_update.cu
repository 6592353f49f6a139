// Negotiated-congestion prices as fused integer kernels.
//
// accumulate: one block per net adds a usage unit for every cell of its
// packed reverse path (integer atomics, so the result is order independent).
// price update: one thread per resource computes overuse, the allocator
// epoch present / history / total prices and the CS-RR next-pass snapshot
// cost in one pass with checked uint64 arithmetic (reference
// negotiated_regeneration_plan.cc:676-760, cpu_sequential_negotiated_routing.cc
// :299-505 and :1300-1330, resource_accounting.cc:212-213).
#include <cuda_runtime.h>

#include <cstdint>

#include "apgar_b200.h"

namespace apgar_b200 {
namespace {

struct PriceParams {
  uint64_t factor;       // initial + epoch * increment (checked on the host)
  uint64_t next_factor;  // initial + (epoch + 1) * increment
  uint64_t hist_inc;
  uint64_t capacity;
  uint64_t max_value;
};

__device__ __forceinline__ bool mul_checked(uint64_t a, uint64_t b, uint64_t* out) {
  if (a != 0 && b > ~0ull / a) return false;
  *out = a * b;
  return true;
}

__device__ __forceinline__ bool add_checked(uint64_t a, uint64_t b, uint64_t* out) {
  if (a > ~0ull - b) return false;
  *out = a + b;
  return true;
}

__global__ void price_update_kernel(uint32_t count, const uint32_t* __restrict__ usage,
                                    PriceParams pp, uint64_t* __restrict__ present,
                                    uint64_t* __restrict__ history, uint64_t* __restrict__ total,
                                    uint64_t* __restrict__ next_cost,
                                    uint32_t* __restrict__ next_cost32,
                                    uint32_t* __restrict__ next_cost_own32, uint32_t* status,
                                    unsigned long long* stats) {
  uint32_t flags = 0;
  unsigned long long overused = 0, overuse_sum = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint64_t u = usage[i];
    const uint64_t over = u > pp.capacity ? u - pp.capacity : 0;
    overused += over != 0 ? 1ull : 0ull;
    overuse_sum += over;
    uint64_t h = history[i];
    uint64_t p = 0;
    if (over != 0) {
      uint64_t inc;
      if (!mul_checked(pp.factor, over, &p) || !mul_checked(pp.hist_inc, over, &inc) ||
          !add_checked(h, inc, &h)) {
        flags |= APGAR_B200_PRICE_OVERFLOW;
        p = ~0ull;
        h = ~0ull;
      } else if (h > pp.max_value) {
        flags |= APGAR_B200_PRICE_BOUND;
      }
    }
    uint64_t t;
    if (!add_checked(p, h, &t)) {
      flags |= APGAR_B200_PRICE_OVERFLOW;
      t = ~0ull;
    }
    if (present != nullptr) present[i] = p;
    history[i] = h;
    if (total != nullptr) total[i] = t;
    if (next_cost != nullptr || next_cost32 != nullptr) {
      const uint64_t predicted = u + 1;
      const uint64_t pover = predicted > pp.capacity ? predicted - pp.capacity : 0;
      uint64_t c, pc;
      if (!mul_checked(pp.next_factor, pover, &pc) || !add_checked(h, pc, &c)) {
        flags |= APGAR_B200_PRICE_OVERFLOW;
        c = ~0ull;
      } else if (c > pp.max_value) {
        flags |= APGAR_B200_PRICE_BOUND;
      }
      if (next_cost != nullptr) next_cost[i] = c;
      // the search reads a 32-bit entry price; a larger cost saturates to the
      // label sentinel, so any path through the cell is rejected, never wrong
      if (next_cost32 != nullptr) next_cost32[i] = c < 0x7FFFFFFFull ? static_cast<uint32_t>(c) : 0x7FFFFFFFu;
      if (next_cost_own32 != nullptr) {
        // the same snapshot for a net whose own previous path holds one of
        // the u units: the reference rips that net up before pricing, so it
        // sees u - 1 other uses (u - 1 + 1 - capacity).  c_own <= c, so no
        // new overflow or bound can arise here.
        const uint64_t oover = u > pp.capacity ? u - pp.capacity : 0;
        uint64_t co, opc;
        if (!mul_checked(pp.next_factor, oover, &opc) || !add_checked(h, opc, &co)) co = ~0ull;
        next_cost_own32[i] = co < 0x7FFFFFFFull ? static_cast<uint32_t>(co) : 0x7FFFFFFFu;
      }
    }
  }
  flags = __reduce_or_sync(0xFFFFFFFFu, flags);
  if (flags != 0u && (threadIdx.x & 31) == 0) atomicOr(status, flags);
  if (stats != nullptr) {
    for (int o = 16; o > 0; o >>= 1) {
      overused += __shfl_xor_sync(0xFFFFFFFFu, overused, o);
      overuse_sum += __shfl_xor_sync(0xFFFFFFFFu, overuse_sum, o);
    }
    if ((threadIdx.x & 31) == 0 && (overused | overuse_sum) != 0ull) {
      atomicAdd(stats, overused);
      atomicAdd(stats + 1, overuse_sum);
    }
  }
}

__global__ void accumulate_cells_kernel(const apgar_b200_lattice_result* __restrict__ results,
                                        uint32_t count, const uint32_t* __restrict__ paths,
                                        uint32_t* usage, uint64_t cell_count) {
  for (uint32_t n = blockIdx.x; n < count; n += gridDim.x) {
    const apgar_b200_lattice_result r = results[n];
    if (r.completion != APGAR_B200_COMPLETION_REACHED) continue;
    for (uint32_t j = threadIdx.x; j < r.path_len; j += blockDim.x) {
      const uint32_t c = paths[r.path_offset + j];
      if (c < cell_count) atomicAdd(usage + c, 1u);
    }
  }
}

// Partial rip-up: a net keeps its route (skip = 1) when it reached its goal
// and no cell of its path is overused; otherwise it is rerouted.
__global__ void mark_dirty_kernel(const apgar_b200_lattice_result* __restrict__ results,
                                  uint32_t count, const uint32_t* __restrict__ paths,
                                  const uint32_t* __restrict__ usage, uint64_t cell_count,
                                  uint32_t capacity, uint8_t* __restrict__ skip) {
  const int lane = threadIdx.x & 31;
  for (uint32_t n = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); n < count;
       n += gridDim.x * (blockDim.x / 32)) {
    const apgar_b200_lattice_result r = results[n];
    bool dirty = r.completion != APGAR_B200_COMPLETION_REACHED;
    for (uint32_t j = lane; !dirty && j < r.path_len; j += 32) {
      const uint32_t c = paths[r.path_offset + j];
      if (c >= cell_count || usage[c] > capacity) dirty = true;
    }
    dirty = __any_sync(0xFFFFFFFFu, dirty);
    if (lane == 0) skip[n] = dirty ? 0u : 1u;
  }
}

}  // namespace

cudaError_t launch_mark_dirty(const apgar_b200_lattice_result* results, uint32_t count,
                              const uint32_t* paths, const uint32_t* usage, uint64_t cell_count,
                              uint32_t capacity, uint8_t* skip, int sm_count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  const uint32_t warps = 8;
  const uint32_t cap = static_cast<uint32_t>(sm_count > 0 ? sm_count * 16 : 2048);
  const uint32_t blocks = (count + warps - 1) / warps;
  mark_dirty_kernel<<<blocks < cap ? blocks : cap, warps * 32, 0, stream>>>(
      results, count, paths, usage, cell_count, capacity, skip);
  return cudaGetLastError();
}

cudaError_t launch_price_update(uint32_t count, const uint32_t* usage, uint64_t factor,
                                uint64_t next_factor, uint64_t hist_inc, uint64_t capacity,
                                uint64_t max_value, uint64_t* present, uint64_t* history,
                                uint64_t* total, uint64_t* next_cost, uint32_t* next_cost32,
                                uint32_t* next_cost_own32, uint32_t* status,
                                unsigned long long* stats, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
  if (e == cudaSuccess && stats != nullptr) {
    e = cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), stream);
  }
  if (e != cudaSuccess || count == 0) return e;
  PriceParams pp{factor, next_factor, hist_inc, capacity, max_value};
  const uint32_t blocks = (count + 255u) / 256u;
  price_update_kernel<<<blocks < 148u * 16u ? blocks : 148u * 16u, 256, 0, stream>>>(
      count, usage, pp, present, history, total, next_cost, next_cost32, next_cost_own32, status,
      stats);
  return cudaGetLastError();
}

cudaError_t launch_accumulate_cells(const apgar_b200_lattice_result* results, uint32_t count,
                                    const uint32_t* paths, uint32_t* usage, uint64_t cell_count,
                                    int sm_count, cudaStream_t stream) {
  if (count == 0) return cudaSuccess;
  const uint32_t cap = static_cast<uint32_t>(sm_count > 0 ? sm_count * 8 : 1024);
  accumulate_cells_kernel<<<count < cap ? count : cap, 128, 0, stream>>>(results, count, paths,
                                                                        usage, cell_count);
  return cudaGetLastError();
}

}  // namespace apgar_b200
