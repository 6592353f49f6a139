// Host entry points of the congestion-price kernels (price_update.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "host_common.h"

namespace apgar_b200 {
cudaError_t launch_price_update(uint32_t count, const uint32_t* usage, uint64_t factor,
                                uint64_t next_factor, uint64_t hist_inc, uint64_t capacity,
                                uint64_t max_value, uint64_t* present, uint64_t* history,
                                uint64_t* total, uint64_t* next_cost, uint32_t* next_cost32,
                                uint32_t* next_cost_own32, uint32_t* status,
                                unsigned long long* stats, cudaStream_t stream);
namespace {

// factor = initial + epoch * increment with checked arithmetic
// (NextPresentFactor, negotiated_regeneration_plan.cc:430-442).
bool present_factor(const apgar_b200_price_policy& p, uint64_t epoch, uint64_t* out) {
  const unsigned __int128 f =
      static_cast<unsigned __int128>(epoch) * p.present_factor_increment + p.initial_present_factor;
  if (f > static_cast<unsigned __int128>(~0ull)) return false;
  *out = static_cast<uint64_t>(f);
  return true;
}

}  // namespace
}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" int apgar_b200_price_update_device(uint32_t count, const uint32_t* usage,
                                              const apgar_b200_price_policy* policy, uint64_t epoch,
                                              uint64_t* present, uint64_t* history, uint64_t* total,
                                              uint64_t* next_cost, uint32_t* status, void* stream) {
  if (policy == nullptr || status == nullptr ||
      (count > 0 && (usage == nullptr || present == nullptr || history == nullptr || total == nullptr))) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "price update received a null argument");
  }
  uint64_t factor = 0, next_factor = 0;
  if (!present_factor(*policy, epoch, &factor) ||
      !present_factor(*policy, epoch + 1, &next_factor)) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "present-price schedule overflowed uint64");
  }
  APGAR_B200_CUDA("price update launch",
                  launch_price_update(count, usage, factor, next_factor,
                                      policy->historical_price_increment, policy->capacity,
                                      policy->maximum_value, present, history, total, next_cost,
                                      nullptr, nullptr, status, nullptr,
                                      static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_price_update(uint32_t count, const uint32_t* usage,
                                       const apgar_b200_price_policy* policy, uint64_t epoch,
                                       uint64_t* present, uint64_t* history, uint64_t* total,
                                       uint64_t* next_cost, uint32_t* status) {
  if (policy == nullptr || status == nullptr ||
      (count > 0 && (usage == nullptr || present == nullptr || history == nullptr || total == nullptr))) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "price update received a null argument");
  }
  const size_t n = count;
  DeviceBuffer<uint32_t> d_usage, d_status;
  DeviceBuffer<uint64_t> d_present, d_history, d_total, d_next;
  APGAR_B200_CUDA("cudaMalloc(usage)", d_usage.ensure(n > 0 ? n : 1));
  APGAR_B200_CUDA("cudaMalloc(status)", d_status.ensure(1));
  APGAR_B200_CUDA("cudaMalloc(present)", d_present.ensure(n > 0 ? n : 1));
  APGAR_B200_CUDA("cudaMalloc(history)", d_history.ensure(n > 0 ? n : 1));
  APGAR_B200_CUDA("cudaMalloc(total)", d_total.ensure(n > 0 ? n : 1));
  if (next_cost != nullptr) APGAR_B200_CUDA("cudaMalloc(next)", d_next.ensure(n > 0 ? n : 1));
  if (n > 0) {
    APGAR_B200_CUDA("cudaMemcpy(usage)", cudaMemcpy(d_usage.get(), usage, n * 4, cudaMemcpyHostToDevice));
    APGAR_B200_CUDA("cudaMemcpy(history)", cudaMemcpy(d_history.get(), history, n * 8, cudaMemcpyHostToDevice));
  }
  if (int rc = apgar_b200_price_update_device(count, d_usage.get(), policy, epoch, d_present.get(),
                                              d_history.get(), d_total.get(),
                                              next_cost != nullptr ? d_next.get() : nullptr,
                                              d_status.get(), nullptr);
      rc != APGAR_B200_OK) {
    return rc;
  }
  APGAR_B200_CUDA("cudaMemcpy(status)", cudaMemcpy(status, d_status.get(), 4, cudaMemcpyDeviceToHost));
  if (n > 0) {
    APGAR_B200_CUDA("cudaMemcpy(present)", cudaMemcpy(present, d_present.get(), n * 8, cudaMemcpyDeviceToHost));
    APGAR_B200_CUDA("cudaMemcpy(history)", cudaMemcpy(history, d_history.get(), n * 8, cudaMemcpyDeviceToHost));
    APGAR_B200_CUDA("cudaMemcpy(total)", cudaMemcpy(total, d_total.get(), n * 8, cudaMemcpyDeviceToHost));
    if (next_cost != nullptr) {
      APGAR_B200_CUDA("cudaMemcpy(next)", cudaMemcpy(next_cost, d_next.get(), n * 8, cudaMemcpyDeviceToHost));
    }
  }
  clear_error();
  return APGAR_B200_OK;
}
