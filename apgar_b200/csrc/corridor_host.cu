// C ABI of the corridor CNN's plan-independent operations (corridor_net.cu).
#include <cuda_runtime.h>

#include <cstdint>

#include "apgar_b200.h"
#include "host_common.h"

namespace apgar_b200 {
uint32_t cnn_param_count();
uint32_t cnn_operand_count();
cudaError_t launch_prepare(const float* params, void* operands, cudaStream_t stream);
cudaError_t launch_forward(const float* params, const void* operands, const void* rasters,
                           const uint32_t* dims, uint32_t count, void* const acts[5], float* logits,
                           uint32_t* error, int sm_count, cudaStream_t stream);
cudaError_t launch_backward(const float* params, const void* operands, const void* rasters,
                            const uint32_t* dims, uint32_t count, void* const acts[5],
                            const float* logits, const uint8_t* labels, float pos_weight,
                            float* dlogit, void* scratch0, void* scratch1, float* grads, float* loss,
                            uint32_t* error, int sm_count, cudaStream_t stream);
cudaError_t launch_adam(float* params, const float* grads, float* m, float* v, uint32_t step,
                        float lr, float beta1, float beta2, float eps, cudaStream_t stream);

namespace {
int sm_count_now() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return sms;
}
}  // namespace
}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" uint32_t apgar_b200_cnn_param_count(void) { return cnn_param_count(); }
extern "C" uint32_t apgar_b200_cnn_operand_count(void) { return cnn_operand_count(); }

extern "C" int apgar_b200_cnn_prepare(const float* params, void* operands, void* stream) {
  if (params == nullptr || operands == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "null params or operands");
  }
  APGAR_B200_CUDA("cnn prepare launch", launch_prepare(params, operands, static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_cnn_forward(const float* params, const void* operands, const void* rasters,
                                      const uint32_t* dims, uint32_t count, void* const acts[5],
                                      float* logits, uint32_t* error, void* stream) {
  if (params == nullptr || operands == nullptr || rasters == nullptr || dims == nullptr ||
      acts == nullptr || logits == nullptr || error == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "cnn forward received a null argument");
  }
  for (int l = 0; l < 5; ++l) {
    if (acts[l] == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "null activation buffer");
    if (l > 0 && acts[l] == acts[l - 1]) {
      return set_error(APGAR_B200_INTERNAL_INVARIANT, "consecutive layers need distinct buffers");
    }
  }
  APGAR_B200_CUDA("cnn forward launch",
                  launch_forward(params, operands, rasters, dims, count, acts, logits, error,
                                 sm_count_now(), static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_cnn_backward(const float* params, const void* operands, const void* rasters,
                                       const uint32_t* dims, uint32_t count, void* const acts[5],
                                       const float* logits, const uint8_t* labels, float pos_weight,
                                       float* dlogit, void* scratch0, void* scratch1, float* grads,
                                       float* loss, uint32_t* error, void* stream) {
  if (params == nullptr || operands == nullptr || rasters == nullptr || dims == nullptr ||
      acts == nullptr || logits == nullptr || labels == nullptr || dlogit == nullptr ||
      scratch0 == nullptr || scratch1 == nullptr || scratch0 == scratch1 || grads == nullptr ||
      loss == nullptr || error == nullptr) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "cnn backward received a null or aliased argument");
  }
  for (int l = 0; l < 5; ++l) {
    for (int k = 0; k < l; ++k) {
      if (acts[l] == acts[k]) return set_error(APGAR_B200_INTERNAL_INVARIANT, "training needs five distinct activations");
    }
  }
  const auto s = static_cast<cudaStream_t>(stream);
  APGAR_B200_CUDA("cudaMemsetAsync(grads)", cudaMemsetAsync(grads, 0, cnn_param_count() * sizeof(float), s));
  APGAR_B200_CUDA("cnn backward launch",
                  launch_backward(params, operands, rasters, dims, count, acts, logits, labels,
                                  pos_weight, dlogit, scratch0, scratch1, grads, loss, error,
                                  sm_count_now(), s));
  clear_error();
  return APGAR_B200_OK;
}

extern "C" int apgar_b200_cnn_adam(float* params, const float* grads, float* m, float* v, uint32_t step,
                                   float lr, float beta1, float beta2, float eps, void* stream) {
  if (params == nullptr || grads == nullptr || m == nullptr || v == nullptr || step == 0) {
    return set_error(APGAR_B200_INTERNAL_INVARIANT, "adam needs buffers and a step >= 1");
  }
  APGAR_B200_CUDA("adam launch", launch_adam(params, grads, m, v, step, lr, beta1, beta2, eps,
                                             static_cast<cudaStream_t>(stream)));
  clear_error();
  return APGAR_B200_OK;
}
