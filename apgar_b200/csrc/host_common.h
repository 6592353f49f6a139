// Host-side helpers shared by the C-ABI translation units: error reporting,
// CUDA status mapping and an owning device buffer.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>

#include "apgar_b200.h"

namespace apgar_b200 {

// Records the calling thread's last error detail and returns `status`.
int set_error(int status, const std::string& detail);
void clear_error();

// cudaErrorMemoryAllocation -> kResourceExhausted, every other failure ->
// kBackendFailure (the mapping of gpu/cuda/planar_router.cu:73-78).
int cuda_failure(const char* operation, cudaError_t status);

#define APGAR_B200_CUDA(op, expr)                              \
  do {                                                         \
    const cudaError_t apgar_b200_e_ = (expr);                  \
    if (apgar_b200_e_ != cudaSuccess) return cuda_failure(op, apgar_b200_e_); \
  } while (0)

template <typename T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept
      : ptr_(std::exchange(o.ptr_, nullptr)), count_(std::exchange(o.count_, 0)) {}
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      reset();
      ptr_ = std::exchange(o.ptr_, nullptr);
      count_ = std::exchange(o.count_, 0);
    }
    return *this;
  }
  ~DeviceBuffer() { reset(); }

  // Grows to at least `count` elements (contents are not preserved).
  cudaError_t ensure(size_t count) {
    if (count <= count_) return cudaSuccess;
    reset();
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) return e;
    ptr_ = static_cast<T*>(p);
    count_ = count;
    return cudaSuccess;
  }
  void reset() noexcept {
    if (ptr_ != nullptr) cudaFree(ptr_);
    ptr_ = nullptr;
    count_ = 0;
  }
  T* get() const noexcept { return ptr_; }
  size_t count() const noexcept { return count_; }
  size_t bytes() const noexcept { return count_ * sizeof(T); }

 private:
  T* ptr_ = nullptr;
  size_t count_ = 0;
};

}  // namespace apgar_b200
