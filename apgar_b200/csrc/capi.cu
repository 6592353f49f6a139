// C-ABI plumbing shared by every entry point: version, thread-local error
// detail, CUDA status mapping and device metadata.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>

#include "host_common.h"

namespace apgar_b200 {
namespace {
thread_local std::string g_last_error;
}

int set_error(int status, const std::string& detail) {
  g_last_error = detail;
  return status;
}

void clear_error() { g_last_error.clear(); }

int cuda_failure(const char* operation, cudaError_t status) {
  const int code = status == cudaErrorMemoryAllocation ? APGAR_B200_RESOURCE_EXHAUSTED
                                                       : APGAR_B200_BACKEND_FAILURE;
  return set_error(code, std::string(operation) + " failed: " + cudaGetErrorString(status));
}

}  // namespace apgar_b200

using namespace apgar_b200;

extern "C" uint32_t apgar_b200_abi_version(void) { return APGAR_B200_ABI_VERSION; }

extern "C" size_t apgar_b200_last_error(char* buffer, size_t capacity) {
  const std::string& e = g_last_error;
  if (buffer != nullptr && capacity > 0) {
    const size_t n = e.size() < capacity - 1 ? e.size() : capacity - 1;
    std::memcpy(buffer, e.data(), n);
    buffer[n] = '\0';
  }
  return e.size();
}

extern "C" int apgar_b200_query_metadata(apgar_b200_metadata* out) {
  if (out == nullptr) return set_error(APGAR_B200_INTERNAL_INVARIANT, "metadata output is null");
  int device = 0;
  APGAR_B200_CUDA("cudaGetDevice", cudaGetDevice(&device));
  cudaDeviceProp prop{};
  APGAR_B200_CUDA("cudaGetDeviceProperties", cudaGetDeviceProperties(&prop, device));
  int runtime = 0, driver = 0;
  APGAR_B200_CUDA("cudaRuntimeGetVersion", cudaRuntimeGetVersion(&runtime));
  APGAR_B200_CUDA("cudaDriverGetVersion", cudaDriverGetVersion(&driver));
  std::memset(out, 0, sizeof(*out));
  std::snprintf(out->device_name, sizeof(out->device_name), "%s", prop.name);
  for (int i = 0; i < 16; ++i) {
    std::snprintf(out->device_uuid + 2 * i, 3, "%02x",
                  static_cast<unsigned>(static_cast<unsigned char>(prop.uuid.bytes[i])));
  }
  out->compute_capability_major = static_cast<uint32_t>(prop.major);
  out->compute_capability_minor = static_cast<uint32_t>(prop.minor);
  out->runtime_version = static_cast<uint32_t>(runtime);
  out->driver_version = static_cast<uint32_t>(driver);
  out->global_memory_bytes = prop.totalGlobalMem;
  out->multiprocessor_count = static_cast<uint32_t>(prop.multiProcessorCount);
  clear_error();
  return APGAR_B200_OK;
}
