// Host helpers shared by the library's translation units: the thread-local
// error slot behind bssn_b200_last_error and the cached SM count.
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace bssn_host {
constexpr int kMaxDev = 64;  // device ordinals with per-device caches
int fail(int code, const std::string& msg);
int cuda_fail(const char* what, cudaError_t e);
int device_sms(int* sms);
}  // namespace bssn_host
