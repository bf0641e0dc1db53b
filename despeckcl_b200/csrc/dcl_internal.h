// Internal helpers shared by the host translation units of the library.
#pragma once

#include <cuda_runtime.h>

namespace dcl {

// Record a message for dcl_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
// Map a CUDA error to a dcl_status (recording the message).
int cuda_error(cudaError_t e, const char* where);
// Current device, its stream-ordered pool set to keep freed scratch between
// calls (once per device).
int ensure_device_ready(int& dev);
// Devices a process may use (per-device caches are sized by it).
constexpr int kMaxDevices = 64;
// Allows `func` up to `bytes` of dynamic shared memory on the current device
// (the limit is a per-device attribute); `cache` holds, per device, the
// largest size already allowed, so repeated launches skip the call.
cudaError_t allow_dynamic_smem(const void* func, size_t bytes, size_t* cache);
// Count `n` kernel launches of the calling thread while dcl_profile_begin is active.
void profile_count(int n);

}  // namespace dcl
