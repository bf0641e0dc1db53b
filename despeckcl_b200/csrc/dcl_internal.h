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
// Count `n` kernel launches of the calling thread while dcl_profile_begin is active.
void profile_count(int n);

}  // namespace dcl
