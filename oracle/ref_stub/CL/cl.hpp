// TEST INFRASTRUCTURE ONLY: the few OpenCL C++ names that the reference's
// host-side smoothing step (src/compute/nlinsar/smoothing.cpp) uses, over host
// memory, so that file compiles and runs on the CPU in oracle/_ref.
#pragma once
#include <cstddef>
#include <cstring>

#ifndef CL_TRUE
#define CL_TRUE 1
#endif

namespace cl {
struct Buffer {
  void* host = nullptr;
  Buffer() {}
  explicit Buffer(void* p) : host(p) {}
};
struct CommandQueue {
  int enqueueReadBuffer(const Buffer& b, int, size_t off, size_t n, void* dst, const void* = nullptr,
                        void* = nullptr) const {
    std::memcpy(dst, static_cast<char*>(b.host) + off, n);
    return 0;
  }
  int enqueueWriteBuffer(const Buffer& b, int, size_t off, size_t n, const void* src, const void* = nullptr,
                         void* = nullptr) const {
    std::memcpy(static_cast<char*>(b.host) + off, src, n);
    return 0;
  }
};
}  // namespace cl
