// Shared definitions for the UW12 B200 engine: status codes, error helpers,
// stream-ordered device buffers and launch accounting.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace uw12b {

// Status codes of the C-ABI (mirrors the exception classes of libuw12).
enum Status : int {
  kOk = 0,
  kErrRuntime = 1,  // std::runtime_error in libuw12 (user-input errors)
  kErrLogic = 2,    // std::logic_error in libuw12 (shape errors)
  kErrCuda = 3,
  kErrAlloc = 4,
  kErrInvalid = 5,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void throw_runtime(const std::string& m) { throw Error(kErrRuntime, m); }
[[noreturn]] inline void throw_logic(const std::string& m) { throw Error(kErrLogic, m); }

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    const int code = (e == cudaErrorMemoryAllocation) ? kErrAlloc : kErrCuda;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" +
                          std::to_string(line) + ")");
  }
}

#define UW12_CUDA(expr) ::uw12b::cuda_check((expr), #expr, __FILE__, __LINE__)
#define UW12_LAUNCHED() ::uw12b::note_launch(__FILE__, __LINE__)

// Counts this library's kernel launches (used by benchmarks to report how many
// native launches a call made) and surfaces launch-configuration errors.
void note_launch(const char* file, int line);
unsigned long long launch_count();

// Stream used by every launch of the calling host thread.
cudaStream_t current_stream();
void set_current_stream(cudaStream_t s);

// The library's own stream-ordered memory pool on the current device.  It
// keeps freed memory reserved (release threshold = max) so repeated calls do
// not map and unmap pages; trim_pools() returns it to the system.
cudaMemPool_t library_pool();
void trim_pools();

// Device memory from the library's stream-ordered pool of the current device.
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(size_t n_doubles, cudaStream_t s = nullptr) { alloc(n_doubles, s); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) { release(); p_ = o.p_; n_ = o.n_; s_ = o.s_; o.p_ = nullptr; o.n_ = 0; }
    return *this;
  }
  ~DevBuf() { release(); }

  void alloc(size_t n_doubles, cudaStream_t s = nullptr) {
    release();
    s_ = s ? s : current_stream();
    n_ = n_doubles;
    if (n_)
      UW12_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p_), n_ * sizeof(double),
                                        library_pool(), s_));
  }
  void zero() {
    if (n_) UW12_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(double), s_));
  }
  void release() noexcept {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
  }
  double* get() const { return p_; }
  size_t size() const { return n_; }

 private:
  double* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};

inline size_t packed_size(size_t n) { return n * (n + 1) / 2; }

}  // namespace uw12b
