// device.hpp -- host-side CUDA plumbing: error checks and owned device arrays.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>
#include <string>
#include <utility>

namespace gample {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define GP_CUDA(call)                                                                               \
  do {                                                                                              \
    cudaError_t gp_err_ = (call);                                                                   \
    if (gp_err_ != cudaSuccess)                                                                     \
      throw ::gample::CudaError(gp_err_, std::string(#call) + " failed at " + __FILE__ + ":" +      \
                                             std::to_string(__LINE__) + ": " +                      \
                                             cudaGetErrorString(gp_err_));                           \
  } while (0)

// Every kernel launch is followed by GP_LAUNCH_CHECK(), which also counts it
// (gp_kernel_launches() in the C ABI).
void note_kernel_launch();
void add_kernel_launches(long long n);  // graph launches; negative to uncount captured kernels
unsigned long long kernel_launches();
unsigned long long thread_kernel_launches();  // launches issued by the calling host thread
#define GP_LAUNCH_CHECK()              \
  do {                                 \
    ::gample::note_kernel_launch();    \
    GP_CUDA(cudaGetLastError());       \
  } while (0)

// Device memory comes from the current device's default stream-ordered pool
// with an unbounded release threshold: a freed block stays with the process
// and serves a later allocation of the same size without the driver mapping
// (or, on free, unmapping) the memory again, which for the multi-GB particle
// stores costs tens of milliseconds to seconds per simulation created or
// closed. device_free() first waits for the device, as cudaFree does, since
// the library's streams do not synchronise with the default stream.
// release_cached_device_memory() returns the cached blocks to the driver.
void* device_alloc(size_t bytes);

// A CUDA event with timing, destroyed with its owner.
class TimingEvent {
 public:
  TimingEvent() { GP_CUDA(cudaEventCreate(&e_)); }
  ~TimingEvent() {
    if (e_) cudaEventDestroy(e_);
  }
  TimingEvent(const TimingEvent&) = delete;
  TimingEvent& operator=(const TimingEvent&) = delete;
  cudaEvent_t get() const { return e_; }

 private:
  cudaEvent_t e_ = nullptr;
};
void device_free(void* p);
void release_cached_device_memory();

// Page-locked host memory for the small diagnostics read-backs. Freed blocks
// are kept per size and handed out again: cudaMallocHost costs 1-3 ms per
// call, which every simulation created would pay for each of its read-back
// buffers. release_cached_device_memory() frees the kept blocks as well.
void* pinned_alloc(size_t bytes);
void pinned_free(void* p, size_t bytes);

// Owned device allocation of n elements of T (not initialised unless asked).
template <typename T>
class DeviceArray {
 public:
  DeviceArray() = default;
  explicit DeviceArray(size_t n, bool zero = false) { resize(n, zero); }
  ~DeviceArray() { release(); }
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  DeviceArray& operator=(DeviceArray&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_;
      n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  void resize(size_t n, bool zero = false) {
    release();
    if (n) {
      p_ = static_cast<T*>(device_alloc(n * sizeof(T)));
      n_ = n;
      if (zero) GP_CUDA(cudaMemset(p_, 0, n * sizeof(T)));
    }
  }
  // Grow to at least n elements keeping the first `keep` elements.
  void grow(size_t n, size_t keep, cudaStream_t s) {
    if (n <= n_) return;
    T* q = static_cast<T*>(device_alloc(n * sizeof(T)));
    if (p_ && keep) GP_CUDA(cudaMemcpyAsync(q, p_, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
    GP_CUDA(cudaStreamSynchronize(s));
    release();
    p_ = q;
    n_ = n;
  }
  void zero(cudaStream_t s) {
    if (n_) GP_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  size_t bytes() const { return n_ * sizeof(T); }

 private:
  void release() {
    if (p_) device_free(p_);
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  size_t n_ = 0;
};

// Pinned host buffer for asynchronous diagnostics read-back.
template <typename T>
class PinnedArray {
 public:
  PinnedArray() = default;
  explicit PinnedArray(size_t n) { resize(n); }
  ~PinnedArray() {
    if (p_) pinned_free(p_, n_ * sizeof(T));
  }
  PinnedArray(const PinnedArray&) = delete;
  PinnedArray& operator=(const PinnedArray&) = delete;
  void resize(size_t n) {
    if (p_) pinned_free(p_, n_ * sizeof(T));
    p_ = nullptr;
    n_ = 0;
    if (n) p_ = static_cast<T*>(pinned_alloc(n * sizeof(T)));
    n_ = n;
  }
  T* get() const { return p_; }
  T& operator[](size_t i) { return p_[i]; }
  size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  size_t n_ = 0;
};

}  // namespace gample
