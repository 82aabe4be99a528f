// Shared host/device helpers: status errors, CUDA/cuBLAS/cuSOLVER checks,
// RAII device buffers and complex arithmetic on double2/float2.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace hb {

enum Status : int {
  kSuccess = 0,
  kInvalidArgument = 1,
  kIO = 2,
  kInvalidHandle = 3,
  kCapacity = 4,
  kUnavailable = 5,
  kInternal = 6
};

// Every failure inside the library surfaces as one of these; the C ABI layer
// turns it into a status code and an error string (the reference aborts the
// process on device errors instead, src/half_cuda_assembly.cuf:477-479).
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(int status, const std::string& msg) { throw Error(status, msg); }

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) fail(kInternal, std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
}
inline void cublas_check(cublasStatus_t s, const char* what) {
  if (s != CUBLAS_STATUS_SUCCESS) fail(kInternal, std::string("cuBLAS ") + what + " failed (" + std::to_string(int(s)) + ")");
}
inline void cusolver_check(cusolverStatus_t s, const char* what) {
  if (s != CUSOLVER_STATUS_SUCCESS) fail(kInternal, std::string("cuSOLVER ") + what + " failed (" + std::to_string(int(s)) + ")");
}
#define HALF_CUDA(x) ::hb::cuda_check((x), #x)
#define HALF_LAUNCH(what) ::hb::cuda_check(cudaGetLastError(), what)

// With HALF_TRACE_ALLOC set, device allocations and frees slower than 5 ms are
// reported (they synchronise the device and stall the host).
struct AllocTimer {
  const char* what;
  size_t bytes;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  AllocTimer(const char* w, size_t b) : what(w), bytes(b) {}
  ~AllocTimer() {
    static const bool on = std::getenv("HALF_TRACE_ALLOC") != nullptr;
    if (!on) return;
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ms > 5.0) std::fprintf(stderr, "HALF slow %s: %.1f ms (%zu bytes)\n", what, ms, bytes);
  }
};

void* device_alloc(size_t bytes, size_t* granted);   // devmem.cpp: caching allocator
void device_free(void* p, size_t granted);

// Owning device allocation through the caching allocator (devmem.h).
// Allocation failure is reported, never fatal.
template <typename T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t n) { resize(n); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : p_(o.p_), n_(o.n_), cap_(o.cap_) { o.p_ = nullptr; o.n_ = o.cap_ = 0; }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_; n_ = o.n_; cap_ = o.cap_;
      o.p_ = nullptr; o.n_ = o.cap_ = 0;
    }
    return *this;
  }
  void resize(size_t n) {
    if (n == n_) return;
    release();
    if (n) p_ = static_cast<T*>(device_alloc(n * sizeof(T), &cap_));
    n_ = n;
  }
  void release() {
    if (p_) device_free(p_, cap_);
    p_ = nullptr;
    n_ = cap_ = 0;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }
  void upload(const T* h, size_t n, cudaStream_t s = 0) {
    if (n > n_) resize(n);
    HALF_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& v, cudaStream_t s = 0) { upload(v.data(), v.size(), s); }
  std::vector<T> download(cudaStream_t s = 0) const {
    std::vector<T> h(n_);
    if (n_) {
      HALF_CUDA(cudaMemcpyAsync(h.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s));
      HALF_CUDA(cudaStreamSynchronize(s));
    }
    return h;
  }
  void zero(cudaStream_t s = 0) {
    if (n_) HALF_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }

 private:
  T* p_ = nullptr;
  size_t n_ = 0, cap_ = 0;   // elements, granted bytes
};

// ---- complex helpers (double2 / float2) -----------------------------------
template <typename R> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };
template <typename R> using cplx_t = typename Cplx<R>::type;

__host__ __device__ inline double2 cmake(double x, double y) { return make_double2(x, y); }
__host__ __device__ inline float2 cmake(float x, float y) { return make_float2(x, y); }
template <typename C> __host__ __device__ inline C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __host__ __device__ inline C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __host__ __device__ inline C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <typename C> __host__ __device__ inline C cconjmul(C a, C b) {  // conj(a)*b
  C r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
template <typename C, typename R> __host__ __device__ inline C cscale(C a, R s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }

inline int ceil_div(long long a, long long b) { return int((a + b - 1) / b); }

// Raise, never lower, a kernel's dynamic shared-memory limit on the current
// device.  The limit is a property of the function shared by every thread of
// the process, so concurrent callers with different launch sizes (k points
// whose sphere spans a different number of planes) must not shrink each
// other's limit between the set and the launch.
template <typename F>
void raise_smem_limit(F* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> limits;
  if (bytes <= 48 * 1024) return;
  int dev = 0;
  HALF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  size_t& cur = limits[{dev, reinterpret_cast<const void*>(kernel)}];
  if (bytes <= cur) return;
  HALF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  cur = bytes;
}

}  // namespace hb
