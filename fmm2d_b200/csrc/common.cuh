// Shared helpers for the fmm2d_b200 CUDA library (sm_100a).
#pragma once
#include <mutex>
#include <utility>
#include <vector>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <atomic>
#include <stdexcept>
#include <string>
#include <vector>

namespace b2 {

// Error codes returned through `ier` (the reference uses 0 = ok,
// 4 = allocation failure, 13 = expansion order too large).
enum {
  IER_OK = 0,
  IER_ALLOC = 4,
  IER_NTERMS = 13,
  IER_HIGHFREQ = 20,  // Helmholtz boxes above 16 wavelengths (wideband translations)
  IER_BADARG = 100,  // invalid argument (sizes, flags)
  IER_CUDA = 101,    // CUDA runtime error
  IER_TIMEOUT = 102,  // a bounded device wait gave up
  IER_NOALLOC_TOO_LARGE = 103,  // problem exceeds a fixed static scratch array
  IER_TREE_LIMIT = 104  // an asynchronous call's tree needed more boxes or levels than a
                        // call without read-back allows: repeat it synchronously
};

struct CudaError : public std::runtime_error {
  int ier;
  CudaError(const std::string& m, int code) : std::runtime_error(m), ier(code) {}
};

#define B2_CHECK(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      throw ::b2::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_),          \
                            e_ == cudaErrorMemoryAllocation ? ::b2::IER_ALLOC            \
                                                            : ::b2::IER_CUDA);           \
    }                                                                                    \
  } while (0)

// Every kernel launch of the library is followed by B2_LAUNCH_CHECK(), which
// also counts it (b2fmm_kernel_launches()).
extern std::atomic<unsigned long long> g_launches;
#define B2_LAUNCH_CHECK()                                         \
  do {                                                            \
    ::b2::g_launches.fetch_add(1, std::memory_order_relaxed);     \
    B2_CHECK(cudaGetLastError());                                 \
  } while (0)

// Test hook: true exactly once, on the allocation that b2fmm_test_fail_alloc
// asked to fail (the library then reports IER_ALLOC as for a real failure).
bool alloc_fault_due();

// Stream-ordered device buffer (cudaMallocAsync from the device's default pool).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DBuf() {}
  explicit DBuf(cudaStream_t st) : s(st) {}
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; s = o.s;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count, cudaStream_t st) {
    release();
    s = st;
    n = count;
    if (count) {
      if (alloc_fault_due()) throw CudaError("injected allocation failure (test hook)", IER_ALLOC);
      B2_CHECK(cudaMallocAsync((void**)&p, count * sizeof(T), st));
    }
  }
  // grow to at least `count` elements keeping the first `keep` elements
  void grow(size_t count, size_t keep) {
    if (count <= n) return;
    T* q = nullptr;
    if (alloc_fault_due()) throw CudaError("injected allocation failure (test hook)", IER_ALLOC);
    B2_CHECK(cudaMallocAsync((void**)&q, count * sizeof(T), s));
    if (p && keep) B2_CHECK(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
    if (p) cudaFreeAsync(p, s);
    p = q;
    n = count;
  }
  void zero(size_t count) {
    if (count) B2_CHECK(cudaMemsetAsync(p, 0, count * sizeof(T), s));
  }
  void fill_bytes(int v, size_t count) {
    if (count) B2_CHECK(cudaMemsetAsync(p, v, count * sizeof(T), s));
  }
};

// Raise a kernel's dynamic shared-memory limit when a launch needs more than
// the default 48 KB.  Each (kernel, device) pair is set once per size, so
// repeated launches (and launches under stream capture) make no further calls.
template <typename K>
void set_smem_attr(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return;
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, int>, size_t>> done;
  int dev = 0;
  B2_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  for (auto& e : done)
    if (e.first.first == (const void*)kernel && e.first.second == dev && e.second >= bytes) return;
  B2_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  done.push_back({{(const void*)kernel, dev}, bytes});
}

// Keep freed memory in the pool between calls so repeated FMMs do not pay
// for cudaMalloc (the pool is per device and shared by all streams).
void configure_mempool(int device);

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// complex helpers on double2 / float2
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}
// a += b*c
__host__ __device__ __forceinline__ void cfma(double2& a, double2 b, double2 c) {
  a.x += b.x * c.x - b.y * c.y;
  a.y += b.x * c.y + b.y * c.x;
}
// complex reciprocal 1/z (one division: conj(z) * (1 / |z|^2))
__host__ __device__ __forceinline__ double2 crcp(double2 z) {
  const double id = 1.0 / (z.x * z.x + z.y * z.y);
  return make_double2(z.x * id, -z.y * id);
}
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, crcp(b)); }

__host__ __device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// 64-bit Morton-style digit of a point at tree level lev (1-based):
// digit = 2*(y >= cy) + (x >= cx) of the box being split at lev-1.
__host__ __device__ __forceinline__ int key_digit(uint64_t hi, uint64_t lo, int lev) {
  return lev <= 32 ? (int)((hi >> (64 - 2 * lev)) & 3ull)
                   : (int)((lo >> (64 - 2 * (lev - 32))) & 3ull);
}

}  // namespace b2
