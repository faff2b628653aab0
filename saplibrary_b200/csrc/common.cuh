// Shared utilities of the sap_b200 library: error plumbing, device buffers,
// launch accounting and the asynchronous-copy PTX wrappers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <unordered_map>
#include <utility>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sap_b200.h"

namespace sapb {

// Library failure carrying a C-ABI status code.  Reference failures use the
// sap::system_error::Reason values (sap/exception.h:16-23).
#ifndef SAPB_ERROR_DEFINED
#define SAPB_ERROR_DEFINED
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
#endif

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? SAP_ERR_OUT_OF_MEMORY : SAP_ERR_CUDA;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define SAPB_CUDA(x) ::sapb::cuda_check((x), #x)

// Message returned by sap_last_error() on the calling thread.
void set_last_error(const std::string& msg);

// Number of kernels enqueued by this library (reported by the bench).
extern std::atomic<int64_t> g_launches;
extern std::atomic<int64_t> g_lib_calls;
inline void count_launch(int k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }
inline void count_lib_call() { g_lib_calls.fetch_add(1, std::memory_order_relaxed); }
#define SAPB_LAUNCHED() do { ::sapb::count_launch(); SAPB_CUDA(cudaGetLastError()); } while (0)

// Event bracketing of the launches of one selected kernel (sap_profile_*).
struct ProfScope {
  bool on = false;
  cudaStream_t s = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(const char* name, cudaStream_t st);
  ~ProfScope();
};
#define SAPB_PROF(name, stream) ::sapb::ProfScope _sapb_prof_scope(name, stream)

// Owning device buffer (stream-ordered allocation on the solver's stream).
template <typename T>
class DBuf {
 public:
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept { swap(o); }
  DBuf& operator=(DBuf&& o) noexcept { release(); swap(o); return *this; }
  ~DBuf() { release(); }

  void alloc(size_t n) {
    if (n == n_ && p_) return;
    release();
    n_ = n;
    if (n) SAPB_CUDA(cudaMalloc(&p_, n * sizeof(T)));
  }
  // grow-only: at least n elements (a smaller request keeps the buffer)
  void ensure(size_t n) {
    if (n > n_ || !p_) alloc(n);
  }
  // ensure(n) and copy n host elements to the front
  void put(const T* h, size_t n, cudaStream_t s) {
    ensure(n);
    if (n) SAPB_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void put(const std::vector<T>& h, cudaStream_t s) { put(h.data(), h.size(), s); }
  void zero(cudaStream_t s) {
    if (n_) SAPB_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }
  void upload(const T* h, size_t n, cudaStream_t s) {
    alloc(n);
    if (n) SAPB_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
  void download(std::vector<T>& h, cudaStream_t s) const {
    h.resize(n_);
    if (n_) SAPB_CUDA(cudaMemcpyAsync(h.data(), p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  void release() {
    if (p_) cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  T* get() const { return p_; }
  size_t size() const { return n_; }

 private:
  void swap(DBuf& o) { std::swap(p_, o.p_); std::swap(n_, o.n_); }
  T* p_ = nullptr;
  size_t n_ = 0;
};

// Allocator whose value construction leaves trivially constructible elements
// uninitialised: a HostVec resized to hold a copy is first touched by the
// (parallel) copy itself instead of being zero-filled by one thread.
template <typename T>
struct DefaultInitAllocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = DefaultInitAllocator<U>;
  };
  DefaultInitAllocator() = default;
  template <typename U>
  DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <typename T>
using HostVec = std::vector<T, DefaultInitAllocator<T>>;

// Page-locked host blocks kept for reuse (PinnedPoolAllocator): a block
// released by one host copy of a matrix is taken by the next copy that fits
// in it (at most twice its size), so repeated copies neither fault in fresh
// pages nor go through the driver's pageable staging when they are
// uploaded.  Free blocks beyond kMaxFreeBytes go back to the driver, largest
// first.  Where page-locked memory cannot be had, blocks come from malloc.
// The pool is never destroyed (no driver call during static teardown).
class PinnedPool {
 public:
  static PinnedPool& instance() {
    static PinnedPool* pool = new PinnedPool();
    return *pool;
  }
  void* take(size_t bytes) {
    if (bytes == 0) bytes = 1;
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first / 2 <= bytes) {
        void* p = it->second;
        used_[p] = it->first;
        free_bytes_ -= it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) == cudaSuccess && p) {
      std::lock_guard<std::mutex> lk(mu_);
      used_[p] = bytes;
      return p;
    }
    (void)cudaGetLastError();  // a failed allocation is not sticky: clear it
    p = std::malloc(bytes);
    if (!p) throw std::bad_alloc();
    std::lock_guard<std::mutex> lk(mu_);
    plain_[p] = bytes;
    return p;
  }
  void give(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu_);
    auto pl = plain_.find(p);
    if (pl != plain_.end()) {
      plain_.erase(pl);
      std::free(p);
      return;
    }
    auto it = used_.find(p);
    if (it == used_.end()) return;
    free_.emplace(it->second, p);
    free_bytes_ += it->second;
    used_.erase(it);
    while (free_bytes_ > kMaxFreeBytes && !free_.empty()) {
      auto big = std::prev(free_.end());
      free_bytes_ -= big->first;
      cudaFreeHost(big->second);
      free_.erase(big);
    }
  }

 private:
  static constexpr size_t kMaxFreeBytes = size_t(1) << 31;
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  std::unordered_map<void*, size_t> used_, plain_;
  size_t free_bytes_ = 0;
};

// Allocator over PinnedPool with the construction of DefaultInitAllocator
// (elements left uninitialised until the copy writes them).
template <typename T>
struct PinnedPoolAllocator {
  using value_type = T;
  PinnedPoolAllocator() = default;
  template <typename U>
  PinnedPoolAllocator(const PinnedPoolAllocator<U>&) noexcept {}
  T* allocate(size_t n) { return static_cast<T*>(PinnedPool::instance().take(n * sizeof(T))); }
  void deallocate(T* p, size_t) noexcept { PinnedPool::instance().give(p); }
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
  template <typename U>
  bool operator==(const PinnedPoolAllocator<U>&) const noexcept { return true; }
  template <typename U>
  bool operator!=(const PinnedPoolAllocator<U>&) const noexcept { return false; }
};
template <typename T>
using PinnedHostVec = std::vector<T, PinnedPoolAllocator<T>>;

// Page-locked host buffer (grow-only) for device->host copies at full speed.
template <typename T>
class PinnedBuf {
 public:
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p_) cudaFreeHost(p_);
  }
  T* reserve(size_t n) {
    if (n > cap_ || !p_) {
      if (p_) cudaFreeHost(p_);
      p_ = nullptr;
      cap_ = 0;
      SAPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p_), (n ? n : 1) * sizeof(T)));
      cap_ = n;
    }
    return p_;
  }
  T* get() const { return p_; }

 private:
  T* p_ = nullptr;
  size_t cap_ = 0;
};

// --- asynchronous global->shared copies (sm_80+ cp.async) ---------------------
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
template <typename T>
__device__ __forceinline__ void cp_async_val(T* smem, const T* gmem) {
  if constexpr (sizeof(T) == 8) cp_async8(smem, gmem);
  else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// a / b from y = 1 / b (itself correctly rounded) with one multiply and two
// FMAs: Markstein's quotient correction (P. Markstein, IBM J. Res. Dev.
// 34(1), 1990; Muller et al., Handbook of Floating-Point Arithmetic,
// Markstein's theorem): q0 = RN(a y) is within one ulp of a / b, the
// remainder r = a - b q0 is exact through the FMA, and RN(q0 + r y) =
// RN(a / b) as long as nothing underflows or overflows; for a = 0, q0 = +-0
// is the quotient.  `ok` is false outside exponent ranges that guarantee
// this (non-finite, subnormal, very large or very small operands), where the
// caller must use the division; with ok true the result equals a / b.
template <typename T>
struct DivRange;
template <>
struct DivRange<double> {
  static constexpr double lo_a = 0x1p-960, lo = 0x1p-1000, hi = 0x1p1000;
};
template <>
struct DivRange<float> {
  static constexpr float lo_a = 0x1p-96f, lo = 0x1p-120f, hi = 0x1p120f;
};
template <typename T>
__device__ __forceinline__ T div_rcp_fast(T a, T b, T y, bool& ok) {
  using L = DivRange<T>;
  const T q0 = a * y;
  const T r = fma(-q0, b, a);
  const T q = fma(r, y, q0);
  const T aa = fabs(a), aq = fabs(q0), ay = fabs(y);
  ok = ay >= L::lo && ay <= L::hi && (a == T(0) || (aa >= L::lo_a && aq >= L::lo && aq <= L::hi));
  return a == T(0) ? q0 : q;
}

// boostValue (sap/device/factor_band_const.cuh:29-40): pivots with
// |p| <= BURST_VALUE are replaced by +-BURST_NEW_VALUE.
template <typename T>
__device__ __forceinline__ T boost_pivot(T v) {
  const T thr = (T)1e-7, nv = (T)1e-4;
  if (v > thr || v < -thr) return v;
  return v < (T)0 ? -nv : nv;
}

}  // namespace sapb
