// Shared plumbing for the mguso sm_100a library: status codes, error capture, device
// buffers and the PTX wrappers (mbarrier, 1-D TMA bulk copy) the staged kernels use.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <stdint.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <cstdlib>
#include <vector>

#include "../../include/mguso_cuda.h"

namespace mg {

// Per-thread last error message, read through mguso_last_error().
void set_error(const std::string& msg);
const std::string& get_error();

#define MG_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) {                                                                   \
      ::mg::set_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " @" __FILE__ ":" + \
                      std::to_string(__LINE__));                                               \
      return e_ == cudaErrorMemoryAllocation ? MGUSO_ERR_OOM : MGUSO_ERR_CUDA;                 \
    }                                                                                          \
  } while (0)

#define MG_CHECK_ARG(cond, msg)    \
  do {                             \
    if (!(cond)) {                 \
      ::mg::set_error(msg);        \
      return MGUSO_ERR_INVALID_ARG; \
    }                              \
  } while (0)

#define MG_TRY(expr)          \
  do {                        \
    int s_ = (expr);          \
    if (s_ != MGUSO_OK) return s_; \
  } while (0)

// A typed device allocation that grows on demand and frees itself.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;  // elements
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  // Ensures room for n elements plus `pad_bytes` of slack (bulk copies may over-read up
  // to 16 bytes past the last element). Contents are not preserved.
  int reserve(size_t n, size_t pad_bytes = 32) {
    if (n <= cap && p) return MGUSO_OK;
    release();
    size_t bytes = n * sizeof(T) + pad_bytes;
    cudaError_t e = cudaMalloc((void**)&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      set_error(std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
      return MGUSO_ERR_OOM;
    }
    cap = n;
    return MGUSO_OK;
  }
  // reserve for buffers sized by a count that varies between calls (contact stencils,
  // sort lengths): a cudaMalloc of tens of MB takes milliseconds to tens of milliseconds,
  // so the capacity at least doubles when it has to grow
  int grow(size_t n) { return reserve(n <= cap && p ? n : std::max(n, 2 * cap)); }
  int upload(const T* h, size_t n, cudaStream_t s) {
    MG_TRY(reserve(n));
    if (n && h) MG_CUDA(cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return MGUSO_OK;
  }
};

// A typed page-locked host allocation (the target of device-to-host copies that must not
// block the host), grown on demand and freed with the object.
template <class T>
struct PinnedBuf {
  T* p = nullptr;
  size_t cap = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  int reserve(size_t n) {
    if (n <= cap && p) return MGUSO_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    MG_CUDA(cudaMallocHost((void**)&p, n * sizeof(T)));
    cap = n;
    return MGUSO_OK;
  }
};

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

inline unsigned int f2u_host(float f) {
  unsigned int u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline float u2f_host(unsigned int u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

int device_sm_count();

// MGUSO_PLAIN_LAUNCHES=1: the step's device-driven loops (the PCG solve and the CCD schedule,
// conditional-while CUDA graphs) run as plain kernel launches driven by the host instead, with
// the same kernels and iterations; for profilers, which cannot see the kernels of graphs with
// conditional nodes.
inline bool plain_launches() {
  static const bool on = [] {
    const char* e = std::getenv("MGUSO_PLAIN_LAUNCHES");
    return e && e[0] && e[0] != '0';
  }();
  return on;
}

// ---------------------------------------------------------------------------------------
// PTX wrappers: mbarrier + 1-D bulk (TMA) global -> shared copies.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 1-D bulk copy; src, dst and bytes must all be multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase. Returns false after `max_tries` polls; the caller
// records an error status instead of spinning forever.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint32_t max_tries = (1u << 24)) {
  uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < max_tries; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(addr), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Device status word bits (written by kernels, read by the host).
enum : uint32_t {
  ST_WAIT_TIMEOUT = 1u << 0,
  ST_NONFINITE = 1u << 1,
  ST_PAIR_OVERFLOW = 1u << 2,
  ST_STACK_OVERFLOW = 1u << 3,
  ST_PCG_BREAKDOWN = 1u << 4,
  ST_CCD_CAP = 1u << 5,
  ST_CAPACITY = 1u << 6,
};

}  // namespace mg
