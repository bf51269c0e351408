// common.cuh -- device-side helpers shared by the engine's kernels.
#ifndef NIDO_COMMON_CUH_
#define NIDO_COMMON_CUH_
#include <cuda_runtime.h>
#include <stdint.h>

#include "nido_b200.h"
#include "nido_internal.h"

#define NIDO_FULL_MASK 0xffffffffu

// MAX_FLOAT of the reference (cuda_wrapper.hpp:94): the initial best gain.
#define NIDO_MAX_FLOAT 1.0E+308

#define NIDO_CUDA_TRY(expr)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return nido_set_error(NIDO_E_CUDA, "%s failed: %s (%s:%d)", #expr,                \
                            cudaGetErrorString(e_), __FILE__, __LINE__);                 \
  } while (0)

#define NIDO_TRY(expr)       \
  do {                       \
    int s_ = (expr);         \
    if (s_ != NIDO_OK) return s_; \
  } while (0)

// Follows every kernel launch: counts it and reports a launch error (bad
// configuration) without a sync.
extern "C" void nido_count_launch(void);
extern "C" void nido_count_launches(uint64_t n);  // kernels of a replayed CUDA graph
#define NIDO_LAUNCH_CHECK()                     \
  do {                                          \
    nido_count_launch();                        \
    NIDO_CUDA_TRY(cudaPeekAtLastError());       \
  } while (0)

namespace nido {

// 148 SMs on B200; the grid sizes below are multiples of the SM count.
constexpr int kSMs = 148;

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Multiplicative (Fibonacci) hash of a community id into a power-of-two table
// of mask+1 >= 2 slots: the top log2(mask+1) bits of c * 2^32/phi.  (The low
// bits of the product would only permute c mod 2^k, so ids that agree in
// their low bits would collide.)
__device__ __forceinline__ unsigned hash_slot(int c, unsigned mask) {
  return ((unsigned)c * 0x9E3779B1u) >> __clz(mask);
}

// 3-bit bit reversal: the order in which the reference's 8-lane shuffle-down
// tree (graph_cuda.cu:1515-1526) prefers lanes on equal gains.
__device__ __forceinline__ unsigned bitrev3(unsigned x) {
  return ((x & 1u) << 2) | (x & 2u) | ((x & 4u) >> 2);
}

// "a beats b": larger gain, then smaller tie key (community id for the
// smallest-id rule, the reference's lane order for the nido rule).
__device__ __forceinline__ bool better(double ga, unsigned long long ka, double gb,
                                       unsigned long long kb) {
  return ga > gb || (ga == gb && ka < kb);
}

}  // namespace nido
#endif
