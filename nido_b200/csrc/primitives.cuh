// primitives.cuh -- device-wide exclusive scan and stable LSD radix sort.
#ifndef NIDO_PRIMITIVES_CUH_
#define NIDO_PRIMITIVES_CUH_
#include <cuda_runtime.h>
#include <stdint.h>

namespace nido {

constexpr int kScanThreads = 256;
constexpr int kScanIpt = 8;
constexpr int kScanTile = kScanThreads * kScanIpt;

// int64 temp elements needed by scan_exclusive for n inputs
int64_t scan_temp_elems(int64_t n);
// out[i] = sum_{j<i} in[j] for i in [0, n], i.e. out has n+1 entries and
// out[n] is the total.  in and out may alias.  temp: scan_temp_elems(n).
int scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* temp,
                       cudaStream_t s);
int scan_exclusive_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* temp,
                       cudaStream_t s);

constexpr int kRadixThreads = 256;
constexpr int kRadixIpt = 16;
constexpr int kRadixTile = kRadixThreads * kRadixIpt;

// int64 temp elements needed by radix_sort_pairs for n inputs
int64_t radix_temp_elems(int64_t n);
// Stable sort of (keys, vals) by the low `bits` bits of keys, 8 bits per pass.
// keys_tmp / vals_tmp are ping-pong buffers of n entries; the result is left
// in keys / vals.
int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                     int64_t n, int bits, int64_t* temp, cudaStream_t s);

}  // namespace nido
#endif
