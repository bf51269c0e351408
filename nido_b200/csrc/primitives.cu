// primitives.cu -- device-wide exclusive scan (reduce-then-scan, recursive
// over tile sums) and stable LSD radix sort of 32-bit (key, value) pairs.
// These replace the Thrust inclusive_scan / stable_sort_by_key calls of the
// reference (graph_gpu.cpp:484, 515, 1168).
#include "common.cuh"
#include "primitives.cuh"

namespace nido {
namespace {

template <typename T>
__device__ __forceinline__ int64_t warp_incl_scan(int64_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(NIDO_FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) scan_tile_sums(const TIn* __restrict__ in,
                                                               int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t ws[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanIpt;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < kScanIpt; ++i)
    if (base + i < n) s += (int64_t)in[base + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int i = 0; i < kScanThreads / 32; ++i) t += ws[i];
    sums[blockIdx.x] = t;
  }
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) scan_tile_apply(const TIn* in, int64_t* out, int64_t n,
                                                                const int64_t* __restrict__ tile_off) {
  __shared__ int64_t ws[kScanThreads / 32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanIpt;
  int64_t x[kScanIpt];
  int64_t tot = 0;
#pragma unroll
  for (int i = 0; i < kScanIpt; ++i) {
    x[i] = (base + i < n) ? (int64_t)in[base + i] : 0;
    tot += x[i];
  }
  const int64_t incl = warp_incl_scan<int64_t>(tot);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 31) ws[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int64_t v = (lane < kScanThreads / 32) ? ws[lane] : 0;
    v = warp_incl_scan<int64_t>(v);
    if (lane < kScanThreads / 32) ws[lane] = v;
  }
  __syncthreads();
  int64_t run = (tile_off ? tile_off[blockIdx.x] : 0) + (wid > 0 ? ws[wid - 1] : 0) + incl - tot;
#pragma unroll
  for (int i = 0; i < kScanIpt; ++i) {
    if (base + i < n) {
      out[base + i] = run;
      run += x[i];
      if (base + i == n - 1) out[n] = run;
    }
  }
}

template <typename TIn>
int scan_impl(const TIn* in, int64_t* out, int64_t n, int64_t* temp, cudaStream_t s) {
  if (n <= 0) {
    NIDO_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    return NIDO_OK;
  }
  const int64_t nt = (n + kScanTile - 1) / kScanTile;
  if (nt == 1) {
    scan_tile_apply<TIn><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
    NIDO_LAUNCH_CHECK();
    return NIDO_OK;
  }
  scan_tile_sums<TIn><<<(unsigned)nt, kScanThreads, 0, s>>>(in, n, temp);
  NIDO_LAUNCH_CHECK();
  // temp[0..nt] receives the exclusive offsets of the tiles (temp[nt] = total)
  NIDO_TRY(scan_impl<int64_t>(temp, temp, nt, temp + nt + 1, s));
  scan_tile_apply<TIn><<<(unsigned)nt, kScanThreads, 0, s>>>(in, out, n, temp);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}

// ---- radix sort ---------------------------------------------------------------
__global__ void __launch_bounds__(kRadixThreads) radix_hist(const uint32_t* __restrict__ keys, int64_t n,
                                                            int shift, int64_t* __restrict__ hist,
                                                            int nblocks) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int i = threadIdx.x; i < kRadixTile; i += kRadixThreads) {
    const int64_t idx = base + i;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: elements of a tile are ranked in index order within each
// digit (warp match + per-warp digit counts), on top of the digit's global
// offset for this tile.
__global__ void __launch_bounds__(kRadixThreads) radix_scatter(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, int64_t n, int shift,
    const int64_t* __restrict__ offs, int nblocks, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout) {
  constexpr int W = kRadixThreads / 32;
  __shared__ int64_t run[256];
  __shared__ unsigned wcnt[W][257];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  run[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixIpt; ++r) {
    const int64_t idx = base + (int64_t)r * kRadixThreads + threadIdx.x;
    const bool valid = idx < n;
    const uint32_t k = valid ? kin[idx] : 0u;
    const uint32_t v = valid ? vin[idx] : 0u;
    const unsigned d = valid ? ((k >> shift) & 255u) : 256u;
#pragma unroll
    for (int w = 0; w < W; ++w) wcnt[w][threadIdx.x] = 0;
    if (threadIdx.x == 0) {
#pragma unroll
      for (int w = 0; w < W; ++w) wcnt[w][256] = 0;
    }
    __syncthreads();
    const unsigned peers = __match_any_sync(NIDO_FULL_MASK, d);
    const unsigned rank = __popc(peers & lanemask_lt());
    if (lane == __ffs(peers) - 1) wcnt[wid][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int64_t pos = run[d] + rank;
      for (int w = 0; w < wid; ++w) pos += wcnt[w][d];
      kout[pos] = k;
      vout[pos] = v;
    }
    __syncthreads();
    unsigned add = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) add += wcnt[w][threadIdx.x];
    run[threadIdx.x] += add;
    __syncthreads();
  }
}

}  // namespace

int64_t scan_temp_elems(int64_t n) {
  int64_t t = 0;
  while (n > kScanTile) {
    n = (n + kScanTile - 1) / kScanTile;
    t += n + 1;
  }
  return t + 1;
}

int scan_exclusive_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* temp, cudaStream_t s) {
  return scan_impl<int64_t>(in, out, n, temp, s);
}
int scan_exclusive_i32(const int32_t* in, int64_t* out, int64_t n, int64_t* temp, cudaStream_t s) {
  return scan_impl<int32_t>(in, out, n, temp, s);
}

int64_t radix_temp_elems(int64_t n) {
  const int64_t nb = (n + kRadixTile - 1) / kRadixTile;
  const int64_t h = 256 * (nb > 0 ? nb : 1);
  return h + 1 + scan_temp_elems(h);
}

int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                     int64_t n, int bits, int64_t* temp, cudaStream_t s) {
  if (n <= 1 || bits <= 0) return NIDO_OK;
  const int64_t nb64 = (n + kRadixTile - 1) / kRadixTile;
  if (nb64 > (1ll << 30)) return nido_set_error(NIDO_E_TOO_LARGE, "radix sort: too many elements");
  const int nb = (int)nb64;
  const int64_t h = 256 * nb64;
  int64_t* hist = temp;
  int64_t* stemp = temp + h + 1;
  uint32_t *ki = keys, *vi = vals, *ko = keys_tmp, *vo = vals_tmp;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, ++passes) {
    radix_hist<<<nb, kRadixThreads, 0, s>>>(ki, n, shift, hist, nb);
    NIDO_LAUNCH_CHECK();
    NIDO_TRY(scan_exclusive_i64(hist, hist, h, stemp, s));
    radix_scatter<<<nb, kRadixThreads, 0, s>>>(ki, vi, n, shift, hist, nb, ko, vo);
    NIDO_LAUNCH_CHECK();
    uint32_t* t = ki; ki = ko; ko = t;
    t = vi; vi = vo; vo = t;
  }
  if (passes & 1) {
    NIDO_CUDA_TRY(cudaMemcpyAsync(keys, ki, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    NIDO_CUDA_TRY(cudaMemcpyAsync(vals, vi, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
  }
  return NIDO_OK;
}

}  // namespace nido
