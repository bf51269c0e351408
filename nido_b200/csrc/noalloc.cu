// noalloc.cu -- modularity of a partition from caller-owned device arrays,
// with no memory allocation at all.
//
// Who needs this: code that runs where cudaMalloc is not allowed or not
// wanted -- while a CUDA stream is being captured into a graph, inside a
// custom device-memory allocator or a memory-pool callback, or in a serving
// process that has handed all of the GPU's memory to a fixed pool.  Such
// callers hold their graph and partition in device memory already and only
// need the number back.
//
// Design: the reference's reduction (compute_modularity_reduce_kernel<128,16>
// and reduce_vector_kernel, graph_cuda.cu:2078-2134, 1806-1835) writes one
// partial per 16-thread group into a buffer it cudaMallocs on every call
// (graph_gpu.cpp:872-875).  Here that buffer is a file-scope __device__
// array of the reference's maximum size, 65535 blocks * 128 / 16 = 524,280
// doubles (4 MiB), which every GPU that loads this library holds until the
// process exits.  Every partial that the final reduction reads is written
// earlier in the same call, so nothing has to be cleared between calls.  All
// calls on a device share the array: calls that overlap on the GPU (for
// example on two streams at once) race and give wrong results.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int64_t kMaxGroups = 524280;  // 65535 * 128 / 16
constexpr int64_t kNoallocMaxVertices = ((int64_t)1 << 31) - 2;  // the library's vertex limit
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_group_partials[kMaxGroups];

std::mutex g_setup_mutex;
double* g_scratch[kMaxDevices] = {};  // device address of g_group_partials, per device

// Thread slot t folds the in-community edge weights of vertices t, t+S, ...
// in edge order and ac = fma(a_v, a_v, ac); 16-lane shuffle trees; lane 0 of
// every group writes self/(2m) - ac/(4m*m).
__global__ void k_noalloc_groups(int64_t nv, int64_t S, int64_t ngroups, const int64_t* __restrict__ off,
                                 const int64_t* __restrict__ adj, const double* __restrict__ w,
                                 const int64_t* __restrict__ comm, const double* __restrict__ a, double m,
                                 double* __restrict__ partials) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t g = t >> 4;
  double s = 0., ac = 0.;
  if (g < ngroups) {
    for (int64_t v = t; v < nv; v += S) {
      const int64_t own = comm[v];
      for (int64_t j = off[v]; j < off[v + 1]; ++j)
        if (comm[adj[j]] == own) s += w[j];
      ac = fma(a[v], a[v], ac);
    }
  }
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) {
    s += __shfl_down_sync(NIDO_FULL_MASK, s, o, 16);
    ac += __shfl_down_sync(NIDO_FULL_MASK, ac, o, 16);
  }
  if ((t & 15) == 0 && g < ngroups) {
    double x = __ddiv_rn(s, __dmul_rn(2., m));
    x = __dsub_rn(x, __ddiv_rn(ac, __dmul_rn(__dmul_rn(4., m), m)));
    partials[g] = __dadd_rn(0., x);
  }
}

// one block of 1024 threads: strided fold, then warp trees
__global__ void __launch_bounds__(1024) k_noalloc_reduce(const double* __restrict__ partials, int64_t n,
                                                         double* __restrict__ q) {
  __shared__ double ws[32];
  double s = 0.;
  for (int64_t i = threadIdx.x; i < n; i += 1024) s += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = ws[threadIdx.x];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(NIDO_FULL_MASK, s, o);
    if (threadIdx.x == 0) *q = s;
  }
}

// Looks up (once per device, with that device current) the device address of
// the scratch array; host code must not use the symbol itself as a pointer.
int scratch_for_current_device(double** out) {
  int dev = -1;
  NIDO_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return nido_set_error(NIDO_E_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_group_partials);
    if (e != cudaSuccess)
      return nido_set_error(NIDO_E_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    g_scratch[dev] = static_cast<double*>(p);
  }
  *out = g_scratch[dev];
  return NIDO_OK;
}

}  // namespace

extern "C" int nido_modularity_noalloc(void* stream, int64_t nv, const int64_t* d_off, const int64_t* d_adj,
                                       const double* d_w, const int64_t* d_comm, const double* d_a, double m,
                                       double* d_q) {
  // every array the kernels may read must be given once there are vertices;
  // a caller whose graph has no edges passes any non-null d_adj and d_w
  if (nv < 0 || !d_q || (nv > 0 && (!d_off || !d_adj || !d_w || !d_comm || !d_a)))
    return nido_set_error(NIDO_E_INVALID, "nido_modularity_noalloc: bad arguments");
  if (nv > kNoallocMaxVertices)
    return nido_set_error(NIDO_E_TOO_LARGE, "nido_modularity_noalloc: %lld vertices exceed the limit of %lld",
                          (long long)nv, (long long)kNoallocMaxVertices);
  double* partials = nullptr;
  NIDO_TRY(scratch_for_current_device(&partials));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int64_t grid = (nv + 7) / 8;
  if (grid > 65535) grid = 65535;
  if (grid < 1) grid = 1;
  const int64_t S = 128 * grid;
  const int64_t nslots = nv < S ? nv : S;
  const int64_t ngroups = (nslots + 15) / 16;  // <= kMaxGroups for every nv
  if (ngroups > kMaxGroups) return nido_set_error(NIDO_E_TOO_LARGE, "too many groups");
  if (ngroups > 0) {
    k_noalloc_groups<<<(unsigned)((ngroups * 16 + 255) / 256), 256, 0, s>>>(nv, S, ngroups, d_off, d_adj, d_w,
                                                                           d_comm, d_a, m, partials);
    NIDO_LAUNCH_CHECK();
  }
  k_noalloc_reduce<<<1, 1024, 0, s>>>(partials, ngroups, d_q);
  NIDO_LAUNCH_CHECK();
  return NIDO_OK;
}
