// cuda_wrapper.hpp -- the device helpers a program written against sg0/nido
// calls itself (cuda_wrapper.hpp of the reference: CudaSetDevice, CudaCall).
// libnido_b200.so owns the device: its objects release what they hold when
// they are destroyed, and everything runs on device 0, so these are checks
// rather than runtime calls.
#ifndef NIDO_COMPAT_CUDA_WRAPPER_HPP_
#define NIDO_COMPAT_CUDA_WRAPPER_HPP_
#include "../nido_host.hpp"

// status of a wrapped call: 0 is success (cudaSuccess and NIDO_OK alike)
#define CudaCall(ans) nido_check((int)(ans), #ans)
inline void nido_compat_set_device(int id) {
  if (id != 0) {
    fprintf(stderr, "CudaSetDevice(%d): this build runs on one GPU (device 0)\n", id);
    exit(EXIT_FAILURE);
  }
}
#define CudaSetDevice(id) nido_compat_set_device(id)
#define CudaDeviceSynchronize() ((void)0)

#if !defined(__CUDA_RUNTIME_API_H__)
// the reference program ends with a device reset; the engine's objects have
// already released the device by then
inline int cudaDeviceReset() { return NIDO_OK; }
#endif
#endif
