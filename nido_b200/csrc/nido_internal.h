// nido_internal.h -- error reporting shared by the host and device code of
// libnido_b200.so.  Every C-ABI entry point returns a status and records a
// message for nido_last_error() on the calling thread.
#ifndef NIDO_INTERNAL_H_
#define NIDO_INTERNAL_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
/* records (code, message) for nido_last_error(); returns code */
int nido_set_error(int code, const char* fmt, ...);
#ifdef __cplusplus
}
#endif
#endif
