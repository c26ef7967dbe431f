// Shared helpers for the tomocupy_b200 C-ABI library: status codes, the
// thread-local last-error message, and checked CUDA / cuFFT calls.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/tomocupy_b200.h"

namespace tcb {

void set_error(const char *fmt, ...);

// Evaluate a CUDA runtime call; on failure record the message and return
// TCB_ERR_CUDA (or TCB_ERR_OUT_OF_MEMORY) from the enclosing function.
#define TCB_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t _e = (call);                                                    \
    if (_e != cudaSuccess) {                                                    \
      ::tcb::set_error("%s:%d: %s failed: %s", __FILE__, __LINE__, #call,       \
                       cudaGetErrorString(_e));                                 \
      return _e == cudaErrorMemoryAllocation ? TCB_ERR_OUT_OF_MEMORY            \
                                             : TCB_ERR_CUDA;                    \
    }                                                                           \
  } while (0)

#define TCB_CUFFT(call)                                                         \
  do {                                                                          \
    cufftResult _r = (call);                                                    \
    if (_r != CUFFT_SUCCESS) {                                                  \
      ::tcb::set_error("%s:%d: %s failed: cufftResult %d", __FILE__, __LINE__,  \
                       #call, (int)_r);                                         \
      return _r == CUFFT_ALLOC_FAILED ? TCB_ERR_OUT_OF_MEMORY : TCB_ERR_CUFFT;  \
    }                                                                           \
  } while (0)

#define TCB_CHECK_ARG(cond, ...)                                                \
  do {                                                                          \
    if (!(cond)) {                                                              \
      ::tcb::set_error(__VA_ARGS__);                                            \
      return TCB_ERR_INVALID_ARGUMENT;                                          \
    }                                                                           \
  } while (0)

// After a launch: report configuration errors immediately (launch failures
// such as an invalid grid) without synchronising the stream.
#define TCB_LAUNCH_CHECK()                                                      \
  do {                                                                          \
    cudaError_t _e = cudaPeekAtLastError();                                     \
    if (_e != cudaSuccess) {                                                    \
      cudaGetLastError();                                                       \
      ::tcb::set_error("%s:%d: kernel launch failed: %s", __FILE__, __LINE__,   \
                       cudaGetErrorString(_e));                                 \
      return TCB_ERR_CUDA;                                                      \
    }                                                                           \
  } while (0)

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// Launch counter and optional per-stage event timing (see tcb_profile_*).
void count_launch(unsigned k = 1);
struct StageTimer {
  // Records a start event on `s` when profiling is on; the destructor records
  // the end.  bytes / flops: the stage's algorithmic DRAM bytes and FLOPs of
  // this launch (0 = not stated), summed per stage in the report.
  StageTimer(const char *name, cudaStream_t s, double bytes = 0.0, double flops = 0.0);
  ~StageTimer();
  const char *name;
  cudaStream_t stream;
  int slot;
};

// Number of SMs of the current device (cached per process; one device per
// process is the deployment model).
int sm_count();

}  // namespace tcb
