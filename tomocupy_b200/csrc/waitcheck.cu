// Failure-detection check of the bounded mbarrier waits.
//
// The tensor-core filter, the tensor-core gridding and the TMA-staged line
// backprojection wait on mbarriers with tc::mbar_wait, which gives up after a
// clock budget, sets the handle's error flag and lets the kernel finish.
// This entry point runs that same wait on an mbarrier that nothing arrives
// on, with a short budget chosen by the caller, so a test can see the wait
// run out, the status come back and the context stay usable.  No copy or
// MMA is in flight and no TMEM is held while it waits.
#include "common.cuh"
#include "tcgen05.cuh"

namespace {

__global__ void bounded_wait_check(long long budget, int *status, long long *cycles) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tcb::tc::mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const long long t0 = clock64();
    const bool ok = tcb::tc::mbar_wait_budget(&bar, 0, budget);  // phase 0 never completes
    cycles[0] = clock64() - t0;
    status[0] = ok ? 0 : 1;
  }
}

}  // namespace

extern "C" int tcb_check_bounded_wait(long long budget_cycles, int *timed_out,
                                      long long *waited_cycles, void *stream) {
  TCB_CHECK_ARG(timed_out && waited_cycles, "tcb_check_bounded_wait: null pointer");
  TCB_CHECK_ARG(budget_cycles >= 1 && budget_cycles <= 20000000000LL,
                "tcb_check_bounded_wait: budget %lld outside [1, 2e10] cycles", budget_cycles);
  cudaStream_t s = (cudaStream_t)stream;
  void *buf = nullptr;
  TCB_CUDA(cudaMalloc(&buf, 16));
  int *st = static_cast<int *>(buf);
  long long *cyc = reinterpret_cast<long long *>(static_cast<char *>(buf) + 8);
  bounded_wait_check<<<1, 32, 0, s>>>(budget_cycles, st, cyc);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(timed_out, st, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(waited_cycles, cyc, sizeof(long long), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  tcb::count_launch();
  cudaFree(buf);
  if (e != cudaSuccess) {
    tcb::set_error("tcb_check_bounded_wait: %s", cudaGetErrorString(e));
    return TCB_ERR_CUDA;
  }
  return TCB_OK;
}
