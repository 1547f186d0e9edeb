// dv_selftest.cu -- makes the solve kernels' bounded waits run out on
// purpose, without a fault: a cooperative launch of two CTAs where CTA 1
// never arrives at the grid barrier, and an mbarrier that expects 16 bytes no
// copy will bring.  The waits are the ones the solve kernels use (grid_sync,
// bounded_mbar_wait); each must end after the limit with its error bit set,
// and the context stays usable.
#include "dv_solve.cuh"

#include "dvide.h"

namespace dv {

namespace {

struct WaitTestArgs {
  EngineWords* ew;
};

__global__ void __launch_bounds__(kThreads) k_selftest_waits(WaitTestArgs a, int* out) {
  __shared__ __align__(8) uint64_t bar[1];
  if (blockIdx.x != 0) return;  // the CTA that never reaches the barrier
  const bool barrier_ok = grid_sync(a, kPhaseSetup, NoCtl{});
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  bool copy_ok = true;
  if (threadIdx.x < 32) {
    if (threadIdx.x == 0) mbar_arrive_expect_tx(bar, 16u);  // no copy follows
    __syncwarp();
    copy_ok = __all_sync(0xffffffffu, bounded_mbar_wait(bar, 0u, &a.ew->wait_limit_ns));
  }
  if (threadIdx.x == 0) {
    if (!copy_ok) atomicOr(&a.ew->err, kErrCopyTimeout);
    out[0] = barrier_ok ? 0 : 1;
    out[1] = copy_ok ? 0 : 1;
  }
}

}  // namespace

}  // namespace dv

using namespace dv;

DV_API int dv_selftest_bounded_waits(int32_t limit_ms, int32_t* barrier_timed_out,
                                     int32_t* copy_timed_out, uint32_t* error_bits) {
  if (limit_ms <= 0) return DV_ERR_ARG;
  EngineWords* ew = nullptr;
  int* out = nullptr;
  if (cudaMalloc(&ew, sizeof(EngineWords)) != cudaSuccess) return DV_ERR_OOM;
  if (cudaMalloc(&out, 2 * sizeof(int)) != cudaSuccess) {
    cudaFree(ew);
    return DV_ERR_OOM;
  }
  EngineWords h;
  memset(&h, 0, sizeof(h));
  h.wait_limit_ns = (unsigned long long)limit_ms * 1000000ull;
  int host_out[2] = {-1, -1};
  cudaMemcpy(ew, &h, sizeof(h), cudaMemcpyHostToDevice);
  cudaMemcpy(out, host_out, sizeof(host_out), cudaMemcpyHostToDevice);
  WaitTestArgs a{ew};
  void* params[] = {&a, &out};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_selftest_waits, 2, kThreads, params, 0, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(host_out, out, sizeof(host_out), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&h, ew, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(out);
  cudaFree(ew);
  if (e != cudaSuccess) return dv_record_cuda_error(e, "dv_selftest_bounded_waits", __FILE__, __LINE__);
  if (barrier_timed_out) *barrier_timed_out = host_out[0];
  if (copy_timed_out) *copy_timed_out = host_out[1];
  if (error_bits) *error_bits = h.err;
  return DV_OK;
}
