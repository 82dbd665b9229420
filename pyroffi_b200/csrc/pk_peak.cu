// FP32 FMA-pipe microbenchmark: the SIMT roof of the kinematics kernels.
//
// Every thread runs `iters` rounds of 8 independent FMA chains (enough
// instruction-level parallelism to fill the pipe at full occupancy); the
// result is written so nothing is dead code.  FLOPs = 2 * 8 * iters * threads.
#include "pk_common.cuh"

namespace pk {

__global__ void __launch_bounds__(256) fma_peak_kernel(float* out, int iters, float s) {
  float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
  float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
  const float m = 0.999999f;
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    a0 = fmaf(a0, m, s); a1 = fmaf(a1, m, s); a2 = fmaf(a2, m, s); a3 = fmaf(a3, m, s);
    a4 = fmaf(a4, m, s); a5 = fmaf(a5, m, s); a6 = fmaf(a6, m, s); a7 = fmaf(a7, m, s);
  }
  const float r = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (r == 1234.5f) out[blockIdx.x] = r;  // practically never taken; keeps the chains live
}

}  // namespace pk

extern "C" int pk_fp32_fma_peak(void* stream, float* out, int32_t iters, int32_t blocks) {
  PK_CHECK_ARG(iters > 0 && blocks > 0 && out, "bad arguments");
  pk::fma_peak_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 1e-9f);
  return pk::cuda_status(cudaGetLastError(), "fma_peak_kernel launch");
}
