// probe.cu - the FP64 fused multiply-add rate of the device (cb_probe_fp64), the denominator of
// the FP64-pipe fraction that the benchmark reports beside its HBM fraction.
//
// Each thread runs kChains independent FMA chains (a = a * m + c) for `iterations` rounds, so the
// issue of one chain's FMA never waits on the previous one's result; the grid is a multiple of the
// SM count with enough warps per SM to hide the FMA latency. The chains' sum is stored so nothing
// is dead code. FLOPs = 2 x kChains x iterations x threads.

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cells_b200.h"
#include "handle.h"

namespace {

using namespace cbk;

constexpr int kChains = 8;
constexpr int kThreads = 256;
constexpr int kCtasPerSm = 8;

__global__ void __launch_bounds__(kThreads) fma_chains(int64_t iterations, double m, double c,
                                                       double *out) {
  double a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
  for (int64_t i = 0; i < iterations; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], m, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  out[blockIdx.x * kThreads + threadIdx.x] = s;
}

}  // namespace

using cbk::cuda_fail;
using cbk::fail;

extern "C" int cb_probe_fp64(int device, int64_t iterations, double *flops_per_second,
                             double *milliseconds) {
  if (!flops_per_second || iterations <= 0) return fail(CB_ERR_ARGUMENT, "probe: bad argument");
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  int sms = 0;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
    return cuda_fail(e, "cudaDeviceGetAttribute");
  const int ctas = sms * kCtasPerSm;
  double *out = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  if ((e = cudaMalloc(&out, sizeof(double) * ctas * kThreads)) != cudaSuccess)
    return cuda_fail(e, "cudaMalloc");
  int rc = CB_OK;
  float ms = 0.0f;
  if ((e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess) {
    rc = cuda_fail(e, "cudaEventCreate");
  } else {
    // m slightly below 1 and c small keep every chain finite for any iteration count.
    fma_chains<<<ctas, kThreads>>>(iterations / 8 + 1, 0.999999, 1e-6, out);  // warm-up
    cudaEventRecord(a);
    fma_chains<<<ctas, kThreads>>>(iterations, 0.999999, 1e-6, out);
    cudaEventRecord(b);
    if ((e = cudaEventSynchronize(b)) != cudaSuccess ||
        (e = cudaEventElapsedTime(&ms, a, b)) != cudaSuccess)
      rc = cuda_fail(e, "fp64 probe");
  }
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(out);
  if (rc) return rc;
  const double flops = 2.0 * kChains * (double)iterations * (double)ctas * kThreads;
  *flops_per_second = flops / (ms * 1e-3);
  if (milliseconds) *milliseconds = ms;
  return CB_OK;
}
