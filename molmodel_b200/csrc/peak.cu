// FP32 FMA throughput of the current GPU, measured, for roofline reports of
// the pair kernels (whose bound is the FP32 pipe).  No counterpart in the
// reference.  Every thread runs 8 independent FMA chains; the grid fills the
// device several times over; the result is the best of a few timed launches.

#include "mmnb_internal.cuh"

namespace mmnb {

constexpr int kPeakThreads = 256;
constexpr int kPeakIters = 4096;

__global__ void __launch_bounds__(kPeakThreads) k_fma_peak(float *out, float a, float b)
{
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; k++)
    x[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < kPeakIters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++)
      x[k] = fmaf(x[k], a, b);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++)
    s += x[k];
  if (s == 12345.f)  // never true for these inputs; keeps the chains live
    out[threadIdx.x] = s;
}

}  // namespace mmnb

extern "C" int mmnb_measure_fp32_peak(int device, double *tflops)
{
  using namespace mmnb;
  if (!tflops)
    return MMNB_ERR_ARG;
  if (device >= 0 && cudaSetDevice(device) != cudaSuccess)
    return MMNB_ERR_CUDA;
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return MMNB_ERR_CUDA;
  float *out = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s = nullptr;
  int status = MMNB_OK;
  if (cudaMalloc(&out, kPeakThreads * sizeof(float)) != cudaSuccess || cudaEventCreate(&a) != cudaSuccess ||
      cudaEventCreate(&b) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    status = MMNB_ERR_CUDA;
  const int blocks = nsm * 8 * 4;
  double best = 0;
  for (int rep = 0; rep < 5 && status == MMNB_OK; rep++) {
    cudaEventRecord(a, s);
    k_fma_peak<<<blocks, kPeakThreads, 0, s>>>(out, 0.999f, 1e-3f);
    cudaEventRecord(b, s);
    float ms = 0;
    if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
      status = MMNB_ERR_CUDA;
      break;
    }
    const double flop = 2.0 * 8 * kPeakIters * (double) blocks * kPeakThreads;
    if (rep > 0)  // the first launch warms up
      best = std::max(best, flop / (ms * 1e-3) / 1e12);
  }
  if (out)
    cudaFree(out);
  if (a)
    cudaEventDestroy(a);
  if (b)
    cudaEventDestroy(b);
  if (s)
    cudaStreamDestroy(s);
  *tflops = best;
  return status;
}
