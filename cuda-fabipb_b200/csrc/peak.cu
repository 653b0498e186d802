// peak.cu -- the FP32 and FP64 SIMT rates of this device, measured.
//
// The near-field P2P and the mixed-precision direct sums are bound by the FP32
// FMA pipe (not a memory stream, not a tensor-core contraction), so their
// roofline denominator is the FP32 FMA rate.  It is measured here rather than
// derived from the clock: every thread runs long chains of independent packed
// f32x2 FMAs (FFMA2, the instruction the near field issues) on values the
// compiler cannot fold, timed with CUDA events over a grid of several waves;
// the FP64 pipe (the FP64 operator's denominator) likewise with DFMAs.
#include <cuda_runtime.h>

#include "common.cuh"

namespace fb {

constexpr int kPeakChains = 8;     // independent accumulators per thread
constexpr int kPeakIters = 4096;   // FMA steps per chain

__global__ void __launch_bounds__(256) fp32_peak_kernel(float seed, float *sink) {
  float2 acc[kPeakChains];
  const float2 m = make_float2(0.999f + 1e-7f * threadIdx.x, 0.998f);
  const float2 a = make_float2(seed, -seed);
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) acc[k] = make_float2(seed * (k + 1), seed * (k + 2));
  for (int it = 0; it < kPeakIters; it++) {
#pragma unroll
    for (int k = 0; k < kPeakChains; k++) acc[k] = __ffma2_rn(acc[k], m, a);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) s += acc[k].x + acc[k].y;
  if (s == 12345.678f) sink[threadIdx.x] = s;   // never true for these inputs; keeps the chains live
}

// the same chains in scalar FP32 FMAs (twice the chains, half the steps)
__global__ void __launch_bounds__(256) fp32s_peak_kernel(float seed, float *sink) {
  float acc[2 * kPeakChains];
  const float m = 0.999f + 1e-7f * threadIdx.x;
#pragma unroll
  for (int k = 0; k < 2 * kPeakChains; k++) acc[k] = seed * (k + 1);
  for (int it = 0; it < kPeakIters; it++) {
#pragma unroll
    for (int k = 0; k < 2 * kPeakChains; k++) acc[k] = fmaf(acc[k], m, seed);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 2 * kPeakChains; k++) s += acc[k];
  if (s == 12345.678f) sink[threadIdx.x] = s;
}

// the FP64 pipe: the same chains in scalar double FMAs (a quarter of the steps)
__global__ void __launch_bounds__(256) fp64_peak_kernel(double seed, float *sink) {
  double acc[kPeakChains];
  const double m = 0.999 + 1e-7 * threadIdx.x;
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) acc[k] = seed * (k + 1);
  for (int it = 0; it < kPeakIters / 4; it++) {
#pragma unroll
    for (int k = 0; k < kPeakChains; k++) acc[k] = fma(acc[k], m, seed);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kPeakChains; k++) s += acc[k];
  if (s == 12345.678) sink[threadIdx.x] = (float)s;
}

// TFLOP/s of the FP32 (fp64 = 0: the better of packed and scalar FMA chains)
// or FP64 FMA pipe (2 flop per lane FMA), the best of `reps` event-timed
// launches after about 200 ms of warm-up launches (clocks up to speed)
static bool simt_peak_variant(int device, int variant, int reps, double *tflops);

bool measure_simt_peak(int device, int fp64, int reps, double *tflops) {
  if (fp64) return simt_peak_variant(device, 2, reps, tflops);
  double a = 0.0, b = 0.0;
  if (!simt_peak_variant(device, 0, reps, &a) || !simt_peak_variant(device, 1, reps, &b)) return false;
  *tflops = std::max(a, b);
  return true;
}

static bool simt_peak_variant(int device, int variant, int reps, double *tflops) {
  FB_CUDA(cudaSetDevice(device));
  int sms = 0;
  FB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *sink = nullptr;
  FB_CUDA(cudaMalloc(&sink, 256 * sizeof(float)));
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess;
  const int blocks = sms * 8 * 4;   // eight resident 256-thread blocks per SM, four waves
  const double flop = variant == 2 ? 2.0 * kPeakChains * (double)(kPeakIters / 4) * 256.0 * blocks
                                    : 2.0 * 2.0 * kPeakChains * (double)kPeakIters * 256.0 * blocks;
  double best = 0.0, warm = 0.0;
  int r = 0, warmLaunches = 0;
  while (ok && r <= reps) {
    ok = cudaEventRecord(e0, st) == cudaSuccess;
    if (variant == 2) fp64_peak_kernel<<<blocks, 256, 0, st>>>(1e-3, sink);
    else if (variant == 1) fp32s_peak_kernel<<<blocks, 256, 0, st>>>(1e-3f, sink);
    else fp32_peak_kernel<<<blocks, 256, 0, st>>>(1e-3f, sink);
    ok = ok && cudaGetLastError() == cudaSuccess && cudaEventRecord(e1, st) == cudaSuccess &&
         cudaEventSynchronize(e1) == cudaSuccess;
    float ms = 0.f;
    if (!ok || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) break;
    if (r == 0 && warm < 200.0 && warmLaunches++ < 1000) {   // warm-up launches, not timed
      warm += ms;
      continue;
    }
    if (r > 0 && ms > 0.f) best = std::max(best, flop / (ms * 1e-3) / 1e12);
    r++;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(sink);
  FB_CHECK(ok, "SIMT peak measurement failed: %s", cudaGetErrorString(cudaGetLastError()));
  *tflops = best;
  return true;
}

}  // namespace fb

extern "C" int fabipb_b200_simt_peak(int device, int fp64, double *tflops) {
  if (tflops == nullptr) {
    fb::set_error("fabipb_b200_simt_peak: null output");
    return 0;
  }
  return fb::measure_simt_peak(device, fp64, 5, tflops) ? 1 : 0;
}
