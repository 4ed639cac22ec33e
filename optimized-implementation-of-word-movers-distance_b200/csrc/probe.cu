// Roofline probes: the measured denominators of the solve's roofline.
//
// The iteration kernels read their K rows from an L2-resident panel and then
// from registers and shared memory, so neither the HBM copy bandwidth nor the
// tensor-core peak bounds them; the bounds are the L2 read bandwidth (for the
// row gathers) and the FP32 FMA rate (for the dot products and updates).
// These two kernels measure both on the running GPU with CUDA events:
//
//   l2_read_kernel   every thread streams 16-byte loads over a buffer small
//                    enough to stay in L2 (warmed first), summing them so the
//                    loads cannot be dropped; bytes / time.
//   fma_kernel       every thread runs 8 independent chains of packed FP32
//                    FMAs (FFMA2) on registers (fma1_kernel: 16 scalar
//                    chains); 2 flops per lane-FMA / the faster time.
//
// No reference counterpart (the reference has no GPU code).  Not on any
// solve path: they allocate their own buffers.
#include <cuda_runtime.h>
#include <stdint.h>

#include "wmd_b200.h"
#include "wmd_internal.cuh"

namespace wmd {
namespace {

__global__ void l2_read_kernel(const float4* __restrict__ buf, uint64_t n4, int passes,
                               float* __restrict__ sink) {
  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (int p = 0; p < passes; ++p) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += 4 * stride) {
      float4 v[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint64_t j = i + k * stride;
        v[k] = j < n4 ? __ldcg(buf + j) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        acc.x += v[k].x;
        acc.y += v[k].y;
        acc.z += v[k].z;
        acc.w += v[k].w;
      }
    }
  }
  // Never true for the zero-filled buffer, but the compiler cannot know.
  if (acc.x + acc.y + acc.z + acc.w == 1.2345f) sink[0] = acc.x;
}

constexpr int kFmaChains = 8;

// Scalar form of the same chains (16 per thread), in case the packed form
// does not reach the pipe's rate.
__global__ void fma1_kernel(int iters, float seed, float* __restrict__ sink) {
  float a[2 * kFmaChains];
#pragma unroll
  for (int c = 0; c < 2 * kFmaChains; ++c) a[c] = seed + threadIdx.x * 1e-7f + c;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 2 * kFmaChains; ++c) a[c] = fmaf(a[c], 0.999999f, 1e-7f);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < 2 * kFmaChains; ++c) s += a[c];
  if (s == 1.2345f) sink[threadIdx.x] = s;
}

__global__ void fma_kernel(int iters, float seed, float* __restrict__ sink) {
  float2 a[kFmaChains];
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c)
    a[c] = make_float2(seed + threadIdx.x * 1e-7f + c, seed - c);
  const float2 m = make_float2(0.999999f, 0.999998f), b = make_float2(1e-7f, 2e-7f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kFmaChains; ++c) a[c] = __ffma2_rn(a[c], m, b);
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kFmaChains; ++c) s += a[c].x + a[c].y;
  if (s == 1.2345f) sink[threadIdx.x] = s;
}

}  // namespace
}  // namespace wmd

extern "C" wmd_status wmd_probe_roofline(int device, uint64_t l2_bytes,
                                         double* l2_read_gbs, double* fp32_tflops) {
  using namespace wmd;
  if (!l2_read_gbs || !fp32_tflops || l2_bytes < (1u << 20) || l2_bytes > (96ull << 20))
    return WMD_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return WMD_ERR_NO_DEVICE;
  }
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* buf = nullptr;
  float* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  wmd_status st = WMD_OK;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && st == WMD_OK) {
      set_last_error(cudaGetErrorString(e));
      st = WMD_ERR_CUDA;
    }
    return st == WMD_OK;
  };
  const uint64_t n4 = l2_bytes / 16;
  if (ok(cudaMalloc(&buf, n4 * 16)) && ok(cudaMalloc(&sink, 1024 * sizeof(float))) &&
      ok(cudaMemset(buf, 0, n4 * 16)) && ok(cudaEventCreate(&e0)) &&
      ok(cudaEventCreate(&e1))) {
    // L2 read: warm the buffer into L2, then time several passes over it.
    const unsigned grid = (unsigned)sms * 8;
    const int passes = 20;
    l2_read_kernel<<<grid, 256>>>(reinterpret_cast<const float4*>(buf), n4, 2, sink);
    float best = 1e30f;
    for (int rep = 0; rep < 5 && ok(cudaGetLastError()); ++rep) {
      cudaEventRecord(e0);
      l2_read_kernel<<<grid, 256>>>(reinterpret_cast<const float4*>(buf), n4, passes, sink);
      cudaEventRecord(e1);
      float ms = 0.f;
      if (ok(cudaEventSynchronize(e1)) && ok(cudaEventElapsedTime(&ms, e0, e1)))
        best = ms < best ? ms : best;
    }
    *l2_read_gbs = (double)n4 * 16 * passes / (best * 1e-3) / 1e9;
    // FP32 FMA rate: 4 CTAs of 256 threads per SM, 8 packed chains each.
    const int iters = 20000;
    fma_kernel<<<sms * 4, 256>>>(iters / 10, 1.f, sink);
    best = 1e30f;
    for (int rep = 0; rep < 5 && ok(cudaGetLastError()); ++rep) {
      cudaEventRecord(e0);
      fma_kernel<<<sms * 4, 256>>>(iters, 1.f, sink);
      cudaEventRecord(e1);
      float ms = 0.f;
      if (ok(cudaEventSynchronize(e1)) && ok(cudaEventElapsedTime(&ms, e0, e1)))
        best = ms < best ? ms : best;
    }
    // scalar chains: the same flops per launch
    fma1_kernel<<<sms * 4, 256>>>(iters / 10, 1.f, sink);
    for (int rep = 0; rep < 5 && ok(cudaGetLastError()); ++rep) {
      cudaEventRecord(e0);
      fma1_kernel<<<sms * 4, 256>>>(iters, 1.f, sink);
      cudaEventRecord(e1);
      float ms = 0.f;
      if (ok(cudaEventSynchronize(e1)) && ok(cudaEventElapsedTime(&ms, e0, e1)))
        best = ms < best ? ms : best;
    }
    const double flops = (double)sms * 4 * 256 * iters * kFmaChains * 2 /*lanes*/ * 2;
    *fp32_tflops = flops / (best * 1e-3) / 1e12;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (buf) cudaFree(buf);
  if (sink) cudaFree(sink);
  cudaGetLastError();
  if (st == WMD_OK) set_last_error("");
  return st;
}
