// Word-major Sinkhorn solve: the reference's own traversal order on the GPU.
//
// The reference's fused solver walks the target matrix word by word
// (word-major CSR, sinkhorn_wmd_fused.cpp:249-292): each thread takes an
// nnz-balanced chunk of entries, finds its first row by binary search
// (p_binary_search, fused:88-109, 165-179), and for every entry (word w,
// document j, weight c) computes s = K_w . u_j, v = c / s and scatters
// x_j += K_w v with atomics (fused:284); then u = 1 / x (fused:304-319).
// Each K row is read once per pass, at the price of gathering u_j and
// scattering into x_j per entry.  This file is that order on the GPU:
//
//   wm_pass_kernel     one warp per nnz-balanced chunk of word-major entries
//                      (start row by binary search on the row pointers), lanes
//                      over source dimensions; the warp keeps the current word's
//                      K row in registers while consecutive entries share it,
//                      gathers u_j (coalesced, ld floats), reduces s with
//                      shuffles and adds K_w v into x_j with red.global.add
//                      (vector atomics, no return);
//   wm_update_kernel   u = 1 / (x / r), x = 0 for the next pass;
//   wm_final_kernel    the final half-step: v from the last u, and
//                      WMD_j += v sum_i K_wi M_wi u_ji (FP64 atomics),
//                      K.*M = K ln K / expo (fused:339-393);
//   wm_finish_kernel   a document whose u is not finite scores NaN (the
//                      reference's sum meets u = inf there), an empty source 0.
//
// The document-major solves (solve.cu, solve_block.cu) keep u_j and x_j on
// chip and read each document's rows once per solve; this form instead
// re-reads u and re-writes x through L2/HBM every pass (N * v_r * 8 bytes of
// state), which is what it costs to stream the panel one row at a time.
// Fixed update count only (tol = 0, omega = 1, cold start), FP32 panel.
#include "wmd_internal.cuh"

namespace wmd {
namespace {

constexpr int kWmThreads = 256;
constexpr int kWmMaxQ = 32;  // dimensions per lane: v_r <= 1024

// Row pointers are 64-bit; the first row whose range contains entry e.
__device__ __forceinline__ int64_t row_of(const int64_t* __restrict__ rp, int64_t V,
                                          int64_t e) {
  int64_t lo = 0, hi = V;  // rp[lo] <= e < rp[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (rp[mid] <= e) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int Q>
__global__ void __launch_bounds__(kWmThreads)
wm_pass_kernel(const float* __restrict__ K, int ld, const int64_t* __restrict__ rp,
               int64_t V, const uint2* __restrict__ went,  // {doc, float bits c}
               int64_t nnz, int64_t chunk, const float* __restrict__ u,
               float* __restrict__ x, int ldu) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t e0 = warp * chunk;
  if (e0 >= nnz) return;
  const int64_t e1 = min(nnz, e0 + chunk);
  int64_t w = row_of(rp, V, e0);
  int64_t wend = rp[w + 1];
  float kr[Q];
  auto load_row = [&](int64_t ww) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = lane + 32 * q;
      kr[q] = i < ld ? __ldg(&K[(size_t)ww * ld + i]) : 0.f;
    }
  };
  load_row(w);
  for (int64_t e = e0; e < e1; ++e) {
    while (e >= wend) {  // next non-empty row
      ++w;
      wend = rp[w + 1];
      if (e < wend) load_row(w);
    }
    const uint2 en = __ldg(&went[e]);
    const float* uj = u + (size_t)en.x * ldu;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = lane + 32 * q;
      if (i < ld) s = fmaf(kr[q], __ldg(&uj[i]), s);
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    const float v = __fdividef(__uint_as_float(en.y), s);
    float* xj = x + (size_t)en.x * ldu;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = lane + 32 * q;
      if (i < ld) atomicAdd(&xj[i], kr[q] * v);
    }
  }
}

__global__ void wm_init_kernel(float* __restrict__ u, float* __restrict__ x, int ldu,
                               int64_t N, const uint32_t* __restrict__ vr_dev) {
  const int vr = (int)*vr_dev;
  const int64_t total = N * ldu;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldu);
    u[k] = i < vr ? (float)vr : 0.f;  // cold start u = v_r (fused:188-191)
    x[k] = 0.f;
  }
}

__global__ void wm_update_kernel(float* __restrict__ u, float* __restrict__ x, int ldu,
                                 int64_t N, const uint32_t* __restrict__ vr_dev,
                                 const float* __restrict__ rinv) {
  const int vr = (int)*vr_dev;
  const int64_t total = N * ldu;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(k % ldu);
    u[k] = i < vr ? __frcp_rn(rinv[i] * x[k]) : 0.f;  // u = 1 / x (fused:304-319)
    x[k] = 0.f;
  }
}

template <int Q>
__global__ void __launch_bounds__(kWmThreads)
wm_final_kernel(const float* __restrict__ K, int ld, float expo,
                const int64_t* __restrict__ rp, int64_t V,
                const uint2* __restrict__ went, int64_t nnz, int64_t chunk,
                const float* __restrict__ u, int ldu, const float* __restrict__ mrow,
                double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t e0 = warp * chunk;
  if (e0 >= nnz) return;
  const int64_t e1 = min(nnz, e0 + chunk);
  int64_t w = row_of(rp, V, e0);
  int64_t wend = rp[w + 1];
  float kr[Q], kl[Q];  // K and K log2 K of the current row
  auto load_row = [&](int64_t ww) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = lane + 32 * q;
      kr[q] = i < ld ? __ldg(&K[(size_t)ww * ld + i]) : 0.f;
      kl[q] = kr[q] > 0.f ? kr[q] * __log2f(kr[q]) : 0.f;
    }
  };
  load_row(w);
  const float km_scale = 0.69314718f / expo;  // K.*M = K ln K / expo
  for (int64_t e = e0; e < e1; ++e) {
    while (e >= wend) {
      ++w;
      wend = rp[w + 1];
      if (e < wend) load_row(w);
    }
    const uint2 en = __ldg(&went[e]);
    const float* uj = u + (size_t)en.x * ldu;
    float s = 0.f, t = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int i = lane + 32 * q;
      if (i < ld) {
        const float ui = __ldg(&uj[i]);
        s = fmaf(kr[q], ui, s);
        t = fmaf(kl[q], ui, t);
      }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, off);
      t += __shfl_xor_sync(0xffffffffu, t, off);
    }
    if (lane == 0) {
      const float c = __uint_as_float(en.y);
      const float v = __fdividef(c, s);
      double add = (double)v * (double)(t * km_scale);
      if (mrow) add += (double)c * (double)__ldg(&mrow[w]);  // row-scaled panel
      atomicAdd(&out[en.x], add);
    }
  }
}

__global__ void wm_finish_kernel(const float* __restrict__ u, int ldu, int64_t N,
                                 const uint32_t* __restrict__ vr_dev,
                                 double* __restrict__ out, bool scaled) {
  const int vr = (int)*vr_dev;
  const int lane = threadIdx.x & 31;
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= N) return;
  bool bad = false;
  for (int i = lane; i < vr; i += 32) {
    const float ui = u[(size_t)j * ldu + i];
    bad |= !isfinite(ui) || (scaled && ui > kScaledUMax);  // see solve.cu
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    if (vr == 0) out[j] = 0.0;  // no source word: an empty sum (fused:387)
    else if (bad) out[j] = __longlong_as_double(0x7ff8000000000000ll);
  }
}

template <int Q>
int launch_word_t(const float* K, int ld, float expo, const SourceSel& s,
                  const WordMajor& wm, int64_t N, int max_iter, float* u, float* x,
                  int num_sms, double* out, cudaStream_t st) {
  const int ldu = ld;
  const int sms = num_sms > 0 ? num_sms : 148;
  // nnz-balanced chunks: about 8 warps of work per SM slot, each chunk long
  // enough that consecutive entries share K rows
  const int64_t warps = (int64_t)sms * (kWmThreads / 32) * 4;
  int64_t chunk = (wm.nnz + warps - 1) / warps;
  if (chunk < 16) chunk = 16;
  const int64_t nwarp = (wm.nnz + chunk - 1) / chunk;
  const unsigned pgrid = (unsigned)((nwarp * 32 + kWmThreads - 1) / kWmThreads);
  const unsigned egrid = (unsigned)sms * 8;
  wm_init_kernel<<<egrid, 256, 0, st>>>(u, x, ldu, N, s.vr);
  cudaMemsetAsync(out, 0, (size_t)N * sizeof(double), st);
  int n = 2;
  for (int it = 0; it < max_iter; ++it) {
    wm_pass_kernel<Q><<<pgrid, kWmThreads, 0, st>>>(K, ld, wm.row_ptr, wm.V, wm.ent,
                                                    wm.nnz, chunk, u, x, ldu);
    wm_update_kernel<<<egrid, 256, 0, st>>>(u, x, ldu, N, s.vr, s.rinv);
    n += 2;
  }
  wm_final_kernel<Q><<<pgrid, kWmThreads, 0, st>>>(K, ld, expo, wm.row_ptr, wm.V, wm.ent,
                                                   wm.nnz, chunk, u, ldu, wm.mrow, out);
  wm_finish_kernel<<<(unsigned)((N * 32 + 255) / 256), 256, 0, st>>>(u, ldu, N, s.vr, out,
                                                                     wm.mrow != nullptr);
  return n + 2;
}

}  // namespace

int launch_solve_word(const float* K, int ld, float expo, uint32_t vr_cap,
                      const SourceSel& s, const WordMajor& wm, int64_t N, int max_iter,
                      float* u, float* x, int num_sms, double* out, cudaStream_t st) {
  if (N <= 0) return 0;
  if (wm.nnz == 0) {
    cudaMemsetAsync(u, 0xff, (size_t)N * ld * sizeof(float), st);  // NaN: empty
    wm_finish_kernel<<<(unsigned)((N * 32 + 255) / 256), 256, 0, st>>>(u, ld, N, s.vr, out,
                                                                       false);
    return 1;
  }
  const int q = (int)((vr_cap + 31) / 32);
  if (q <= 1) return launch_word_t<1>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  if (q <= 2) return launch_word_t<2>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  if (q <= 4) return launch_word_t<4>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  if (q <= 8) return launch_word_t<8>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  if (q <= 16) return launch_word_t<16>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  if (q <= kWmMaxQ)
    return launch_word_t<kWmMaxQ>(K, ld, expo, s, wm, N, max_iter, u, x, num_sms, out, st);
  return -1;
}

}  // namespace wmd
