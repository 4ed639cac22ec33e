// FP64 re-solve of the documents a row-scaled FP32 panel cannot carry.
//
// The row scaling of panel_rescale.cu keeps every vocabulary row's largest K
// entry at 1, which removes the underflow of whole documents; what it cannot
// remove is a source word that is far (by more than ~87 / lambda in M) from
// every word of one document relative to those words' nearest source words:
// its column of the document's rows then underflows to 0 in FP32, x_i = 0 and
// the document's score is not finite, where the reference's FP64
// K = exp(lamda M) (sinkhorn_wmd_fused.cpp:217) is still finite.  Those
// documents are listed after the FP32 solve and solved again here in FP64,
// with M recomputed exactly from the embeddings (sqrt(sum_t (E_wt - S_it)^2),
// the reference's euclidean_distance, fused:35-43) and K = exp(-lambda M) in
// FP64, by the reference's recurrence (fused:188-393):
//
//   u = v_r;  repeat: s_k = K_k . u, v_k = c_k / s_k, x_i = (K^T v)_i / r_i,
//   u = 1 / x;  final: s, v as above, WMD = sum_k v_k sum_i K_ki M_ki u_i
//
// with the same stopping rule as the FP32 solves (tol > 0: stop after the
// first update whose marginal residual sum_i |u_i (K v)_i - r_i| is <= tol),
// unrelaxed.  A document the FP64 recurrence cannot carry either (lambda M
// beyond ~708) stays NaN, as in the reference.  One CTA per listed document;
// M is recomputed on every use (d FMAs per entry), which is affordable only
// because the list is short.  Used only in the row-scaled form.
#include "wmd_internal.cuh"

namespace wmd {
namespace {

constexpr int kXT = 256;          // threads per document
constexpr int kXD = 4;            // source words per thread (v_r <= 1024)

__global__ void list_nonfinite_kernel(const double* __restrict__ out,
                                      const int64_t* __restrict__ col_ptr, int64_t N,
                                      const uint32_t* __restrict__ vr_dev,
                                      int32_t* __restrict__ list,
                                      unsigned* __restrict__ count, unsigned cap) {
  const int vr = (int)*vr_dev;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < N;
       j += (int64_t)gridDim.x * blockDim.x) {
    if (vr > 0 && !isfinite(out[j]) && col_ptr[j + 1] > col_ptr[j]) {
      const unsigned pos = atomicAdd(count, 1u);
      if (pos < cap) list[pos] = (int32_t)j;
    }
  }
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();  // red is free (its previous readers are done)
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < kXT / 32; ++w) t += red[w];
  return t;
}

__global__ void __launch_bounds__(kXT)
solve_exact_f64_kernel(const float* __restrict__ E32, int d, const float* __restrict__ S,
                       const float* __restrict__ rinv, const uint32_t* __restrict__ vr_dev,
                       const int64_t* __restrict__ col_ptr, const uint2* __restrict__ ent,
                       const int32_t* __restrict__ list, const unsigned* __restrict__ count,
                       unsigned cap, double lambda, int max_iter, float tol,
                       int* __restrict__ iters_out, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* red = reinterpret_cast<double*>(smem_raw);          // [kXT / 32]
  float* Ek = reinterpret_cast<float*>(red + kXT / 32);       // [d]
  double* vk = reinterpret_cast<double*>(Ek + ((d + 1) & ~1));  // [n]
  const int tid = threadIdx.x;
  const int vr = (int)*vr_dev;
  const unsigned listed = min(*count, cap);
  double r[kXD];
  for (int q = 0; q < kXD; ++q) {
    const int i = tid + q * kXT;
    r[q] = i < vr ? 1.0 / (double)rinv[i] : 0.0;
  }
  // M and K of (document word held in Ek, source word i)
  auto mk = [&](int i, double& M, double& K) {
    const float* s = S + (size_t)i * d;
    float a = 0.f;
    for (int t = 0; t < d; ++t) {
      const float z = Ek[t] - s[t];
      a = fmaf(z, z, a);
    }
    M = (double)sqrtf(a);
    K = exp(-lambda * M);
  };
  auto load_row = [&](uint32_t w) {
    __syncthreads();  // previous users of Ek are done
    for (int t = tid; t < d; t += kXT) Ek[t] = E32[(size_t)w * d + t];
    __syncthreads();
  };
  for (unsigned e = blockIdx.x; e < listed; e += gridDim.x) {
    const int64_t j = list[e];
    const int64_t b = col_ptr[j];
    const int n = (int)(col_ptr[j + 1] - b);
    double u[kXD];
    for (int q = 0; q < kXD; ++q) u[q] = tid + q * kXT < vr ? (double)vr : 0.0;
    // s-step: v_k = c_k / (K_k . u) for every document word
    auto sstep = [&]() {
      for (int k = 0; k < n; ++k) {
        const uint2 en = ent[b + k];
        load_row(en.x);
        double p = 0.0;
        for (int q = 0; q < kXD; ++q) {
          const int i = tid + q * kXT;
          if (i < vr) {
            double M, K;
            mk(i, M, K);
            p += K * u[q];
          }
        }
        const double s = block_sum(p, red);
        if (tid == 0) vk[k] = (double)__uint_as_float(en.y) / s;
      }
      __syncthreads();
    };
    int it = 0;
    double res = 0.0;
    while (it < max_iter && !(it > 0 && tol > 0.f && res <= (double)tol)) {
      sstep();
      double x[kXD] = {0.0, 0.0, 0.0, 0.0};
      for (int k = 0; k < n; ++k) {
        load_row(ent[b + k].x);
        const double v = vk[k];
        for (int q = 0; q < kXD; ++q) {
          const int i = tid + q * kXT;
          if (i < vr) {
            double M, K;
            mk(i, M, K);
            x[q] += K * v;
          }
        }
      }
      double pr = 0.0;
      for (int q = 0; q < kXD; ++q) {
        const int i = tid + q * kXT;
        if (i < vr) {
          pr += fabs(u[q] * x[q] - r[q]);  // u_i (K v)_i - r_i
          u[q] = r[q] / x[q];              // 1 / (x_i / r_i)
        }
      }
      res = block_sum(pr, red);
      ++it;
    }
    // Final half-step and the FP64 reduction (fused:339-393).
    sstep();
    double acc = 0.0;
    for (int k = 0; k < n; ++k) {
      load_row(ent[b + k].x);
      double p = 0.0;
      for (int q = 0; q < kXD; ++q) {
        const int i = tid + q * kXT;
        if (i < vr) {
          double M, K;
          mk(i, M, K);
          p += K * M * u[q];
        }
      }
      acc += vk[k] * p;  // this thread's share
    }
    bool bad = false;
    for (int q = 0; q < kXD; ++q) bad |= (tid + q * kXT < vr) && !isfinite(u[q]);
    const double tot = block_sum(acc, red);
    bad = __syncthreads_or(bad);
    if (tid == 0) {
      out[j] = bad ? __longlong_as_double(0x7ff8000000000000ll) : tot;
      if (iters_out) iters_out[j] = it;
    }
  }
}

}  // namespace

size_t exact_f64_list_cap() { return 4096; }

int launch_exact_f64(const float* E32, uint64_t d, const SourceSel& s, const Targets& t,
                     float expo, const SolveCtl& ctl, int max_doc_len, int32_t* list,
                     unsigned* count, int num_sms, double* out, cudaStream_t st) {
  if (t.N <= 0 || expo == 0.f) return 0;
  const unsigned cap = (unsigned)exact_f64_list_cap();
  int64_t g = (t.N + 255) / 256;
  if (g > 4 * (int64_t)(num_sms > 0 ? num_sms : 148)) g = 4 * (int64_t)(num_sms > 0 ? num_sms : 148);
  cudaMemsetAsync(count, 0, sizeof(unsigned), st);
  list_nonfinite_kernel<<<(unsigned)g, 256, 0, st>>>(out, t.col_ptr, t.N, s.vr, list,
                                                     count, cap);
  const size_t smem = (kXT / 32) * sizeof(double) + (((size_t)d + 1) & ~(size_t)1) * 4 +
                      (size_t)max_doc_len * sizeof(double);
  if (smem > 200 * 1024) return -1;  // documents too long for the FP64 re-solve
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    cudaFuncSetAttribute(solve_exact_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    attr[dev] = true;
  }
  solve_exact_f64_kernel<<<num_sms > 0 ? num_sms : 148, kXT, smem, st>>>(
      E32, (int)d, s.S, s.rinv, s.vr, t.col_ptr, t.ent, list, count, cap,
      -(double)expo, ctl.max_iter, ctl.tol, ctl.iters, out);
  return 2;
}

}  // namespace wmd
