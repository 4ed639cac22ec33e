// Learned warm start: training side.
//
// No reference counterpart (the reference always starts from u = v_r,
// sinkhorn_wmd_fused.cpp:188-191, and runs a fixed iteration count).  A small
// MLP predicts log u_i for (source word i, target document j); Sinkhorn then
// starts from exp(prediction) instead of the cold start.  Because the
// iteration is invariant to a per-document scaling of u (u -> a u gives
// v -> v / a and the same plan), the training loss ignores each document's
// mean offset: per (source, document) group the error e_i = y_i - t_i is
// centred, L = sum (e_i - mean_group e)^2 / rows.
//
// Features of a row (width F = 2d + 5 rounded up to 16):
//   [0, d)      embedding of source word i
//   [d, 2d)     target centroid: c-weighted mean of the document's embeddings
//   2d, 2d+1    r_i, log r_i
//   2d+2..2d+4  min / mean / max of M(i, w) over the document's words w,
//               M read back from the cost panel as ln(K) / expo
// Network: standardise (per-feature shift/scale), 256 GELU, 256 GELU, 1.
// GELU is the tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
//
// Labels come from the plain solver itself run to convergence in FP64 over
// the FP32 cost panel (solve_f64_kernel): log of the converged u for
// documents whose marginal residual reached the label tolerance.
//
// Training kernels are FP32 CUDA-core kernels: a generic tiled GEMM with
// bias+GELU and GELU'-gating epilogues, the head/loss kernel, column
// reductions for the bias gradients, and Adam.  The fused inference kernel
// (BF16 tensor cores) is in ws_infer.cu.
#include <math.h>

#include "wmd_internal.cuh"

namespace wmd {

WsLayout ws_layout(int d) {
  WsLayout L;
  L.d = d;
  L.F = ((2 * d + 5) + 15) & ~15;
  size_t o = 0;
  L.shift = o; o += L.F;
  L.scale = o; o += L.F;
  L.W1 = o; o += (size_t)kWsH * L.F;
  L.b1 = o; o += kWsH;
  L.W2 = o; o += (size_t)kWsH * kWsH;
  L.b2 = o; o += kWsH;
  L.w3 = o; o += kWsH;
  L.b3 = o; o += 4;
  L.count = o;
  return L;
}

__device__ __forceinline__ float gelu_t(float z) {
  const float a = 0.7978845608f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.f + tanhf(a));
}
__device__ __forceinline__ float gelu_t_grad(float z) {
  const float a = 0.7978845608f * (z + 0.044715f * z * z * z);
  const float t = tanhf(a);
  return 0.5f * (1.f + t) +
         0.5f * z * (1.f - t * t) * 0.7978845608f * (1.f + 3.f * 0.044715f * z * z);
}

// ---------------------------------------------------------------------------
// Target centroids: C[j] = sum_w c_w E_w / sum_w c_w (zero for an empty
// document).  One warp per document.
__global__ void centroid_kernel(const float* __restrict__ E32, int d,
                                const int64_t* __restrict__ col_ptr,
                                const uint2* __restrict__ ent, int64_t N,
                                float* __restrict__ C) {
  const int lane = threadIdx.x & 31;
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= N) return;
  const int64_t b = col_ptr[j], e = col_ptr[j + 1];
  float wsum = 0.f;
  for (int64_t k = b; k < e; ++k) wsum += __uint_as_float(ent[k].y);
  const float inv = wsum > 0.f ? 1.f / wsum : 0.f;
  for (int c = lane; c < d; c += 32) {
    float acc = 0.f;
    for (int64_t k = b; k < e; ++k) {
      const uint2 en = ent[k];
      acc = fmaf(__uint_as_float(en.y), E32[(size_t)en.x * d + c], acc);
    }
    C[(size_t)j * d + c] = acc * inv;
  }
}

// ---------------------------------------------------------------------------
// Converged FP64 solve of listed documents (label generation).  One warp per
// document; lane owns source dimensions lane + 32 t (v_r <= 512).  Same
// recurrence as the plain solve (fused:246-335) in FP64, iterated until the
// marginal residual sum_i |u_i (K v)_i - r_i| <= tol or `cap` updates.
// Outputs the scaling u after the last update, the update count and the last
// residual measured.
__global__ void solve_f64_kernel(const float* __restrict__ K, int ld, int vr,
                                 const double* __restrict__ r,
                                 const int64_t* __restrict__ col_ptr,
                                 const uint2* __restrict__ ent,
                                 const int32_t* __restrict__ docs, int ndocs,
                                 double tol, int cap, double* __restrict__ u_out,
                                 int* __restrict__ it_out,
                                 double* __restrict__ res_out) {
  constexpr int T = 16;
  const int lane = threadIdx.x & 31;
  const int q = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (q >= ndocs) return;
  const int64_t j = docs[q];
  const int64_t b = col_ptr[j];
  const int n = (int)(col_ptr[j + 1] - b);
  double u[T], rr[T];
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int D = lane + 32 * t;
    rr[t] = D < vr ? r[D] : 0.0;
    u[t] = D < vr ? (double)vr : 0.0;
  }
  int it = 0;
  double res = INFINITY;
  while (it < cap) {
    double x[T];
#pragma unroll
    for (int t = 0; t < T; ++t) x[t] = 0.0;
    for (int k = 0; k < n; ++k) {
      const uint2 en = ent[b + k];
      const float* row = K + (size_t)en.x * ld;
      double kv[T];
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < T; ++t) {
        const int D = lane + 32 * t;
        kv[t] = D < vr ? (double)row[D] : 0.0;
        s = fma(kv[t], u[t], s);
      }
#pragma unroll
      for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
      const double v = (double)__uint_as_float(en.y) / s;
#pragma unroll
      for (int t = 0; t < T; ++t) x[t] = fma(kv[t], v, x[t]);
    }
    double rs = 0.0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const int D = lane + 32 * t;
      if (D < vr) {
        rs += fabs(u[t] * x[t] - rr[t]);
        u[t] = rr[t] / x[t];
      }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, off);
    res = rs;
    ++it;
    if (!(res > tol)) break;  // also stops on NaN
  }
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int D = lane + 32 * t;
    if (D < vr) u_out[(size_t)q * vr + D] = u[t];
  }
  if (lane == 0) {
    it_out[q] = it;
    res_out[q] = res;
  }
}

// ---------------------------------------------------------------------------
// Training rows for one source: row `row0[q] + m` holds the features of
// (source word sel[q*G + m], document docs[q]) and the label log u.  One warp
// per row; the M statistics are reduced over the document's words by the
// lanes.
__global__ void ws_rows_kernel(const float* __restrict__ E32, int d,
                               const float* __restrict__ C,
                               const float* __restrict__ K, int ld, float expo,
                               const uint32_t* __restrict__ src_ids,
                               const double* __restrict__ r, int vr,
                               const int64_t* __restrict__ col_ptr,
                               const uint2* __restrict__ ent,
                               const int32_t* __restrict__ docs,
                               const double* __restrict__ u, int ndocs,
                               const int32_t* __restrict__ sel, int G,
                               const int64_t* __restrict__ row0, int F,
                               float* __restrict__ X, float* __restrict__ y,
                               const float* __restrict__ mrow) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gw >= (int64_t)ndocs * G) return;
  const int q = (int)(gw / G), m = (int)(gw % G);
  const int i = sel[(size_t)q * G + m];
  if (i < 0 || row0[q] < 0) return;
  const int64_t row = row0[q] + m;
  const int64_t j = docs[q];
  float* xr = X + (size_t)row * F;
  const uint32_t wi = src_ids[i];
  for (int c = lane; c < d; c += 32) {
    xr[c] = E32[(size_t)wi * d + c];
    xr[d + c] = C[(size_t)j * d + c];
  }
  const int64_t b = col_ptr[j];
  const int n = (int)(col_ptr[j + 1] - b);
  float mn = INFINITY, mx = -INFINITY, sm = 0.f;
  for (int k = lane; k < n; k += 32) {
    const uint32_t w = ent[b + k].x;
    const float kv = K[(size_t)w * ld + i];
    const float Mv = fmaxf(logf(fmaxf(kv, 1e-38f)) / expo, 0.f) + (mrow ? mrow[w] : 0.f);
    mn = fminf(mn, Mv);
    mx = fmaxf(mx, Mv);
    sm += Mv;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, off));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    sm += __shfl_xor_sync(0xffffffffu, sm, off);
  }
  if (lane == 0) {
    const double ri = r[i];
    xr[2 * d] = (float)ri;
    xr[2 * d + 1] = (float)log(ri);
    xr[2 * d + 2] = n > 0 ? mn : 0.f;
    xr[2 * d + 3] = n > 0 ? sm / (float)n : 0.f;
    xr[2 * d + 4] = n > 0 ? mx : 0.f;
    y[row] = (float)log(u[(size_t)q * vr + i]);
  }
  for (int c = 2 * d + 5 + lane; c < F; c += 32) xr[c] = 0.f;
}

// Per-feature sums and sums of squares over row chunks (FP64 partials
// [chunks][F] each), for the standardisation.
__global__ void ws_colstats_kernel(const float* __restrict__ X, int64_t P, int F,
                                   int64_t rows_per_chunk, double* __restrict__ s1,
                                   double* __restrict__ s2) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= F) return;
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_chunk;
  const int64_t r1 = min(P, r0 + rows_per_chunk);
  double a = 0.0, b = 0.0;
  for (int64_t rr = r0; rr < r1; ++rr) {
    const double v = X[(size_t)rr * F + c];
    a += v;
    b += v * v;
  }
  s1[(size_t)blockIdx.x * F + c] = a;
  s2[(size_t)blockIdx.x * F + c] = b;
}

// X <- (X - shift) * scale, in place.
__global__ void ws_standardize_kernel(float* __restrict__ X, int64_t P, int F,
                                      const float* __restrict__ shift,
                                      const float* __restrict__ scale) {
  const int64_t total = P * (int64_t)F;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % F);
    X[i] = (X[i] - shift[c]) * scale[c];
  }
}

// ---------------------------------------------------------------------------
// Generic FP32 GEMM: C[m][n] = epi(sum_k A(m,k) B(k,n)) with
// A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn].  64x64 tiles, 16-deep
// k-slices in shared memory, 4x4 outputs per thread.
enum { EPI_STORE = 0, EPI_BIAS_GELU = 1, EPI_GELU_GRAD = 2 };

template <int EPI>
__global__ void __launch_bounds__(256)
ws_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int64_t sam,
               int64_t sak, const float* __restrict__ B, int64_t sbk, int64_t sbn,
               float* __restrict__ Cm, int64_t ldc, const float* __restrict__ bias,
               const float* __restrict__ aux, float* __restrict__ Z) {
  __shared__ float As[16][65];
  __shared__ float Bs[16][65];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int e = tid + 256 * r;
      int ml, kl;
      if (sak == 1) { kl = e & 15; ml = e >> 4; } else { ml = e & 63; kl = e >> 6; }
      const int m = m0 + ml, k = k0 + kl;
      As[kl][ml] = (m < M && k < K) ? A[(int64_t)m * sam + (int64_t)k * sak] : 0.f;
      int nl, kb;
      if (sbn == 1) { nl = e & 63; kb = e >> 6; } else { kb = e & 15; nl = e >> 4; }
      const int n = n0 + nl, kk = k0 + kb;
      Bs[kb][nl] = (n < N && kk < K) ? B[(int64_t)kk * sbk + (int64_t)n * sbn] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) bb[jj] = Bs[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fmaf(a[i], bb[jj], acc[i][jj]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int n = n0 + tx + 16 * jj;
      if (n >= N) continue;
      float v = acc[i][jj];
      if (EPI == EPI_BIAS_GELU) {
        v += bias[n];
        Z[(int64_t)m * ldc + n] = v;
        v = gelu_t(v);
      } else if (EPI == EPI_GELU_GRAD) {
        v *= gelu_t_grad(aux[(int64_t)m * ldc + n]);
      }
      Cm[(int64_t)m * ldc + n] = v;
    }
  }
}

template <int EPI>
static void gemm(int M, int N, int K, const float* A, int64_t sam, int64_t sak,
                 const float* B, int64_t sbk, int64_t sbn, float* C, int64_t ldc,
                 const float* bias, const float* aux, float* Z, cudaStream_t st) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  ws_gemm_kernel<EPI><<<grid, 256, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C,
                                            ldc, bias, aux, Z);
}

// y[m] = H2[m] . w3 + b3; one warp per row.
__global__ void ws_head_kernel(const float* __restrict__ H2, int64_t P,
                               const float* __restrict__ w3, const float* __restrict__ b3,
                               float* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int64_t m = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (m >= P) return;
  float s = 0.f;
  for (int c = lane; c < kWsH; c += 32) s = fmaf(H2[(size_t)m * kWsH + c], w3[c], s);
#pragma unroll
  for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) y[m] = s + b3[0];
}

// Group-centred squared error: per group g (rows gptr[g]..gptr[g+1]),
// e = y - t, dy = 2 (e - mean e) / P, loss_g = sum (e - mean e)^2 / P.
// One warp per group.
__global__ void ws_loss_kernel(const float* __restrict__ y, const float* __restrict__ t,
                               const int64_t* __restrict__ gptr, int64_t ngroups,
                               int64_t P, float* __restrict__ dy,
                               double* __restrict__ loss_g) {
  const int lane = threadIdx.x & 31;
  const int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (g >= ngroups) return;
  const int64_t a = gptr[g], b = gptr[g + 1];
  double s = 0.0;
  for (int64_t m = a + lane; m < b; m += 32) s += (double)y[m] - (double)t[m];
#pragma unroll
  for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  const double mean = b > a ? s / (double)(b - a) : 0.0;
  double l = 0.0;
  for (int64_t m = a + lane; m < b; m += 32) {
    const double e = (double)y[m] - (double)t[m] - mean;
    l += e * e;
    dy[m] = (float)(2.0 * e / (double)P);
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
  if (lane == 0) loss_g[g] = l / (double)P;
}

// dZ2[m][n] = dy[m] w3[n] GELU'(Z2[m][n]).
__global__ void ws_dz2_kernel(const float* __restrict__ dy, const float* __restrict__ w3,
                              const float* __restrict__ Z2, int64_t P,
                              float* __restrict__ dZ2) {
  const int64_t total = P * kWsH;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t m = i / kWsH;
    const int n = (int)(i % kWsH);
    dZ2[i] = dy[m] * w3[n] * gelu_t_grad(Z2[i]);
  }
}

// Column sums out[c] = sum_m X[m][c] * (wrow ? wrow[m] : 1), deterministic:
// partials over fixed row chunks, then a fixed-order sum.
__global__ void ws_colsum_partial_kernel(const float* __restrict__ X, int64_t P, int N,
                                         const float* __restrict__ wrow,
                                         int64_t rows_per_chunk,
                                         float* __restrict__ part) {
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_chunk;
  const int64_t r1 = min(P, r0 + rows_per_chunk);
  float s = 0.f;
  for (int64_t m = r0; m < r1; ++m) s = fmaf(X[(size_t)m * N + c], wrow ? wrow[m] : 1.f, s);
  part[(size_t)blockIdx.x * N + c] = s;
}
__global__ void ws_colsum_final_kernel(const float* __restrict__ part, int chunks, int N,
                                       float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  float s = 0.f;
  for (int k = 0; k < chunks; ++k) s += part[(size_t)k * N + c];
  out[c] = s;
}

// Adam on params[lo, hi) (the trainable range), bias-corrected.
__global__ void ws_adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                               float* __restrict__ m1, float* __restrict__ m2,
                               int64_t lo, int64_t hi, float lr, float b1, float b2,
                               float eps, float c1, float c2) {
  for (int64_t i = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

// Gathers whole groups into a contiguous batch: rows of group perm[g] for
// g in [g0, g1) -> Xb, tb; batch group pointers -> gb.
__global__ void ws_gather_kernel(const float* __restrict__ X, const float* __restrict__ t,
                                 const int64_t* __restrict__ gptr,
                                 const int64_t* __restrict__ perm,
                                 const int64_t* __restrict__ bptr, int64_t g0,
                                 int64_t ng, int F, float* __restrict__ Xb,
                                 float* __restrict__ tb) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gw >= ng) return;
  const int64_t g = perm[g0 + gw];
  const int64_t a = gptr[g], b = gptr[g + 1];
  const int64_t o = bptr[gw];
  for (int64_t m = a; m < b; ++m) {
    for (int c = lane; c < F; c += 32) Xb[(size_t)(o + m - a) * F + c] = X[(size_t)m * F + c];
    if (lane == 0) tb[o + m - a] = t[m];
  }
}

// ---------------------------------------------------------------------------
// Host launchers.
int launch_centroids(const float* E32, int d, const int64_t* col_ptr,
                     const uint2* ent, int64_t N, float* C, cudaStream_t st) {
  const int64_t threads = N * 32;
  centroid_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(E32, d, col_ptr,
                                                                      ent, N, C);
  return 1;
}

int launch_solve_f64(const float* K, int ld, int vr, const double* r,
                     const int64_t* col_ptr, const uint2* ent, const int32_t* docs,
                     int ndocs, double tol, int cap, double* u_out, int* it_out,
                     double* res_out, cudaStream_t st) {
  if (ndocs <= 0) return 0;
  if (vr > 512) return -1;
  const int64_t threads = (int64_t)ndocs * 32;
  solve_f64_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(
      K, ld, vr, r, col_ptr, ent, docs, ndocs, tol, cap, u_out, it_out, res_out);
  return 1;
}

int launch_ws_rows(const float* E32, int d, const float* C, const float* K, int ld,
                   float expo, const uint32_t* src_ids, const double* r, int vr,
                   const int64_t* col_ptr, const uint2* ent, const int32_t* docs,
                   const double* u, int ndocs, const int32_t* sel, int G,
                   const int64_t* row0, int F, float* X, float* y, cudaStream_t st,
                   const float* mrow) {
  const int64_t threads = (int64_t)ndocs * G * 32;
  if (threads == 0) return 0;
  ws_rows_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      E32, d, C, K, ld, expo, src_ids, r, vr, col_ptr, ent, docs, u, ndocs, sel, G,
      row0, F, X, y, mrow);
  return 1;
}

int launch_ws_colstats(const float* X, int64_t P, int F, double* s1, double* s2,
                       int chunks, cudaStream_t st) {
  const int64_t rpc = (P + chunks - 1) / chunks;
  dim3 grid((unsigned)chunks, (unsigned)((F + 255) / 256));
  ws_colstats_kernel<<<grid, 256, 0, st>>>(X, P, F, rpc, s1, s2);
  return 1;
}

int launch_ws_standardize(float* X, int64_t P, int F, const float* shift,
                          const float* scale, cudaStream_t st) {
  ws_standardize_kernel<<<1184, 256, 0, st>>>(X, P, F, shift, scale);
  return 1;
}

static void colsum(const float* X, int64_t P, int N, const float* wrow, float* part,
                   float* out, cudaStream_t st) {
  const int chunks = 64;
  const int64_t rpc = (P + chunks - 1) / chunks;
  dim3 grid(chunks, (unsigned)((N + 255) / 256));
  ws_colsum_partial_kernel<<<grid, 256, 0, st>>>(X, P, N, wrow, rpc, part);
  ws_colsum_final_kernel<<<(N + 255) / 256, 256, 0, st>>>(part, chunks, N, out);
}

size_t ws_scratch_floats(int64_t P, int F) {
  // Z1, H1, Z2, H2, dZ2, dZ1 [P][H]; y, dy [P]; colsum partials 64 x max(F, H)
  return (size_t)P * kWsH * 6 + 2 * (size_t)P + 64 * (size_t)(F > kWsH ? F : kWsH) + 64;
}

// Forward + backward of a batch of P standardised rows X [P][F] with targets
// t and groups gptr [ngroups + 1] (rows contiguous per group).  grad gets
// the gradient of every parameter (zero for shift/scale); loss_g the
// per-group loss terms.  Returns launches.
int launch_ws_fwd_bwd(const WsLayout& L, const float* params, const float* X,
                      const float* t, const int64_t* gptr, int64_t ngroups,
                      int64_t P, float* grad, double* loss_g, float* scratch,
                      cudaStream_t st) {
  const int F = L.F, H = kWsH;
  float* Z1 = scratch;
  float* H1 = Z1 + (size_t)P * H;
  float* Z2 = H1 + (size_t)P * H;
  float* H2 = Z2 + (size_t)P * H;
  float* dZ2 = H2 + (size_t)P * H;
  float* dZ1 = dZ2 + (size_t)P * H;
  float* y = dZ1 + (size_t)P * H;
  float* dy = y + P;
  float* part = dy + P;
  const float* W1 = params + L.W1;
  const float* W2 = params + L.W2;
  // forward
  gemm<EPI_BIAS_GELU>((int)P, H, F, X, F, 1, W1, 1, F, H1, H, params + L.b1, nullptr, Z1, st);
  gemm<EPI_BIAS_GELU>((int)P, H, H, H1, H, 1, W2, 1, H, H2, H, params + L.b2, nullptr, Z2, st);
  ws_head_kernel<<<(unsigned)((P * 32 + 255) / 256), 256, 0, st>>>(H2, P, params + L.w3,
                                                                  params + L.b3, y);
  ws_loss_kernel<<<(unsigned)((ngroups * 32 + 255) / 256), 256, 0, st>>>(
      y, t, gptr, ngroups, P, dy, loss_g);
  // backward
  cudaMemsetAsync(grad, 0, (L.W1) * sizeof(float), st);  // shift/scale: not trained
  cudaMemsetAsync(grad + L.b3, 0, 4 * sizeof(float), st);
  colsum(H2, P, H, dy, part, grad + L.w3, st);           // dw3 = H2^T dy
  colsum(dy, P, 1, nullptr, part, grad + L.b3, st);      // db3 = sum dy
  ws_dz2_kernel<<<1184, 256, 0, st>>>(dy, params + L.w3, Z2, P, dZ2);
  colsum(dZ2, P, H, nullptr, part, grad + L.b2, st);     // db2
  gemm<EPI_STORE>(H, H, (int)P, dZ2, 1, H, H1, H, 1, grad + L.W2, H, nullptr, nullptr,
                  nullptr, st);                          // dW2 = dZ2^T H1
  gemm<EPI_GELU_GRAD>((int)P, H, H, dZ2, H, 1, W2, H, 1, dZ1, H, nullptr, Z1, nullptr,
                      st);                               // dZ1 = (dZ2 W2) * GELU'(Z1)
  colsum(dZ1, P, H, nullptr, part, grad + L.b1, st);     // db1
  gemm<EPI_STORE>(H, F, (int)P, dZ1, 1, H, X, F, 1, grad + L.W1, F, nullptr, nullptr,
                  nullptr, st);                          // dW1 = dZ1^T X
  return 15;
}

int launch_ws_adam(const WsLayout& L, float* params, const float* grad, float* m1,
                   float* m2, float lr, int step, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  ws_adam_kernel<<<592, 256, 0, st>>>(params, grad, m1, m2, (int64_t)L.W1,
                                      (int64_t)L.count, lr, b1, b2, 1e-8f, c1, c2);
  return 1;
}

int launch_ws_gather(const float* X, const float* t, const int64_t* gptr,
                     const int64_t* perm, const int64_t* bptr, int64_t g0, int64_t ng,
                     int F, float* Xb, float* tb, cudaStream_t st) {
  if (ng <= 0) return 0;
  ws_gather_kernel<<<(unsigned)((ng * 32 + 255) / 256), 256, 0, st>>>(
      X, t, gptr, perm, bptr, g0, ng, F, Xb, tb);
  return 1;
}

}  // namespace wmd
