// FP32 CUDA-core cost panel.
//
// For every vocabulary word w and selected source word i this computes
//   M[w,i] = ||E_w - S_i||,  K[w,i] = exp(expo * M),  KM[w,i] = K * M
// and stores K and KM in the word-major layout [V][ld] that the reference's
// fused solver uses for K and K_over_r (sinkhorn_wmd_fused.cpp:197-223), so a
// target document's gather of one word is one contiguous ld-float row.
//
// M comes from the GEMM form ||E_w||^2 + ||S_i||^2 - 2 E_w.S_i (a BM x 32
// register-tiled SIMT GEMM over d).  That form cancels catastrophically for
// close pairs (a word against itself gives M ~ 1e-3 instead of 0, i.e. a 1%
// error in K at lambda = 10), so pairs whose GEMM-form M^2 falls below
// max(0.25, (|E_w|^2 + |S_i|^2) / 30) are listed for near_fixup_kernel, which
// recomputes them directly as sqrt(sum_k (E_wk - S_ik)^2), the reference's
// formula (fused:35-43), in FP32.
// Padding columns i >= v_r are written as K = KM = 0.  KM is written only when
// the caller passes a buffer for it (the solve needs it only for expo = 0).
//
// Row-scaled form (mrow given, expo != 0): the panel receives M itself and
// mrow[w] the smallest M of row w (atomicMin on the float bits, M >= 0);
// panel_rescale_kernel then turns M into K' = exp(expo (M - mrow[w])) once
// the near pairs are fixed.  See panel_rescale.cu for why.
#include "wmd_internal.cuh"

namespace wmd {

// Rows per thread (tile height BM = 16 * RPT) and resident CTAs per SM: a
// build-time tuning knob.
#ifndef WMD_CDIST_RPT
#define WMD_CDIST_RPT 8
#endif
#ifndef WMD_CDIST_MINB
#define WMD_CDIST_MINB 1
#endif

namespace {
constexpr int RPT = WMD_CDIST_RPT;
constexpr int BM = 16 * RPT;   // vocabulary rows per CTA
constexpr int BN = 32;         // source words per CTA
constexpr int BK = 16;         // d-slice per stage
constexpr int THREADS = 128;   // 16 x 8 threads, each RPT rows x 4 sources
constexpr int AS = BM + 4;     // padded smem row (floats)
constexpr int ALOADS = BM * BK / 4 / THREADS;  // float4 A slots per thread
static_assert(RPT % 4 == 0 || RPT == 6 || RPT == 2, "RPT");
static_assert(BM * BK / 4 == ALOADS * THREADS, "A tile load split");

}  // namespace

template <bool VEC4>
__global__ void __launch_bounds__(THREADS, WMD_CDIST_MINB)
cdist_fp32_kernel(const float* __restrict__ E, const float* __restrict__ nE,
                  uint64_t V, int d, const float* __restrict__ S,
                  const float* __restrict__ nS,
                  const uint32_t* __restrict__ vr_dev, float expo,
                  float* __restrict__ Kout, float* __restrict__ KMout, int ld,
                  const NearList near, float* __restrict__ mrow) {
  __shared__ __align__(16) float As[2][BK][AS];
  __shared__ __align__(16) float Bs[2][BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid & 7, ty = tid >> 3;
  const uint64_t m0 = (uint64_t)blockIdx.x * BM;
  const int n0 = blockIdx.y * BN;
  const int vr = (int)*vr_dev;

  float acc[RPT][4];
#pragma unroll
  for (int i = 0; i < RPT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;

  const bool active = n0 < vr;  // tiles of pure padding only write zeros
  if (active) {
    float4 ra[ALOADS];
    float4 rb;
    auto load_tile = [&](int k0) {
#pragma unroll
      for (int p = 0; p < ALOADS; ++p) {
        const int f = tid + p * THREADS;  // BM rows x 4 float4 slots
        const int row = f >> 2, kq = f & 3;
        const uint64_t gr = m0 + row;
        const int k = k0 + kq * 4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gr < V) {
          const float* src = E + gr * (uint64_t)d + k;
          if (VEC4) {
            if (k < d) v = __ldg(reinterpret_cast<const float4*>(src));
          } else {
            if (k + 0 < d) v.x = __ldg(src + 0);
            if (k + 1 < d) v.y = __ldg(src + 1);
            if (k + 2 < d) v.z = __ldg(src + 2);
            if (k + 3 < d) v.w = __ldg(src + 3);
          }
        }
        ra[p] = v;
      }
      {
        const int row = tid >> 2, kq = tid & 3;  // 128 slots: 32 sources x 4
        const int gi = n0 + row;
        const int k = k0 + kq * 4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gi < vr) {
          const float* src = S + (uint64_t)gi * d + k;
          if (VEC4) {
            if (k < d) v = *reinterpret_cast<const float4*>(src);
          } else {
            if (k + 0 < d) v.x = src[0];
            if (k + 1 < d) v.y = src[1];
            if (k + 2 < d) v.z = src[2];
            if (k + 3 < d) v.w = src[3];
          }
        }
        rb = v;
      }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
      for (int p = 0; p < ALOADS; ++p) {
        const int f = tid + p * THREADS;
        const int row = f >> 2, kq = f & 3;
        As[buf][kq * 4 + 0][row] = ra[p].x;
        As[buf][kq * 4 + 1][row] = ra[p].y;
        As[buf][kq * 4 + 2][row] = ra[p].z;
        As[buf][kq * 4 + 3][row] = ra[p].w;
      }
      const int row = tid >> 2, kq = tid & 3;
      Bs[buf][kq * 4 + 0][row] = rb.x;
      Bs[buf][kq * 4 + 1][row] = rb.y;
      Bs[buf][kq * 4 + 2][row] = rb.z;
      Bs[buf][kq * 4 + 3][row] = rb.w;
    };

    const int nk = (d + BK - 1) / BK;
    load_tile(0);
    store_tile(0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
      const int buf = kt & 1;
      if (kt + 1 < nk) load_tile((kt + 1) * BK);
#pragma unroll
      for (int k = 0; k < BK; ++k) {
        float av[RPT];
        if constexpr (RPT % 4 == 0) {
#pragma unroll
          for (int i = 0; i < RPT; i += 4) {
            const float4 a = *reinterpret_cast<const float4*>(&As[buf][k][ty * RPT + i]);
            av[i] = a.x;
            av[i + 1] = a.y;
            av[i + 2] = a.z;
            av[i + 3] = a.w;
          }
        } else {
#pragma unroll
          for (int i = 0; i < RPT; i += 2) {
            const float2 a = *reinterpret_cast<const float2*>(&As[buf][k][ty * RPT + i]);
            av[i] = a.x;
            av[i + 1] = a.y;
          }
        }
        const float4 b = *reinterpret_cast<const float4*>(&Bs[buf][k][tx * 4]);
        const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int i = 0; i < RPT; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
      }
      if (kt + 1 < nk) {
        store_tile(buf ^ 1);
        __syncthreads();
      }
    }
  }

  // Epilogue: M^2 from the GEMM form (near pairs listed for the exact
  // fix-up pass), K = exp(expo*M), KM = K*M.
  const int c0 = n0 + tx * 4;
  if (c0 >= ld) return;
#pragma unroll
  for (int i = 0; i < RPT; ++i) {
    const uint64_t w = m0 + ty * RPT + i;
    if (w >= V) break;
    const float ne = active ? nE[w] : 0.f;
    float kv[4], kmv[4];
    float mmin = __int_as_float(0x7f7f7f7f);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      kv[j] = 0.f;
      kmv[j] = 0.f;
      const int c = c0 + j;
      if (c < vr) {
        const float ns = nS[c];
        const float m2 = fmaxf(ne + ns - 2.f * acc[i][j], 0.f);
        if (m2 < near_threshold(ne, ns)) near_pair(near, w, c);
        const float m = sqrtf(m2);
        if (mrow) {  // row-scaled form: M now, K' after the fix-up
          kv[j] = m;
          mmin = fminf(mmin, m);
        } else {
          const float k = expf(expo * m);
          kv[j] = k;
          kmv[j] = k * m;
        }
      }
    }
    if (mrow && c0 < vr) atomicMin(reinterpret_cast<int*>(mrow + w), __float_as_int(mmin));
    *reinterpret_cast<float4*>(Kout + w * (uint64_t)ld + c0) =
        make_float4(kv[0], kv[1], kv[2], kv[3]);
    if (KMout && !mrow)
      *reinterpret_cast<float4*>(KMout + w * (uint64_t)ld + c0) =
          make_float4(kmv[0], kmv[1], kmv[2], kmv[3]);
  }
}

int launch_cdist_fp32(const float* E32, const float* nE, uint64_t V, uint64_t d,
                      const SourceSel& s, float expo, float* K, float* KM,
                      int ld, const NearList& near, cudaStream_t st, float* mrow) {
  dim3 grid((unsigned)((V + BM - 1) / BM), (unsigned)((ld + BN - 1) / BN));
  if (d % 4 == 0)
    cdist_fp32_kernel<true><<<grid, THREADS, 0, st>>>(E32, nE, V, (int)d, s.S, s.nS,
                                                      s.vr, expo, K, KM, ld, near, mrow);
  else
    cdist_fp32_kernel<false><<<grid, THREADS, 0, st>>>(E32, nE, V, (int)d, s.S, s.nS,
                                                       s.vr, expo, K, KM, ld, near, mrow);
  return 1;
}

}  // namespace wmd
