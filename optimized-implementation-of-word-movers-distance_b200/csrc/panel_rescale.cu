// Row-scaled K panel: regularisers and distances whose product lambda * M
// would underflow FP32.
//
// The reference keeps K = exp(-lambda M) in FP64 (sinkhorn_wmd_fused.cpp:217),
// finite down to lambda M ~ 708.  In FP32, exp(-lambda M) underflows to 0 past
// lambda M ~ 87 (~103 with subnormals); a document whose every word is that
// far from every source word would then see s = K^T u = 0 and v = c / 0.
//
// Each vocabulary row w is scaled by its own factor:
//     K'[w, i] = K[w, i] exp(lambda m_w) = exp(expo (M[w, i] - m_w)),
//     m_w = min_i M[w, i]          (expo = -lambda)
// so the row's largest entry is 1.  The scale cancels exactly in the
// iteration: v_w = c_w / (K'^T u)_w is v_w exp(-lambda m_w), and every use of
// K' multiplies such a v (x = K' v, s = K' u then v = c / s), so u, x and the
// scores are unchanged in exact arithmetic.  The final sum needs K.*M:
//     v'_w (K'.*M)_w . u = v'_w m_w (K' u)_w + v'_w (K' ln K' / expo)_w . u
//                        = c_w m_w          + (what the solve already sums)
// so the solves add c_w m_w per document word (FP64) when given m.
//
// Used only when the host sees that lambda * M can exceed ~80 for this
// vocabulary (lambda * 2 max_w |E_w| > 80); otherwise the cost panel writes K
// directly and nothing here runs.  Pipeline in the row-scaled form: cost panel
// writes M and atomically the row minima -> near-pair fix-up writes exact M ->
// panel_rescale_kernel writes K'.
#include "wmd_internal.cuh"

namespace wmd {
namespace {

__global__ void panel_rescale_kernel(float* __restrict__ K, int ld, uint64_t V,
                                     const uint32_t* __restrict__ vr_dev,
                                     const float* __restrict__ mrow, float expo) {
  const int vr = (int)*vr_dev;
  const int ld4 = ld >> 2;  // ld is a multiple of 4
  const uint64_t total = V * (uint64_t)ld4;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = e / ld4;
    const int c = (int)(e - w * ld4) * 4;
    float4* p = reinterpret_cast<float4*>(K + w * (uint64_t)ld) + (c >> 2);
    float4 m = *p;
    const float mw = __ldg(&mrow[w]);
    m.x = c + 0 < vr ? expf(expo * (m.x - mw)) : 0.f;
    m.y = c + 1 < vr ? expf(expo * (m.y - mw)) : 0.f;
    m.z = c + 2 < vr ? expf(expo * (m.z - mw)) : 0.f;
    m.w = c + 3 < vr ? expf(expo * (m.w - mw)) : 0.f;
    *p = m;
  }
}

// Largest squared row norm (float bits; norms are >= 0, so the integer
// maximum is the float maximum).
__global__ void max_norm_kernel(const float* __restrict__ nE, uint64_t V,
                                unsigned* __restrict__ out) {
  float mx = 0.f;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < V;
       w += (uint64_t)gridDim.x * blockDim.x)
    mx = fmaxf(mx, nE[w]);
#pragma unroll
  for (int off = 16; off; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(mx));
}

}  // namespace

int launch_panel_rescale(float* K, int ld, uint64_t V, const uint32_t* vr,
                         const float* mrow, float expo, int num_sms, cudaStream_t st) {
  const uint64_t total = V * (uint64_t)(ld >> 2);
  uint64_t blocks = (total + 255) / 256;
  const uint64_t cap = (uint64_t)(num_sms > 0 ? num_sms : 148) * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  panel_rescale_kernel<<<(unsigned)blocks, 256, 0, st>>>(K, ld, V, vr, mrow, expo);
  return 1;
}

int launch_max_norm(const float* nE, uint64_t V, unsigned* out, cudaStream_t st) {
  cudaMemsetAsync(out, 0, sizeof(unsigned), st);
  uint64_t blocks = (V + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  if (blocks < 1) blocks = 1;
  max_norm_kernel<<<(unsigned)blocks, 256, 0, st>>>(nE, V, out);
  return 1;
}

}  // namespace wmd
