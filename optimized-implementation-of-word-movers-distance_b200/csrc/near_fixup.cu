// Exact recompute of the cancellation-prone cost-panel entries.
//
// Both cost-panel kernels compute M^2 = |E_w|^2 + |S_i|^2 - 2 E_w.S_i, which
// loses all precision for close pairs (a word against itself: M ~ 1e-3
// instead of 0, a 1% error in K at lambda = 10).  Their epilogues append every
// pair below the near threshold to a list; this kernel recomputes those
// entries as sqrt(sum_k (E_wk - S_ik)^2) in FP32 — the reference's formula,
// sinkhorn_wmd_fused.cpp:35-43 — one warp per pair with the lanes splitting the
// d coordinates, and rewrites K (and K.*M when stored).
//
// In the row-scaled form (scaled = true) the panel still holds M at this
// point: the exact M is written instead of K, and panel_rescale_kernel turns
// every entry into K' afterwards.
//
// Near pairs are few (a source word against itself, true near-duplicates), so
// the list is normally short.  If more pairs turned up than the list holds,
// the kernel falls back to scanning the whole panel for near entries (M is
// recovered from the stored K as ln(K)/expo, or read from K.*M when expo = 0).
#include "wmd_internal.cuh"

namespace wmd {

__global__ void near_fixup_kernel(NearList nl, float expo, float* __restrict__ K,
                                  float* __restrict__ KM, int ld, uint64_t V,
                                  const float* __restrict__ nE,
                                  const float* __restrict__ nS,
                                  const uint32_t* __restrict__ vr_dev, bool scaled) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  grid_dep_launch();
  grid_dep_wait();  // the cost panel's list and panel
  const unsigned total = *nl.count;
  const unsigned listed = total < nl.cap ? total : nl.cap;
  auto fix = [&](uint64_t w, int i) {
    const float m2 = warp_sqdist(nl.E32 + w * (uint64_t)nl.d,
                                 nl.S32 + (uint64_t)i * nl.d, nl.d, lane);
    if (lane == 0) {
      const float m = sqrtf(m2);
      if (scaled) {
        K[w * (uint64_t)ld + i] = m;
      } else {
        const float k = expf(expo * m);
        K[w * (uint64_t)ld + i] = k;
        if (KM) KM[w * (uint64_t)ld + i] = k * m;
      }
    }
  };
  for (uint64_t p = gw; p < listed; p += nw) {
    const uint2 pr = nl.pairs[p];
    fix(pr.x, (int)pr.y);
  }
  if (total <= nl.cap) return;
  // Overflow: scan every entry of the panel (one warp per vocabulary row).
  const int vr = (int)*vr_dev;
  for (uint64_t w = gw; w < V; w += nw) {
    const float ne = nE[w];
    for (int i0 = 0; i0 < vr; i0 += 32) {
      const int i = i0 + lane;
      bool near = false;
      if (i < vr) {
        const float kv = K[w * (uint64_t)ld + i];
        const float m = scaled ? kv : expo != 0.f ? logf(kv) / expo : KM[w * (uint64_t)ld + i];
        near = m * m < near_threshold(ne, nS[i]);
      }
      unsigned msk = __ballot_sync(0xffffffffu, near);
      while (msk) {
        const int l = __ffs(msk) - 1;
        msk &= msk - 1;
        fix(w, i0 + l);
      }
    }
  }
}

int launch_near_fixup(const NearList& near, float expo, float* K, float* KM,
                      int ld, uint64_t V, const float* nE, const float* nS,
                      const uint32_t* vr, int num_sms, cudaStream_t st, bool scaled) {
  const int threads = 256;
  launch_pdl(near_fixup_kernel, dim3(num_sms > 0 ? num_sms : 148), dim3(threads), 0, st,
             near, expo, K, KM, ld, V, nE, nS, vr, scaled);
  return 1;
}

}  // namespace wmd
