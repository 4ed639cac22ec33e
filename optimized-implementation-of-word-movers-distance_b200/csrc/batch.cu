// Stacked batch groups: many source documents against one target set with a
// fixed number of launches per group, independent of the number of sources.
//
// The reference solves one source per call (sinkhorn_wmd_fused.cpp:112-114)
// and builds that source's K panel from every embedding row each time
// (:197-223).  A batch here is split into groups of sources of one width
// class (the lane layout of the warp solve, or the BF16 panel width of the
// CTA-per-document solve) whose panels fit a memory budget; per group:
//
//   group_gather_kernel      the selected embedding rows of every source of
//                            the group, stacked (each source padded to whole
//                            N-tiles of the cost panel), with their norms;
//   cdist_tc_kernel          one cost-panel launch over all stacked rows, each
//                            N-tile writing its own source's panel (tile table);
//   near_fixup_group_kernel  the cancellation-prone pairs of every source;
//   panel_to_bf16_group      (block-solve classes) every panel to BF16;
//   solve (stacked form)     one persistent launch over every (source,
//                            document) pair, source-major.
//
// Sources keep their own panels ([V][ld_s] FP32, [V][ld16] BF16) in one pool;
// the solves find them, with each source's weights and output rows, in a
// GroupSrc table.
#include <cuda_bf16.h>

#include "wmd_internal.cuh"

namespace wmd {
namespace {

// Stacked source rows: row g is embedding row rowword[g] (or zeros when -1).
__global__ void group_gather_kernel(const int32_t* __restrict__ rowword, int rows,
                                    const float* __restrict__ E32,
                                    const float* __restrict__ nE, int d,
                                    float* __restrict__ S, float* __restrict__ nS,
                                    const uint16_t* __restrict__ E16,
                                    uint16_t* __restrict__ S16, int dp) {
  const int lane = threadIdx.x & 31;
  const int64_t g0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t gs = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t g = g0; g < rows; g += gs) {
    const int w = rowword[g];
    for (int k = lane; k < d; k += 32)
      S[g * d + k] = w >= 0 ? E32[(size_t)w * d + k] : 0.f;
    if (S16)
      for (int k = lane; k < dp; k += 32)
        S16[g * dp + k] = w >= 0 ? E16[(size_t)w * dp + k] : (uint16_t)0;
    if (lane == 0) nS[g] = w >= 0 ? nE[w] : 0.f;
  }
}

// Exact recompute of the listed near pairs {word, stacked row} of a group
// (the same formula as near_fixup_kernel); when the list overflowed, every
// source's panel is scanned for near entries instead.
__global__ void near_fixup_group_kernel(NearList nl, float expo,
                                        const int32_t* __restrict__ rowsrc,
                                        const GroupSrc* __restrict__ grp, int nsrc,
                                        uint64_t V, const float* __restrict__ nE,
                                        const float* __restrict__ nS) {
  const int lane = threadIdx.x & 31;
  const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const unsigned total = *nl.count;
  const unsigned listed = total < nl.cap ? total : nl.cap;
  auto fix = [&](uint64_t w, int row, const GroupSrc& gs) {
    const float m2 = warp_sqdist(nl.E32 + w * (uint64_t)nl.d,
                                 nl.S32 + (uint64_t)row * nl.d, nl.d, lane);
    if (lane == 0) gs.K[w * (uint64_t)gs.ld + (row - gs.row0)] = expf(expo * sqrtf(m2));
  };
  for (uint64_t p = gw; p < listed; p += nw) {
    const uint2 pr = nl.pairs[p];
    fix(pr.x, (int)pr.y, grp[rowsrc[pr.y]]);
  }
  if (total <= nl.cap) return;
  for (int s = 0; s < nsrc; ++s) {
    const GroupSrc& gs = grp[s];
    for (uint64_t w = gw; w < V; w += nw) {
      const float ne = nE[w];
      for (int i0 = 0; i0 < gs.vr; i0 += 32) {
        const int i = i0 + lane;
        bool near = false;
        if (i < gs.vr) {
          const float m = logf(gs.K[w * (uint64_t)gs.ld + i]) / expo;
          near = m * m < near_threshold(ne, nS[gs.row0 + i]);
        }
        unsigned msk = __ballot_sync(0xffffffffu, near);
        while (msk) {
          const int l = __ffs(msk) - 1;
          msk &= msk - 1;
          fix(w, gs.row0 + i0 + l, gs);
        }
      }
    }
  }
}

// Every source's FP32 panel to its BF16 panel [V][ld16] (zero past v_r).
__global__ void panel_to_bf16_group_kernel(const GroupSrc* __restrict__ grp, int nsrc,
                                           uint64_t V, int ldq) {
  const uint64_t per = V * (uint64_t)ldq;
  const uint64_t total = per * (uint64_t)nsrc;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const int s = (int)(e / per);
    const uint64_t i = e - (uint64_t)s * per;
    const GroupSrc& gs = grp[s];
    const uint64_t w = i / ldq;
    const int D0 = 4 * (int)(i % ldq);
    unsigned h[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int D = D0 + k;
      const float v = D < gs.vr ? gs.K[w * gs.ld + D] : 0.f;
      h[k] = (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
    static_cast<uint2*>(gs.K16)[i] = make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
  }
}

}  // namespace

int launch_group_gather(const int32_t* rowword, int rows, const float* E32,
                        const float* nE, uint64_t d, float* S, float* nS,
                        const void* E16, void* S16, int dp, int num_sms, cudaStream_t st) {
  int64_t g = ((int64_t)rows * 32 + 255) / 256;
  const int64_t cap = (int64_t)(num_sms > 0 ? num_sms : 148) * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  group_gather_kernel<<<(unsigned)g, 256, 0, st>>>(
      rowword, rows, E32, nE, (int)d, S, nS, static_cast<const uint16_t*>(E16),
      static_cast<uint16_t*>(S16), dp);
  return 1;
}

int launch_near_fixup_group(const NearList& near, float expo, const int32_t* rowsrc,
                            const GroupSrc* grp, int nsrc, uint64_t V, const float* nE,
                            const float* nS, int num_sms, cudaStream_t st) {
  near_fixup_group_kernel<<<num_sms > 0 ? num_sms : 148, 256, 0, st>>>(
      near, expo, rowsrc, grp, nsrc, V, nE, nS);
  return 1;
}

int launch_panel_to_bf16_group(const GroupSrc* grp, int nsrc, uint64_t V, int ld16,
                               int num_sms, cudaStream_t st) {
  panel_to_bf16_group_kernel<<<(num_sms > 0 ? num_sms : 148) * 8, 256, 0, st>>>(
      grp, nsrc, V, ld16 / 4);
  return 1;
}

}  // namespace wmd
