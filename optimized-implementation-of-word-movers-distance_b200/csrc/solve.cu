// Fused Sinkhorn solve, one warp per target document.
//
// Restates the reference's loop (sinkhorn_wmd_fused.cpp:246-393) column by
// column.  For target document j with words w_1..w_n and weights c_1..c_n:
//
//   u = v_r                                           (fused:188-191)
//   repeat max_iter:                                  (fused:246-335)
//     s_k = K[w_k,:] . u          v_k = c_k / s_k     (SDDMM, fused:267-276)
//     x   = diag(1/r) sum_k K[w_k,:] v_k              (SpMM,  fused:278-289)
//     u   = 1 / x                                     (fused:304-319)
//   s_k = K[w_k,:] . u,  v_k = c_k / s_k              (fused:339-366)
//   WMD_j = sum_i u_i sum_k KM[w_k,i] v_k   (FP64)    (fused:367-393)
//
// A document's scalings depend only on its own column, so the whole loop runs
// inside one warp with u and x in registers: no atomics (the reference needs
// `omp atomic`, fused:284), no global u/x traffic and no per-iteration
// launches.  The document's K rows (n x v_r, gathered from the L2-resident
// panel) are staged once in shared memory and re-read from there by every
// iteration; rows beyond the per-warp staging capacity are re-gathered from
// L2.  KM rows are read once, by the final half-step.
//
// Lane layout: LPW lanes share one word (a "group"), 32/LPW words are in
// flight per warp step.  Lane q of a group owns DPL source dimensions, as the
// float4 chunks q, q+LPW, q+2*LPW, ... of the row, so a group's lanes read
// consecutive 16-byte chunks (one coalesced segment in L2, conflict-free in
// shared memory; the two words of a 4-lane phase are separated by an XOR
// swizzle of the staged row).
#include "wmd_internal.cuh"

namespace wmd {

namespace {
constexpr int kWarps = 8;                 // warps per CTA
constexpr int kSmemBudget = 200 * 1024;   // dynamic shared memory per CTA

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
}  // namespace

template <int LPW, int DPL>
struct SolveShape {
  static constexpr int WPS = 32 / LPW;  // words per warp step
  static constexpr int RL = LPW * DPL;  // padded row length (floats)
  static constexpr int NCH = RL / 4;    // float4 chunks per padded row
  static constexpr int CPL = DPL / 4;   // chunks per lane
  static_assert(LPW >= 4 && LPW <= 32 && (LPW & (LPW - 1)) == 0, "LPW");
  static_assert(DPL % 4 == 0, "DPL");
  // Swizzle so the two words of an 8-lane shared-memory phase (LPW = 4) hit
  // disjoint banks.  Wider groups already cover a full 128-byte phase.
  static __device__ __forceinline__ int swz(int kk) {
    return LPW == 4 ? ((kk & 1) << 2) : 0;
  }
};

template <int LPW, int DPL>
__global__ void __launch_bounds__(kWarps * 32)
solve_kernel(const float* __restrict__ K, const float* __restrict__ KM, int ld,
             const uint32_t* __restrict__ vr_dev,
             const float* __restrict__ rinv,
             const int64_t* __restrict__ col_ptr,
             const uint2* __restrict__ ent,
             const int32_t* __restrict__ order, int64_t N, int max_iter,
             int stage_rows, double* __restrict__ out) {
  using Sh = SolveShape<LPW, DPL>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = lane & (LPW - 1), g = lane / LPW;
  float4* sK = reinterpret_cast<float4*>(smem_raw) +
               (size_t)warp * stage_rows * Sh::NCH;
  uint2* sE = reinterpret_cast<uint2*>(reinterpret_cast<float4*>(smem_raw) +
                                       (size_t)kWarps * stage_rows * Sh::NCH) +
              (size_t)warp * stage_rows;
  const int vr = (int)*vr_dev;
  const int ldc = ld >> 2;  // float4 chunks per global panel row

  // Per-lane constants: validity of each owned dimension and 1/r there.
  static_assert(DPL <= 32, "validity mask is 32 bits");
  float rv[DPL];
  unsigned vmask = 0;
#pragma unroll
  for (int t = 0; t < Sh::CPL; ++t)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int i = 4 * (q + t * LPW) + e;
      const bool ok = i < vr;
      rv[t * 4 + e] = ok ? rinv[i] : 0.f;
      vmask |= ok ? (1u << (t * 4 + e)) : 0u;
    }

  const int64_t total_warps = (int64_t)gridDim.x * kWarps;
  for (int64_t idx = (int64_t)blockIdx.x * kWarps + warp; idx < N;
       idx += total_warps) {
    const int64_t j = order ? (int64_t)order[idx] : idx;
    const int64_t b = col_ptr[j];
    const int n = (int)(col_ptr[j + 1] - b);
    const int ns = n < stage_rows ? n : stage_rows;

    // Stage this document's entries and K rows [0, ns).
    __syncwarp();
    for (int k = lane; k < ns; k += 32) sE[k] = ent[b + k];
    __syncwarp();
    for (int c = lane; c < ns * Sh::NCH; c += 32) {
      const int kk = c / Sh::NCH, ch = c % Sh::NCH;
      float4* dst = sK + kk * Sh::NCH + (ch ^ Sh::swz(kk));
      if (ch < ldc)
        cp_async16(dst, K + (size_t)sE[kk].x * ld + 4 * ch);
      else
        *dst = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    cp_async_wait_all();
    __syncwarp();

    // Row loader: staged rows from shared memory, the rest from L2.
    auto load_row = [&](int kk, const float* __restrict__ P, bool use_stage,
                        float (&kc)[DPL], float& cval) {
      if (kk >= n) {
#pragma unroll
        for (int t = 0; t < DPL; ++t) kc[t] = 0.f;
        cval = 0.f;
        return;
      }
      if (use_stage && kk < ns) {
        const uint2 en = sE[kk];
        cval = __uint_as_float(en.y);
#pragma unroll
        for (int t = 0; t < Sh::CPL; ++t) {
          const float4 v = sK[kk * Sh::NCH + ((q + t * LPW) ^ Sh::swz(kk))];
          kc[4 * t + 0] = v.x; kc[4 * t + 1] = v.y;
          kc[4 * t + 2] = v.z; kc[4 * t + 3] = v.w;
        }
      } else {
        const uint2 en = kk < ns ? sE[kk] : __ldg(&ent[b + kk]);
        cval = __uint_as_float(en.y);
        const float* row = P + (size_t)en.x * ld;
#pragma unroll
        for (int t = 0; t < Sh::CPL; ++t) {
          const int ch = q + t * LPW;
          float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
          if (ch < ldc) v = __ldg(reinterpret_cast<const float4*>(row) + ch);
          kc[4 * t + 0] = v.x; kc[4 * t + 1] = v.y;
          kc[4 * t + 2] = v.z; kc[4 * t + 3] = v.w;
        }
      }
    };
    auto group_sum = [&](float s) {
#pragma unroll
      for (int off = 1; off < LPW; off <<= 1)
        s += __shfl_xor_sync(0xffffffffu, s, off);
      return s;
    };
    auto cross_group_sum = [&](float (&x)[DPL]) {
#pragma unroll
      for (int off = LPW; off < 32; off <<= 1)
#pragma unroll
        for (int t = 0; t < DPL; ++t) x[t] += __shfl_xor_sync(0xffffffffu, x[t], off);
    };

    float u[DPL], x[DPL];
#pragma unroll
    for (int t = 0; t < DPL; ++t) u[t] = ((vmask >> t) & 1u) ? (float)vr : 0.f;

    for (int it = 0; it < max_iter; ++it) {
#pragma unroll
      for (int t = 0; t < DPL; ++t) x[t] = 0.f;
#pragma unroll 2
      for (int k0 = 0; k0 < n; k0 += Sh::WPS) {
        const int kk = k0 + g;
        float kc[DPL], cval;
        load_row(kk, K, true, kc, cval);
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < DPL; ++t) s = fmaf(kc[t], u[t], s);
        s = group_sum(s);
        const float v = kk < n ? cval / s : 0.f;
#pragma unroll
        for (int t = 0; t < DPL; ++t) x[t] = fmaf(kc[t], v, x[t]);
      }
      cross_group_sum(x);
#pragma unroll
      for (int t = 0; t < DPL; ++t)
        u[t] = ((vmask >> t) & 1u) ? 1.f / (rv[t] * x[t]) : 0.f;
    }

    // Final half-step with K.*M, then the FP64 reduction (fused:339-393).
#pragma unroll
    for (int t = 0; t < DPL; ++t) x[t] = 0.f;
    for (int k0 = 0; k0 < n; k0 += Sh::WPS) {
      const int kk = k0 + g;
      float kc[DPL], km[DPL], cval, cdup;
      load_row(kk, K, true, kc, cval);
      float s = 0.f;
#pragma unroll
      for (int t = 0; t < DPL; ++t) s = fmaf(kc[t], u[t], s);
      s = group_sum(s);
      const float v = kk < n ? cval / s : 0.f;
      load_row(kk, KM, false, km, cdup);
#pragma unroll
      for (int t = 0; t < DPL; ++t) x[t] = fmaf(km[t], v, x[t]);
    }
    cross_group_sum(x);
    double acc = 0.0;
#pragma unroll
    for (int t = 0; t < DPL; ++t)
      if ((vmask >> t) & 1u) acc += (double)u[t] * (double)x[t];
#pragma unroll
    for (int off = 1; off < LPW; off <<= 1)
      acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (lane == 0) out[j] = acc;
  }
}

template <int LPW, int DPL>
static int launch_solve_t(const float* K, const float* KM, int ld,
                          const SourceSel& s, const Targets& t, int max_iter,
                          double* out, cudaStream_t st) {
  using Sh = SolveShape<LPW, DPL>;
  const int per_row = Sh::RL * 4 + 8;
  int stage_rows = kSmemBudget / kWarps / per_row;
  const size_t smem = (size_t)kWarps * stage_rows * per_row;
  // Per-device one-time set-up: opt in to the large shared-memory carve-out
  // and size the persistent grid.
  constexpr int kMaxDev = 64;
  static int per_sm_cache[kMaxDev] = {0};
  static int sms_cache[kMaxDev] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) dev = 0;
  if (per_sm_cache[dev] == 0) {
    cudaFuncSetAttribute(solve_kernel<LPW, DPL>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSmemBudget);
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, solve_kernel<LPW, DPL>, kWarps * 32, smem);
    sms_cache[dev] = sms > 0 ? sms : 1;
    per_sm_cache[dev] = per_sm > 0 ? per_sm : 1;
  }
  const int sms = sms_cache[dev], per_sm = per_sm_cache[dev];
  int64_t want = (t.N + kWarps - 1) / kWarps;
  int64_t grid = (int64_t)sms * per_sm;
  if (grid > want) grid = want;
  if (grid < 1) grid = 1;
  solve_kernel<LPW, DPL><<<(unsigned)grid, kWarps * 32, smem, st>>>(
      K, KM, ld, s.vr, s.rinv, t.col_ptr, t.ent, t.order, t.N, max_iter,
      stage_rows, out);
  return 1;
}

int launch_solve(const float* K, const float* KM, int ld, uint32_t vr_cap,
                 const SourceSel& s, const Targets& t, int max_iter,
                 double* out, cudaStream_t st) {
  if (t.N <= 0) return 0;
  if (vr_cap <= 32) return launch_solve_t<4, 8>(K, KM, ld, s, t, max_iter, out, st);
  if (vr_cap <= 64) return launch_solve_t<8, 8>(K, KM, ld, s, t, max_iter, out, st);
  if (vr_cap <= 128) return launch_solve_t<16, 8>(K, KM, ld, s, t, max_iter, out, st);
  if (vr_cap <= 256) return launch_solve_t<32, 8>(K, KM, ld, s, t, max_iter, out, st);
  if (vr_cap <= 512) return launch_solve_t<32, 16>(K, KM, ld, s, t, max_iter, out, st);
  if (vr_cap <= 1024) return launch_solve_t<32, 32>(K, KM, ld, s, t, max_iter, out, st);
  return -1;
}

}  // namespace wmd
