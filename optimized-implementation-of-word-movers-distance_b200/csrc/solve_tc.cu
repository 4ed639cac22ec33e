// Sinkhorn solve on the tensor cores: one CTA per target document, the
// document's BF16 K rows in shared memory, both matrix-vector products of a
// pass as warp-level BF16 MMAs (mma.sync m16n8k16, FP32 accumulation).
//
// Same recurrence as solve.cu / solve_block.cu (sinkhorn_wmd_fused.cpp:
// 246-393 restated per column).  Per pass, with K the document's n x v_r
// block:
//   s = K u        M = rows, N = 8, K = source dimensions
//   v = c ./ s
//   x = K^T v      M = source dimensions, N = 8, K = rows
//   u = 1 / (x / r)
// A matrix-vector product uses one column of an MMA; here u (and v) enter as
// three columns, its BF16 split u = hi + mid + lo (hi = bf16(u), mid =
// bf16(u - hi), lo = bf16(u - hi - mid): 24 significant bits, the FP32
// operand to within 2^-24 relative), and the three column sums are added in
// FP32.  Each K x hi product is exact in FP32, so the products carry FP32
// accuracy over the BF16 K panel; the remaining 5 of the 8 columns are zero.
//
// K tiles come from shared memory with ldmatrix (row pitch padded by 16
// bytes: the 8 rows of an 8x8 matrix land in 8 distinct bank groups); the
// transposed operand of x = K^T v is ldmatrix.trans of the same rows.
// s = K u is split into (row tile, quarter of the dimension tiles) units so
// that all warps share a short document; the four partial sums meet in
// shared memory.  x = K^T v is split by dimension tiles: each warp owns whole
// dimensions, sums over all rows itself and updates u for them.
//
// Documents whose rows exceed the shared-memory capacity are solved by the
// CUDA-core block kernel (the caller splits the length-ordered documents).
// The final half-step reads K.*M = K ln K / expo from the staged rows on the
// CUDA cores in FP32 with an FP64 sum, as solve_block.cu does.
#include <cuda_bf16.h>

#include "wmd_internal.cuh"

namespace wmd {

namespace {
constexpr int kTW = 8;  // warps per CTA
constexpr int kTT = kTW * 32;

__device__ __forceinline__ void tcp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void tcp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ void ldsm_x4(uint32_t (&a)[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(s));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&a)[4], const void* p) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
               : "r"(s));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4],
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// BF16 split of an FP32 value: hi + mid + lo.
__device__ __forceinline__ void split3(float v, __nv_bfloat16& h, __nv_bfloat16& m,
                                       __nv_bfloat16& l) {
  h = __float2bfloat16_rn(v);
  const float r1 = v - __bfloat162float(h);
  m = __float2bfloat16_rn(r1);
  const float r2 = r1 - __bfloat162float(m);
  l = __float2bfloat16_rn(r2);
}
__device__ __forceinline__ float4 tq_to_f32(uint2 q) {
  return make_float4(__uint_as_float(q.x << 16), __uint_as_float(q.x & 0xffff0000u),
                     __uint_as_float(q.y << 16), __uint_as_float(q.y & 0xffff0000u));
}
}  // namespace

template <int NQ>
struct TcShape {
  static constexpr int RL = 128 * NQ;     // padded row length (elements)
  static constexpr int RP = RL * 2 + 16;  // row pitch in shared memory (bytes)
  static constexpr int KT = RL / 16;      // dimension tiles
  static constexpr int DPW = KT / kTW;    // dimension tiles per warp (x = K^T v)
  static_assert(KT % kTW == 0, "dimension tiles per warp");
  // rows [cap][RP], then per row: c (f32), 4 partial sums (f32), v split
  // (3 x bf16, padded to 8 bytes); per dimension: u split (3 x bf16 + pad),
  // two u buffers (f32); per warp: residual partial (f64).
  static __host__ __device__ size_t bytes(int cap) {
    return (size_t)cap * RP + (size_t)cap * (4 + 16 + 8) + (size_t)RL * (8 + 8) +
           (size_t)kTW * 8;
  }
};

template <int NQ>
__global__ void __launch_bounds__(kTT, 1)
solve_tc_kernel(const uint2* __restrict__ K16, int ldq, float expo,
                const uint32_t* __restrict__ vr_dev, const float* __restrict__ rinv,
                const int64_t* __restrict__ col_ptr, const uint2* __restrict__ ent,
                const int32_t* __restrict__ order, int64_t N, int max_iter, float tol,
                int* __restrict__ iters_out, const float* __restrict__ u0, int64_t ldu,
                int cap, float omega, float* __restrict__ vstate,
                const float* __restrict__ mrow, double* __restrict__ out) {
  using Sh = TcShape<NQ>;
  constexpr int RL = Sh::RL, RP = Sh::RP, KT = Sh::KT, DPW = Sh::DPW;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* sRows = smem_raw;
  float* sC = reinterpret_cast<float*>(smem_raw + (size_t)cap * RP);
  float* sS = sC + cap;                                         // [4][cap]
  __nv_bfloat16* sV = reinterpret_cast<__nv_bfloat16*>(sS + 4 * cap);  // [4][cap]
  __nv_bfloat16* sU = sV + 4 * cap;                             // [4][RL]
  float* ubufA = reinterpret_cast<float*>(sU + 4 * RL);
  float* ubufB = ubufA + RL;
  double* red = reinterpret_cast<double*>(ubufB + RL);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int col = lane >> 2, quad = lane & 3;  // MMA fragment coordinates
  const int vr = (int)*vr_dev;

  for (int64_t idx = blockIdx.x; idx < N; idx += gridDim.x) {
    const int64_t j = order ? (int64_t)order[idx] : idx;
    const int64_t b = col_ptr[j];
    const int n = (int)(col_ptr[j + 1] - b);
    if (n > cap) {  // the caller routes longer documents elsewhere
      if (tid == 0) out[j] = __longlong_as_double(0x7ff8000000000000ll);
      continue;
    }
    // Over-relaxation of both half-steps (vstate: each word's previous v).
    const bool relax = vstate != nullptr;
    RelaxGuard g;
    g.init(omega);
    float resv = 0.f;  // this thread's c-side residual of the current pass
    const int RT = (n + 15) >> 4, npad = RT << 4;
    const bool warm = u0 != nullptr && max_iter > 0;

    __syncthreads();  // the previous document is done with shared memory
    for (int k = tid; k < npad; k += kTT) sC[k] = k < n ? __uint_as_float(__ldg(&ent[b + k]).y) : 0.f;
    for (int D = tid; D < RL; D += kTT) {
      ubufA[D] = D < vr ? (float)vr : 0.f;  // cold start (fused:188-191)
      if (warm) ubufB[D] = D < vr ? __ldg(&u0[j * ldu + D]) : 0.f;
    }
    constexpr int CPR = RL / 8;  // 16-byte chunks per row
    for (int c = tid; c < npad * CPR; c += kTT) {
      const int k = c / CPR, ch = c % CPR;
      unsigned char* dst = sRows + (size_t)k * RP + ch * 16;
      if (k < n) {
        const uint32_t w = __ldg(&ent[b + k]).x;
        tcp_async16(dst, K16 + (size_t)w * ldq + 2 * ch);
      } else {
        *reinterpret_cast<uint4*>(dst) = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    tcp_async_wait_all();
    __syncthreads();

    // s = K u for the rows, u given as its split in sU; partial sums of the
    // four dimension-tile quarters in sS[q][row].
    auto product_s = [&]() {
      // A warp always takes the same quarter q = warp % 4 of the dimension
      // tiles (units advance by kTW, a multiple of 4): its B fragments (the
      // u split at those tiles) are loaded once per pass.
      constexpr int KQ = KT / 4;
      const int q = warp & 3;
      uint32_t bq[KQ][2];
#pragma unroll
      for (int i = 0; i < KQ; ++i) {
        bq[i][0] = bq[i][1] = 0u;
        if (col < 3) {
          const __nv_bfloat16* us = sU + col * RL + 16 * (q + 4 * i) + 2 * quad;
          bq[i][0] = *reinterpret_cast<const uint32_t*>(us);
          bq[i][1] = *reinterpret_cast<const uint32_t*>(us + 8);
        }
      }
      for (int unit = warp; unit < RT * 4; unit += kTW) {
        const int rt = unit >> 2;
        // two accumulator chains (even / odd k-tiles), every A tile of the
        // unit loaded before its MMA is needed
        float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
        const unsigned char* arow =
            sRows + (size_t)(16 * rt + (lane & 7) + ((lane >> 3) & 1) * 8) * RP +
            (lane >> 4) * 16;
        uint32_t a[KQ][4];
#pragma unroll
        for (int i = 0; i < KQ; ++i) ldsm_x4(a[i], arow + 32 * (q + 4 * i));
#pragma unroll
        for (int i = 0; i < KQ; ++i) {
          if (i & 1)
            mma_bf16(c1, a[i], bq[i][0], bq[i][1]);
          else
            mma_bf16(c0, a[i], bq[i][0], bq[i][1]);
        }
        // columns 0,1 (hi, mid) in quad 0, column 2 (lo) in quad 1
        const float lo_r = (c0[0] + c1[0]) + (c0[1] + c1[1]);
        const float hi_r = (c0[2] + c1[2]) + (c0[3] + c1[3]);
        const float lo_o = __shfl_down_sync(0xffffffffu, lo_r, 1);
        const float hi_o = __shfl_down_sync(0xffffffffu, hi_r, 1);
        if (quad == 0) {
          sS[q * cap + 16 * rt + col] = lo_r + lo_o;
          sS[q * cap + 16 * rt + col + 8] = hi_r + hi_o;
        }
      }
    };
    auto split_u = [&](const float* src) {
      for (int D = tid; D < RL; D += kTT) {
        __nv_bfloat16 h, m, l;
        split3(src[D], h, m, l);
        sU[D] = h;
        sU[RL + D] = m;
        sU[2 * RL + D] = l;
      }
    };
    auto weight = [](float c, float s) { return c != 0.f ? __fdividef(c, s) : 0.f; };

    // One pass: u from `src` -> new u into `dst` (may alias); returns the
    // marginal residual of `src` (CTA-uniform) when want_res.
    auto pass = [&](const float* src, float* dst, bool want_res) -> float {
      // Previous v of this thread's first rows, loaded before the products
      // (off the s -> v critical path).
      float vp[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = tid + i * kTT;
        vp[i] = (relax && !g.vfirst && k < n) ? vstate[b + k] : 0.f;
      }
      split_u(src);
      __syncthreads();
      product_s();
      __syncthreads();
      resv = 0.f;
      auto row_v = [&](int k, float vold) {
        const float s = sS[k] + sS[cap + k] + sS[2 * cap + k] + sS[3 * cap + k];
        __nv_bfloat16 h, m, l;
        // padding rows (k >= n) have c = 0: v = 0 and no state touched
        split3(relax ? relaxed_v_pre(sC[k], s, vold, vstate + b + k, g.vfirst, g.omega, resv)
                     : weight(sC[k], s),
               h, m, l);
        sV[k] = h;
        sV[cap + k] = m;
        sV[2 * cap + k] = l;
      };
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int k = tid + i * kTT;
        if (k < npad) row_v(k, vp[i]);
      }
      for (int k = tid + 4 * kTT; k < npad; k += kTT)
        row_v(k, (relax && !g.vfirst && k < n) ? vstate[b + k] : 0.f);
      __syncthreads();
      // x = K^T v: this warp's dimension tiles, all row tiles.
      float c[DPW][4];
#pragma unroll
      for (int t = 0; t < DPW; ++t) c[t][0] = c[t][1] = c[t][2] = c[t][3] = 0.f;
      const int brow = (lane & 7) + (lane >> 4) * 8;
      const int bcol = ((lane >> 3) & 1) * 8;
#pragma unroll 2
      for (int rt = 0; rt < RT; ++rt) {
        uint32_t b0 = 0u, b1 = 0u;
        if (col < 3) {
          const __nv_bfloat16* vs = sV + col * cap + 16 * rt + 2 * quad;
          b0 = *reinterpret_cast<const uint32_t*>(vs);
          b1 = *reinterpret_cast<const uint32_t*>(vs + 8);
        }
        const unsigned char* rowp = sRows + (size_t)(16 * rt + brow) * RP;
        uint32_t a[DPW][4];
#pragma unroll
        for (int t = 0; t < DPW; ++t) ldsm_x4_t(a[t], rowp + (16 * (warp + kTW * t) + bcol) * 2);
#pragma unroll
        for (int t = 0; t < DPW; ++t) mma_bf16(c[t], a[t], b0, b1);
      }
      float res = resv;
#pragma unroll
      for (int t = 0; t < DPW; ++t) {
        const int dt = warp + kTW * t;
        const float lo_x = c[t][0] + c[t][1], hi_x = c[t][2] + c[t][3];
        const float lo_o = __shfl_down_sync(0xffffffffu, lo_x, 1);
        const float hi_o = __shfl_down_sync(0xffffffffu, hi_x, 1);
        if (quad == 0) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int D = 16 * dt + col + 8 * h;
            const float x = h ? hi_x + hi_o : lo_x + lo_o;
            if (D < vr) {
              const float rvD = __ldg(&rinv[D]);
              const float uo = src[D];
              res += fabsf(uo * x - __frcp_rn(rvD));
              dst[D] = relaxed_update(uo, __frcp_rn(rvD * x), g.omega);
            } else {
              dst[D] = 0.f;
            }
          }
        }
      }
      if (want_res) {
#pragma unroll
        for (int off = 16; off; off >>= 1) res += __shfl_xor_sync(0xffffffffu, res, off);
        if (lane == 0) red[warp] = (double)res;
      }
      __syncthreads();
      float total = 0.f;
      if (want_res) {
#pragma unroll
        for (int w = 0; w < kTW; ++w) total += (float)red[w];
      }
      return total;
    };

    float* cur = ubufA;
    int it = 0;
    float res = 0.f;
    const bool want_res = tol > 0.f || relax;
    if (warm) {
      const float rc = pass(ubufA, ubufA, true);
      const float rwm = pass(ubufB, ubufB, true);
      // Keep u0 unless its first-update residual is worse than the cold
      // start's or not finite, or its update is not finite (a prediction far
      // off the cold start's scale can underflow v = c / (K^T u0) to 0).
      bool fin = true;
      for (int D = tid; D < vr; D += kTT) fin &= (bool)isfinite(ubufB[D]);
      fin = __syncthreads_and(fin) != 0;
      const bool use_warm = fin && isfinite(rwm) && !(rc < rwm);
      cur = use_warm ? ubufB : ubufA;
      res = use_warm ? rwm : rc;
      it = 1;
      g.vfirst = true;  // the stored v are the last candidate's
    }
    while (it < max_iter && !(it > 0 && tol > 0.f && res <= tol)) {
      res = pass(cur, cur, want_res);
      ++it;
      bool reset_u = false;
      if (relax && g.step(res, it, &reset_u) && reset_u) {
        for (int D = tid; D < RL; D += kTT) cur[D] = D < vr ? (float)vr : 0.f;
        __syncthreads();
      }
    }
    if (iters_out && tid == 0) iters_out[j] = it;

    // Final half-step (fused:339-393): s = K u on the tensor cores, then
    // WMD = sum_k v_k (KM_k . u), KM_k = K_k ln(K_k) / expo, FP64 sum.
    split_u(cur);
    __syncthreads();
    product_s();
    __syncthreads();
    for (int k = tid; k < npad; k += kTT) {
      const float s = sS[k] + sS[cap + k] + sS[2 * cap + k] + sS[3 * cap + k];
      sS[k] = weight(sC[k], s);  // v
    }
    __syncthreads();
    float4 u[NQ];
#pragma unroll
    for (int t = 0; t < NQ; ++t) u[t] = reinterpret_cast<const float4*>(cur)[lane + 32 * t];
    const float km_scale = 0.69314718f / expo;  // ln 2 / expo
    double acc = 0.0;
    for (int k = warp; k < n; k += kTW) {
      const uint2* rp = reinterpret_cast<const uint2*>(sRows + (size_t)k * RP);
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < NQ; ++t) {
        const float4 kk = tq_to_f32(rp[lane + 32 * t]);
        const float l0 = kk.x > 0.f ? __log2f(kk.x) : 0.f;
        const float l1 = kk.y > 0.f ? __log2f(kk.y) : 0.f;
        const float l2 = kk.z > 0.f ? __log2f(kk.z) : 0.f;
        const float l3 = kk.w > 0.f ? __log2f(kk.w) : 0.f;
        a = __ffma2_rn(make_float2(u[t].x * kk.x, u[t].y * kk.y), make_float2(l0, l1), a);
        a = __ffma2_rn(make_float2(u[t].z * kk.z, u[t].w * kk.w), make_float2(l2, l3), a);
      }
      float tk = a.x + a.y;
#pragma unroll
      for (int off = 16; off; off >>= 1) tk += __shfl_xor_sync(0xffffffffu, tk, off);
      if (lane == 0) {
        acc += (double)sS[k] * (double)(tk * km_scale);
        if (mrow)  // row-scaled panel: + c_w m_w (panel_rescale.cu)
          acc += (double)sC[k] * (double)__ldg(&mrow[__ldg(&ent[b + k]).x]);
      }
    }
    // A non-finite u_i (x_i = 0: an empty document) makes the reference's
    // sum over dimensions NaN (fused:382-393).
    bool bad = false;
    for (int D = tid; D < vr; D += kTT)
      bad |= !isfinite(cur[D]) || (mrow && cur[D] > kScaledUMax);  // see solve.cu
    __syncthreads();  // every warp has read the last u before red is reused
    if (lane == 0) red[warp] = acc;
    bad = __syncthreads_or(bad);
    if (tid == 0) {
      double tot = 0.0;
      for (int w = 0; w < kTW; ++w) tot += red[w];
      out[j] = bad ? __longlong_as_double(0x7ff8000000000000ll) : tot;
    }
  }
}

// Rows of one document the tensor-core solve holds (a multiple of 16) when
// `cps` CTAs share an SM's shared memory; 0 if the width is not supported.
// More CTAs per SM keep more documents in flight (a pass is a latency
// chain of MMAs, barriers and reductions) but send more of the longest
// documents to the CUDA-core kernel.
template <int NQ>
static int tc_capacity_t(int cps) {
  using Sh = TcShape<NQ>;
  const size_t budget = 227 * 1024 / (cps > 0 ? cps : 1) - 1024;
  int cap = (int)(budget / (Sh::RP + 28)) & ~15;
  while (cap > 0 && Sh::bytes(cap) > budget) cap -= 16;
  return cap;
}

int tc_solve_capacity(int ld16, int cps) {
  switch (ld16 / 128) {
    case 1: return tc_capacity_t<1>(cps);
    case 2: return tc_capacity_t<2>(cps);
    case 3: return tc_capacity_t<3>(cps);
    case 4: return tc_capacity_t<4>(cps);
    default: return 0;
  }
}

template <int NQ>
static int launch_tc_t(const void* K16, int ld16, float expo, const SourceSel& s,
                       const Targets& t, const SolveCtl& ctl, const float* u0,
                       int64_t ldu, double* out, cudaStream_t st, int cps) {
  using Sh = TcShape<NQ>;
  constexpr int kMaxDev = 64;
  static int sms_cache[kMaxDev] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) dev = 0;
  const int cap = tc_capacity_t<NQ>(cps);
  if (cap < 16) return -1;
  if (sms_cache[dev] == 0) {
    // the largest footprint (one CTA per SM) once; smaller ones fit under it
    cudaFuncSetAttribute(solve_tc_kernel<NQ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Sh::bytes(tc_capacity_t<NQ>(1)));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms_cache[dev] = sms > 0 ? sms : 1;
  }
  int64_t grid = (int64_t)sms_cache[dev] * cps;
  if (grid > t.N) grid = t.N;
  if (grid < 1) grid = 1;
  solve_tc_kernel<NQ><<<(unsigned)grid, kTT, Sh::bytes(cap), st>>>(
      static_cast<const uint2*>(K16), ld16 / 4, expo, s.vr, s.rinv, t.col_ptr, t.ent,
      t.order, t.N, ctl.max_iter, ctl.tol, ctl.iters, u0, ldu, cap, ctl.omega,
      ctl.omega != 1.f ? ctl.vstate : nullptr, ctl.mrow, out);
  return 1;
}

// Documents order[0 .. n_long) (the longest, beyond the tensor-core
// capacity) are solved by the CUDA-core block kernel, the rest on the tensor
// cores.
int launch_solve_tc(const void* K16, int ld16, float expo, uint32_t vr_cap,
                    const SourceSel& s, const Targets& t, const SolveCtl& ctl,
                    const float* u0, int64_t ldu, double* out, cudaStream_t st,
                    int cps, int64_t n_long) {
  if (t.N <= 0) return 0;
  if (expo == 0.f || ld16 != block_panel_width(vr_cap) || !t.order) return -1;
  if (n_long < 0 || n_long > t.N) return -1;
  if (ctl.omega != 1.f && !ctl.vstate) return -1;
  int launches = 0;
  if (n_long > 0) {
    Targets tl = t;
    tl.N = n_long;
    const int l = launch_solve_block(K16, ld16, expo, vr_cap, s, tl, ctl, u0, ldu, out, st, -1);
    if (l < 0) return -1;
    launches += l;
  }
  if (n_long < t.N) {
    Targets ts = t;
    ts.order = t.order + n_long;
    ts.N = t.N - n_long;
    int l = -1;
    switch (ld16 / 128) {
      case 1: l = launch_tc_t<1>(K16, ld16, expo, s, ts, ctl, u0, ldu, out, st, cps); break;
      case 2: l = launch_tc_t<2>(K16, ld16, expo, s, ts, ctl, u0, ldu, out, st, cps); break;
      case 3: l = launch_tc_t<3>(K16, ld16, expo, s, ts, ctl, u0, ldu, out, st, cps); break;
      case 4: l = launch_tc_t<4>(K16, ld16, expo, s, ts, ctl, u0, ldu, out, st, cps); break;
      default: l = -1;
    }
    if (l < 0) return -1;
    launches += l;
  }
  return launches;
}

}  // namespace wmd
