// Sinkhorn solve for wide sources (64 < v_r <= 512): one CTA per target
// document, the document's K rows resident in shared memory as BF16.
//
// Same recurrence as solve.cu (sinkhorn_wmd_fused.cpp:246-393 restated per
// column; see there), different resource plan.  With a few hundred source
// words a document's K block (n words x v_r) no longer fits one warp's share
// of registers and shared memory, and the warp-per-document kernel re-gathers
// most rows from L2 on every pass.  Here the whole CTA works on one document:
// its rows are gathered once into shared memory (BF16, half the bytes of the
// FP32 panel) and every pass reads them from there; rows beyond the
// shared-memory capacity are read from the L2-resident BF16 panel.
//
// Per pass the warps split the rows in pairs.  Each lane owns 4*NQ source
// dimensions (quads lane + 32t), so a row is one 8-byte load per quad, the
// dot product K_w . u is a lane-local FMA chain plus a warp reduction, and
// the two rows of a pair share that reduction (one exchange across the warp
// halves, then a 16-lane butterfly).  The per-warp x slices are summed
// through shared memory in a fixed order (bitwise reproducible), after which
// each thread updates u = 1 / (x / r) for its dimensions and the marginal
// residual sum_i |u_i (K v)_i - r_i| is reduced across the CTA.
//
// Arithmetic: K in BF16 (converted to FP32 in registers), u, v, x and all
// sums in FP32, the final per-document reduction in FP64.
//
// Warm start: when an initial scaling u0 is given, the first update is
// evaluated from both the cold start (u = v_r) and u0, and the one with the
// smaller marginal residual is kept; the cold start is the fallback.
#include <cuda_bf16.h>

#include "wmd_internal.cuh"

namespace wmd {

// Launch shape per panel width (warps per CTA, CTAs per SM), a build-time
// tuning table.  Measured on B200 (N = 1e5 documents, 15 iterations): four
// documents in flight per SM beat one or two documents with more shared
// memory each at every width, even when most rows of the widest panels then
// come from L2 -- each pass is bound by its barrier and reduction latency,
// which other documents' work hides.
#ifndef WMD_BLK_W1  // NQ = 1 (v_r <= 128)
#define WMD_BLK_W1 4
#define WMD_BLK_C1 4
#endif
#ifndef WMD_BLK_W2  // NQ = 2 (v_r <= 256)
#define WMD_BLK_W2 8
#define WMD_BLK_C2 2
#endif
#ifndef WMD_BLK_W3  // NQ = 3 (v_r <= 384)
#define WMD_BLK_W3 4
#define WMD_BLK_C3 4
#endif
#ifndef WMD_BLK_W4  // NQ = 4 (v_r <= 512)
#define WMD_BLK_W4 4
#define WMD_BLK_C4 4
#endif

namespace {
__device__ __forceinline__ void bcp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void bcp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
// Four BF16 values (one 8-byte quad) -> FP32 (exact: BF16 is the top half
// of an FP32 bit pattern).
__device__ __forceinline__ float4 quad_to_f32(uint2 q) {
  return make_float4(__uint_as_float(q.x << 16), __uint_as_float(q.x & 0xffff0000u),
                     __uint_as_float(q.y << 16), __uint_as_float(q.y & 0xffff0000u));
}
}  // namespace

template <int NQ, int kBW>
struct BlockShape {
  static constexpr int RL = 128 * NQ;  // padded row length (elements)
  static constexpr int RB = RL * 2;    // bytes per staged row
  static constexpr int QPR = RL / 4;   // quads per row
  static __host__ __device__ size_t ent_bytes(int rows) {
    return ((size_t)rows * 8 + 15) & ~(size_t)15;
  }
  // staged rows, staged entries, per-warp x slices, two u buffers, the
  // per-warp partial sums.
  static __host__ __device__ size_t bytes(int rows) {
    return (size_t)rows * RB + ent_bytes(rows) + (size_t)kBW * RL * 4 +
           2 * (size_t)RL * 4 + (size_t)kBW * 8;
  }
};

// GRP: stacked batch group (batch.cu): work items are (source, document)
// pairs, source-major, the per-source arguments taken from grp[] item by item.
template <int NQ, int kBW, int kCPS, bool RLX, bool GRP = false>
__global__ void __launch_bounds__(kBW * 32, kCPS)
solve_block_kernel(const uint2* __restrict__ K16, int ldq, float expo,
                   const uint32_t* __restrict__ vr_dev,
                   const float* __restrict__ rinv,
                   const int64_t* __restrict__ col_ptr,
                   const uint2* __restrict__ ent,
                   const int32_t* __restrict__ order, int64_t N, int max_iter,
                   float tol, int* __restrict__ iters_out,
                   const float* __restrict__ u0, int64_t ldu, int max_rows,
                   float omega, float* __restrict__ vstate,
                   const float* __restrict__ mrow, double* __restrict__ out,
                   const GroupSrc* __restrict__ grp = nullptr, int nsrc = 0) {
  using Sh = BlockShape<NQ, kBW>;
  constexpr int kBT = kBW * 32;
  constexpr int RL = Sh::RL;
  constexpr int QPR = Sh::QPR;
  constexpr int DPT = (RL + kBT - 1) / kBT;  // dimensions per thread (update)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint2* sRows = reinterpret_cast<uint2*>(smem_raw);
  uint2* sEnt = reinterpret_cast<uint2*>(smem_raw + (size_t)max_rows * Sh::RB);
  float* xbuf = reinterpret_cast<float*>(smem_raw + (size_t)max_rows * Sh::RB +
                                         Sh::ent_bytes(max_rows));
  float* ubufA = xbuf + kBW * RL;
  float* ubufB = ubufA + RL;
  double* red = reinterpret_cast<double*>(ubufB + RL);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool lo = lane < 16;
  // GRP: the current source's arguments, one copy per CTA in shared memory,
  // read where they are used instead of being held in registers for the
  // whole document loop (which spilled the widest instantiation).
  __shared__ __align__(16) unsigned char gs_raw[GRP ? sizeof(GroupSrc) : 16];
  GroupSrc& gs = *reinterpret_cast<GroupSrc*>(gs_raw);
  const int vr_arg = GRP ? 0 : (int)*vr_dev;
  auto VR = [&]() -> int {
    if constexpr (GRP) return gs.vr;
    else return vr_arg;
  };
  auto KP = [&]() -> const uint2* {
    if constexpr (GRP) return static_cast<const uint2*>(gs.K16);
    else return K16;
  };
  auto VSTATE = [&]() -> float* {
    if constexpr (GRP) return gs.vstate;
    else return vstate;
  };
  auto MROW = [&]() -> const float* {
    if constexpr (GRP) return gs.mrow;
    else return mrow;
  };

  float rv[DPT], rw[DPT];  // 1/r_i and r_i of this thread's update dimensions
  auto set_dims = [&]() {
    const int vr = VR();
    const float* ri = GRP ? gs.rinv : rinv;
#pragma unroll
    for (int i = 0; i < DPT; ++i) {
      const int D = tid + i * kBT;
      rv[i] = D < vr ? ri[D] : 0.f;
      rw[i] = D < vr ? __frcp_rn(rv[i]) : 0.f;
    }
  };
  if constexpr (!GRP) set_dims();
  int cur_src = -1;
  const int64_t NI = GRP ? N * (int64_t)nsrc : N;  // work items

  for (int64_t idx = blockIdx.x; idx < NI; idx += gridDim.x) {
    const int64_t pos = GRP ? idx % N : idx;
    const int64_t j = order ? (int64_t)order[pos] : pos;
    const int64_t b = col_ptr[j];
    const int n = (int)(col_ptr[j + 1] - b);
    const int ns = n < max_rows ? n : max_rows;  // rows staged in shared memory
    const bool warm = u0 != nullptr && max_iter > 0;
    // Over-relaxation of both half-steps (vstate: each word's previous v),
    // compiled only into the RLX instantiations.
    constexpr bool relax = RLX;
    RelaxGuard g;
    g.init(omega);
    float resv = 0.f;  // this thread's c-side residual of the current pass

    __syncthreads();  // the previous document is done with shared memory
    if constexpr (GRP) {
      const int src = (int)(idx / N);
      if (src != cur_src) {  // this source's panel, weights and outputs
        if (tid == 0) gs = grp[src];
        __syncthreads();
        set_dims();
        cur_src = src;
      }
    }
    const int vr = VR();
    const uint2* const Kd = KP();  // this source's panel (rows past the staged ones)
    for (int k = tid; k < ns; k += kBT) sEnt[k] = __ldg(&ent[b + k]);
    for (int D = tid; D < RL; D += kBT) {
      ubufA[D] = D < vr ? (float)vr : 0.f;  // cold start (fused:188-191)
      if (warm) ubufB[D] = D < vr ? __ldg(&u0[j * ldu + D]) : 0.f;
    }
    __syncthreads();
    for (int c = tid; c < ns * (QPR / 2); c += kBT) {
      const int k = c / (QPR / 2), ch = c % (QPR / 2);
      bcp_async16(sRows + (size_t)k * QPR + 2 * ch,
                  Kd + (size_t)sEnt[k].x * ldq + 2 * ch);
    }
    bcp_async_wait_all();
    __syncthreads();

    // This warp's rows: a contiguous, even-sized share of the document.
    const int per = (((n + kBW - 1) / kBW) + 1) & ~1;
    const int r0 = min(n, warp * per), r1 = min(n, r0 + per);
    auto load_row = [&](int k, uint2 (&q)[NQ], float& c) {
      if (k >= r1) {
        c = 0.f;
#pragma unroll
        for (int t = 0; t < NQ; ++t) q[t] = make_uint2(0u, 0u);
      } else if (k < ns) {
        c = __uint_as_float(sEnt[k].y);
        const uint2* rp = sRows + (size_t)k * QPR;
#pragma unroll
        for (int t = 0; t < NQ; ++t) q[t] = rp[lane + 32 * t];
      } else {
        const uint2 e = __ldg(&ent[b + k]);
        c = __uint_as_float(e.y);
        const uint2* rp = Kd + (size_t)e.x * ldq;
#pragma unroll
        for (int t = 0; t < NQ; ++t) q[t] = __ldg(rp + lane + 32 * t);
      }
    };
    auto dot = [&](const uint2 (&q)[NQ], const float4 (&u)[NQ]) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < NQ; ++t) {
        const float4 k = quad_to_f32(q[t]);
        a = __ffma2_rn(make_float2(k.x, k.y), make_float2(u[t].x, u[t].y), a);
        a = __ffma2_rn(make_float2(k.z, k.w), make_float2(u[t].z, u[t].w), a);
      }
      return a.x + a.y;
    };
    // Sum of a per-lane partial over the warp for two rows at once: lanes
    // 0-15 end with row a's total, lanes 16-31 with row b's.
    auto pair_sum = [&](float pa, float pb) {
      float keep = lo ? pa : pb;
      const float send = lo ? pb : pa;
      keep += __shfl_xor_sync(0xffffffffu, send, 16);
#pragma unroll
      for (int off = 8; off; off >>= 1) keep += __shfl_xor_sync(0xffffffffu, keep, off);
      return keep;
    };
    auto weight = [](float c, float s) { return c != 0.f ? __fdividef(c, s) : 0.f; };
    // v of a row pair (rows ka, ka + 1) from its pair_sum: (v_a, v_b) in
    // every lane.  Relaxed: lanes 0 and 16 own the rows' states (vold: the
    // row's previous v, prefetched by vold_of).
    auto vold_of = [&](int kr) -> float {
      return (relax && !g.vfirst && (lane & 15) == 0 && kr < r1) ? VSTATE()[b + kr] : 0.f;
    };
    auto pair_weights = [&](float s, float ca, float cb, int ka, float vold, float2& va,
                            float2& vb) {
      float vm;
      if (relax) {
        float v = 0.f;
        if ((lane & 15) == 0)
          v = relaxed_v_pre(lo ? ca : cb, s, vold, VSTATE() + b + ka + (lo ? 0 : 1),
                            g.vfirst, g.omega, resv);
        vm = __shfl_sync(0xffffffffu, v, lane & 16);
      } else {
        vm = weight(lo ? ca : cb, s);
      }
      const float vo = __shfl_xor_sync(0xffffffffu, vm, 16);
      va = make_float2(lo ? vm : vo, lo ? vm : vo);
      vb = make_float2(lo ? vo : vm, lo ? vo : vm);
    };
    auto axpy = [&](const uint2 (&q)[NQ], float2 v, float4 (&x)[NQ]) {
#pragma unroll
      for (int t = 0; t < NQ; ++t) {
        const float4 k = quad_to_f32(q[t]);
        const float2 x01 = __ffma2_rn(make_float2(k.x, k.y), v, make_float2(x[t].x, x[t].y));
        const float2 x23 = __ffma2_rn(make_float2(k.z, k.w), v, make_float2(x[t].z, x[t].w));
        x[t] = make_float4(x01.x, x01.y, x23.x, x23.y);
      }
    };

    // One pass: x = K^T (c ./ (K u)) over the document's rows, summed over
    // the warps, then u <- 1 / (x / r) into `dst` (which may be `src`).
    // Returns the marginal residual of `src` (CTA-uniform) when `want_res`.
    auto pass = [&](const float* src, float* dst, bool want_res) -> float {
      float4 u[NQ], x[NQ];
      resv = 0.f;
#pragma unroll
      for (int t = 0; t < NQ; ++t) {
        u[t] = reinterpret_cast<const float4*>(src)[lane + 32 * t];
        x[t] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      int k = r0;
      // Four rows per step: two independent reduction chains in flight
      // (measured faster than converting each row to FP32 once and reusing
      // it: the reductions' latency, not the instruction count, bounds a
      // pass).
      for (; k + 2 < r1; k += 4) {
        uint2 qa[NQ], qb[NQ], qc[NQ], qd[NQ];
        float ca, cb, cc, cd;
        load_row(k, qa, ca);
        load_row(k + 1, qb, cb);
        load_row(k + 2, qc, cc);
        load_row(k + 3, qd, cd);
        const float o0 = vold_of(k + (lo ? 0 : 1)), o1 = vold_of(k + 2 + (lo ? 0 : 1));
        const float s0 = pair_sum(dot(qa, u), dot(qb, u));
        const float s1 = pair_sum(dot(qc, u), dot(qd, u));
        float2 va, vb, vc, vd;
        pair_weights(s0, ca, cb, k, o0, va, vb);
        pair_weights(s1, cc, cd, k + 2, o1, vc, vd);
        axpy(qa, va, x);
        axpy(qb, vb, x);
        axpy(qc, vc, x);
        axpy(qd, vd, x);
      }
      for (; k < r1; k += 2) {
        uint2 qa[NQ], qb[NQ];
        float ca, cb;
        load_row(k, qa, ca);
        load_row(k + 1, qb, cb);
        const float o0 = vold_of(k + (lo ? 0 : 1));
        float2 va, vb;
        pair_weights(pair_sum(dot(qa, u), dot(qb, u)), ca, cb, k, o0, va, vb);
        axpy(qa, va, x);
        axpy(qb, vb, x);
      }
#pragma unroll
      for (int t = 0; t < NQ; ++t)
        reinterpret_cast<float4*>(xbuf + warp * RL)[lane + 32 * t] = x[t];
      __syncthreads();
      float res = resv;
#pragma unroll
      for (int i = 0; i < DPT; ++i) {
        const int D = tid + i * kBT;
        if (D < RL) {
          float tot = 0.f;
#pragma unroll
          for (int w = 0; w < kBW; ++w) tot += xbuf[w * RL + D];
          if (D < vr) {
            const float uo = src[D];
            res += fabsf(uo * tot - rw[i]);
            dst[D] = relaxed_update(uo, __frcp_rn(rv[i] * tot), g.omega);
          } else {
            dst[D] = 0.f;
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
        for (int w = 0; w < kBW; ++w) total += (float)red[w];
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
      for (int D = tid; D < vr; D += kBT) fin &= (bool)isfinite(ubufB[D]);
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
        for (int D = tid; D < RL; D += kBT) cur[D] = D < vr ? (float)vr : 0.f;
        __syncthreads();
      }
    }
    int* const iters_p = GRP ? gs.iters : iters_out;
    if (iters_p && tid == 0) iters_p[j] = it;

    // Final half-step (fused:339-393): WMD = sum_k v_k (KM_k . u), FP64 sum,
    // KM_k = K_k ln(K_k) / expo from the staged BF16 row.
    float4 u[NQ];
#pragma unroll
    for (int t = 0; t < NQ; ++t) u[t] = reinterpret_cast<const float4*>(cur)[lane + 32 * t];
    const float km_scale = 0.69314718f / expo;  // ln 2 / expo
    auto kmdot = [&](const uint2 (&q)[NQ]) {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < NQ; ++t) {
        const float4 k = quad_to_f32(q[t]);
        const float l0 = k.x > 0.f ? __log2f(k.x) : 0.f;
        const float l1 = k.y > 0.f ? __log2f(k.y) : 0.f;
        const float l2 = k.z > 0.f ? __log2f(k.z) : 0.f;
        const float l3 = k.w > 0.f ? __log2f(k.w) : 0.f;
        a = __ffma2_rn(make_float2(u[t].x * k.x, u[t].y * k.y), make_float2(l0, l1), a);
        a = __ffma2_rn(make_float2(u[t].z * k.z, u[t].w * k.w), make_float2(l2, l3), a);
      }
      return a.x + a.y;
    };
    double acc = 0.0;
    for (int k = r0; k < r1; k += 2) {
      uint2 qa[NQ], qb[NQ];
      float ca, cb;
      load_row(k, qa, ca);
      load_row(k + 1, qb, cb);
      const float s = pair_sum(dot(qa, u), dot(qb, u));
      const float v = weight(lo ? ca : cb, s);
      const float tk = pair_sum(kmdot(qa), kmdot(qb)) * km_scale;
      if (lane == 0 || (lane == 16 && k + 1 < r1)) {
        acc += (double)v * (double)tk;
        if (MROW())  // row-scaled panel: + c_w m_w (panel_rescale.cu)
          acc += (double)(lo ? ca : cb) *
                 (double)__ldg(&MROW()[__ldg(&ent[b + k + (lo ? 0 : 1)]).x]);
      }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    // A non-finite u_i (x_i = 0: an empty document) makes the reference's
    // sum over dimensions NaN (fused:382-393).
    bool bad = false;
    for (int D = tid; D < vr; D += kBT)
      bad |= !isfinite(cur[D]) || (MROW() && cur[D] > kScaledUMax);  // see solve.cu
    __syncthreads();  // every warp has read the last u before red is reused
    if (lane == 0) red[warp] = acc;
    bad = __syncthreads_or(bad);
    if (tid == 0) {
      double tot = 0.0;
      for (int w = 0; w < kBW; ++w) tot += red[w];
      (GRP ? gs.out : out)[j] = bad ? __longlong_as_double(0x7ff8000000000000ll) : tot;
    }
  }
}

// FP32 panel [V][ld] -> BF16 panel [V][ld16] (round to nearest even), zero
// past the v_r source words so that the padded dimensions contribute nothing.
__global__ void panel_to_bf16_kernel(const float* __restrict__ K, int ld,
                                     uint2* __restrict__ K16, int ldq,
                                     uint64_t V, const uint32_t* __restrict__ vr_dev) {
  const int vr = (int)*vr_dev;
  const uint64_t total = V * (uint64_t)ldq;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = i / ldq;
    const int D0 = 4 * (int)(i % ldq);
    unsigned h[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int D = D0 + e;
      const float v = D < vr ? K[w * ld + D] : 0.f;
      h[e] = (unsigned)__bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
    K16[i] = make_uint2(h[0] | (h[1] << 16), h[2] | (h[3] << 16));
  }
}

int block_panel_width(uint32_t vr_cap) {
  if (vr_cap <= 64 || vr_cap > 512) return 0;
  return 128 * (int)((vr_cap + 127) / 128);
}

int launch_panel_to_bf16(const float* K, int ld, void* K16, int ld16, uint64_t V,
                         const uint32_t* vr, int num_sms, cudaStream_t st) {
  panel_to_bf16_kernel<<<(num_sms > 0 ? num_sms : 148) * 8, 256, 0, st>>>(
      K, ld, static_cast<uint2*>(K16), ld16 / 4, V, vr);
  return 1;
}

template <int NQ, int kBW, int kCPS, bool RLX, bool GRP = false>
static int launch_block_t(const void* K16, int ld16, float expo,
                          const SourceSel& s, const Targets& t,
                          const SolveCtl& ctl, const float* u0, int64_t ldu,
                          double* out, cudaStream_t st,
                          const GroupSrc* grp = nullptr, int nsrc = 0) {
  using Sh = BlockShape<NQ, kBW>;
  constexpr int kMaxDev = 64;
  static int sms_cache[kMaxDev] = {0};
  static int rows_cache[kMaxDev] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) dev = 0;
  if (sms_cache[dev] == 0) {
    const size_t budget = 227 * 1024 / kCPS - 1024;
    int rows = (int)((budget - Sh::bytes(0)) / (Sh::RB + 8));
    while (rows > 0 && Sh::bytes(rows) > budget) --rows;
    if (rows < 2) return -1;
    cudaFuncSetAttribute(solve_block_kernel<NQ, kBW, kCPS, RLX, GRP>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)Sh::bytes(rows));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms_cache[dev] = sms > 0 ? sms : 1;
    rows_cache[dev] = rows;
  }
  const int rows = rows_cache[dev];
  const int64_t items = GRP ? t.N * (int64_t)nsrc : t.N;
  int64_t grid = (int64_t)sms_cache[dev] * kCPS;
  if (grid > items) grid = items;
  if (grid < 1) grid = 1;
  solve_block_kernel<NQ, kBW, kCPS, RLX, GRP>
      <<<(unsigned)grid, kBW * 32, Sh::bytes(rows), st>>>(
          static_cast<const uint2*>(K16), ld16 / 4, expo, s.vr, s.rinv, t.col_ptr,
          t.ent, t.order, t.N, ctl.max_iter, ctl.tol, ctl.iters, u0, ldu, rows,
          ctl.omega, ctl.vstate, ctl.mrow, out, grp, nsrc);
  return 1;
}

// Stacked batch group on the BF16 panels (all of panel width ld16): one
// persistent launch over every (source, document) pair, in the launch shape
// `shape` (0: 4 warps x 4 CTAs/SM, 1: 8 x 2, 2: 16 x 1).
template <int NQ>
static int launch_block_group_nq(const GroupSrc* grp, int nsrc, int ld16, float expo,
                                 const Targets& t, const SolveCtl& ctl, int shape,
                                 cudaStream_t st) {
  SourceSel none;
  const bool r = ctl.omega != 1.f;
  switch (shape) {
    case 1:
      return r ? launch_block_t<NQ, 8, 2, true, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc)
               : launch_block_t<NQ, 8, 2, false, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc);
    case 2:
      return r ? launch_block_t<NQ, 16, 1, true, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc)
               : launch_block_t<NQ, 16, 1, false, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc);
    default:
      return r ? launch_block_t<NQ, 4, 4, true, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc)
               : launch_block_t<NQ, 4, 4, false, true>(nullptr, ld16, expo, none, t, ctl, nullptr, 0, nullptr, st, grp, nsrc);
  }
}

int launch_block_group(const GroupSrc* grp, int nsrc, int ld16, float expo,
                       const Targets& t, const SolveCtl& ctl, int shape, cudaStream_t st) {
  if (t.N <= 0 || nsrc <= 0) return 0;
  switch (ld16 / 128) {
    case 1: return launch_block_group_nq<1>(grp, nsrc, ld16, expo, t, ctl, shape, st);
    case 2: return launch_block_group_nq<2>(grp, nsrc, ld16, expo, t, ctl, shape, st);
    case 3: return launch_block_group_nq<3>(grp, nsrc, ld16, expo, t, ctl, shape, st);
    case 4: return launch_block_group_nq<4>(grp, nsrc, ld16, expo, t, ctl, shape, st);
  }
  return -1;
}

// Over-relaxed solves (omega != 1) run the instantiation that keeps each
// word's v; the plain one compiles without that state.
template <int NQ, int kBW, int kCPS>
static int launch_block_r(const void* K16, int ld16, float expo, const SourceSel& s,
                          const Targets& t, const SolveCtl& ctl, const float* u0,
                          int64_t ldu, double* out, cudaStream_t st) {
  if (ctl.omega != 1.f) {
    if (!ctl.vstate) return -1;
    return launch_block_t<NQ, kBW, kCPS, true>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
  }
  return launch_block_t<NQ, kBW, kCPS, false>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
}

// Launch shapes the autotuner chooses from (warps per CTA, CTAs per SM).
// shape < 0 selects the build-time table above.
// Indices 3-5 are the tensor-core form (solve_tc.cu) with 1, 2 or 4 CTAs
// per SM, launched by the caller.
int block_shape_count() { return 6; }
const char* block_shape_name(int shape) {
  static const char* names[] = {"4 warps x 4 CTAs/SM", "8 warps x 2 CTAs/SM",
                                "16 warps x 1 CTA/SM",
                                "tensor cores, 1 CTA/SM (longest documents on CUDA cores)",
                                "tensor cores, 2 CTAs/SM (longest documents on CUDA cores)",
                                "tensor cores, 4 CTAs/SM (longest documents on CUDA cores)"};
  return shape >= 0 && shape < 6 ? names[shape] : "build-time table";
}

template <int NQ, int W, int C>
static int launch_nq_default(const void* K16, int ld16, float expo, const SourceSel& s,
                             const Targets& t, const SolveCtl& ctl, const float* u0,
                             int64_t ldu, double* out, cudaStream_t st, int shape) {
  switch (shape) {
    case 0: return launch_block_r<NQ, 4, 4>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
    case 1: return launch_block_r<NQ, 8, 2>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
    case 2: return launch_block_r<NQ, 16, 1>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
    default: return launch_block_r<NQ, W, C>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st);
  }
}

int launch_solve_block(const void* K16, int ld16, float expo, uint32_t vr_cap,
                       const SourceSel& s, const Targets& t, const SolveCtl& ctl,
                       const float* u0, int64_t ldu, double* out, cudaStream_t st,
                       int shape) {
  if (t.N <= 0) return 0;
  if (expo == 0.f || ld16 != block_panel_width(vr_cap)) return -1;
  switch (ld16 / 128) {
    case 1: return launch_nq_default<1, WMD_BLK_W1, WMD_BLK_C1>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st, shape);
    case 2: return launch_nq_default<2, WMD_BLK_W2, WMD_BLK_C2>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st, shape);
    case 3: return launch_nq_default<3, WMD_BLK_W3, WMD_BLK_C3>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st, shape);
    case 4: return launch_nq_default<4, WMD_BLK_W4, WMD_BLK_C4>(K16, ld16, expo, s, t, ctl, u0, ldu, out, st, shape);
    default: return -1;
  }
}

}  // namespace wmd
