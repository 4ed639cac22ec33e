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
// The last line is evaluated as  WMD_j = sum_k v_k (KM[w_k,:] . u)  (the same
// sum, regrouped by word, accumulated in FP64), and because K = exp(expo*M)
// the K.*M entries are recovered from the K rows already on chip as
// K ln(K) / expo; only expo = 0 (K = 1, M unrecoverable) reads a K.*M panel.
//
// A document's scalings depend only on its own column, so the whole loop runs
// inside one warp with u and x in registers: no atomics (the reference needs
// `omp atomic`, fused:284), no global u/x traffic and no per-iteration
// launches.  The document's K rows are gathered once from the L2-resident
// panel and re-used by every iteration from the fastest place they fit:
// the first one to three rounds of rows stay in registers, the next ones are
// staged in shared memory, any remainder is re-gathered from L2.  A
// document's word ids and weights are staged first (independent loads), so
// every row gather is issued from on-chip addresses without a dependent L2
// round trip.
//
// Lane layout: LPW lanes share one word and each owns 32 consecutive source
// dimensions (lane q of the group: dimensions 32q..32q+31), so 32/LPW words
// ("a round") are in flight per warp.  For v_r <= 32 (LPW = 1) each lane holds
// a whole K row: the dot product K_w . u needs no shuffle and the 64 FMAs per
// word run as 32 packed FFMA2.  The x accumulators of the word slots are
// combined once per iteration through a 4.5 KB shared-memory transpose
// (rows padded to 36 floats), after which every lane recomputes u for its
// dimensions.
#include "wmd_internal.cuh"

namespace wmd {

// Launch shape (warps per CTA, CTAs per SM) and arithmetic form: build-time
// tuning knobs, the defaults being the measured best on B200.
// Wide sources (LPW > 1): 4 warps x 2 CTAs per SM, two staged rounds in
// flight.  v_r <= 32 (LPW = 1): one-warp CTAs, eight per SM, two staged
// rounds in flight and three rounds of rows in registers (eight rounds on
// chip: every document of up to 256 words without an L2 re-gather) -- the
// same occupancy; one-warp CTAs measured 6 % faster there and 12-27 %
// slower for the wide instantiations.
#ifndef WMD_SOLVE_WARPS
#define WMD_SOLVE_WARPS 4
#endif
#ifndef WMD_SOLVE_CTAS_PER_SM
#define WMD_SOLVE_CTAS_PER_SM 2
#endif
#ifndef WMD_SOLVE_WARPS_1
#define WMD_SOLVE_WARPS_1 1
#endif
#ifndef WMD_SOLVE_CTAS_PER_SM_1
#define WMD_SOLVE_CTAS_PER_SM_1 8
#endif
#ifndef WMD_SOLVE_UNROLL_1
#define WMD_SOLVE_UNROLL_1 2
#endif
#ifndef WMD_SOLVE_PACKED_FMA
#define WMD_SOLVE_PACKED_FMA 1
#endif
#ifndef WMD_SOLVE_REG_ROUNDS  // rounds of K rows kept in registers, 2 <= LPW <= 4
#define WMD_SOLVE_REG_ROUNDS 2
#endif
#ifndef WMD_SOLVE_REG_ROUNDS_1  // the same for LPW = 1 (v_r <= 32), unrelaxed
#define WMD_SOLVE_REG_ROUNDS_1 3
#endif
#ifndef WMD_SOLVE_UNROLL  // staged rounds in flight per step
#define WMD_SOLVE_UNROLL 2
#endif
#ifndef WMD_SOLVE_SKIP_PAD  // documents shorter than the register rounds skip the rest
#define WMD_SOLVE_SKIP_PAD 1
#endif
#ifndef WMD_SOLVE_DOT_CHAINS  // independent accumulators per dot product
#define WMD_SOLVE_DOT_CHAINS 2
#endif

namespace {
// Launch shape per lane layout: warps per CTA, CTAs per SM, staged rounds
// in flight per step.
template <int LPW>
struct SolveCfg {
  static constexpr int kWarps = LPW == 1 ? WMD_SOLVE_WARPS_1 : WMD_SOLVE_WARPS;
  static constexpr int kCtas = LPW == 1 ? WMD_SOLVE_CTAS_PER_SM_1 : WMD_SOLVE_CTAS_PER_SM;
  static constexpr int kUnroll = LPW == 1 ? WMD_SOLVE_UNROLL_1 : WMD_SOLVE_UNROLL;
};

// 16-byte copy global -> shared through L1 (.ca): a lane stages a row in
// 16-byte pieces, so the second half of each 32-byte sector hits L1.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) {
#if WMD_SOLVE_PACKED_FMA
  return __ffma2_rn(a, b, c);
#else
  return make_float2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y));
#endif
}

// Packed add (FADD2): each half rounded as the scalar add.
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) {
#if WMD_SOLVE_PACKED_FMA
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}

// The hardware base-2 logarithm with subnormal inputs flushed to zero.
__device__ __forceinline__ float lg2_ftz(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

struct Row {  // one lane's 32-dimension slice of a K (or KM) row
  float4 c[8];
};

__device__ __forceinline__ void zero_row(Row& r) {
#pragma unroll
  for (int t = 0; t < 8; ++t) r.c[t] = make_float4(0.f, 0.f, 0.f, 0.f);
}
// Rows of padding words (past the end of a document) are all ones with
// weight c = 0: then s = K_w . u > 0 for any u > 0 and v = c / s is exactly
// 0, so they add nothing to x and need no test for c = 0.
__device__ __forceinline__ void ones_row(Row& r) {
#pragma unroll
  for (int t = 0; t < 8; ++t) r.c[t] = make_float4(1.f, 1.f, 1.f, 1.f);
}
}  // namespace

template <int LPW, bool RLX = false>
struct SolveShape {
  static constexpr int WPS = 32 / LPW;  // words per round
  static constexpr int RL = 32 * LPW;   // padded row length (floats)
  static constexpr int NCH = RL / 4;    // float4 chunks per padded row
  static constexpr int SROW = NCH;  // float4 slots per staged row
  // Row pitch (floats) of the 32 x 32 transpose buffer: 36 puts the rows of
  // the 8 lanes of a 16-byte shared-memory phase on distinct bank groups
  // with no address arithmetic per access.
  static constexpr int RP = 36;
  // Rounds of K rows kept in registers (fewer when the per-lane dimension
  // arrays of wide sources, or the relaxation state, already use the
  // register budget).
  static constexpr int RR = LPW == 1 ? (RLX ? 2 : WMD_SOLVE_REG_ROUNDS_1)
                                     : (LPW <= 4 ? WMD_SOLVE_REG_ROUNDS : 1);
  static_assert(LPW >= 1 && LPW <= 32 && (LPW & (LPW - 1)) == 0, "LPW");
  // Per-warp shared memory: staged rows (whole rounds), staged entries
  // {word id, weight} of the register and staged rounds, 32x32 transpose
  // buffer, u broadcast buffer.  Every term is a multiple of 16 bytes.
  static __host__ __device__ size_t entries_bytes(int srounds) {
    return ((size_t)(srounds + RR) * WPS * 8 + 15) & ~(size_t)15;
  }
  static __host__ __device__ size_t staged_bytes(int srounds) {
    return (size_t)srounds * WPS * SROW * 16;
  }
  static __host__ __device__ size_t warp_bytes(int srounds) {
    return staged_bytes(srounds) + entries_bytes(srounds) + 32 * RP * 4 + RL * 4;
  }
};

// GRP: the stacked form of a batch (batch.cu): the work items are (source,
// document) pairs, source-major, over `nsrc` sources whose panel, weights and
// outputs come from grp[]; the per-source arguments below are then replaced
// item by item.
// kW, kC: warps per CTA and CTAs per SM of this instantiation (the
// build-time default shape, or an autotuner candidate).
template <int LPW, bool FROM_KM, bool RLX, bool GRP, int kW = SolveCfg<LPW>::kWarps,
          int kC = SolveCfg<LPW>::kCtas>
__global__ void __launch_bounds__(kW * 32, kC)
solve_kernel(const float* __restrict__ K, const float* __restrict__ KM, int ld_arg,
             float expo, const uint32_t* __restrict__ vr_dev,
             const float* __restrict__ rinv,
             const int64_t* __restrict__ col_ptr,
             const uint2* __restrict__ ent,
             const int32_t* __restrict__ order, int64_t N, int max_iter,
             float tol, int* __restrict__ iters_out, int srounds,
             const float* __restrict__ u0, int64_t ldu, float omega,
             float* __restrict__ vstate, const float* __restrict__ mrow,
             double* __restrict__ out, const GroupSrc* __restrict__ grp, int nsrc) {
  using Sh = SolveShape<LPW, RLX>;
  constexpr int WPS = Sh::WPS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = lane & (LPW - 1), g = lane / LPW;
  const int srows = srounds * WPS;
  unsigned char* wbase = smem_raw + (size_t)warp * Sh::warp_bytes(srounds);
  float4* sK = reinterpret_cast<float4*>(wbase);
  uint2* sE = reinterpret_cast<uint2*>(wbase + Sh::staged_bytes(srounds));
  float* red = reinterpret_cast<float*>(wbase + Sh::staged_bytes(srounds) +
                                        Sh::entries_bytes(srounds));
  float* ubuf = red + 32 * Sh::RP;
  // GRP: the current source's arguments, one copy per warp in shared
  // memory, read where they are used instead of being held in registers for
  // the whole document loop (which spilled the wide instantiations).
  __shared__ __align__(16) unsigned char gs_raw[GRP ? kW * sizeof(GroupSrc) : 16];
  GroupSrc& gs = reinterpret_cast<GroupSrc*>(gs_raw)[GRP ? warp : 0];
  grid_dep_wait();  // the panel (cost panel, fix-up) and the selection
  const int vr_arg = GRP ? 0 : (int)*vr_dev;
  auto KP = [&]() -> const float* {
    if constexpr (GRP) return gs.K;
    else return K;
  };
  auto VSTATE = [&]() -> float* {
    if constexpr (GRP) return gs.vstate;
    else return vstate;
  };
  auto MROW = [&]() -> const float* {
    if constexpr (GRP) return gs.mrow;
    else return mrow;
  };
  // Staged rounds are chunk-major: chunk t (dimensions 4t..4t+3 of the
  // lane's slice) of the row lane L holds in staged round s sits at float4
  // s * 256 + t * 32 + L.  A lane stages and reads only its own rows; the 8
  // lanes of a 16-byte shared-memory phase touch 8 consecutive slots (no
  // bank conflict), and every load is at an immediate offset from the
  // lane's base sK + L (rounds 4 KB apart, chunks 512 bytes apart).
  const float4* const sKl = sK + lane;

  // Dimensions this lane finalises after the transpose: 32*qq + own, with
  // own = 2 (lane % 16) + lane / 16 when the slot sums run in pairs
  // (LPW < 32), else own = lane.
  constexpr bool kPairSum = LPW < 32;
  const int own = kPairSum ? 2 * (lane & 15) + (lane >> 4) : lane;
  float rv[LPW], rw[LPW];  // 1/r_i and r_i
  unsigned dmask = 0;
  auto set_dims = [&]() {
    const int vr = GRP ? gs.vr : vr_arg;
    const float* ri = GRP ? gs.rinv : rinv;
    dmask = 0;
#pragma unroll
    for (int qq = 0; qq < LPW; ++qq) {
      const int D = 32 * qq + own;
      const bool ok = D < vr;
      rv[qq] = ok ? ri[D] : 0.f;
      rw[qq] = ok ? __frcp_rn(rv[qq]) : 0.f;
      dmask |= ok ? (1u << qq) : 0u;
    }
  };
  if constexpr (!GRP) set_dims();
  int cur_src = -1;
  const int64_t NI = GRP ? N * (int64_t)nsrc : N;  // work items

  constexpr int kWarps = kW;
  const int64_t total_warps = (int64_t)gridDim.x * kWarps;
  // Persistent warps over the documents in decreasing-length order, in
  // "snake" order: in lap p over the grid, warp w takes position
  // p*W + w for even p and p*W + (W-1-w) for odd p, so a warp that drew one
  // of the longest documents of a lap draws one of the shortest of the
  // next.  A plain stride hands warp 0 the longest document of every lap
  // (about 22 % above the mean load at the single-source workload).
  // Positions grow strictly with p, so the loop ends at the first >= NI.
  const int64_t wid = (int64_t)blockIdx.x * kWarps + warp;
  auto position = [&](int64_t p) -> int64_t {
    return p * total_warps + ((p & 1) ? total_warps - 1 - wid : wid);
  };
  int64_t lap = 0;
  int64_t idx = position(0);
  // Item -> (source, position in the document order).
  auto doc_of = [&](int64_t it) -> int64_t {
    const int64_t pos = GRP ? it % N : it;
    return order ? (int64_t)__ldg(&order[pos]) : pos;
  };
  // Pointers of the current document; the next one's are prefetched while
  // this one is processed.
  int64_t j = 0, b = 0;
  int n = 0;
  if (idx < NI) {
    j = doc_of(idx);
    b = col_ptr[j];
    n = (int)(col_ptr[j + 1] - b);
  }
  for (; idx < NI; idx = position(++lap)) {
    if constexpr (GRP) {
      const int src = (int)(idx / N);
      if (src != cur_src) {  // this source's panel, weights and outputs
        __syncwarp();
        if (lane == 0) gs = grp[src];
        __syncwarp();
        set_dims();
        cur_src = src;
      }
    }
    const int vr = GRP ? gs.vr : vr_arg;
    const int ld = GRP ? gs.ld : ld_arg;
    const int ldc = ld >> 2;  // float4 chunks per global panel row
    const float* const Kd = KP();  // this source's panel
    RelaxGuard rg;  // over-relaxation of this document (RLX instantiations)
    rg.init(omega);
    float resv = 0.f;  // this lane's c-side residual of the current pass
    const int64_t nidx = position(lap + 1);
    int64_t jn = 0;
    if (nidx < NI) jn = doc_of(nidx);
    const int rounds = (n + WPS - 1) / WPS;
    constexpr int RR = Sh::RR;
    const int rr = rounds < RR ? rounds : RR;                   // in registers
    const int sr = min(rounds - rr, srounds);                   // staged
    const int lr = rounds - rr - sr;                            // from L2
    const int ne = (rr + sr) * WPS;                             // staged entries

    // Entries of the register and staged rounds (zero past the document).
    __syncwarp();
#pragma unroll 4
    for (int k = lane; k < ne; k += 32)
      sE[k] = k < n ? __ldg(&ent[b + k]) : make_uint2(0u, 0u);
    __syncwarp();
    // Register rows: rounds [0, rr); padding rows (ones, c = 0) elsewhere.
    // Chunks past the panel width stay zero (their u is 0).
    Row reg[RR];
    float creg[RR];
#pragma unroll
    for (int t = 0; t < RR; ++t) {
      creg[t] = 0.f;
      const int k = t * WPS + g;
      if (t < rr && k < n) {
        zero_row(reg[t]);
        const uint2 en = sE[k];
        creg[t] = __uint_as_float(en.y);
        const float4* rp = reinterpret_cast<const float4*>(Kd + (size_t)en.x * ld);
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (8 * q + c < ldc) reg[t].c[c] = __ldg(rp + 8 * q + c);
      } else {
        ones_row(reg[t]);
      }
    }
    // Staged rows: rounds [rr, rr + sr), each lane its own row slice, padded
    // with ones rows to whole rounds; chunks past the panel width are zero.
    for (int r = 0; r < sr; ++r) {
      const int k = (rr + r) * WPS + g;
      float4* dst = sK + r * (WPS * Sh::NCH) + lane;
      if (k < n) {
        const float* src = Kd + (size_t)sE[k].x * ld + 32 * q;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          if (8 * q + t < ldc)
            cp_async16(dst + 32 * t, src + 4 * t);
          else
            dst[32 * t] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      } else {
#pragma unroll
        for (int t = 0; t < 8; ++t) dst[32 * t] = make_float4(1.f, 1.f, 1.f, 1.f);
      }
    }
    // Next document's pointers (the order[] load has landed by now).
    int64_t bn = 0;
    int nn = 0;
    if (nidx < NI) {
      bn = __ldg(&col_ptr[jn]);
      nn = (int)(__ldg(&col_ptr[jn + 1]) - bn);
    }
    cp_async_wait_all();
    __syncwarp();

    const uint2* const sEl = sE + rr * WPS + g;  // entries of staged round 0
    auto load_staged = [&](int s_round, Row& r, float& cval) {
      cval = __uint_as_float(sEl[s_round * WPS].y);
      const float4* rp = sKl + s_round * (WPS * Sh::NCH);
#pragma unroll
      for (int t = 0; t < 8; ++t) r.c[t] = rp[32 * t];
    };
    // A row from L2 (pad: the padding row for k >= n, else zeros).
    auto load_global = [&](const float* __restrict__ P, int k, Row& r,
                           float& cval, bool pad) {
      cval = 0.f;
      if (k < n) {
        zero_row(r);
        const uint2 en = __ldg(&ent[b + k]);
        cval = __uint_as_float(en.y);
        const float4* rp = reinterpret_cast<const float4*>(P + (size_t)en.x * ld);
#pragma unroll
        for (int t = 0; t < 8; ++t)
          if (8 * q + t < ldc) r.c[t] = __ldg(rp + 8 * q + t);
      } else if (pad) {
        ones_row(r);
      } else {
        zero_row(r);
      }
    };
    auto dot = [&](const Row& r, const float2 (&u2)[16]) {
      constexpr int NC = WMD_SOLVE_DOT_CHAINS;
      float2 a[NC];
#pragma unroll
      for (int i = 0; i < NC; ++i) a[i] = make_float2(0.f, 0.f);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        a[(2 * t) % NC] = ffma2(make_float2(r.c[t].x, r.c[t].y), u2[2 * t], a[(2 * t) % NC]);
        a[(2 * t + 1) % NC] =
            ffma2(make_float2(r.c[t].z, r.c[t].w), u2[2 * t + 1], a[(2 * t + 1) % NC]);
      }
#pragma unroll
      for (int w = NC / 2; w >= 1; w >>= 1)
#pragma unroll
        for (int i = 0; i < w; ++i) a[i] = fadd2(a[i], a[i + w]);
      float s = a[0].x + a[0].y;
#pragma unroll
      for (int off = 1; off < LPW; off <<= 1)
        s += __shfl_xor_sync(0xffffffffu, s, off);
      return s;
    };
    auto axpy = [&](const Row& r, float v, float2 (&x2)[16]) {
      const float2 vv = make_float2(v, v);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        x2[2 * t] = ffma2(make_float2(r.c[t].x, r.c[t].y), vv, x2[2 * t]);
        x2[2 * t + 1] = ffma2(make_float2(r.c[t].z, r.c[t].w), vv, x2[2 * t + 1]);
      }
    };
    // The first word slot of a pass starts the accumulators (x = K_w v).
    auto axpy_first = [&](const Row& r, float v, float2 (&x2)[16]) {
      const float2 vv = make_float2(v, v);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        x2[2 * t] = __fmul2_rn(make_float2(r.c[t].x, r.c[t].y), vv);
        x2[2 * t + 1] = __fmul2_rn(make_float2(r.c[t].z, r.c[t].w), vv);
      }
    };
    // v = c / s; exactly 0 for the padding words (c = 0, s > 0).
    auto weight = [](float c, float s) { return __fdividef(c, s); };
    // v of word k in a pass; over-relaxed (RLX) against the word's previous v
    // (vold, prefetched by vold_at with the word's row), which lane q = 0 of
    // the word's group keeps in vstate and broadcasts.
    auto vold_at = [&](int k) -> float {
      if constexpr (RLX) return (q == 0 && k < n && !rg.vfirst) ? VSTATE()[b + k] : 0.f;
      else return 0.f;
    };
    auto vweight = [&](float c, float s, int k, float vold) -> float {
      if constexpr (!RLX) {
        return weight(c, s);
      } else {
        float v = 0.f;
        if (q == 0 && k < n)
          v = relaxed_v_pre(c, s, vold, VSTATE() + b + k, rg.vfirst, rg.omega, resv);
        if constexpr (LPW > 1) v = __shfl_sync(0xffffffffu, v, lane & ~(LPW - 1));
        return v;
      }
    };
    // Sum the x slices of all word slots: lane writes its 32 values as row
    // `lane` of a 32x32 buffer (row pitch RP), then each lane sums, for
    // each of its LPW dimension groups, the slots' values of its dimension.
    // Paired form (LPW < 32): lanes L and L ^ 16 sum the dimension pair
    // (2p, 2p + 1), p = L % 16, over the two halves of the slots with 8-byte
    // loads and packed adds, combine the halves with one shuffle, and keep
    // dimension 2p + L / 16 (= own): tot[qq] is dimension 32*qq + own.
    auto reduce_slots = [&](const float2 (&x2)[16], float (&tot)[LPW]) {
      float4* rw = reinterpret_cast<float4*>(red + lane * Sh::RP);
#pragma unroll
      for (int t = 0; t < 8; ++t)
        rw[t] = make_float4(x2[2 * t].x, x2[2 * t].y, x2[2 * t + 1].x, x2[2 * t + 1].y);
      __syncwarp();
      if constexpr (kPairSum) {
        constexpr int HALF = WPS / 2;
        const int p = lane & 15, h = lane >> 4;
        const float* redp = red + h * HALF * LPW * Sh::RP + 2 * p;
#pragma unroll
        for (int qq = 0; qq < LPW; ++qq) {
          float2 part[HALF];
#pragma unroll
          for (int i = 0; i < HALF; ++i)
            part[i] = *reinterpret_cast<const float2*>(redp + (i * LPW + qq) * Sh::RP);
#pragma unroll
          for (int w = HALF / 2; w >= 1; w >>= 1)
#pragma unroll
            for (int i = 0; i < w; ++i)
              part[i] = fadd2(part[i], part[i + w]);
          const float2 o = make_float2(__shfl_xor_sync(0xffffffffu, part[0].x, 16),
                                       __shfl_xor_sync(0xffffffffu, part[0].y, 16));
          tot[qq] = h ? part[0].y + o.y : part[0].x + o.x;
        }
      } else {
#pragma unroll
        for (int qq = 0; qq < LPW; ++qq) {
          float part[WPS];
#pragma unroll
          for (int gg = 0; gg < WPS; ++gg) part[gg] = red[(gg * LPW + qq) * Sh::RP + lane];
#pragma unroll
          for (int w = WPS / 2; w >= 1; w >>= 1)
#pragma unroll
            for (int i = 0; i < w; ++i) part[i] += part[i + w];
          tot[qq] = part[0];
        }
      }
      __syncwarp();
    };
    auto broadcast_u = [&](const float (&uval)[LPW], float2 (&u2)[16]) {
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq) ubuf[32 * qq + own] = uval[qq];
      __syncwarp();
      const float4* ub = reinterpret_cast<const float4*>(ubuf + 32 * q);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const float4 v = ub[t];
        u2[2 * t] = make_float2(v.x, v.y);
        u2[2 * t + 1] = make_float2(v.z, v.w);
      }
      __syncwarp();
    };
    // One pass of v = c ./ (K^T u), x += K v over all rounds of the document.
    auto pass = [&](const float2 (&u2)[16], float2 (&x2)[16]) {
      if constexpr (RLX) resv = 0.f;
      {
        float sreg[RR], oreg[RR];
#pragma unroll
        for (int t = 0; t < RR; ++t) oreg[t] = vold_at(t * WPS + g);
        if (WMD_SOLVE_SKIP_PAD && RR > 1 && rr < RR) {
          // A document of fewer rounds than the register rounds: only the
          // rounds it fills (the others hold padding rows, whose v = 0 adds
          // exactly nothing to x).  Round 0 always runs: it starts x.
          sreg[0] = dot(reg[0], u2);
          axpy_first(reg[0], vweight(creg[0], sreg[0], g, oreg[0]), x2);
#pragma unroll
          for (int t = 1; t < RR; ++t)
            if (t < rr)
              axpy(reg[t], vweight(creg[t], dot(reg[t], u2), t * WPS + g, oreg[t]), x2);
        } else {
#pragma unroll
          for (int t = 0; t < RR; ++t) sreg[t] = dot(reg[t], u2);
          axpy_first(reg[0], vweight(creg[0], sreg[0], g, oreg[0]), x2);
#pragma unroll
          for (int t = 1; t < RR; ++t)
            axpy(reg[t], vweight(creg[t], sreg[t], t * WPS + g, oreg[t]), x2);
        }
      }
      constexpr int U = SolveCfg<LPW>::kUnroll;
      int t = 0;
      for (; t + U <= sr; t += U) {
        Row ra[U];
        float ca[U], sa[U], oa[U];
#pragma unroll
        for (int i = 0; i < U; ++i) {
          load_staged(t + i, ra[i], ca[i]);
          oa[i] = vold_at((rr + t + i) * WPS + g);
        }
#pragma unroll
        for (int i = 0; i < U; ++i) sa[i] = dot(ra[i], u2);
#pragma unroll
        for (int i = 0; i < U; ++i)
          axpy(ra[i], vweight(ca[i], sa[i], (rr + t + i) * WPS + g, oa[i]), x2);
      }
      for (; t < sr; ++t) {
        Row ra;
        float ca;
        load_staged(t, ra, ca);
        const float oa = vold_at((rr + t) * WPS + g);
        axpy(ra, vweight(ca, dot(ra, u2), (rr + t) * WPS + g, oa), x2);
      }
      for (int l = 0; l < lr; ++l) {
        Row ra;
        float ca;
        load_global(Kd, (rr + sr + l) * WPS + g, ra, ca, true);
        const float oa = vold_at((rr + sr + l) * WPS + g);
        axpy(ra, vweight(ca, dot(ra, u2), (rr + sr + l) * WPS + g, oa), x2);
      }
    };

    float2 u2[16];
    {
      float uval[LPW];
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq) uval[qq] = ((dmask >> qq) & 1u) ? (float)vr : 0.f;
      broadcast_u(uval, u2);
    }
    // One x-update from the u in u2 / ubuf: the new u into unew, and the
    // marginal residual |u_i (K v)_i - r_i| of the u entering it (read from
    // the broadcast buffer: each lane reads only entries it wrote itself),
    // warp-reduced when want_res.
    auto step = [&](float (&unew)[LPW], bool want_res) {
      float2 x2[16];
      pass(u2, x2);
      float tot[LPW];
      reduce_slots(x2, tot);
      float res = 0.f;
      if constexpr (RLX) res = resv;
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq) {
        const bool ok = (dmask >> qq) & 1u;
        const float uo = ubuf[32 * qq + own];
        if (want_res && ok) res += fabsf(uo * tot[qq] - rw[qq]);
        // u = 1 / (x / r), on the per-pass serial chain: the hardware's
        // approximate reciprocal (about 1 ulp; 2-4 % of the solve against
        // the round-to-nearest one, results within 1e-7 of each other),
        // except for the row-scaled panel, whose extreme scalings may need
        // the subnormal range that the approximation flushes to zero.
        const float xr = rv[qq] * tot[qq];
        const float uh = MROW() ? __frcp_rn(xr) : __fdividef(1.f, xr);
        unew[qq] = ok ? relaxed_update(uo, uh, RLX ? rg.omega : 1.f)
                      : 0.f;
      }
      if (want_res) {
#pragma unroll
        for (int off = 16; off; off >>= 1) res += __shfl_xor_sync(0xffffffffu, res, off);
      }
      return res;
    };

    int it = 0;
    float res = 0.f;
    if (u0 && max_iter > 0) {
      // Warm start: the first update from both the cold start and u0; keep
      // u0's unless its residual is worse than the cold start's or not
      // finite.
      float uc[LPW], uw[LPW], uval[LPW];
      const float rc = step(uc, true);
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq)
        uval[qq] = ((dmask >> qq) & 1u) ? __ldg(&u0[j * ldu + 32 * qq + own]) : 0.f;
      broadcast_u(uval, u2);
      const float rwm = step(uw, true);
      // The warm candidate must also leave a finite u.
      bool fin = true;
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq) fin &= !((dmask >> qq) & 1u) || isfinite(uw[qq]);
      fin = __all_sync(0xffffffffu, fin);
      const bool use_warm = fin && isfinite(rwm) && !(rc < rwm);
#pragma unroll
      for (int qq = 0; qq < LPW; ++qq) uval[qq] = use_warm ? uw[qq] : uc[qq];
      broadcast_u(uval, u2);
      res = use_warm ? rwm : rc;
      it = 1;
      if constexpr (RLX) rg.vfirst = true;  // the stored v are the last candidate's
    }
    while (it < max_iter && !(it > 0 && tol > 0.f && res <= tol)) {
      float uval[LPW];
      res = step(uval, tol > 0.f || RLX);
      ++it;
      if constexpr (RLX) {
        bool reset_u = false;
        if (rg.step(res, it, &reset_u) && reset_u) {
#pragma unroll
          for (int qq = 0; qq < LPW; ++qq) uval[qq] = ((dmask >> qq) & 1u) ? (float)vr : 0.f;
        }
      }
      broadcast_u(uval, u2);
    }
    int* const iters_p = GRP ? gs.iters : iters_out;
    if (iters_p && lane == 0) iters_p[j] = it;

    // Final half-step (fused:339-393): WMD = sum_k v_k (KM_k . u), FP64 sum.
    const float km_scale = FROM_KM ? 1.f : 0.69314718f / expo;  // ln 2 / expo
    double acc = 0.0;
    // KM_k . u with KM_i = K_i M_i = K_i log2(K_i) ln2 / expo.  Outside the
    // row-scaled panel every K entry is 0 (padding) or normal (lambda M stays
    // below the scaling limit, K >= e^-80), so the flush-to-zero hardware
    // logarithm of max(K, 2^-126) gives log2 K exactly as the subnormal-aware
    // form and 0 x (-126) = 0 for the zeros; the row-scaled panel's subnormal
    // entries (weighted by a large u) keep the subnormal-aware form.
    auto km_dot = [&](const Row& rk, bool exact) -> float {
      float2 a = make_float2(0.f, 0.f);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const float4 kk = rk.c[c];
        float l0, l1, l2, l3;
        if (exact) {
          l0 = kk.x > 0.f ? __log2f(kk.x) : 0.f;
          l1 = kk.y > 0.f ? __log2f(kk.y) : 0.f;
          l2 = kk.z > 0.f ? __log2f(kk.z) : 0.f;
          l3 = kk.w > 0.f ? __log2f(kk.w) : 0.f;
        } else {
          l0 = lg2_ftz(fmaxf(kk.x, 0x1p-126f));
          l1 = lg2_ftz(fmaxf(kk.y, 0x1p-126f));
          l2 = lg2_ftz(fmaxf(kk.z, 0x1p-126f));
          l3 = lg2_ftz(fmaxf(kk.w, 0x1p-126f));
        }
        const float2 uk0 = __fmul2_rn(u2[2 * c], make_float2(kk.x, kk.y));
        const float2 uk1 = __fmul2_rn(u2[2 * c + 1], make_float2(kk.z, kk.w));
        a = ffma2(uk0, make_float2(l0, l1), a);
        a = ffma2(uk1, make_float2(l2, l3), a);
      }
      return a.x + a.y;
    };
    // exact: the row-scaled panel (its subnormal-aware logarithm and the
    // + c_w m_w term).
    auto final_word = [&](const Row& rk, float ck, int k, bool exact) {
      const float v = weight(ck, dot(rk, u2));
      float tk;
      if (FROM_KM) {
        Row rm;
        float cm;
        load_global(KM, k, rm, cm, false);
        tk = dot(rm, u2);
      } else {
        tk = km_dot(rk, exact);
#pragma unroll
        for (int off = 1; off < LPW; off <<= 1)
          tk += __shfl_xor_sync(0xffffffffu, tk, off);
        tk *= km_scale;
      }
      if (q == 0 && k < n) {
        acc += (double)v * (double)tk;
        if (exact) {  // row-scaled panel: + c_w m_w (panel_rescale.cu)
          const uint32_t id = k < ne ? sE[k].x : __ldg(&ent[b + k]).x;
          acc += (double)ck * (double)__ldg(&MROW()[id]);
        }
      }
    };
    if (MROW()) {
      // Row-scaled panel: one copy of the word body (the register rows
      // selected per round), which keeps the final half-step's code small.
      for (int t = 0; t < rounds; ++t) {
        Row rk;
        float ck;
        if (t < rr) {
          rk = reg[0];
          ck = creg[0];
#pragma unroll
          for (int i = 1; i < RR; ++i)
            if (t == i) {
              rk = reg[i];
              ck = creg[i];
            }
        } else if (t < rr + sr) {
          load_staged(t - rr, rk, ck);
        } else {
          load_global(Kd, t * WPS + g, rk, ck, true);
        }
        final_word(rk, ck, t * WPS + g, true);
      }
    } else {
      // Register rounds by their fixed registers, then the staged and L2 ones.
#pragma unroll
      for (int t = 0; t < RR; ++t)
        if (t < rr) final_word(reg[t], creg[t], t * WPS + g, false);
      for (int t = rr; t < rounds; ++t) {
        Row rk;
        float ck;
        if (t < rr + sr)
          load_staged(t - rr, rk, ck);
        else
          load_global(Kd, t * WPS + g, rk, ck, true);
        final_word(rk, ck, t * WPS + g, false);
      }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    // The reference sums u_i x'_i over dimensions (fused:382-393): a
    // non-finite u_i (x_i = 0, e.g. an empty document) meets x'_i = 0 there
    // and makes the document NaN, which the regrouped sum above cannot see.
    bool bad = false;
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int d0 = 32 * q + 2 * t;
      bad |= (d0 < vr && !isfinite(u2[t].x)) || (d0 + 1 < vr && !isfinite(u2[t].y));
      // Row-scaled panel: a u this large means a source word whose K entries
      // in this document are at the FP32 floor (subnormal, few significant
      // bits): the document goes to the FP64 re-solve (exact_f64.cu).
      if (MROW())
        bad |= (d0 < vr && u2[t].x > kScaledUMax) || (d0 + 1 < vr && u2[t].y > kScaledUMax);
    }
    if (__any_sync(0xffffffffu, bad)) acc = __longlong_as_double(0x7ff8000000000000ll);
    if (vr == 0) acc = 0.0;  // no source word: an empty sum (fused:387)
    if (lane == 0) (GRP ? gs.out : out)[j] = acc;
    j = jn;
    b = bn;
    n = nn;
  }
}

template <int LPW, bool FROM_KM, bool RLX, bool GRP = false,
          int kW = SolveCfg<LPW>::kWarps, int kC = SolveCfg<LPW>::kCtas>
static int launch_solve_t(const float* K, const float* KM, int ld, float expo,
                          const SourceSel& s, const Targets& t,
                          const SolveCtl& ctl, double* out, cudaStream_t st,
                          const GroupSrc* grp = nullptr, int nsrc = 0) {
  using Sh = SolveShape<LPW, RLX>;
  constexpr int kMaxDev = 64;
  constexpr int kBlocksPerSm = kC;
  constexpr int kWarps = kW;
  constexpr size_t kSmemPerSm = 227 * 1024;
  static int sms_cache[kMaxDev] = {0};
  static int srounds_cache[kMaxDev] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) dev = 0;
  if (sms_cache[dev] == 0) {
    const size_t per_warp = (kSmemPerSm / kBlocksPerSm - 1024) / kWarps;
    const size_t fixed = Sh::warp_bytes(0);
    const size_t per_round = Sh::staged_bytes(1) + (size_t)Sh::WPS * 8;
    int sr = per_warp > fixed ? (int)((per_warp - fixed) / per_round) : 0;
    while (sr > 0 && Sh::warp_bytes(sr) > per_warp) --sr;
    cudaFuncSetAttribute(solve_kernel<LPW, FROM_KM, RLX, GRP, kW, kC>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(kWarps * Sh::warp_bytes(sr)));
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms_cache[dev] = sms > 0 ? sms : 1;
    srounds_cache[dev] = sr;
  }
  const int sr = srounds_cache[dev];
  const size_t smem = (size_t)kWarps * Sh::warp_bytes(sr);
  const int64_t items = GRP ? t.N * (int64_t)nsrc : t.N;
  int64_t want = (items + kWarps - 1) / kWarps;
  int64_t grid = (int64_t)sms_cache[dev] * kBlocksPerSm;
  if (grid > want) grid = want;
  if (grid < 1) grid = 1;
  launch_pdl(solve_kernel<LPW, FROM_KM, RLX, GRP, kW, kC>, dim3((unsigned)grid),
             dim3(kWarps * 32), smem, st, K, KM, ld, expo, s.vr, s.rinv, t.col_ptr, t.ent,
             t.order, t.N, ctl.max_iter, ctl.tol, ctl.iters, sr, ctl.u0, ctl.ldu, ctl.omega,
             ctl.vstate, ctl.mrow, out, grp, nsrc);
  return 1;
}

// Stacked batch group: one persistent launch over every (source, document)
// pair of `nsrc` sources of one lane-layout class (v_r <= vr_max), source-
// major so that the grid works on one or two sources' panels at a time.
template <int LPW>
static int launch_group_t(const GroupSrc* grp, int nsrc, float expo, const Targets& t,
                          const SolveCtl& ctl, cudaStream_t st, int shape) {
  SourceSel none;
  if (ctl.omega != 1.f)
    return launch_solve_t<LPW, false, true, true>(nullptr, nullptr, 4, expo, none, t, ctl,
                                                  nullptr, st, grp, nsrc);
  switch (shape) {  // the candidates of solve_shape_name()
    case 0:
      return launch_solve_t<LPW, false, false, true, 1, 8>(nullptr, nullptr, 4, expo, none, t,
                                                           ctl, nullptr, st, grp, nsrc);
    case 1:
      return launch_solve_t<LPW, false, false, true, 2, 4>(nullptr, nullptr, 4, expo, none, t,
                                                           ctl, nullptr, st, grp, nsrc);
    case 2:
      return launch_solve_t<LPW, false, false, true, 4, 2>(nullptr, nullptr, 4, expo, none, t,
                                                           ctl, nullptr, st, grp, nsrc);
  }
  return launch_solve_t<LPW, false, false, true>(nullptr, nullptr, 4, expo, none, t, ctl,
                                                 nullptr, st, grp, nsrc);
}

int launch_solve_group(uint32_t vr_max, const GroupSrc* grp, int nsrc, float expo,
                       const Targets& t, const SolveCtl& ctl, cudaStream_t st, int shape) {
  if (t.N <= 0 || nsrc <= 0) return 0;
  SolveCtl c = ctl;
  c.u0 = nullptr;  // cold start only in the stacked form
  if (vr_max <= 32) return launch_group_t<1>(grp, nsrc, expo, t, c, st, shape);
  if (vr_max <= 64) return launch_group_t<2>(grp, nsrc, expo, t, c, st, shape);
  if (vr_max <= 128) return launch_group_t<4>(grp, nsrc, expo, t, c, st, shape);
  if (vr_max <= 256) return launch_group_t<8>(grp, nsrc, expo, t, c, st, shape);
  if (vr_max <= 512) return launch_group_t<16>(grp, nsrc, expo, t, c, st, shape);
  if (vr_max <= 1024) return launch_group_t<32>(grp, nsrc, expo, t, c, st, shape);
  return -1;
}

template <bool FROM_KM, bool RLX>
static int dispatch_solve(const float* K, const float* KM, int ld, float expo,
                          uint32_t vr_cap, const SourceSel& s, const Targets& t,
                          const SolveCtl& c, double* out, cudaStream_t st) {
  if (vr_cap <= 32) return launch_solve_t<1, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  if (vr_cap <= 64) return launch_solve_t<2, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  if (vr_cap <= 128) return launch_solve_t<4, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  if (vr_cap <= 256) return launch_solve_t<8, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  if (vr_cap <= 512) return launch_solve_t<16, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  if (vr_cap <= 1024) return launch_solve_t<32, FROM_KM, RLX>(K, KM, ld, expo, s, t, c, out, st);
  return -1;
}

// Autotuner candidates of the plain (unrelaxed, lambda != 0) warp solve:
// warps per CTA x CTAs per SM at the same eight warps per SM.
int solve_shape_count() { return 3; }
const char* solve_shape_name(int shape) {
  switch (shape) {
    case 0: return "1 warp x 8 CTAs/SM";
    case 1: return "2 warps x 4 CTAs/SM";
    case 2: return "4 warps x 2 CTAs/SM";
  }
  return "build-time default";
}

template <int LPW>
static int launch_plain_shape(const float* K, int ld, float expo, const SourceSel& s,
                              const Targets& t, const SolveCtl& c, double* out,
                              cudaStream_t st, int shape) {
  switch (shape) {
    case 0: return launch_solve_t<LPW, false, false, false, 1, 8>(K, nullptr, ld, expo, s, t, c, out, st);
    case 1: return launch_solve_t<LPW, false, false, false, 2, 4>(K, nullptr, ld, expo, s, t, c, out, st);
    case 2: return launch_solve_t<LPW, false, false, false, 4, 2>(K, nullptr, ld, expo, s, t, c, out, st);
  }
  return launch_solve_t<LPW, false, false>(K, nullptr, ld, expo, s, t, c, out, st);
}

int launch_solve(const float* K, const float* KM, int ld, float expo,
                 uint32_t vr_cap, const SourceSel& s, const Targets& t,
                 const SolveCtl& ctl, double* out, cudaStream_t st, int shape) {
  if (t.N <= 0) return 0;
  if (shape >= 0 && !KM && ctl.omega == 1.f) {
    if (vr_cap <= 32) return launch_plain_shape<1>(K, ld, expo, s, t, ctl, out, st, shape);
    if (vr_cap <= 64) return launch_plain_shape<2>(K, ld, expo, s, t, ctl, out, st, shape);
    if (vr_cap <= 128) return launch_plain_shape<4>(K, ld, expo, s, t, ctl, out, st, shape);
    if (vr_cap <= 256) return launch_plain_shape<8>(K, ld, expo, s, t, ctl, out, st, shape);
    if (vr_cap <= 512) return launch_plain_shape<16>(K, ld, expo, s, t, ctl, out, st, shape);
    if (vr_cap <= 1024) return launch_plain_shape<32>(K, ld, expo, s, t, ctl, out, st, shape);
    return -1;
  }
  // lambda = 0 (KM read from a panel: K = 1 everywhere) runs unrelaxed.
  if (KM)
    return dispatch_solve<true, false>(K, KM, ld, expo, vr_cap, s, t, ctl, out, st);
  if (ctl.omega != 1.f) {
    if (!ctl.vstate) return -1;
    return dispatch_solve<false, true>(K, KM, ld, expo, vr_cap, s, t, ctl, out, st);
  }
  return dispatch_solve<false, false>(K, KM, ld, expo, vr_cap, s, t, ctl, out, st);
}

}  // namespace wmd
