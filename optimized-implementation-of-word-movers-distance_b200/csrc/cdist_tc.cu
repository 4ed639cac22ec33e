// Tensor-core cost panel (tcgen05, sm_100a).
//
// Same output as cdist_fp32.cu — K[w,i] = exp(expo * M[w,i]) and
// KM = K * M in the word-major [V][ld] layout of the reference's fused solver
// (sinkhorn_wmd_fused.cpp:197-223) — but the dot products E_w . S_i run on
// the 5th-generation tensor cores (16-bit or split-TF32 operands, below) with
// FP32 accumulation in tensor memory:
//
//   warp 0      TMA producer: the source tile S (all K-chunks) once, then a
//               ring of 128-row x 128-byte vocabulary tiles (128-byte
//               swizzle), one mbarrier pair per stage; the ring is as deep
//               as the shared memory left by S allows (up to 12 stages), as
//               the bytes in flight per SM bound this streaming kernel;
//   warp 1      allocates TMEM; one thread issues tcgen05.mma
//               (M=128, N=NT, 32 bytes of K per instruction) into a
//               double-buffered FP32 accumulator and tcgen05.commit's
//               stage-release / accumulator-ready barriers;
//   warps 2-9   epilogue: tcgen05.ld of one accumulator row per thread (two
//               warps per TMEM lane quarter, splitting the columns),
//               M^2 = |E_w|^2 + |S_i|^2 - 2 E_w.S_i with FP32 norms of the FP32
//               embeddings, then K = exp(expo*M), KM = K*M.  Pairs below
//               max(0.25, (|E_w|^2+|S_i|^2)/30) (the cancellation-prone ones)
//               are appended to a list that near_fixup_kernel recomputes
//               exactly afterwards, one warp per pair.
//
// Persistent grid: each CTA owns one N-tile of source words and walks the
// vocabulary M-tiles blockIdx.x, blockIdx.x + gridDim.x, ...  No TMA
// multicast is used.  Every mbarrier wait gives up after a wall-clock bound
// (globaltimer), sets ERR_TIMEOUT in the error word and lets the CTA exit.
//
// Operand forms: 16-bit copies of the embeddings (BF16 or FP16, kind::f16),
// or the FP32-accurate split form (X3 = true, kind::tf32) that reads the FP32
// embeddings themselves (128 rows x 32 floats per 128-byte swizzle row).  In
// the split form four more warps (10-13) take every landed tile, release its
// ring stage at once, and write it into one of two slots as a TF32 high part
// hi = x with the low 13 mantissa bits cleared and the remainder lo = x - hi
// (exact in FP32), both in the tile's swizzled layout; the source tile is
// split the same way once and stacked as one N = 2 NT operand [hi | lo].  Per
// 8-element K step the MMA issuer accumulates hi.[hi | lo] (columns [0, NT)
// and [NT, 2 NT)) and lo.hi (columns [0, NT)), and the epilogue adds the two
// halves: hi.hi + hi.lo + lo.hi, the split-operand "3xTF32" product (the
// dropped lo.lo term is below 2^-22 relative), which carries about 21 of FP32's 24 mantissa
// bits, so the epilogue and the near-pair fix-up give the FP32 panel's
// results.  Only the FP32 embeddings are read: no 16-bit or split copies are
// kept in HBM.
#include <cuda.h>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tcgen05.cuh"
#include "wmd_internal.cuh"

namespace wmd {
namespace tc {

constexpr int BM = 128;          // vocabulary rows per tile (UMMA M)
constexpr int BK = 64;           // 16-bit elements per 128-byte swizzle row
constexpr int kTileBytesA = BM * 128;  // 16 KB: 128 rows of 128 bytes

// Per-form constants.  Both forms step K by 32 bytes per instruction (16
// 16-bit or 8 TF32 elements), four steps per 128-byte chunk.  The ring depth
// is chosen per launch from the shared memory the source tile leaves
// (kMaxStages at most): the deeper the ring, the more HBM bytes are in flight
// per SM, which is what bounds this streaming kernel.
#ifndef WMD_TC_MAX_STAGES
#define WMD_TC_MAX_STAGES 12
#endif
#ifndef WMD_TC_X3_SLOTS  // split (hi, lo) tile slots between converters and MMA
#define WMD_TC_X3_SLOTS 2
#endif
constexpr int kMaxStages = WMD_TC_MAX_STAGES;
constexpr int kSlots = WMD_TC_X3_SLOTS;
// H2: the split-FP16 form (kind::f16 on FP16 high and scaled low parts of
// the embeddings, both read from HBM by TMA: two vocabulary tiles per ring
// stage, no converter warps).
template <bool X3, bool H2 = false>
struct Form {
  static_assert(!(X3 && H2), "one split form");
  static constexpr int kThreads = X3 ? 448 : 320;   // + 4 converter warps
  static constexpr int kChunk = X3 ? 32 : BK;       // elements per chunk row
  static constexpr int kMult = (X3 || H2) ? 2 : 1;  // B buffers (hi, lo)
  static constexpr int kSlotBytes = X3 ? kSlots * 2 * kTileBytesA : 0;
  static constexpr int kStageBytes = (H2 ? 2 : 1) * kTileBytesA;  // ring stage
};

struct Params {
  const float* E32;   // [V][d]
  const float* nE;    // [V]
  const float* S32;   // [cap][d]
  const float* nS;    // [cap]
  const uint32_t* vr; // device v_r
  float* K;           // [V][ld]
  float* KM;          // [V][ld] or null (then K*M is not stored)
  NearList near;      // cancellation-prone pairs for the exact fix-up pass
  float* mrow;        // row-scaled form: [V] row minima of M (else null)
  // Stacked batch group (null: one source): N-tile blockIdx.y covers rows
  // [tiles[y].y, + NT) of the stacked source rows, which are columns
  // [tiles[y].z, + NT) of source tiles[y].x's panel (grp[]).
  const int4* tiles;
  const GroupSrc* grp;
  // Split-FP16 form: 1/s of each vocabulary row (esc) and of each source row
  // (ssc), one FP32 value every sc_stride floats (inside the split rows).
  const float* esc;
  const float* ssc;
  int sc_stride;
  unsigned* err;
  uint64_t V;
  int d, ld, NT, KT, tmem_cols, stages;
  float expo;
};

// Dynamic shared memory layout (base rounded up to 1024 bytes):
//   A ring   stages x 16 KB       TMA destination (X3: raw FP32 tiles)
//   slots    kSlots x 32 KB       X3 only: split tiles, hi then lo
//   B        KT x NT x 128 B      (X3: per chunk NT hi rows, then NT lo
//                                 rows: one N = 2 NT operand [hi | lo])
//   barriers full[stages], empty[stages], conv[kSlots], mfree[kSlots],
//            bfull, bconv, accf[2], acce[2]
//   tmem address slot, nS copy [NT] (H2: + source scales [NT])
// H2: each ring stage holds the high then the low tile (2 x 16 KB), and B
// per chunk NT high rows then NT low rows, both loaded by TMA.
template <bool X3, bool H2 = false>
__host__ __device__ inline size_t smem_fixed_bytes(int NT, int KT) {
  return 1024 + (size_t)Form<X3, H2>::kSlotBytes +
         (size_t)KT * NT * 128 * Form<X3, H2>::kMult + (2 * kSlots + 6) * 8 + 16 +
         (size_t)NT * 4 * (H2 ? 2 : 1);
}
template <bool X3, bool H2 = false>
__host__ __device__ inline size_t smem_bytes(int NT, int KT, int stages) {
  return smem_fixed_bytes<X3, H2>(NT, KT) +
         (size_t)stages * (Form<X3, H2>::kStageBytes + 16);
}
// Deepest ring that fits in `budget` bytes (0 if not even two stages fit).
template <bool X3, bool H2 = false>
inline int ring_stages(int NT, int KT, size_t budget) {
  const size_t fixed = smem_fixed_bytes<X3, H2>(NT, KT);
  if (fixed >= budget) return 0;
  int st = (int)((budget - fixed) / (Form<X3, H2>::kStageBytes + 16));
  if (st > kMaxStages) st = kMaxStages;
  return st >= 2 ? st : 0;
}

// hi = x with the 13 low mantissa bits cleared (an exact TF32 value),
// lo = x - hi (exact in FP32).
__device__ __forceinline__ void split_tf32(const float4 x, float4& hi, float4& lo) {
  hi.x = __uint_as_float(__float_as_uint(x.x) & 0xFFFFE000u);
  hi.y = __uint_as_float(__float_as_uint(x.y) & 0xFFFFE000u);
  hi.z = __uint_as_float(__float_as_uint(x.z) & 0xFFFFE000u);
  hi.w = __uint_as_float(__float_as_uint(x.w) & 0xFFFFE000u);
  lo = make_float4(x.x - hi.x, x.y - hi.y, x.z - hi.z, x.w - hi.w);
}
// Orders this thread's generic-proxy shared-memory accesses before later
// async-proxy accesses of the same bytes (tensor-core reads of what it wrote,
// TMA writes over what it read).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// tmA2 / tmB2: the low parts of the split-FP16 form (H2; unused otherwise).
template <bool X3, bool H2 = false>
__global__ void __launch_bounds__(Form<X3, H2>::kThreads, 1)
cdist_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                const __grid_constant__ CUtensorMap tmB,
                const __grid_constant__ CUtensorMap tmA2,
                const __grid_constant__ CUtensorMap tmB2, const Params p,
                const uint32_t idesc, const uint32_t idesc2) {
  using Fm = Form<X3, H2>;
  constexpr int MU = Fm::kMult;
  constexpr int CH = Fm::kChunk;
  constexpr int SB = Fm::kStageBytes;
  const int ST = p.stages;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = base;
  unsigned char* sSlot = sA + (size_t)ST * SB;  // X3 only
  unsigned char* sB = sSlot + Fm::kSlotBytes;
  const size_t bbytes = (size_t)p.KT * p.NT * 128;  // bytes TMA loads
  const size_t bchunk = (size_t)MU * p.NT * 128;    // smem per B chunk
  const int accw = MU * p.NT;                       // accumulator columns
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + bbytes * MU);
  uint64_t* full = bars;            // raw tile landed
  uint64_t* empty = bars + ST;      // raw stage free (f16: MMAs retired;
                                    // X3: converters read it)
  uint64_t* conv = bars + 2 * ST;   // X3: slot split, ready for the MMA
  uint64_t* mfree = conv + kSlots;  // X3: slot's MMAs retired
  uint64_t* bfull = mfree + kSlots;
  uint64_t* bconv = bfull + 1;      // X3: source tile split
  uint64_t* accf = bconv + 1;
  uint64_t* acce = accf + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acce + 2);
  float* nS_s = reinterpret_cast<float*>(tmem_slot + 4);
  float* ss_s = nS_s + p.NT;  // H2: source row scales

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  grid_dep_launch();
  // This CTA's N-tile: its first stacked source row (TMA, norms, near-pair
  // ids), its first panel column, and the panel it writes.
  int n0 = blockIdx.y * p.NT, col0 = n0, vr = 0, ldk = p.ld;
  float* Kt = p.K;
  float* mrowt = p.mrow;
  const int ntiles = (int)((p.V + BM - 1) / BM);

  if (threadIdx.x == 0) {
    for (int s = 0; s < ST; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], X3 ? 128 : 1);
    }
    for (int m = 0; m < kSlots; ++m) {
      mbar_init(&conv[m], 128);
      mbar_init(&mfree[m], 1);
    }
    mbar_init(bfull, 1);
    mbar_init(bconv, 128);
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 8 * 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            smem_u32(tmem_slot)),
        "r"((uint32_t)p.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // Everything above touches only this CTA's shared and tensor memory; the
  // source rows, their norms and v_r come from the selection before it.
  grid_dep_wait();
  if (p.tiles) {
    const int4 tl = p.tiles[blockIdx.y];
    const GroupSrc& gs = p.grp[tl.x];
    n0 = tl.y;
    col0 = tl.z;
    vr = gs.vr;
    ldk = gs.ld;
    Kt = gs.K;
    mrowt = gs.mrow;
  } else {
    vr = (int)*p.vr;
  }
  for (int c = threadIdx.x; c < p.NT; c += blockDim.x) {
    nS_s[c] = col0 + c < vr ? p.nS[n0 + c] : 0.f;
    if constexpr (H2) ss_s[c] = col0 + c < vr ? p.ssc[(size_t)(n0 + c) * p.sc_stride] : 0.f;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (col0 < vr) {
    if (warp == 0) {
      if (lane == 0) {
        // ---- TMA producer ----
        mbar_expect_tx(bfull, (uint32_t)(bbytes * (H2 ? 2 : 1)));
        for (int q = 0; q < p.KT; ++q) {
          tma_load_2d(sB + (size_t)q * bchunk, &tmB, bfull, q * CH, n0);
          if constexpr (H2)
            tma_load_2d(sB + (size_t)q * bchunk + (size_t)p.NT * 128, &tmB2, bfull, q * CH, n0);
        }
        uint32_t it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
          for (int q = 0; q < p.KT; ++q, ++it) {
            const uint32_t s = it % ST, ph = (it / ST) & 1u;
            if (!mbar_wait(&empty[s], ph ^ 1u, p.err)) {
              ok = false;
              break;
            }
            mbar_expect_tx(&full[s], SB);
            tma_load_2d(sA + (size_t)s * SB, &tmA, &full[s], q * CH, tile * BM);
            if constexpr (H2)
              tma_load_2d(sA + (size_t)s * SB + kTileBytesA, &tmA2, &full[s], q * CH,
                          tile * BM);
          }
        }
      }
    } else if (warp == 1) {
      if (lane == 0) {
        // ---- MMA issuer ----
        bool ok = mbar_wait(X3 ? bconv : bfull, 0, p.err);
        uint32_t it = 0, t = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++t) {
          const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
          if (!mbar_wait(&acce[b], tph ^ 1u, p.err)) break;
          fence_after();
          const uint32_t dt = tmem + b * (uint32_t)accw;
          for (int q = 0; q < p.KT; ++q, ++it) {
            const uint32_t b0 = smem_u32(sB + (size_t)q * bchunk);
            if constexpr (X3) {
              const uint32_t m = it % kSlots, ph = (it / kSlots) & 1u;
              if (!mbar_wait(&conv[m], ph, p.err)) {
                ok = false;
                break;
              }
              fence_after();
              const uint32_t ah0 = smem_u32(sSlot + (size_t)m * 2 * kTileBytesA);
              const uint32_t al0 = ah0 + kTileBytesA;
              // Columns [0, NT) accumulate hi.hi + lo.hi, columns [NT, 2 NT)
              // hi.lo: one N = 2 NT product of the high tile with the stacked
              // source [hi | lo], one N = NT product of the low tile with hi.
#pragma unroll
              for (int kk = 0; kk < 4; ++kk) {
                const uint64_t bd = sw128_desc(b0 + kk * 32);
                mma_tf32(dt, sw128_desc(ah0 + kk * 32), bd, idesc2,
                         (q > 0 || kk > 0) ? 1u : 0u);
                mma_tf32(dt, sw128_desc(al0 + kk * 32), bd, idesc, 1u);
              }
              mma_commit(&mfree[m]);  // slot free once these MMAs retire
            } else {
              const uint32_t s = it % ST, ph = (it / ST) & 1u;
              if (!mbar_wait(&full[s], ph, p.err)) {
                ok = false;
                break;
              }
              fence_after();
              const uint32_t a0 = smem_u32(sA + (size_t)s * SB);
              if constexpr (H2) {
                // Columns [0, NT) accumulate hi.hi, columns [NT, 2 NT) the
                // cross terms (both scaled by 2^11): hi.[hi | lo'] as one
                // N = 2 NT product, then lo'.hi into the second half.
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                  const uint64_t bd = sw128_desc(b0 + kk * 32);
                  mma_f16(dt, sw128_desc(a0 + kk * 32), bd, idesc2,
                          (q > 0 || kk > 0) ? 1u : 0u);
                  mma_f16(dt + (uint32_t)p.NT, sw128_desc(a0 + kTileBytesA + kk * 32), bd,
                          idesc, 1u);
                }
              } else {
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                  mma_f16(dt, sw128_desc(a0 + kk * 32), sw128_desc(b0 + kk * 32),
                          idesc, (q > 0 || kk > 0) ? 1u : 0u);
              }
              mma_commit(&empty[s]);  // stage free once these MMAs retire
            }
          }
          if (!ok) break;
          mma_commit(&accf[b]);     // accumulator b ready for the epilogue
        }
      }
    } else if (X3 && warp >= 10) {
      // ---- converters: warps 10..13 split each landed FP32 tile into its
      // TF32 high part and the FP32 remainder in a free slot, release the raw
      // stage to the producer at once, then hand the slot to the MMA issuer.
      // The source tile is split first (in place).
      const int c = threadIdx.x - 320;
      bool ok = mbar_wait(bfull, 0, p.err);
      if (ok) {
        const int per = p.NT * 8;  // float4 per chunk of NT rows
        const int nb = p.KT * per;
        for (int k = c; k < nb; k += 128) {
          float4* bh = reinterpret_cast<float4*>(sB + (size_t)(k / per) * bchunk) + k % per;
          float4 h, l;
          split_tf32(*bh, h, l);
          bh[0] = h;
          bh[per] = l;
        }
        fence_proxy_async_smem();
        mbar_arrive(bconv);
      }
      uint32_t it = 0;
      for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        for (int q = 0; q < p.KT; ++q, ++it) {
          const uint32_t s = it % ST, ph = (it / ST) & 1u;
          const uint32_t m = it % kSlots, mph = (it / kSlots) & 1u;
          if (!mbar_wait(&full[s], ph, p.err)) {
            ok = false;
            break;
          }
          constexpr int kPer = kTileBytesA / 16 / 128;  // float4 per thread
          const float4* raw = reinterpret_cast<const float4*>(sA + (size_t)s * SB);
          float4 x[kPer];
#pragma unroll
          for (int k = 0; k < kPer; ++k) x[k] = raw[c + 128 * k];
          // Release the raw stage to the producer at once.  Its next TMA
          // write (async proxy) must be ordered after these generic-proxy
          // reads: without the proxy fence the refill was seen to overtake
          // them (wrong low parts, run-to-run varying results).
          fence_proxy_async_smem();
          mbar_arrive(&empty[s]);
          if (!mbar_wait(&mfree[m], mph ^ 1u, p.err)) {
            ok = false;
            break;
          }
          float4* hi = reinterpret_cast<float4*>(sSlot + (size_t)m * 2 * kTileBytesA);
          float4* lo = hi + kTileBytesA / 16;
#pragma unroll
          for (int k = 0; k < kPer; ++k) {
            float4 h, l;
            split_tf32(x[k], h, l);
            hi[c + 128 * k] = h;
            lo[c + 128 * k] = l;
          }
          fence_proxy_async_smem();
          mbar_arrive(&conv[m]);
        }
      }
    } else {
      // ---- epilogue: warps 2..9.  A warp may only access its TMEM lane
      // quarter (warp % 4); the two warps of a quarter split the columns in
      // 16-column chunks.  One tile row per thread.
      const int quarter = warp & 3;
      const int half = (warp - 2) >> 2;
      const int row = quarter * 32 + lane;
      uint32_t t = 0;
      for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++t) {
        const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
        const uint64_t w = (uint64_t)tile * BM + row;
        const bool wok = w < p.V;
        const float ne = wok ? p.nE[w] : 0.f;  // issued before the wait
        const float sw = H2 && wok ? p.esc[w * (uint64_t)p.sc_stride] : 1.f;
        float mmin = __int_as_float(0x7f7f7f7f);  // row-scaled form
        if (!mbar_wait(&accf[b], tph, p.err)) break;
        fence_after();
        for (int c0 = 16 * half; c0 < p.NT; c0 += 32) {
          float acc[16];
          const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + b * accw + c0;
          tmem_ld16(ta, acc);
          if constexpr (X3) {
            float acc2[16];
            tmem_ld16(ta + p.NT, acc2);
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[j] += acc2[j];
          } else if constexpr (H2) {
            float acc2[16];
            tmem_ld16(ta + p.NT, acc2);
#pragma unroll
            for (int j = 0; j < 16; ++j)
              acc[j] = fmaf(acc2[j], 0x1p-11f, acc[j]) * (sw * ss_s[c0 + j]);
          }
          if (!wok) continue;
          // Straight-line over the 16 entries (no branch inside), so their
          // sqrt / exp latency chains interleave; the cancellation-prone
          // pairs are collected as a bitmask and listed afterwards, and the
          // columns past v_r are zeroed last.
          float kv[16], kmv[16];
          unsigned nearmask = 0;
          const int nval = vr - (col0 + c0);  // valid columns of this chunk
          if (mrowt) {
            // Row-scaled form: M now (and the row minimum), K' after the
            // near-pair fix-up (panel_rescale.cu).
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const float ns = nS_s[c0 + j];
              const float m2 = fmaxf(ne + ns - 2.f * acc[j], 0.f);
              nearmask |= (m2 < near_threshold(ne, ns) ? 1u : 0u) << j;
              const float m = sqrtf(m2);
              kv[j] = m;
              kmv[j] = 0.f;
              if (j < nval) mmin = fminf(mmin, m);
            }
          } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const float ns = nS_s[c0 + j];
              const float m2 = fmaxf(ne + ns - 2.f * acc[j], 0.f);
              nearmask |= (m2 < near_threshold(ne, ns) ? 1u : 0u) << j;
              const float m = sqrtf(m2);
              const float kx = expf(p.expo * m);
              kv[j] = kx;
              kmv[j] = kx * m;
            }
          }
          if (nval < 16) {
#pragma unroll
            for (int j = 0; j < 16; ++j)
              if (j >= nval) {
                kv[j] = 0.f;
                kmv[j] = 0.f;
              }
            nearmask &= nval <= 0 ? 0u : (1u << nval) - 1u;
          }
          while (nearmask) {
            const int j = __ffs(nearmask) - 1;
            nearmask &= nearmask - 1u;
            near_pair(p.near, w, n0 + c0 + j);
          }
          float* krow = Kt + w * (uint64_t)ldk;
          float* kmrow = p.KM + w * (uint64_t)ldk;
#pragma unroll
          for (int j4 = 0; j4 < 4; ++j4) {
            const int c = col0 + c0 + 4 * j4;
            if (c < ldk) {
              *reinterpret_cast<float4*>(krow + c) = make_float4(
                  kv[4 * j4], kv[4 * j4 + 1], kv[4 * j4 + 2], kv[4 * j4 + 3]);
              if (p.KM && !mrowt)
                *reinterpret_cast<float4*>(kmrow + c) = make_float4(
                    kmv[4 * j4], kmv[4 * j4 + 1], kmv[4 * j4 + 2], kmv[4 * j4 + 3]);
            }
          }
        }
        if (mrowt && wok && mmin < __int_as_float(0x7f7f7f7f))
          atomicMin(reinterpret_cast<int*>(mrowt + w), __float_as_int(mmin));
        fence_before();
        mbar_arrive(&acce[b]);
      }
    }
  } else if (warp >= 2 && warp < 6) {
    // Pure padding tile (no source word in it): zero the panel columns.
    const int quarter = warp & 3;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      const uint64_t w = (uint64_t)tile * BM + quarter * 32 + lane;
      if (w >= p.V) continue;
      for (int c = col0; c < col0 + p.NT && c < ldk; c += 4) {
        *reinterpret_cast<float4*>(Kt + w * (uint64_t)ldk + c) = make_float4(0.f, 0.f, 0.f, 0.f);
        if (p.KM)
          *reinterpret_cast<float4*>(p.KM + w * (uint64_t)p.ld + c) = make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
  }

  fence_before();
  __syncthreads();
  fence_after();
  if (warp == 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)p.tmem_cols));
  }
}

// FP32 [V][d] -> 16-bit [V][dp] with zero padding (dp = d rounded up to 8, so
// every row starts on a 16-byte boundary as TMA requires).
template <class T>
__global__ void to16_kernel(const float* __restrict__ src, uint64_t rows, int d,
                            int dp, T* __restrict__ dst) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = rows * (uint64_t)dp;
  if (idx >= total) return;
  const uint64_t r = idx / dp;
  const int k = (int)(idx % dp);
  const float v = k < d ? src[r * d + k] : 0.f;
  if constexpr (sizeof(T) == 2 && std::is_same<T, __nv_bfloat16>::value)
    dst[idx] = __float2bfloat16_rn(v);
  else
    dst[idx] = __float2half_rn(v);
}

// FP32 [V][d] -> split-FP16 rows of the F16X3 panel, one warp per row.
// Row w is scaled by s = 2^(14 - e), e the binary exponent of max_k |E_wk|
// (max < 2^e), so the largest scaled entry lies in [2^13, 2^14); then
//   hi = fp16(x s),  lo = fp16((x s - hi) 2^11)      (x s - hi is exact)
// and the row is stored as [hi: dp halves][lo: dp halves][1/s: FP32][pad to
// 16 bytes], 4 dp + 16 bytes.  hi + 2^-11 lo carries 22 significant bits of
// x s (the scaled remainder keeps lo clear of FP16's subnormal range), so
// hi.hi + 2^-11 (hi.lo + lo.hi) is a dot product to about FP32 accuracy,
// like the split-TF32 form.  A row of zeros keeps s = 1.
__global__ void to_split16_kernel(const float* __restrict__ src, uint64_t rows, int d,
                                  int dp, unsigned char* __restrict__ dst) {
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= rows) return;
  const float* e = src + w * (uint64_t)d;
  float m = 0.f;
  for (int k = lane; k < d; k += 32) m = fmaxf(m, fabsf(e[k]));
#pragma unroll
  for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  int ex = 0;
  if (m > 0.f) frexpf(m, &ex);
  const int sh = max(-126, min(126, 14 - ex));
  const float sc = ldexpf(1.f, sh);
  __half* hrow = reinterpret_cast<__half*>(dst + w * (uint64_t)(4 * dp + 16));
  __half* lrow = hrow + dp;
  for (int k = lane; k < dp; k += 32) {
    const float x = k < d ? e[k] * sc : 0.f;
    const __half h = __float2half_rn(x);
    hrow[k] = h;
    lrow[k] = __float2half_rn((x - __half2float(h)) * 2048.f);
  }
  if (lane < 4) {
    float* tail = reinterpret_cast<float*>(lrow + dp);
    tail[lane] = lane == 0 ? ldexpf(1.f, -sh) : 0.f;
  }
}

}  // namespace tc

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
namespace {
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                                  void*, const cuuint64_t*, const cuuint64_t*,
                                  const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault,
                                &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// stride: bytes between rows (0: dense rows of inner elements).
bool make_map(CUtensorMap* tm, const void* ptr, CUtensorMapDataType dt,
              int esize, uint64_t inner, uint64_t rows, uint32_t box_inner,
              uint32_t box_rows, uint64_t stride = 0) {
  EncodeTiledFn f = encode_fn();
  if (!f) return false;
  const cuuint64_t gdim[2] = {inner, rows};
  const cuuint64_t gstride[1] = {stride ? stride : inner * (uint64_t)esize};
  const cuuint32_t box[2] = {box_inner, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return f(tm, dt, 2, const_cast<void*>(ptr), gdim, gstride, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool X3, bool H2 = false>
void set_smem_attr() {
  static bool done[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !done[dev]) {
    cudaFuncSetAttribute(tc::cdist_tc_kernel<X3, H2>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    done[dev] = true;
  }
}
}  // namespace

int tc_padded_width(uint64_t d) { return (int)((d + 7) & ~7ull); }

namespace {
constexpr size_t kSmemBudget = 227 * 1024;
constexpr int kMinStages = 3;
}  // namespace

int tc_tile_n(uint32_t cap, uint64_t d) {
  const int KT = (int)((tc_padded_width(d) + tc::BK - 1) / tc::BK);
  int nt = (int)(((cap ? cap : 1) + 15) & ~15u);
  if (nt > 128) nt = 128;
  while (nt > 16 && tc::ring_stages<false>(nt, KT, kSmemBudget) < kMinStages) nt -= 16;
  if (tc::ring_stages<false>(nt, KT, kSmemBudget) < kMinStages) return 0;
  return nt;
}

int tc_tile_n_x3(uint32_t cap, uint64_t d) {
  // The FP32 rows are read by TMA in place: their byte stride (4d) must be a
  // multiple of 16.
  if (d == 0 || d % 4 != 0) return 0;
  const int KT = (int)((d + 31) / 32);
  int nt = cap <= 16 ? 16 : 32;
  while (nt > 16 && tc::ring_stages<true>(nt, KT, kSmemBudget) < kMinStages) nt -= 16;
  if (tc::ring_stages<true>(nt, KT, kSmemBudget) < kMinStages) return 0;
  return nt;
}

int tc_tile_n_h2(uint32_t cap, uint64_t d) {
  const int KT = (int)((tc_padded_width(d) + tc::BK - 1) / tc::BK);
  int nt = (int)(((cap ? cap : 1) + 15) & ~15u);
  if (nt > 64) nt = 64;
  while (nt > 16 && tc::ring_stages<false, true>(nt, KT, kSmemBudget) < kMinStages) nt -= 16;
  if (tc::ring_stages<false, true>(nt, KT, kSmemBudget) < kMinStages) return 0;
  return nt;
}

size_t tc_split_row_bytes(uint64_t d) { return 4 * (size_t)tc_padded_width(d) + 16; }

int launch_to_split16(const float* E32, uint64_t rows, uint64_t d, void* Esplit,
                      cudaStream_t st) {
  if (rows == 0) return 0;
  const int threads = 256;
  const unsigned blocks = (unsigned)((rows * 32 + threads - 1) / threads);
  tc::to_split16_kernel<<<blocks, threads, 0, st>>>(E32, rows, (int)d, tc_padded_width(d),
                                                     static_cast<unsigned char*>(Esplit));
  return 1;
}

int launch_to16(const float* E32, uint64_t rows, uint64_t d, void* E16,
                bool bf16, cudaStream_t st) {
  const int dp = tc_padded_width(d);
  const uint64_t total = rows * (uint64_t)dp;
  const int threads = 256;
  const unsigned blocks = (unsigned)((total + threads - 1) / threads);
  if (bf16)
    tc::to16_kernel<__nv_bfloat16><<<blocks, threads, 0, st>>>(
        E32, rows, (int)d, dp, static_cast<__nv_bfloat16*>(E16));
  else
    tc::to16_kernel<__half><<<blocks, threads, 0, st>>>(
        E32, rows, (int)d, dp, static_cast<__half*>(E16));
  return 1;
}

// Returns launches issued, or -1 when the form is unsupported for this
// width or the tensor maps cannot be built.
int launch_cdist_tc(int form, const void* E16, const void* S16,
                    const float* E32, const float* nE, uint64_t V, uint64_t d,
                    const SourceSel& s, float expo, float* K, float* KM, int ld,
                    const NearList& near, unsigned* err, int num_sms,
                    cudaStream_t st, float* mrow, const StackedPanels* grp) {
  const bool x3 = form == TC_TF32X3;
  const bool h2 = form == TC_F16X3;
  // stacked group: s.cap is the number of stacked source rows
  const uint64_t rows_b = s.cap ? s.cap : 1;
  int NT, KT;
  CUtensorMap tmA, tmB, tmA2, tmB2;
  memset(&tmA2, 0, sizeof(tmA2));
  memset(&tmB2, 0, sizeof(tmB2));
  const int dps = tc_padded_width(d);
  const uint64_t rs = tc_split_row_bytes(d);
  if (h2) {
    if (grp) return -1;  // single-source panels only
    NT = tc_tile_n_h2(s.cap, d);
    if (NT == 0) return -1;
    KT = (dps + tc::BK - 1) / tc::BK;
    // High and low halves of the split rows (row stride rs): two maps per
    // operand over the same rows; columns past dp read as zeros.
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const unsigned char* e = static_cast<const unsigned char*>(E16);
    const unsigned char* sp = static_cast<const unsigned char*>(S16);
    if (!make_map(&tmA, e, dt, 2, (uint64_t)dps, V, tc::BK, tc::BM, rs) ||
        !make_map(&tmA2, e + 2 * dps, dt, 2, (uint64_t)dps, V, tc::BK, tc::BM, rs) ||
        !make_map(&tmB, sp, dt, 2, (uint64_t)dps, rows_b, tc::BK, (uint32_t)NT, rs) ||
        !make_map(&tmB2, sp + 2 * dps, dt, 2, (uint64_t)dps, rows_b, tc::BK, (uint32_t)NT, rs))
      return -1;
  } else if (x3) {
    NT = grp ? grp->nt : tc_tile_n_x3(s.cap, d);
    if (NT == 0) return -1;
    KT = (int)((d + 31) / 32);
    // FP32 rows in place, 32-float (128-byte) chunks; the last chunk's
    // columns past d and the source rows past cap read as zeros.
    if (!make_map(&tmA, E32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, d, V, 32, tc::BM))
      return -1;
    if (!make_map(&tmB, s.S, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, d, rows_b, 32,
                  (uint32_t)NT))
      return -1;
  } else {
    const int dp = tc_padded_width(d);
    NT = grp ? grp->nt : tc_tile_n(s.cap, d);
    if (NT == 0) return -1;
    KT = (dp + tc::BK - 1) / tc::BK;
    const CUtensorMapDataType dt = form == TC_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    if (!make_map(&tmA, E16, dt, 2, (uint64_t)dp, V, tc::BK, tc::BM)) return -1;
    // Rows past the allocated cap read as zeros (TMA out-of-bounds fill).
    if (!make_map(&tmB, S16, dt, 2, (uint64_t)dp, rows_b, tc::BK, (uint32_t)NT))
      return -1;
  }
  const int ntn = grp ? grp->ntiles : (ld + NT - 1) / NT;
  tc::Params p;
  p.tiles = grp ? grp->tiles : nullptr;
  p.grp = grp ? grp->src : nullptr;
  p.esc = h2 ? reinterpret_cast<const float*>(static_cast<const unsigned char*>(E16) + 4 * dps)
             : nullptr;
  p.ssc = h2 ? reinterpret_cast<const float*>(static_cast<const unsigned char*>(S16) + 4 * dps)
             : nullptr;
  p.sc_stride = (int)(rs / 4);
  p.E32 = E32;
  p.nE = nE;
  p.S32 = s.S;
  p.nS = s.nS;
  p.vr = s.vr;
  p.K = K;
  p.KM = KM;
  p.near = near;
  p.mrow = mrow;
  p.err = err;
  p.V = V;
  p.d = (int)d;
  p.ld = ld;
  p.NT = NT;
  p.KT = KT;
  int cols = 32;
  while (cols < (x3 || h2 ? 4 : 2) * NT) cols <<= 1;  // two accumulators
  p.tmem_cols = cols;
  p.expo = expo;
  p.stages = x3   ? tc::ring_stages<true>(NT, KT, kSmemBudget)
             : h2 ? tc::ring_stages<false, true>(NT, KT, kSmemBudget)
                  : tc::ring_stages<false>(NT, KT, kSmemBudget);
  if (p.stages < kMinStages) return -1;
  const int ntiles = (int)((V + tc::BM - 1) / tc::BM);
  int gx = num_sms / ntn;
  if (gx < 1) gx = 1;
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)ntn);
  constexpr int BM_ROWS = tc::BM;
  if (x3) {
    set_smem_attr<true>();
    const uint32_t idesc = tc::make_idesc(2, BM_ROWS, NT);
    const uint32_t idesc2 = tc::make_idesc(2, BM_ROWS, 2 * NT);
    launch_pdl(tc::cdist_tc_kernel<true>, grid, dim3(tc::Form<true>::kThreads),
               tc::smem_bytes<true>(NT, KT, p.stages), st, tmA, tmB, tmA2, tmB2, p, idesc,
               idesc2);
  } else if (h2) {
    set_smem_attr<false, true>();
    const uint32_t idesc = tc::make_idesc(0, BM_ROWS, NT);
    const uint32_t idesc2 = tc::make_idesc(0, BM_ROWS, 2 * NT);
    launch_pdl(tc::cdist_tc_kernel<false, true>, grid, dim3(tc::Form<false, true>::kThreads),
               tc::smem_bytes<false, true>(NT, KT, p.stages), st, tmA, tmB, tmA2, tmB2, p,
               idesc, idesc2);
  } else {
    set_smem_attr<false>();
    const uint32_t idesc = tc::make_idesc(form == TC_BF16 ? 1 : 0, BM_ROWS, NT);
    launch_pdl(tc::cdist_tc_kernel<false>, grid, dim3(tc::Form<false>::kThreads),
               tc::smem_bytes<false>(NT, KT, p.stages), st, tmA, tmB, tmA2, tmB2, p, idesc,
               idesc);
  }
  return 1;
}

}  // namespace wmd
