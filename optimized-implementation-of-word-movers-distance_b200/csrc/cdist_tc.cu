// Tensor-core cost panel (tcgen05, sm_100a).
//
// Same output as cdist_fp32.cu — K[w,i] = exp(expo * M[w,i]) and
// KM = K * M in the word-major [V][ld] layout of the reference's fused solver
// (sinkhorn_wmd_fused.cpp:197-223) — but the dot products E_w . S_i run on
// the 5th-generation tensor cores with 16-bit operands (BF16 or FP16) and FP32
// accumulation in tensor memory:
//
//   warp 0      TMA producer: the source tile S (all K-chunks) once, then a
//               6-stage ring of 128-row x 64-element vocabulary tiles
//               (128-byte swizzle), one mbarrier per stage;
//   warp 1      allocates TMEM; one thread issues tcgen05.mma
//               (M=128, N=NT, K=16) into a double-buffered FP32 accumulator
//               and tcgen05.commit's stage-release / accumulator-ready
//               barriers;
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
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tcgen05.cuh"
#include "wmd_internal.cuh"

namespace wmd {
namespace tc {

constexpr int BM = 128;          // vocabulary rows per tile (UMMA M)
constexpr int BK = 64;           // 16-bit elements per 128-byte swizzle row
constexpr int UK = 16;           // UMMA K per instruction
constexpr int STAGES = 6;        // A-tile ring depth
constexpr int kThreads = 320;    // 10 warps: producer, MMA, 8 epilogue
constexpr int kTileBytesA = BM * BK * 2;  // 16 KB

struct Params {
  const float* E32;   // [V][d]
  const float* nE;    // [V]
  const float* S32;   // [cap][d]
  const float* nS;    // [cap]
  const uint32_t* vr; // device v_r
  float* K;           // [V][ld]
  float* KM;          // [V][ld] or null (then K*M is not stored)
  NearList near;      // cancellation-prone pairs for the exact fix-up pass
  unsigned* err;
  uint64_t V;
  int d, ld, NT, KT, tmem_cols;
  float expo;
};

// Dynamic shared memory layout (base rounded up to 1024 bytes):
//   A ring   STAGES x 16 KB
//   B        KT x NT x 128 B
//   barriers full[STAGES], empty[STAGES], bfull, accf[2], acce[2]
//   tmem address slot, nS copy [NT]
__host__ __device__ inline size_t smem_bytes(int NT, int KT) {
  return 1024 + (size_t)STAGES * kTileBytesA + (size_t)KT * NT * 128 +
         (2 * STAGES + 5) * 8 + 16 + (size_t)NT * 4;
}

__global__ void __launch_bounds__(kThreads, 1)
cdist_tc_kernel(const __grid_constant__ CUtensorMap tmA,
                const __grid_constant__ CUtensorMap tmB, const Params p,
                const uint32_t idesc) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = base;
  unsigned char* sB = sA + (size_t)STAGES * kTileBytesA;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + (size_t)p.KT * p.NT * 128);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* bfull = bars + 2 * STAGES;
  uint64_t* accf = bfull + 1;
  uint64_t* acce = accf + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acce + 2);
  float* nS_s = reinterpret_cast<float*>(tmem_slot + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n0 = blockIdx.y * p.NT;
  const int vr = (int)*p.vr;
  const int ntiles = (int)((p.V + BM - 1) / BM);

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(bfull, 1);
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
  for (int c = threadIdx.x; c < p.NT; c += blockDim.x) {
    const int i = n0 + c;
    nS_s[c] = i < vr ? p.nS[i] : 0.f;
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (n0 < vr) {
    if (warp == 0) {
      if (lane == 0) {
        // ---- TMA producer ----
        mbar_expect_tx(bfull, (uint32_t)(p.KT * p.NT * 128));
        for (int q = 0; q < p.KT; ++q)
          tma_load_2d(sB + (size_t)q * p.NT * 128, &tmB, bfull, q * BK, n0);
        uint32_t it = 0;
        bool ok = true;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
          for (int q = 0; q < p.KT; ++q, ++it) {
            const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
            if (!mbar_wait(&empty[s], ph ^ 1u, p.err)) {
              ok = false;
              break;
            }
            mbar_expect_tx(&full[s], kTileBytesA);
            tma_load_2d(sA + (size_t)s * kTileBytesA, &tmA, &full[s], q * BK,
                        tile * BM);
          }
        }
      }
    } else if (warp == 1) {
      if (lane == 0) {
        // ---- MMA issuer ----
        bool ok = mbar_wait(bfull, 0, p.err);
        uint32_t it = 0, t = 0;
        for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++t) {
          const uint32_t b = t & 1u, tph = (t >> 1) & 1u;
          if (!mbar_wait(&acce[b], tph ^ 1u, p.err)) break;
          fence_after();
          const uint32_t dt = tmem + b * (uint32_t)p.NT;
          for (int q = 0; q < p.KT; ++q, ++it) {
            const uint32_t s = it % STAGES, ph = (it / STAGES) & 1u;
            if (!mbar_wait(&full[s], ph, p.err)) {
              ok = false;
              break;
            }
            fence_after();
            const uint32_t a0 = smem_u32(sA + (size_t)s * kTileBytesA);
            const uint32_t b0 = smem_u32(sB + (size_t)q * p.NT * 128);
#pragma unroll
            for (int kk = 0; kk < BK / UK; ++kk)
              mma_f16(dt, sw128_desc(a0 + kk * UK * 2), sw128_desc(b0 + kk * UK * 2),
                      idesc, (q > 0 || kk > 0) ? 1u : 0u);
            mma_commit(&empty[s]);  // stage free once these MMAs retire
          }
          if (!ok) break;
          mma_commit(&accf[b]);     // accumulator b ready for the epilogue
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
        if (!mbar_wait(&accf[b], tph, p.err)) break;
        fence_after();
        for (int c0 = 16 * half; c0 < p.NT; c0 += 32) {
          float acc[16];
          tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + b * p.NT + c0, acc);
          if (!wok) continue;
          float kv[16], kmv[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int i = n0 + c0 + j;
            kv[j] = 0.f;
            kmv[j] = 0.f;
            if (i < vr) {
              const float ns = nS_s[c0 + j];
              const float m2 = fmaxf(ne + ns - 2.f * acc[j], 0.f);
              if (m2 < near_threshold(ne, ns)) near_pair(p.near, w, i);
              const float m = sqrtf(m2);
              const float kx = expf(p.expo * m);
              kv[j] = kx;
              kmv[j] = kx * m;
            }
          }
          float* krow = p.K + w * (uint64_t)p.ld;
          float* kmrow = p.KM + w * (uint64_t)p.ld;
#pragma unroll
          for (int j4 = 0; j4 < 4; ++j4) {
            const int c = n0 + c0 + 4 * j4;
            if (c < p.ld) {
              *reinterpret_cast<float4*>(krow + c) = make_float4(
                  kv[4 * j4], kv[4 * j4 + 1], kv[4 * j4 + 2], kv[4 * j4 + 3]);
              if (p.KM)
                *reinterpret_cast<float4*>(kmrow + c) = make_float4(
                    kmv[4 * j4], kmv[4 * j4 + 1], kmv[4 * j4 + 2], kmv[4 * j4 + 3]);
            }
          }
        }
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
      for (int c = n0; c < n0 + p.NT && c < p.ld; c += 4) {
        *reinterpret_cast<float4*>(p.K + w * (uint64_t)p.ld + c) = make_float4(0.f, 0.f, 0.f, 0.f);
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

bool make_map(CUtensorMap* tm, const void* ptr, bool bf16, uint64_t inner,
              uint64_t rows, uint32_t box_rows) {
  EncodeTiledFn f = encode_fn();
  if (!f) return false;
  const cuuint64_t gdim[2] = {inner, rows};
  const cuuint64_t gstride[1] = {inner * 2};
  const cuuint32_t box[2] = {(cuuint32_t)tc::BK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return f(tm,
           bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
           2, const_cast<void*>(ptr), gdim, gstride, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

int tc_padded_width(uint64_t d) { return (int)((d + 7) & ~7ull); }

int tc_tile_n(uint32_t cap, uint64_t d) {
  const int KT = (int)((tc_padded_width(d) + tc::BK - 1) / tc::BK);
  int nt = (int)(((cap ? cap : 1) + 15) & ~15u);
  if (nt > 128) nt = 128;
  while (nt > 16 && tc::smem_bytes(nt, KT) > 227 * 1024) nt -= 16;
  if (tc::smem_bytes(nt, KT) > 227 * 1024) return 0;
  return nt;
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

// Returns launches issued, or -1 when the tensor maps cannot be built.
int launch_cdist_tc(const void* E16, const void* S16, bool bf16,
                    const float* E32, const float* nE, uint64_t V, uint64_t d,
                    const SourceSel& s, float expo, float* K, float* KM, int ld,
                    const NearList& near, unsigned* err, int num_sms,
                    cudaStream_t st) {
  const int dp = tc_padded_width(d);
  const int KT = (dp + tc::BK - 1) / tc::BK;
  const int NT = tc_tile_n(s.cap, d);
  if (NT == 0) return -1;
  const int ntn = (ld + NT - 1) / NT;
  CUtensorMap tmA, tmB;
  if (!make_map(&tmA, E16, bf16, (uint64_t)dp, V, tc::BM)) return -1;
  // Rows past the allocated cap read as zeros (TMA out-of-bounds fill).
  if (!make_map(&tmB, S16, bf16, (uint64_t)dp, (uint64_t)(s.cap ? s.cap : 1),
                (uint32_t)NT))
    return -1;
  tc::Params p;
  p.E32 = E32;
  p.nE = nE;
  p.S32 = s.S;
  p.nS = s.nS;
  p.vr = s.vr;
  p.K = K;
  p.KM = KM;
  p.near = near;
  p.err = err;
  p.V = V;
  p.d = (int)d;
  p.ld = ld;
  p.NT = NT;
  p.KT = KT;
  int cols = 32;
  while (cols < 2 * NT) cols <<= 1;
  p.tmem_cols = cols;
  p.expo = expo;
  const size_t smem = tc::smem_bytes(NT, KT);
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    cudaFuncSetAttribute(tc::cdist_tc_kernel,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    attr_set[dev] = true;
  }
  const int ntiles = (int)((V + tc::BM - 1) / tc::BM);
  int gx = num_sms / ntn;
  if (gx < 1) gx = 1;
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)ntn);
  constexpr int BM_ROWS = tc::BM;
  const uint32_t idesc = tc::make_idesc(bf16 ? 1 : 0, BM_ROWS, NT);
  tc::cdist_tc_kernel<<<grid, tc::kThreads, smem, st>>>(tmA, tmB, p, idesc);
  return 1;
}

}  // namespace wmd
