// Learned warm start: fused inference of the initial scalings (tcgen05).
//
// For every (target document j, source word i) pair the kernel computes the
// MLP prediction y = log u_i and writes u0[j][i] = exp(y), the starting point
// of the solve (solve.cu / solve_block.cu fall back to the cold start per
// document when the prediction's first-update residual is worse).
//
// The first layer is split by feature group, so no feature row is ever
// materialised: with the standardisation folded into W1f, b1f,
//   z1 = A_i + B_j + W_s [min M, mean M, max M]_ij
//   A_i = W1f_E E_i + W1f_r r_i + W1f_lr log r_i + b1f   (per source word)
//   B_j = W1f_C centroid_j                                (per document)
// Only the three M statistics are per pair.  ws_stats_kernel computes them
// first, document-major (one warp per document, lanes over the source words:
// every K row of the document is read once, coalesced), into a [N][v_r][3]
// table that the fused kernel reads in its own pair order.
//
// Per 128-pair tile (pairs in document-major order p = j * v_r + i):
//   warps 1-8  stats + z1 + GELU, written as BF16 straight into shared memory
//              in the 128-byte-swizzled K-major layout the tensor core reads
//              (the tile is the A operand, 128 x 256);
//   warp 0     one thread issues tcgen05.mma kind::f16 (M=128, N=256, K=16 x
//              16) against W2 (BF16, resident in shared memory for the whole
//              kernel) into a 128 x 256 FP32 accumulator in TMEM;
//   warps 1-8  tcgen05.ld the accumulator rows (two warps per TMEM lane
//              quarter, one row per thread, half the columns each), + b2,
//              GELU, dot w3, + b3, exp -> u0.
// Waits are bounded (globaltimer) and set ERR_TIMEOUT.
#include <cuda_bf16.h>

#include "tcgen05.cuh"
#include "wmd_internal.cuh"

namespace wmd {
namespace wsi {

constexpr int H = kWsH;         // 256
constexpr int BM = 128;         // pairs per tile
constexpr int kThreads = 288;   // warp 0 MMA, warps 1-8 producer/epilogue
constexpr int kTileA = BM * H * 2;   // 64 KB
constexpr int kW2 = H * H * 2;       // 128 KB

__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_fast(float z) {
  return 0.5f * z * (1.f + tanh_fast(0.7978845608f * (z + 0.044715f * z * z * z)));
}
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
  const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
  return lo | (hi << 16);
}
// Byte offset of element (row, k) of a [rows][256] BF16 K-major operand
// stored as four 64-column blocks of 128-byte rows with the 128-byte swizzle
// (16-byte chunk index XOR row % 8).  Blocks are rows * 128 bytes apart.
__device__ __forceinline__ uint32_t sw_off(int row, int k, int rows) {
  const int kb = k >> 6, c = (k & 63) >> 3;
  return (uint32_t)(kb * rows * 128 + row * 128 + ((c ^ (row & 7)) << 4) + (k & 7) * 2);
}

struct Params {
  const float* K;        // FP32 cost panel [V][ld]
  const float* mrow;     // row minima of M of a row-scaled panel, or null
  const float* stats;    // [N][vr][3] min / mean / max of M per pair
  int ld;
  float expo;
  const int64_t* col_ptr;
  const uint2* ent;
  const float* Asrc;     // [vr][H]
  const float* Bdoc;     // [N][H]
  const float* Ws;       // [3][H] weights of (min, mean, max) M
  const uint16_t* W2;    // [H][H] BF16, W2[out][in]
  const float* b2;       // [H]
  const float* w3;       // [H]
  const float* b3;       // [1]
  int vr;
  int64_t N;
  float* u0;             // [N][ldu]
  int64_t ldu;
  unsigned* err;
};

__host__ __device__ inline size_t smem_bytes() {
  return 1024 + (size_t)kTileA + kW2 + (size_t)(3 * H + 2 * H) * 4 + 2 * BM * 4 +
         2 * BM * 3 * 4 + 64;
}

__global__ void __launch_bounds__(kThreads, 1) ws_init_kernel(const Params p,
                                                              const uint32_t idesc) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* sA = base;
  unsigned char* sW = sA + kTileA;
  float* sWs = reinterpret_cast<float*>(sW + kW2);  // [3][H]
  float* sb2 = sWs + 3 * H;
  float* sw3 = sb2 + H;
  float* red = sw3 + H;                             // [2][BM]
  float* sst = red + 2 * BM;                        // [2][BM][3] M statistics
  uint64_t* bars = reinterpret_cast<uint64_t*>(sst + 2 * BM * 3);
  uint64_t* full = bars;      // producers -> MMA: A tile written
  uint64_t* done = bars + 1;  // MMA -> producers: accumulator ready, A free
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t total = p.N * (int64_t)p.vr;
  const int64_t ntiles = (total + BM - 1) / BM;

  if (threadIdx.x == 0) {
    tc::mbar_init(full, 8 * 32);
    tc::mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile(
        "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
            tc::smem_u32(tmem_slot)),
        "r"((uint32_t)H));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // W2 -> shared memory, swizzled (16-byte chunks: 256 rows x 32 chunks).
  for (int c = threadIdx.x; c < H * (H / 8); c += blockDim.x) {
    const int n = c / (H / 8), k = (c % (H / 8)) * 8;
    *reinterpret_cast<uint4*>(sW + sw_off(n, k, H)) =
        *reinterpret_cast<const uint4*>(p.W2 + (size_t)n * H + k);
  }
  for (int c = threadIdx.x; c < H; c += blockDim.x) {
    sWs[c] = p.Ws[c];
    sWs[H + c] = p.Ws[H + c];
    sWs[2 * H + c] = p.Ws[2 * H + c];
    sb2[c] = p.b2[c];
    sw3[c] = p.w3[c];
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      uint32_t t = 0;
      for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++t) {
        if (!tc::mbar_wait(full, t & 1u, p.err)) break;
        tc::fence_after();
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sW);
#pragma unroll
        for (int kb = 0; kb < H / 64; ++kb)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            tc::mma_f16(tmem, tc::sw128_desc(a0 + kb * BM * 128 + kk * 32),
                        tc::sw128_desc(b0 + kb * H * 128 + kk * 32), idesc,
                        (kb > 0 || kk > 0) ? 1u : 0u);
        tc::mma_commit(done);
      }
    }
  } else {
    const int quarter = warp & 3;
    const int half = (warp - 1) >> 2;  // warps 1-4: columns 0-127, 5-8: 128-255
    const int row = quarter * 32 + lane;
    const int c0 = half * (H / 2);
    const float b3 = *p.b3;
    uint32_t t = 0;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++t) {
      const int64_t pr = tile * BM + row;
      const bool ok = pr < total;
      const int64_t j = ok ? pr / p.vr : 0;
      const int i = ok ? (int)(pr % p.vr) : 0;
      // M statistics over the document's words: the two threads of a row
      // (one per column half) take alternate words, four independent loads
      // in flight each, and combine through shared memory.
      int n = 0;
      float lo = INFINITY, hi = -INFINITY, sm = 0.f;
      if (ok && p.stats) {
        // precomputed (ws_stats_kernel): half 0 takes the pair's values,
        // half 1 the neutral ones, so the combine below is unchanged
        n = (int)(p.col_ptr[j + 1] - p.col_ptr[j]);
        if (half == 0 && n > 0) {
          const float* st = p.stats + (size_t)pr * 3;
          lo = st[0];
          sm = st[1] * (float)n;
          hi = st[2];
        }
      } else if (ok) {
        const int64_t b = p.col_ptr[j];
        n = (int)(p.col_ptr[j + 1] - b);
        // M = ln K / expo, plus the row's minimum for a row-scaled panel
        auto acc = [&](float kv, uint32_t w) {
          const float Mv = fmaxf(__logf(fmaxf(kv, 1e-38f)) / p.expo, 0.f) +
                           (p.mrow ? __ldg(&p.mrow[w]) : 0.f);
          lo = fminf(lo, Mv);
          hi = fmaxf(hi, Mv);
          sm += Mv;
        };
        int k = half;
        for (; k + 6 < n; k += 8) {
          const uint32_t w0 = p.ent[b + k].x, w1 = p.ent[b + k + 2].x;
          const uint32_t w2 = p.ent[b + k + 4].x, w3 = p.ent[b + k + 6].x;
          const float k0 = p.K[(size_t)w0 * p.ld + i], k1 = p.K[(size_t)w1 * p.ld + i];
          const float k2 = p.K[(size_t)w2 * p.ld + i], k3 = p.K[(size_t)w3 * p.ld + i];
          acc(k0, w0);
          acc(k1, w1);
          acc(k2, w2);
          acc(k3, w3);
        }
        for (; k < n; k += 2) {
          const uint32_t w = p.ent[b + k].x;
          acc(p.K[(size_t)w * p.ld + i], w);
        }
      }
      sst[(half * BM + row) * 3 + 0] = lo;
      sst[(half * BM + row) * 3 + 1] = hi;
      sst[(half * BM + row) * 3 + 2] = sm;
      asm volatile("bar.sync 1, 256;" ::: "memory");
      float mn = 0.f, mean = 0.f, mx = 0.f;
      if (n > 0) {
        const int o = ((half ^ 1) * BM + row) * 3;
        mn = fminf(lo, sst[o]);
        mx = fmaxf(hi, sst[o + 1]);
        mean = (sm + sst[o + 2]) / (float)n;
      }
      // z1 -> GELU -> BF16 A tile (this thread: row `row`, columns c0..c0+127).
      const float* Ar = p.Asrc + (size_t)i * H;
      const float* Br = p.Bdoc + (size_t)j * H;
      for (int k = c0; k < c0 + H / 2; k += 8) {
        float h[8];
#pragma unroll
        for (int e = 0; e < 8; e += 4) {
          const float4 a = *reinterpret_cast<const float4*>(Ar + k + e);
          const float4 bb = *reinterpret_cast<const float4*>(Br + k + e);
          const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {bb.x, bb.y, bb.z, bb.w};
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int n = k + e + q;
            const float z = av[q] + bv[q] + sWs[n] * mn + sWs[H + n] * mean +
                            sWs[2 * H + n] * mx;
            h[e + q] = ok ? gelu_fast(z) : 0.f;
          }
        }
        uint4 v;
        v.x = pack_bf16(h[0], h[1]);
        v.y = pack_bf16(h[2], h[3]);
        v.z = pack_bf16(h[4], h[5]);
        v.w = pack_bf16(h[6], h[7]);
        *reinterpret_cast<uint4*>(sA + sw_off(row, k, BM)) = v;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      tc::mbar_arrive(full);
      // Epilogue: wait for the accumulator, reduce this thread's half row.
      const bool got = tc::mbar_wait(done, t & 1u, p.err);
      // Leave the loop together (the named barriers below need all 256
      // threads): any thread's timed-out wait ends every thread's loop.
      unsigned any_bad;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\tsetp.eq.u32 p, %1, 0;\n\t"
          "bar.red.or.pred q, 1, 256, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
          : "=r"(any_bad)
          : "r"((unsigned)got)
          : "memory");
      if (any_bad) break;
      tc::fence_after();
      float s = 0.f;
      for (int cc = c0; cc < c0 + H / 2; cc += 16) {
        float acc[16];
        tc::tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)cc, acc);
#pragma unroll
        for (int e = 0; e < 16; ++e) s = fmaf(gelu_fast(acc[e] + sb2[cc + e]), sw3[cc + e], s);
      }
      tc::fence_before();
      red[half * BM + row] = s;
      asm volatile("bar.sync 1, 256;" ::: "memory");
      if (half == 0 && ok) {
        const float y = fminf(fmaxf(s + red[BM + row] + b3, -80.f), 80.f);
        p.u0[(size_t)j * p.ldu + i] = __expf(y);
      }
      asm volatile("bar.sync 1, 256;" ::: "memory");
    }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)H));
}

// A_i = W1f[:, 0:d) S_i + W1f[:, 2d] r_i + W1f[:, 2d+1] log r_i + b1f.
// One thread per (i, n).
__global__ void ws_src_bias_kernel(const float* __restrict__ W1f, int F, int d,
                                   const float* __restrict__ b1f,
                                   const float* __restrict__ S,
                                   const float* __restrict__ rinv, int vr,
                                   float* __restrict__ Asrc) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= vr * H) return;
  const int i = idx / H, n = idx % H;
  const float* w = W1f + (size_t)n * F;
  const float* s = S + (size_t)i * d;
  float a = b1f[n];
  for (int k = 0; k < d; ++k) a = fmaf(w[k], s[k], a);
  const float r = 1.f / rinv[i];
  a = fmaf(w[2 * d], r, a);
  a = fmaf(w[2 * d + 1], logf(r), a);
  Asrc[idx] = a;
}

// B_j = W1f[:, d:2d) C_j for every document.  One warp per (document, 32
// hidden units); the centroid row is read once per warp.
__global__ void ws_doc_bias_kernel(const float* __restrict__ W1f, int F, int d,
                                   const float* __restrict__ C, int64_t N,
                                   float* __restrict__ Bdoc) {
  const int lane = threadIdx.x & 31;
  const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (gw >= N * (H / 32)) return;
  const int64_t j = gw / (H / 32);
  const int n = (int)(gw % (H / 32)) * 32 + lane;
  const float* w = W1f + (size_t)n * F + d;
  const float* c = C + (size_t)j * d;
  float a = 0.f;
  for (int k = 0; k < d; ++k) a = fmaf(w[k], c[k], a);
  Bdoc[(size_t)j * H + n] = a;
}

// Folds the standardisation into layer 1 and converts W2 to BF16:
// W1f[n][f] = W1[n][f] scale[f], b1f[n] = b1[n] - sum_f W1f[n][f] shift[f],
// Ws = W1f[:, 2d+2 .. 2d+4] transposed to [3][H].
__global__ void ws_fold_kernel(const float* __restrict__ prm, WsLayout L,
                               float* __restrict__ W1f, float* __restrict__ b1f,
                               float* __restrict__ Ws, uint16_t* __restrict__ W2b) {
  const int n = blockIdx.x;  // hidden unit
  const int F = L.F;
  __shared__ float part[256];
  float acc = 0.f;
  for (int f = threadIdx.x; f < F; f += blockDim.x) {
    const float w = prm[L.W1 + (size_t)n * F + f] * prm[L.scale + f];
    W1f[(size_t)n * F + f] = w;
    acc = fmaf(w, prm[L.shift + f], acc);
  }
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s; s >>= 1) {
    if ((int)threadIdx.x < s) part[threadIdx.x] += part[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b1f[n] = prm[L.b1 + n] - part[0];
    for (int q = 0; q < 3; ++q)
      Ws[q * H + n] = prm[L.W1 + (size_t)n * F + 2 * L.d + 2 + q] *
                      prm[L.scale + 2 * L.d + 2 + q];
  }
  for (int k = threadIdx.x; k < H; k += blockDim.x)
    W2b[(size_t)n * H + k] = __bfloat16_as_ushort(__float2bfloat16_rn(prm[L.W2 + (size_t)n * H + k]));
}

}  // namespace wsi

size_t ws_folded_floats(const WsLayout& L) {
  // W1f [H][F], b1f [H], Ws [3][H], W2 as BF16 (H*H/2 floats of storage)
  return (size_t)kWsH * L.F + kWsH + 3 * kWsH + (size_t)kWsH * kWsH / 2;
}

int launch_ws_fold(const WsLayout& L, const float* params, float* folded,
                   cudaStream_t st) {
  float* W1f = folded;
  float* b1f = W1f + (size_t)kWsH * L.F;
  float* Ws = b1f + kWsH;
  uint16_t* W2b = reinterpret_cast<uint16_t*>(Ws + 3 * kWsH);
  wsi::ws_fold_kernel<<<kWsH, 256, 0, st>>>(params, L, W1f, b1f, Ws, W2b);
  return 1;
}

int launch_ws_doc_bias(const WsLayout& L, const float* folded, const float* C,
                       int64_t N, float* Bdoc, cudaStream_t st) {
  const int64_t threads = N * kWsH;
  wsi::ws_doc_bias_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(
      folded, L.F, L.d, C, N, Bdoc);
  return 1;
}

namespace wsi {
// Per (document j, source word i): min / mean / max over j's words w of
// M = ln K[w][i] / expo (+ mrow[w] for a row-scaled panel), one warp per
// document, lanes over i: the document's K rows are read once and coalesced.
__global__ void ws_stats_kernel(const float* __restrict__ K, int ld, float expo,
                                const float* __restrict__ mrow,
                                const int64_t* __restrict__ col_ptr,
                                const uint2* __restrict__ ent, int vr, int64_t N,
                                float* __restrict__ stats) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t j = w0; j < N; j += nw) {
    const int64_t b = col_ptr[j];
    const int n = (int)(col_ptr[j + 1] - b);
    for (int i0 = 0; i0 < vr; i0 += 32) {
      const int i = i0 + lane;
      float lo = INFINITY, hi = -INFINITY, sm = 0.f;
      for (int k = 0; k < n; ++k) {
        const uint32_t w = __ldg(&ent[b + k]).x;
        if (i < vr) {
          const float kv = __ldg(&K[(size_t)w * ld + i]);
          const float Mv = fmaxf(__logf(fmaxf(kv, 1e-38f)) / expo, 0.f) +
                           (mrow ? __ldg(&mrow[w]) : 0.f);
          lo = fminf(lo, Mv);
          hi = fmaxf(hi, Mv);
          sm += Mv;
        }
      }
      if (i < vr) {
        float* st = stats + ((size_t)j * vr + i) * 3;
        st[0] = n > 0 ? lo : 0.f;
        st[1] = n > 0 ? sm / (float)n : 0.f;
        st[2] = n > 0 ? hi : 0.f;
      }
    }
  }
}

// The iteration is invariant to u -> a u per document (v -> v / a, the same
// plan and residual), so the prediction fixes u only up to a factor per
// document.  That factor is set here so that the largest entry of each
// document's u0 equals the cold start's value v_r: a prediction far off that
// scale (e.g. every log u near the clamp) would otherwise push v = c / (K^T u)
// toward the FP32 underflow range.  One warp per document.
__global__ void ws_scale_kernel(float* __restrict__ u0, int64_t ldu, int vr, int64_t N) {
  const int64_t j = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= N) return;
  float* row = u0 + j * ldu;
  float mx = 0.f;
  for (int i = lane; i < vr; i += 32) mx = fmaxf(mx, row[i]);
#pragma unroll
  for (int off = 16; off; off >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  if (!(mx > 0.f) || !isfinite(mx)) return;  // the solve's fallback judges it
  const float scale = (float)vr / mx;
  for (int i = lane; i < vr; i += 32) row[i] *= scale;
}
}  // namespace wsi

int launch_ws_init(const WsLayout& L, const float* folded, const float* params,
                   const float* S, const float* rinv, int vr, const float* K, int ld,
                   float expo, const Targets& t, const float* Bdoc, float* Asrc,
                   float* u0, int64_t ldu, unsigned* err, int num_sms,
                   cudaStream_t st, const float* mrow, float* stats) {
  if (vr <= 0 || t.N <= 0) return 0;
  if (stats) {
    int64_t g = (t.N * 32 + 255) / 256;
    const int64_t cap = (int64_t)(num_sms > 0 ? num_sms : 148) * 16;
    if (g > cap) g = cap;
    wsi::ws_stats_kernel<<<(unsigned)g, 256, 0, st>>>(K, ld, expo, mrow, t.col_ptr,
                                                       t.ent, vr, t.N, stats);
  }
  const float* W1f = folded;
  const float* b1f = W1f + (size_t)kWsH * L.F;
  const float* Ws = b1f + kWsH;
  const uint16_t* W2b = reinterpret_cast<const uint16_t*>(Ws + 3 * kWsH);
  wsi::ws_src_bias_kernel<<<(vr * kWsH + 255) / 256, 256, 0, st>>>(
      W1f, L.F, L.d, b1f, S, rinv, vr, Asrc);
  wsi::Params p;
  p.K = K;
  p.mrow = mrow;
  p.stats = stats;
  p.ld = ld;
  p.expo = expo;
  p.col_ptr = t.col_ptr;
  p.ent = t.ent;
  p.Asrc = Asrc;
  p.Bdoc = Bdoc;
  p.Ws = Ws;
  p.W2 = W2b;
  p.b2 = params + L.b2;
  p.w3 = params + L.w3;
  p.b3 = params + L.b3;
  p.vr = vr;
  p.N = t.N;
  p.u0 = u0;
  p.ldu = ldu;
  p.err = err;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    cudaFuncSetAttribute(wsi::ws_init_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)wsi::smem_bytes());
    attr_set[dev] = true;
  }
  const int64_t ntiles = (t.N * (int64_t)vr + wsi::BM - 1) / wsi::BM;
  int64_t grid = num_sms > 0 ? num_sms : 148;
  if (grid > ntiles) grid = ntiles;
  const uint32_t idesc = tc::make_idesc(1, wsi::BM, kWsH);
  wsi::ws_init_kernel<<<(unsigned)grid, wsi::kThreads, wsi::smem_bytes(), st>>>(p, idesc);
  wsi::ws_scale_kernel<<<(unsigned)((t.N * 32 + 255) / 256), 256, 0, st>>>(u0, ldu, vr, t.N);
  return stats ? 4 : 3;
}

}  // namespace wmd
