// Input preparation kernels: embedding conversion, target packing with
// validation, and source-word selection.
//
// Selection restates select_non_empty_entries (sinkhorn_wmd_fused.cpp:45-63):
// every id with r != 0, in ascending id order, with weight r.  The reference
// does it serially; here it is a two-launch stream compaction (count per
// 1024-element chunk, then each chunk scans its flags and writes at the
// offset of the chunks before it), so the order is the reference's.
#include "wmd_internal.cuh"

namespace wmd {

// ---------------------------------------------------------------------------
// Embeddings: FP64 [V][d] -> FP32 [V][d] plus squared norms (one warp per row).
// ---------------------------------------------------------------------------
__global__ void embed_convert_f64_kernel(const double* __restrict__ src,
                                         uint64_t V, uint64_t d,
                                         float* __restrict__ E32,
                                         float* __restrict__ nE) {
  const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= V) return;
  const double* s = src + row * d;
  float* o = E32 + row * d;
  double acc = 0.0;
  for (uint64_t k = lane; k < d; k += 32) {
    const float f = (float)s[k];
    o[k] = f;
    acc += (double)f * (double)f;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) nE[row] = (float)acc;
}

__global__ void embed_norms_kernel(const float* __restrict__ E32, uint64_t V,
                                   uint64_t d, float* __restrict__ nE) {
  const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= V) return;
  const float* s = E32 + row * d;
  double acc = 0.0;
  for (uint64_t k = lane; k < d; k += 32) {
    const double f = (double)s[k];
    acc += f * f;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) nE[row] = (float)acc;
}

int launch_embed_convert_f64(const double* src, uint64_t V, uint64_t d,
                             float* E32, float* nE, cudaStream_t st) {
  const int threads = 256;
  const uint64_t blocks = (V * 32 + threads - 1) / threads;
  embed_convert_f64_kernel<<<(unsigned)blocks, threads, 0, st>>>(src, V, d, E32, nE);
  return 1;
}

// BF16 embeddings [V][d] -> the exact FP32 working copy E32 [V][d] and the
// tensor-core copy E16 [V][dp] (the same BF16 values, zero-padded to dp).
__global__ void embed_from_bf16_kernel(const uint16_t* __restrict__ src, uint64_t V,
                                       int d, int dp, float* __restrict__ E32,
                                       uint16_t* __restrict__ E16) {
  const uint64_t total = V * (uint64_t)dp;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t w = i / dp;
    const int k = (int)(i - w * dp);
    const uint16_t b = k < d ? src[w * d + k] : (uint16_t)0;
    E16[i] = b;
    if (k < d) E32[w * d + k] = __uint_as_float((unsigned)b << 16);
  }
}

int launch_embed_from_bf16(const void* src, uint64_t V, uint64_t d, int dp, float* E32,
                           void* E16, cudaStream_t st) {
  const uint64_t total = V * (uint64_t)dp;
  uint64_t blocks = (total + 255) / 256;
  if (blocks > 65535ull * 16) blocks = 65535ull * 16;
  embed_from_bf16_kernel<<<(unsigned)blocks, 256, 0, st>>>(
      static_cast<const uint16_t*>(src), V, (int)d, dp, E32, static_cast<uint16_t*>(E16));
  return 1;
}

int launch_embed_norms(const float* E32, uint64_t V, uint64_t d, float* nE,
                       cudaStream_t st) {
  const int threads = 256;
  const uint64_t blocks = (V * 32 + threads - 1) / threads;
  embed_norms_kernel<<<(unsigned)blocks, threads, 0, st>>>(E32, V, d, nE);
  return 1;
}

// ---------------------------------------------------------------------------
// Drop-in embedding rows split between the host and the bus (api.cu): the
// rows of words below `wh` are narrowed FP64 -> FP32 by the host threads and
// copied (rows32[w], every word of that id prefix); above it the GPU reads
// the rows of the words a query can touch (flagged in `need`: every target
// word and every source word) straight from the caller's device-mapped host
// memory, and zeroes the others.  Phase 0 handles the words >= wh (it runs
// while the host converts), phase 1 the prefix.  E32 and the norms come out
// as embed_convert_f64_kernel and embed_norms_kernel write them for the whole
// matrix (the same FP64 -> FP32 rounding, the same per-lane order of the FP64
// norm sums), so the results do not depend on the split.  A zero row is
// finite and never near any source row, so the cost panel's unused rows stay
// harmless; the solve never gathers them.
__global__ void mark_needed_kernel(const uint2* __restrict__ ent, uint64_t nnz,
                                   const double* __restrict__ r, uint64_t V,
                                   unsigned char* __restrict__ need) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // (the packing's range check may not have been read yet: skip bad ids)
  if (i < nnz && ent[i].x < V) need[ent[i].x] = 1;
  if (i < V && r[i] != 0.0) need[i] = 1;
}

__global__ void gather_rows_split_kernel(const double* __restrict__ src_mapped,
                                         const unsigned char* __restrict__ need,
                                         uint64_t V, uint64_t d, uint64_t wh,
                                         const float* __restrict__ rows32, int phase,
                                         float* __restrict__ E32, float* __restrict__ nE,
                                         unsigned long long* __restrict__ nrows) {
  const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= V) return;
  if ((phase == 0) == (row < wh)) return;  // the other phase's row
  float* o = E32 + row * d;
  double acc = 0.0;
  if (row < wh) {
    const float* s = rows32 + row * d;
    for (uint64_t k = lane; k < d; k += 32) {
      const float f = s[k];
      o[k] = f;
      acc += (double)f * (double)f;
    }
  } else if (!need[row]) {
    for (uint64_t k = lane; k < d; k += 32) o[k] = 0.f;
    if (lane == 0) nE[row] = 0.f;
    return;
  } else {
    if (lane == 0) atomicAdd(nrows, 1ull);  // rows read over the bus
    const double* s = src_mapped + row * d;
    if (d <= 512) {
      // All of a lane's loads before any use: one bus round trip per row.
      double v[16];
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const uint64_t k = (uint64_t)lane + 32u * t;
        v[t] = k < d ? s[k] : 0.0;
      }
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const uint64_t k = (uint64_t)lane + 32u * t;
        const float f = (float)v[t];
        if (k < d) o[k] = f;
        acc += (double)f * (double)f;
      }
    } else {
      for (uint64_t k = lane; k < d; k += 32) {
        const float f = (float)s[k];
        o[k] = f;
        acc += (double)f * (double)f;
      }
    }
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
  if (lane == 0) nE[row] = (float)acc;
}

int launch_gather_rows_split(const double* src_mapped, const uint2* ent, uint64_t nnz,
                             const double* r_dev, unsigned char* need, uint64_t V,
                             uint64_t d, uint64_t wh, const float* rows32, int phase,
                             float* E32, float* nE, unsigned long long* nrows,
                             cudaStream_t st) {
  const int threads = 256;
  int n = 0;
  if (phase == 0) {
    cudaMemsetAsync(nrows, 0, sizeof(unsigned long long), st);
    if (wh < V) {
      cudaMemsetAsync(need, 0, V, st);
      const uint64_t m = nnz > V ? nnz : V;
      mark_needed_kernel<<<(unsigned)((m + threads - 1) / threads), threads, 0, st>>>(
          ent, nnz, r_dev, V, need);
      ++n;
    }
  }
  gather_rows_split_kernel<<<(unsigned)((V * 32 + threads - 1) / threads), threads, 0, st>>>(
      src_mapped, need, V, d, wh, rows32, phase, E32, nE, nrows);
  return n + 1;
}

// ---------------------------------------------------------------------------
// Targets: validate a CSC triple and pack it for the solver.  The checks are
// those of the reference driver's MTX reader (sinkhorn_wmd_fused.cpp:474-478):
// indices in range and values > 0; plus consistent column pointers.
// ---------------------------------------------------------------------------
__global__ void pack_colptr_kernel(const uint64_t* __restrict__ cp_in,
                                   uint64_t N, uint64_t nnz,
                                   int64_t* __restrict__ cp_out,
                                   unsigned* __restrict__ err) {
  const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j > N) return;
  const uint64_t a = cp_in[j];
  bool bad = a > nnz;
  if (j == 0) bad |= (a != 0);
  if (j == N) bad |= (a != nnz);
  if (j < N) bad |= (cp_in[j + 1] < a);
  if (bad) atomicOr(err, ERR_COLPTR);
  cp_out[j] = (int64_t)(a > nnz ? nnz : a);
}

__global__ void pack_entries_kernel(const uint64_t* __restrict__ rows,
                                    const double* __restrict__ vals,
                                    uint64_t nnz, uint64_t V,
                                    uint2* __restrict__ ent,
                                    unsigned* __restrict__ err) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  uint64_t w = rows[e];
  const double v = vals[e];
  unsigned bad = 0;
  if (w >= V) {
    bad |= ERR_ROW_RANGE;
    w = 0;  // keep every later gather in bounds
  }
  if (!(v > 0.0) || !isfinite(v)) bad |= ERR_BAD_VAL;
  if (bad) atomicOr(err, bad);
  ent[e] = make_uint2((unsigned)w, __float_as_uint((float)v));
}

int launch_pack_targets(const uint64_t* col_ptr_in, const uint64_t* rows_in,
                        const double* vals_in, uint64_t V, uint64_t N,
                        uint64_t nnz, int64_t* col_ptr, uint2* ent,
                        unsigned* err, cudaStream_t st) {
  const int threads = 256;
  pack_colptr_kernel<<<(unsigned)((N + 1 + threads - 1) / threads), threads, 0, st>>>(
      col_ptr_in, N, nnz, col_ptr, err);
  int n = 1;
  if (nnz) {
    pack_entries_kernel<<<(unsigned)((nnz + threads - 1) / threads), threads, 0, st>>>(
        rows_in, vals_in, nnz, V, ent, err);
    n++;
  }
  return n;
}

// ---------------------------------------------------------------------------
// Source selection.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned block_sum_u32(unsigned v, unsigned* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  unsigned t = 0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0u;
#pragma unroll
    for (int off = 16; off; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    if (threadIdx.x == 0) red[32] = t;
  }
  __syncthreads();
  t = red[32];
  __syncthreads();
  return t;
}

// Copy of one embedding row by a warp.  For d <= 512 every lane issues all
// its loads before its stores (one memory round trip for the row instead of
// one per 32 elements: the rows are cold in L2 when a query starts).
// A row of dp 16-bit values, one warp: 16-byte pieces when dp is a multiple
// of 8 (rows then start on 16-byte boundaries), else element by element.
__device__ __forceinline__ void copy_row16(const unsigned short* __restrict__ src,
                                           unsigned short* __restrict__ dst, int dp,
                                           int lane) {
  if (dp % 8 == 0) {
    const uint4* s4 = reinterpret_cast<const uint4*>(src);
    uint4* d4 = reinterpret_cast<uint4*>(dst);
    for (int k = lane; k < dp / 8; k += 32) d4[k] = __ldg(s4 + k);
  } else {
    for (int k = lane; k < dp; k += 32) dst[k] = src[k];
  }
}

__device__ __forceinline__ void copy_row(const float* __restrict__ src,
                                         float* __restrict__ dst, uint64_t d,
                                         int lane);

// One source row for the cost panel, one warp: the FP32 row (d floats) and,
// when s16 is given, its 16-bit (or split) row of dp values, with every load
// issued before the first store (one memory round trip for both).
__device__ __forceinline__ void gather_source_row(const float* __restrict__ src,
                                                  float* __restrict__ dst, uint64_t d,
                                                  const unsigned short* __restrict__ s16,
                                                  unsigned short* __restrict__ d16, int dp,
                                                  int lane) {
  if (d <= 512 && (!s16 || (dp % 8 == 0 && dp <= 1024))) {
    float v[16];
    uint4 h[4];
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const uint64_t k = (uint64_t)lane + 32u * t;
      v[t] = k < d ? __ldg(src + k) : 0.f;
    }
    if (s16) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = lane + 32 * t;
        h[t] = k < dp / 8 ? __ldg(reinterpret_cast<const uint4*>(s16) + k)
                          : make_uint4(0u, 0u, 0u, 0u);
      }
    }
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const uint64_t k = (uint64_t)lane + 32u * t;
      if (k < d) dst[k] = v[t];
    }
    if (s16) {
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = lane + 32 * t;
        if (k < dp / 8) reinterpret_cast<uint4*>(d16)[k] = h[t];
      }
    }
  } else {
    copy_row(src, dst, d, lane);
    if (s16) copy_row16(s16, d16, dp, lane);
  }
}

__device__ __forceinline__ void copy_row(const float* __restrict__ src,
                                         float* __restrict__ dst, uint64_t d,
                                         int lane) {
  if (d <= 512) {
    float v[16];
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const uint64_t k = (uint64_t)lane + 32u * t;
      v[t] = k < d ? __ldg(src + k) : 0.f;
    }
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const uint64_t k = (uint64_t)lane + 32u * t;
      if (k < d) dst[k] = v[t];
    }
  } else {
    for (uint64_t k = lane; k < d; k += 32) dst[k] = src[k];
  }
}

__global__ void __launch_bounds__(kSelectThreads)
select_count_kernel(const double* __restrict__ r, uint64_t V,
                    uint32_t* __restrict__ chunk_counts,
                    unsigned* __restrict__ err, unsigned* __restrict__ zero_word) {
  __shared__ unsigned red[33];
  grid_dep_launch();
  // A counter of a later kernel of the same query (the near-pair list), reset
  // here instead of by a separate memset on the stream.
  if (zero_word && blockIdx.x == 0 && threadIdx.x == 0) *zero_word = 0u;
  const uint64_t base = (uint64_t)blockIdx.x * kSelectChunk;
  unsigned cnt = 0;
  bool neg = false;
#pragma unroll 4
  for (int k = 0; k < kSelectPerThread; ++k) {
    const uint64_t i = base + (uint64_t)k * kSelectThreads + threadIdx.x;
    if (i < V) {
      const double v = r[i];
      cnt += (v != 0.0);
      neg |= (v < 0.0);
    }
  }
  if (neg) atomicOr(err, ERR_NEG_R);
  const unsigned tot = block_sum_u32(cnt, red);
  if (threadIdx.x == 0) chunk_counts[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kSelectThreads)
select_write_kernel(const double* __restrict__ r, uint64_t V,
                    const float* __restrict__ E32, const float* __restrict__ nE,
                    uint64_t d, int nchunks,
                    const uint32_t* __restrict__ chunk_counts,
                    uint32_t cap, uint32_t* __restrict__ ids,
                    float* __restrict__ rinv, float* __restrict__ S,
                    float* __restrict__ nS, uint32_t* __restrict__ vr_out,
                    unsigned* __restrict__ err,
                    const unsigned short* __restrict__ E16,
                    unsigned short* __restrict__ S16, int dp) {
  __shared__ unsigned red[33];
  __shared__ unsigned warp_off[kSelectThreads / 32];
  __shared__ uint32_t list_pos[kSelectChunk];
  __shared__ uint32_t list_id[kSelectChunk];
  grid_dep_launch();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kSelectChunk;
  // This chunk's weights first: their loads overlap the offset computation.
  double rv[kSelectPerThread];
#pragma unroll
  for (int k = 0; k < kSelectPerThread; ++k) {
    const uint64_t i = base + (uint64_t)k * kSelectThreads + threadIdx.x;
    rv[k] = i < V ? r[i] : 0.0;
  }

  // Offset of this chunk = selected count of all chunks before it (the
  // count kernel's output).
  grid_dep_wait();
  unsigned before = 0, all = 0;
  for (int c = threadIdx.x; c < nchunks; c += blockDim.x) {
    const unsigned v = chunk_counts[c];
    all += v;
    if (c < (int)blockIdx.x) before += v;
  }
  const unsigned offset = block_sum_u32(before, red);
  const unsigned total = block_sum_u32(all, red);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *vr_out = total < cap ? total : cap;
    if (total > cap) atomicOr(err, ERR_VR_CAP);
  }

  unsigned running = 0;
#pragma unroll
  for (int k = 0; k < kSelectPerThread; ++k) {
    const uint64_t i = base + (uint64_t)k * kSelectThreads + threadIdx.x;
    const double v = rv[k];
    const bool sel = (i < V) && (v != 0.0);
    const unsigned bal = __ballot_sync(0xffffffffu, sel);
    if (lane == 0) warp_off[warp] = __popc(bal);
    __syncthreads();
    unsigned wpre = 0, ktot = 0;
#pragma unroll
    for (int w = 0; w < kSelectThreads / 32; ++w) {
      const unsigned c = warp_off[w];
      wpre += (w < warp) ? c : 0u;
      ktot += c;
    }
    if (sel) {
      const unsigned local = running + wpre + __popc(bal & ((1u << lane) - 1u));
      const unsigned pos = offset + local;
      list_pos[local] = pos;
      list_id[local] = (uint32_t)i;
      if (pos < cap) {
        ids[pos] = (uint32_t)i;
        rinv[pos] = (float)(1.0 / v);
      }
    }
    running += ktot;
    __syncthreads();
  }
  // Gather the selected rows of E32 (one warp per selected word).
  for (unsigned s = warp; s < running; s += kSelectThreads / 32) {
    const uint32_t pos = list_pos[s];
    if (pos >= cap) continue;
    const uint64_t id = list_id[s];
    if (lane == 0) nS[pos] = nE[id];
    // FP32 row and, for the tensor-core cost panel, its 16-bit (or split) row
    gather_source_row(E32 + id * d, S + (uint64_t)pos * d, d,
                      S16 ? E16 + id * (uint64_t)dp : nullptr,
                      S16 ? S16 + (uint64_t)pos * dp : nullptr, dp, lane);
  }
}

int launch_select_count(const double* r, uint64_t V, uint32_t* chunk_counts,
                        unsigned* err, cudaStream_t st) {
  select_count_kernel<<<select_num_chunks(V), kSelectThreads, 0, st>>>(
      r, V, chunk_counts, err, nullptr);
  return 1;
}

int launch_select(const double* r, uint64_t V, const float* E32,
                  const float* nE, uint64_t d, const SourceSel& s,
                  unsigned* err, cudaStream_t st, const void* E16, void* S16,
                  int dp, unsigned* zero_word) {
  const int nchunks = select_num_chunks(V);
  select_count_kernel<<<nchunks, kSelectThreads, 0, st>>>(r, V, s.chunk_counts, err,
                                                          zero_word);
  launch_pdl(select_write_kernel, dim3(nchunks), dim3(kSelectThreads), 0, st, r, V, E32, nE,
             d, nchunks, (const uint32_t*)s.chunk_counts, s.cap, s.ids, s.rinv, s.S, s.nS,
             s.vr, err, static_cast<const unsigned short*>(E16),
             static_cast<unsigned short*>(S16), dp);
  return 2;
}

}  // namespace wmd

namespace wmd {

// Batched queries: gather the embedding rows of one source document whose
// (ascending, validated) word ids were uploaded with the batch.  One warp per
// source word; also its squared norm and, when S16 is given, its 16-bit row.
__global__ void gather_sources_kernel(const uint32_t* __restrict__ ids, int count,
                                      const float* __restrict__ E32,
                                      const float* __restrict__ nE, uint64_t d,
                                      float* __restrict__ S, float* __restrict__ nS,
                                      const unsigned short* __restrict__ E16,
                                      unsigned short* __restrict__ S16, int dp) {
  const int w = (int)(((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= count) return;
  const uint64_t id = ids[w];
  if (lane == 0) nS[w] = nE[id];
  gather_source_row(E32 + id * d, S + (uint64_t)w * d, d,
                    S16 ? E16 + id * (uint64_t)dp : nullptr,
                    S16 ? S16 + (uint64_t)w * dp : nullptr, dp, lane);
}

int launch_gather_sources(const uint32_t* ids, int count, const float* E32,
                          const float* nE, uint64_t d, float* S, float* nS,
                          const void* E16, void* S16, int dp, cudaStream_t st) {
  if (count <= 0) return 0;
  const int threads = 256;
  const int blocks = (count * 32 + threads - 1) / threads;
  gather_sources_kernel<<<blocks, threads, 0, st>>>(
      ids, count, E32, nE, d, S, nS, static_cast<const unsigned short*>(E16),
      static_cast<unsigned short*>(S16), dp);
  return 1;
}

}  // namespace wmd
