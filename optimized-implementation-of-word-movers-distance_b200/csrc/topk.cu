// Top-k nearest target documents by WMD.
//
// No reference counterpart: the reference only writes the scores
// (main.py:140-143, sinkhorn_wmd_fused.cpp:617-624).  The ranking is defined
// as a stable ascending sort of the FP64 scores with ties broken by document
// index and NaN (empty documents) last — numpy.argsort(scores,
// kind="stable")[:k] — and the kernels reproduce it exactly.
//
// Scores are mapped to order-preserving 64-bit keys (-0.0 folded into +0.0,
// every NaN to the largest key).  Level 0 sorts chunks of 2048 (key, index)
// pairs with a shared-memory bitonic network and keeps the first k of each;
// each further level merges groups of candidate lists the same way until a
// single list of k remains.
#include <utility>

#include "wmd_internal.cuh"

namespace wmd {

namespace {
constexpr int kTile = 2048;     // pairs sorted per CTA
constexpr int kThreads = 1024;

__device__ __forceinline__ uint64_t order_key(double v) {
  if (v != v) return ~0ull;          // NaN last
  if (v == 0.0) v = 0.0;             // -0.0 ties with +0.0
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double key_value(uint64_t k) {
  if (k == ~0ull) return __longlong_as_double(0x7ff8000000000000ll);
  const uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}
__device__ __forceinline__ bool less_pair(uint64_t ka, uint32_t ia, uint64_t kb,
                                          uint32_t ib) {
  return ka < kb || (ka == kb && ia < ib);
}

// Sorts kTile (key, idx) pairs in shared memory (padding = (~0, ~0)).
__device__ void bitonic_sort(uint64_t* key, uint32_t* idx) {
  for (int size = 2; size <= kTile; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      __syncthreads();
      for (int t = threadIdx.x; t < kTile / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint64_t ka = key[lo], kb = key[hi];
        const uint32_t ia = idx[lo], ib = idx[hi];
        const bool swap = up ? less_pair(kb, ib, ka, ia) : less_pair(ka, ia, kb, ib);
        if (swap) {
          key[lo] = kb; key[hi] = ka;
          idx[lo] = ib; idx[hi] = ia;
        }
      }
    }
  }
  __syncthreads();
}
}  // namespace

// Level 0: chunk c of the scores -> its k smallest (key, idx) pairs.
__global__ void __launch_bounds__(kThreads)
topk_chunks_kernel(const double* __restrict__ scores, uint64_t n, int k,
                   uint64_t* __restrict__ out_key, uint32_t* __restrict__ out_idx) {
  __shared__ uint64_t key[kTile];
  __shared__ uint32_t idx[kTile];
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  for (int t = threadIdx.x; t < kTile; t += blockDim.x) {
    const uint64_t i = base + t;
    key[t] = i < n ? order_key(scores[i]) : ~0ull;
    idx[t] = i < n ? (uint32_t)i : ~0u;
  }
  bitonic_sort(key, idx);
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    out_key[(uint64_t)blockIdx.x * k + t] = key[t];
    out_idx[(uint64_t)blockIdx.x * k + t] = idx[t];
  }
}

// Merge level: group g takes `lists` consecutive candidate lists of length k
// (the last group may have fewer) and keeps the k smallest.
__global__ void __launch_bounds__(kThreads)
topk_merge_kernel(const uint64_t* __restrict__ in_key,
                  const uint32_t* __restrict__ in_idx, int nlists, int lists,
                  int k, uint64_t* __restrict__ out_key,
                  uint32_t* __restrict__ out_idx) {
  __shared__ uint64_t key[kTile];
  __shared__ uint32_t idx[kTile];
  const int first = blockIdx.x * lists;
  const int count = min(lists, nlists - first) * k;
  const uint64_t base = (uint64_t)first * k;
  for (int t = threadIdx.x; t < kTile; t += blockDim.x) {
    key[t] = t < count ? in_key[base + t] : ~0ull;
    idx[t] = t < count ? in_idx[base + t] : ~0u;
  }
  bitonic_sort(key, idx);
  for (int t = threadIdx.x; t < k; t += blockDim.x) {
    out_key[(uint64_t)blockIdx.x * k + t] = key[t];
    out_idx[(uint64_t)blockIdx.x * k + t] = idx[t];
  }
}

__global__ void topk_finish_kernel(const uint64_t* __restrict__ key,
                                   const uint32_t* __restrict__ idx, int k,
                                   uint64_t n, uint32_t* __restrict__ out_idx,
                                   double* __restrict__ out_val) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= k) return;
  const bool real = (uint64_t)t < n;
  out_idx[t] = real ? idx[t] : ~0u;
  out_val[t] = real ? key_value(key[t]) : __longlong_as_double(0x7ff8000000000000ll);
}

size_t topk_scratch_bytes(uint64_t n, int k) {
  const uint64_t chunks = (n + kTile - 1) / kTile;
  return 2 * chunks * (uint64_t)k * (sizeof(uint64_t) + sizeof(uint32_t)) + 64;
}

// scratch: topk_scratch_bytes(n, k) bytes.  1 <= k <= 1024.
int launch_topk(const double* scores, uint64_t n, int k, void* scratch,
                uint32_t* out_idx, double* out_val, cudaStream_t st) {
  const uint64_t chunks = (n + kTile - 1) / kTile;
  const uint64_t half = chunks * (uint64_t)k;
  uint64_t* kA = static_cast<uint64_t*>(scratch);
  uint64_t* kB = kA + half;
  uint32_t* iA = reinterpret_cast<uint32_t*>(kB + half);
  uint32_t* iB = iA + half;
  int launches = 0;
  topk_chunks_kernel<<<(unsigned)chunks, kThreads, 0, st>>>(scores, n, k, kA, iA);
  ++launches;
  int nlists = (int)chunks;
  const int lists = kTile / k;  // candidate lists merged per CTA (>= 2 for k <= 1024)
  while (nlists > 1) {
    const int groups = (nlists + lists - 1) / lists;
    topk_merge_kernel<<<groups, kThreads, 0, st>>>(kA, iA, nlists, lists, k, kB, iB);
    ++launches;
    std::swap(kA, kB);
    std::swap(iA, iB);
    nlists = groups;
  }
  topk_finish_kernel<<<(k + 255) / 256, 256, 0, st>>>(kA, iA, k, n, out_idx, out_val);
  return launches + 1;
}

}  // namespace wmd
