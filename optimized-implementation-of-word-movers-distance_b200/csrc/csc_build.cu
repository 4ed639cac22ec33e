// GPU build of the document-major (CSC) target matrix from an edge list.
//
// The reference turns its edge list into word-major CSR with a counting
// sort that keeps file order within a word (sinkhorn_wmd_fused.cpp:460-506);
// the solve here iterates documents, so the host path transposes that CSR
// with a second stable counting sort keyed by document.  The composition is
// a stable sort of the edges by (document, word) with file order breaking
// ties, which is what this file computes on the GPU: one 64-bit key
// doc * 2^wb + word per edge (wb = bits of V), a stable LSD radix sort of
// (key, edge index) pairs over the key's significant bits (CUB
// DeviceRadixSort: a library sort on this one-off conversion, not on the
// query path), then the column pointers from the sorted document ids and a
// gather of the weights.  Invalid edges (word >= V, document >= N,
// weight <= 0 or not finite) set error bits.
#include <cub/device/device_radix_sort.cuh>

#include "wmd_internal.cuh"

namespace wmd {
namespace {

int bits_for(uint64_t n) {  // bits to hold values 0 .. n-1
  int b = 0;
  while (b < 64 && (n - 1) >> b) ++b;
  return b > 0 ? b : 1;
}

__global__ void csc_keys_kernel(const uint64_t* __restrict__ words,
                                const uint64_t* __restrict__ docs,
                                const double* __restrict__ w, uint64_t nnz,
                                uint64_t V, uint64_t N, int wb,
                                uint64_t* __restrict__ keys,
                                uint32_t* __restrict__ idx, unsigned* err) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t a = words[e], b = docs[e];
    const double x = w[e];
    unsigned bad = 0;
    if (a >= V) bad |= ERR_ROW_RANGE;
    if (b >= N) bad |= ERR_DOC_RANGE;
    if (!(x > 0.0) || !isfinite(x)) bad |= ERR_BAD_VAL;
    if (bad) atomicOr(err, bad);
    keys[e] = (bad ? 0ull : (b << wb) | a);
    idx[e] = (uint32_t)e;
  }
}

// col_ptr[j] = first sorted position whose document is >= j.
__global__ void csc_colptr_kernel(const uint64_t* __restrict__ keys, uint64_t nnz,
                                  uint64_t N, int wb, uint64_t* __restrict__ col_ptr) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p <= nnz;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t lo = p == 0 ? 0 : (keys[p - 1] >> wb) + 1;
    const uint64_t hi = p == nnz ? N : (keys[p] >> wb);
    for (uint64_t j = lo; j <= hi && j <= N; ++j) col_ptr[j] = p;
  }
}

__global__ void csc_gather_kernel(const uint64_t* __restrict__ keys,
                                  const uint32_t* __restrict__ idx,
                                  const double* __restrict__ w, uint64_t nnz,
                                  uint64_t wmask, uint64_t* __restrict__ rows,
                                  double* __restrict__ vals) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz;
       p += (uint64_t)gridDim.x * blockDim.x) {
    rows[p] = keys[p] & wmask;
    vals[p] = w[idx[p]];
  }
}

size_t cub_temp(uint64_t nnz, int bits) {
  size_t t = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                  (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int64_t)nnz, 0, bits);
  return t;
}
}  // namespace

// temp layout: keys[2][nnz] u64, idx[2][nnz] u32, CUB temp storage.
size_t csc_build_temp_bytes(uint64_t nnz, uint64_t V, uint64_t N) {
  const int bits = bits_for(V) + bits_for(N);
  return 2 * nnz * 8 + 2 * nnz * 4 + 256 + cub_temp(nnz, bits > 64 ? 64 : bits);
}

int launch_csc_build(const uint64_t* words, const uint64_t* docs, const double* w,
                     uint64_t nnz, uint64_t V, uint64_t N, void* temp,
                     size_t temp_bytes, uint64_t* col_ptr, uint64_t* rows,
                     double* vals, unsigned* err, cudaStream_t st) {
  const int wb = bits_for(V);
  const int bits = wb + bits_for(N);
  if (bits > 64 || nnz > 0xFFFFFFFFull) return -1;
  unsigned char* t = static_cast<unsigned char*>(temp);
  uint64_t* k0 = reinterpret_cast<uint64_t*>(t);
  uint64_t* k1 = k0 + nnz;
  uint32_t* i0 = reinterpret_cast<uint32_t*>(k1 + nnz);
  uint32_t* i1 = i0 + nnz;
  unsigned char* ct = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(i1 + nnz) + 255) & ~uintptr_t(255));
  size_t ct_bytes = temp_bytes - (size_t)(ct - t);
  const unsigned grid = 1184;
  csc_keys_kernel<<<grid, 256, 0, st>>>(words, docs, w, nnz, V, N, wb, k0, i0, err);
  if (cub::DeviceRadixSort::SortPairs(ct, ct_bytes, k0, k1, i0, i1, (int64_t)nnz, 0,
                                      bits, st) != cudaSuccess)
    return -1;
  csc_colptr_kernel<<<grid, 256, 0, st>>>(k1, nnz, N, wb, col_ptr);
  csc_gather_kernel<<<grid, 256, 0, st>>>(k1, i1, w, nnz, (wb >= 64 ? ~0ull : ((1ull << wb) - 1)),
                                          rows, vals);
  return 4;
}

}  // namespace wmd
