// wmd_sinkhorn_noalloc: the full Sinkhorn WMD solve with no device memory
// allocation at all.
//
// Who needs it: callers that may not call cudaMalloc / cudaFree themselves or
// through a library — code running under another runtime's memory discipline
// (an inference server or framework that owns every byte of device memory
// through its own pool and hands plugins only their input and output
// buffers), and latency-critical loops where the implicit device-wide
// synchronisation of cudaMalloc / cudaFree would stall other work on the GPU.
// The regular entry points allocate their working buffers on first use; this
// one uses a fixed scratch area compiled into the library instead.
//
// The scratch is the file-scope array below (kScratchBytes = 64 MiB).  Every
// GPU that loads this library holds it until the process exits.  All calls
// on a device share it and it keeps the previous call's contents, so calls
// that overlap on the GPU (different streams, or different host threads on
// the same device) race and corrupt each other's results: serialise them.
//
// Host code cannot use the array's name as a device address (in host code
// it names a host-side stand-in), so the first call on each device, with that
// device current, looks the address up with cudaGetSymbolAddress and caches
// it.  Make that first call before any stream capture begins on the device.
// The cached address lives as long as the device's primary context: after
// cudaDeviceReset on a device, this entry point must not be called on it
// again in the same process.
//
// The kernels are the library's regular ones (norms, target packing and
// validation, source selection, FP32 cost panel, near-pair fix-up, fused
// solve); only where their working buffers live differs.
#include <stdio.h>

#include <mutex>

#include "wmd_b200.h"
#include "wmd_internal.cuh"

namespace {

constexpr size_t kScratchBytes = 64ull << 20;  // 64 MiB per device
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

wmd_status noalloc_fail(wmd_status s, const char* msg) {
  wmd::set_last_error(msg);
  return s;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Per-device set-up: resolve the device address of the scratch array.
wmd_status scratch_for_current_device(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(WMD_ERR_UNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return noalloc_fail(WMD_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed");
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
  wmd::set_last_error("");
  return WMD_OK;
}

}  // namespace

extern "C" wmd_status wmd_sinkhorn_noalloc(
    const double* r_dev, const float* vecs_dev, uint64_t V, uint64_t d,
    const uint64_t* col_ptr_dev, const uint64_t* row_inds_dev,
    const double* vals_dev, uint64_t N, uint64_t nnz, uint64_t vr_cap,
    double lambda, int max_iter, double* wmd_dev, void* stream) {
  using namespace wmd;
  char msg[256];
  if (!r_dev || !vecs_dev || !col_ptr_dev || !row_inds_dev || !vals_dev || !wmd_dev)
    return noalloc_fail(WMD_ERR_INVALID_ARG, "null pointer argument");
  if (V == 0 || d == 0 || N == 0 || nnz == 0)
    return noalloc_fail(WMD_ERR_INVALID_INPUT, "empty vocabulary, width or target matrix");
  if (max_iter < 0) return noalloc_fail(WMD_ERR_INVALID_ARG, "max_iter < 0");
  if (vr_cap > 1024)
    return noalloc_fail(WMD_ERR_UNSUPPORTED, "vr_cap above 1024");
  if (V > 0xFFFFFFFFull || N >= 0x7FFFFFFFull)
    return noalloc_fail(WMD_ERR_UNSUPPORTED, "vocabulary or document count too large");
  // Each factor of the scratch sizes below is bounded first, so that none of
  // the size products can wrap around: anything larger cannot fit anyway.
  if (d > kScratchBytes / 4 || nnz > kScratchBytes / 8 || N > kScratchBytes / 8) {
    snprintf(msg, sizeof(msg),
             "d, nnz or N too large for the fixed scratch of %zu bytes (64 MiB)",
             kScratchBytes);
    return noalloc_fail(WMD_ERR_INVALID_ARG, msg);
  }
  // The FP32 cost panel reads the embeddings with 16-byte vector loads when
  // d % 4 == 0; a misaligned base would fault, so it is refused here.
  if (d % 4 == 0 && (reinterpret_cast<uintptr_t>(vecs_dev) & 15u) != 0)
    return noalloc_fail(WMD_ERR_INVALID_ARG,
                        "vecs_dev must be 16-byte aligned when d % 4 == 0");

  // Carve the scratch: everything 256-byte aligned.
  const uint32_t cap = (uint32_t)vr_cap;
  const uint32_t cap1 = cap ? cap : 1;
  const int ld = (int)((cap1 + 3u) & ~3u);
  const int nchunks = select_num_chunks(V);
  size_t off = 0;
  const size_t o_err = off;    off += align256(sizeof(unsigned));
  const size_t o_vr = off;     off += align256(sizeof(uint32_t));
  const size_t o_chunk = off;  off += align256((size_t)nchunks * 4);
  const size_t o_ids = off;    off += align256((size_t)cap1 * 4);
  const size_t o_rinv = off;   off += align256((size_t)cap1 * 4);
  const size_t o_nS = off;     off += align256((size_t)cap1 * 4);
  const size_t o_S = off;      off += align256((size_t)cap1 * d * 4);
  const size_t o_nE = off;     off += align256((size_t)V * 4);
  const size_t o_cp = off;     off += align256((size_t)(N + 1) * 8);
  const size_t o_ent = off;    off += align256((size_t)nnz * 8);
  const unsigned near_cap = 4096;  // near-pair list (overflow -> panel scan)
  const size_t o_ncnt = off;   off += align256(sizeof(unsigned));
  const size_t o_npairs = off; off += align256((size_t)near_cap * 8);
  const float expo = (float)(-lambda);
  const bool want_km = expo == 0.f;  // K.*M is needed only for lambda = 0
  const size_t o_K = off;      off += align256((size_t)V * ld * 4);
  const size_t o_KM = off;     off += want_km ? align256((size_t)V * ld * 4) : 0;
  if (off > kScratchBytes) {
    snprintf(msg, sizeof(msg),
             "problem needs %zu bytes of scratch; the fixed scratch holds %zu "
             "bytes (64 MiB): V*round4(vr_cap)*4 (twice for lambda = 0) + V*4 + "
             "nnz*8 + ... too large",
             off, kScratchBytes);
    return noalloc_fail(WMD_ERR_INVALID_ARG, msg);
  }

  // A pending error from earlier, unrelated work on this thread would
  // otherwise be reported as this call's failure by the final check.
  cudaGetLastError();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(WMD_ERR_NO_DEVICE, "no current CUDA device");
  }
  unsigned char* base = nullptr;
  wmd_status s = scratch_for_current_device(dev, &base);
  if (s != WMD_OK) return s;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  unsigned* err = reinterpret_cast<unsigned*>(base + o_err);
  SourceSel sel;
  sel.vr = reinterpret_cast<uint32_t*>(base + o_vr);
  sel.chunk_counts = reinterpret_cast<uint32_t*>(base + o_chunk);
  sel.ids = reinterpret_cast<uint32_t*>(base + o_ids);
  sel.rinv = reinterpret_cast<float*>(base + o_rinv);
  sel.nS = reinterpret_cast<float*>(base + o_nS);
  sel.S = reinterpret_cast<float*>(base + o_S);
  sel.cap = cap;
  float* nE = reinterpret_cast<float*>(base + o_nE);
  int64_t* cp = reinterpret_cast<int64_t*>(base + o_cp);
  uint2* ent = reinterpret_cast<uint2*>(base + o_ent);
  float* K = reinterpret_cast<float*>(base + o_K);
  float* KMp = want_km ? reinterpret_cast<float*>(base + o_KM) : nullptr;

  NearList near;
  near.pairs = reinterpret_cast<uint2*>(base + o_npairs);
  near.count = reinterpret_cast<unsigned*>(base + o_ncnt);
  near.cap = near_cap;
  near.E32 = vecs_dev;
  near.S32 = sel.S;
  near.d = (int)d;

  // The error word and the near-pair counter are the only scratch that must
  // start at zero; every other region is fully written before it is read.
  if (cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess ||
      cudaMemsetAsync(near.count, 0, sizeof(unsigned), st) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(WMD_ERR_CUDA, "cudaMemsetAsync of a scratch counter failed");
  }
  launch_embed_norms(vecs_dev, V, d, nE, st);
  launch_pack_targets(col_ptr_dev, row_inds_dev, vals_dev, V, N, nnz, cp, ent,
                      err, st);
  launch_select(r_dev, V, vecs_dev, nE, d, sel, err, st);
  launch_cdist_fp32(vecs_dev, nE, V, d, sel, expo, K, KMp, ld, near, st);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  launch_near_fixup(near, expo, K, KMp, ld, V, nE, sel.nS, sel.vr, sms, st);
  Targets t;
  t.col_ptr = cp;
  t.ent = ent;
  t.order = nullptr;
  t.N = (int64_t)N;
  t.nnz = (int64_t)nnz;
  SolveCtl ctl;
  ctl.max_iter = max_iter;
  launch_solve(K, KMp, ld, expo, cap, sel, t, ctl, wmd_dev, st);

  unsigned bits = 0;
  cudaError_t e = cudaMemcpyAsync(&bits, err, sizeof(unsigned),
                                  cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaGetLastError();
    snprintf(msg, sizeof(msg), "CUDA error: %s", cudaGetErrorString(e));
    return noalloc_fail(WMD_ERR_CUDA, msg);
  }
  if (bits) {
    snprintf(msg, sizeof(msg),
             "invalid input (device validation bits 0x%x: 1 word index >= V, "
             "2 bad column pointers, 4 negative r, 8 value <= 0, 16 more "
             "non-zeros in r than vr_cap)",
             bits);
    return noalloc_fail(WMD_ERR_INVALID_INPUT, msg);
  }
  wmd::set_last_error("");
  return WMD_OK;
}
