// C ABI (include/wmd_b200.h): handles, device buffers, validation and the
// drop-in replacements of the reference's sinkhorn_wmd.
//
// Every solve runs on the GPU.  There is no host fallback: if the device or a
// kernel launch fails, the call returns an error status.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <random>
#include <vector>

#include <omp.h>

#include <cuda.h>

#include "wmd_b200.h"
#include "wmd_internal.cuh"

using namespace wmd;

namespace {

thread_local std::string g_last_error;

wmd_status fail(wmd_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

wmd_status fail_cuda(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky launch error where possible
  const wmd_status s =
      e == cudaErrorMemoryAllocation ? WMD_ERR_OUT_OF_MEMORY : WMD_ERR_CUDA;
  return fail(s, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return fail_cuda(e_, #call);   \
  } while (0)

// Grow-only pinned host buffer (staging for host -> device copies that run
// while the host keeps working).
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() { release(); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    release();
    const size_t want = bytes ? bytes : 16;
    cudaError_t e = cudaMallocHost(&p, want);
    if (e == cudaSuccess) cap = want;
    else p = nullptr;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = bytes ? bytes : 16;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

std::string describe_err_bits(unsigned bits) {
  std::string s;
  if (bits & ERR_ROW_RANGE) s += " word index >= vocabulary size;";
  if (bits & ERR_COLPTR) s += " column pointers not monotone from 0 to nnz;";
  if (bits & ERR_NEG_R) s += " negative source weight;";
  if (bits & ERR_BAD_VAL) s += " target value <= 0 or not finite;";
  if (bits & ERR_VR_CAP) s += " more non-zero source words than vr_cap;";
  if (bits & ERR_TIMEOUT) s += " device-side wait timed out (kernel aborted);";
  if (bits & ERR_DOC_RANGE) s += " document index >= number of documents;";
  return s;
}

// Everything a captured query graph depends on.
struct QueryKey {
  const void* r = nullptr;
  const void* out = nullptr;
  uint32_t cap = 0;
  float expo = 0.f;
  int max_iter = -1;
  int mode = -1;
  bool timing = false;
  uint64_t epoch = 0;
  float tol = 0.f;
  float omega = 1.f;
  int prec = -1;
  const void* bufs[25] = {};  // every device buffer the graph reads or writes
  bool operator==(const QueryKey& o) const {
    if (!(r == o.r && out == o.out && cap == o.cap && expo == o.expo &&
          max_iter == o.max_iter && mode == o.mode && timing == o.timing &&
          epoch == o.epoch && tol == o.tol && omega == o.omega && prec == o.prec))
      return false;
    for (int i = 0; i < 25; ++i)
      if (bufs[i] != o.bufs[i]) return false;
    return true;
  }
};

}  // namespace

void wmd::set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

struct wmd_handle {
  int device = 0;
  int sms = 0;
  cudaStream_t stream = nullptr;
  wmd_cdist_mode mode = WMD_CDIST_FP32;
  // Storage of the K panel the solve reads for 64 < v_r <= 512 (BF16: the
  // CTA-per-document kernel with the rows staged in shared memory).
  wmd_solve_precision prec = WMD_SOLVE_FP32;
  // Launch-shape autotuner of the block solve: per (panel width, panel
  // beyond L2) the fastest shape measured on this handle's data.
  bool autotune = true;
  int forced_shape = -2;  // wmd_set_block_shape (-2: none)
  int blk_shape[8] = {-2, -2, -2, -2, -2, -2, -2, -2};  // -2: not tuned yet
  // Launch shape of the plain warp solve per lane layout (v_r <= 32, 64, ...,
  // 1024), tuned on this handle's target set; -2: not tuned yet.
  int warp_shape[6] = {-2, -2, -2, -2, -2, -2};
  // Documents longer than the tensor-core solve's capacity, per panel width
  // (-1: not counted yet for this target set).
  int64_t tc_long[4][3] = {{-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}, {-1, -1, -1}};
  // embeddings
  DevBuf E32, nE, E64_stage, E16;
  // Drop-in rows: flags of the needed words and the count of rows read over
  // the bus; pinned staging of the host-narrowed prefix and its device copy.
  DevBuf need, need_count;
  HostBuf hstage;
  DevBuf rows32;
  std::vector<int32_t> ord_host;  // document order of the last target set
  uint64_t dropin_h2d = 0;  // bytes the last drop-in call moved host -> device
  // rows of the last drop-in call narrowed on the host / read by the GPU
  uint64_t dropin_host_rows = 0, dropin_dev_rows = 0;
  uint64_t V = 0, d = 0;
  bool have_E = false;
  int e16_fmt = -1;  // format E16 holds (1 bf16, 2 fp16), -1 = stale
  // Split-FP16 rows of the F16X3 cost panel (tc_split_row_bytes(d) each),
  // built on first use from E32.
  DevBuf Ehl;
  bool ehl_ready = false;
  // targets
  DevBuf col_ptr, ent, order, stage_cp, stage_rows, stage_vals;
  DevBuf edge_words, edge_docs, edge_w, edge_temp;  // edge-list CSC build
  uint64_t tV = 0, N = 0, nnz = 0;
  bool have_T = false;
  // per query
  DevBuf r_dev, sel_ids, sel_rinv, sel_S, sel_nS, sel_S16, sel_vr, sel_chunks,
      K, KM, K16, out_dev, err_dev, near_pairs, near_count, iters;
  DevBuf vstate;  // each target word's previous v (over-relaxed solves)
  // Row-scaled panels (panel_rescale.cu): row minima of M per query, and the
  // largest squared embedding norm, which decides when they are needed.
  DevBuf mrow, emax_dev;
  float emax2 = 0.f;
  DevBuf exact_list, exact_count;  // documents re-solved in FP64 (exact_f64.cu)
  // Word-major solve order (solve_word.cu): the target set as word-major CSR
  // (built on first use per target set) and the u / x state it streams.
  int solve_order = 0;  // 0 document-major, 1 word-major
  // Stacked batch groups (batch.cu): on/off, device memory budget of one
  // group's panels, their pools and tables, and the tuned launch shape of the
  // stacked block solve per BF16 panel width.
  bool stacked = true;
  uint64_t group_budget = 32ull << 30;
  DevBuf g_pool, g_pool16, g_vst, g_S, g_nS, g_S16, g_rowword, g_rowsrc, g_tiles, g_src;
  int grp_shape[4] = {-2, -2, -2, -2};
  int wgrp_shape[6] = {-2, -2, -2, -2, -2, -2};  // stacked warp solve, per lane layout
  int last_groups = 0;
  bool wm_ready = false;
  DevBuf wm_rp, wm_ent, wm_u, wm_x;
  // batched queries
  DevBuf b_ids, b_rinv, b_vr, b_out, b_iters;
  // Second pipeline slot of the batched queries (its own stream and
  // per-source scratch): consecutive sources alternate between the slots, so
  // one source's solve tail overlaps the next source's cost panel and solve.
  struct BatchSlot {
    DevBuf sel_S, sel_nS, sel_S16, near_pairs, near_count, K, KM, K16, vstate,
        ws_Asrc, ws_u0, ws_stats, mrow, exact_list, exact_count;
  } slot1;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t join[2] = {nullptr, nullptr};
  // top-k
  DevBuf topk_scratch, topk_idx, topk_val;
  // learned warm start: model (FP32 parameters, folded inference form),
  // per-target-set tables, per-query scratch
  DevBuf ws_params, ws_folded, ws_C, ws_Bdoc, ws_Asrc, ws_u0, ws_stats;
  bool ws_on = false;       // queries start from the model's prediction
  bool ws_docs_ready = false;  // ws_C / ws_Bdoc match targets + model
  int ws_d = 0;
  // warm-start training set (standardised rows, labels, group pointers)
  DevBuf ws_X, ws_y, ws_gptr;
  std::vector<int64_t> ws_gptr_host;
  std::vector<uint32_t> ws_gsrc, ws_gdoc;  // per group: source index, document
  std::vector<int32_t> ws_rword;           // per row: source word index
  std::vector<float> ws_shift, ws_scale;
  int64_t ws_rows = 0;
  std::vector<uint32_t> doc_len;  // host copy of the target lengths
  float tol = 0.f;  // per-document convergence tolerance (0: fixed count)
  float omega = 1.f;  // over-relaxation of the u update (1: reference)
  unsigned* err_host = nullptr;      // pinned
  uint32_t* chunks_host = nullptr;   // pinned, grown with V
  size_t chunks_host_cap = 0;
  int last_launches = 0;
  // stage timing
  bool timing = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_split = nullptr;  // drop-in: host-row copies done (stream2)
  cudaEvent_t ev_slot[4] = {nullptr, nullptr, nullptr, nullptr};  // staging slots free
  // CUDA-graph replay of device queries; graph_epoch changes whenever a
  // buffer or setting a captured graph depends on changes.
  bool use_graphs = true;
  uint64_t graph_epoch = 0;
  QueryKey seen_key, graph_key;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_launches = 0;
};

namespace {

wmd_status bind(wmd_handle* h) {
  CK(cudaSetDevice(h->device));
  return WMD_OK;
}

wmd_status clear_err(wmd_handle* h) {
  CK(cudaMemsetAsync(h->err_dev.p, 0, sizeof(unsigned), h->stream));
  return WMD_OK;
}

// Synchronise and turn device-side validation bits into a status.
wmd_status finish(wmd_handle* h) {
  CK(cudaMemcpyAsync(h->err_host, h->err_dev.p, sizeof(unsigned),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  const unsigned bits = *h->err_host;
  if (bits) {
    clear_err(h);
    if (bits & ERR_TIMEOUT)
      return fail(WMD_ERR_DEVICE_TIMEOUT, "device error:" + describe_err_bits(bits));
    return fail(WMD_ERR_INVALID_INPUT, "invalid input:" + describe_err_bits(bits));
  }
  return WMD_OK;
}

uint32_t max_doc_len(const wmd_handle* h) {
  uint32_t m = 0;
  for (uint32_t l : h->doc_len) m = std::max(m, l);
  return m;
}

// Largest squared row norm of the embeddings now on the device (synchronises
// the handle's stream once; embeddings are set far less often than queried).
wmd_status update_emax(wmd_handle* h, uint64_t V) {
  CK(h->emax_dev.ensure(sizeof(unsigned)));
  launch_max_norm(h->nE.as<float>(), V, h->emax_dev.as<unsigned>(), h->stream);
  unsigned bits = 0;
  CK(cudaMemcpyAsync(&bits, h->emax_dev.p, sizeof(unsigned), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  memcpy(&h->emax2, &bits, sizeof(float));
  return WMD_OK;
}

// Whether a query with this exponent needs the row-scaled panel: lambda * M
// can exceed kScaleLimit (M <= 2 max |E_w|; FP32 exp underflows near 87).
bool row_scaled(const wmd_handle* h, float expo) {
  return expo != 0.f && -expo * 2.f * sqrtf(h->emax2) > kScaleLimit;
}

wmd_status set_embeddings(wmd_handle* h, const void* vecs, uint64_t V,
                          uint64_t d, int where, bool f64) {
  if (!h || !vecs || V == 0 || d == 0 || (where != 0 && where != 1))
    return fail(WMD_ERR_INVALID_ARG, "set_embeddings: bad argument");
  if (V > 0xFFFFFFFFull)
    return fail(WMD_ERR_UNSUPPORTED, "vocabulary larger than 2^32 words");
  if (d > 65536) return fail(WMD_ERR_UNSUPPORTED, "embedding width above 65536");
  wmd_status s = bind(h);
  if (s) return s;
  const size_t n = (size_t)V * d;
  CK(h->E32.ensure(n * sizeof(float)));
  CK(h->nE.ensure((size_t)V * sizeof(float)));
  int launches = 0;
  if (f64) {
    const double* src = static_cast<const double*>(vecs);
    if (where == 0) {
      CK(h->E64_stage.ensure(n * sizeof(double)));
      CK(cudaMemcpyAsync(h->E64_stage.p, vecs, n * sizeof(double),
                         cudaMemcpyHostToDevice, h->stream));
      src = h->E64_stage.as<double>();
    }
    launches += launch_embed_convert_f64(src, V, d, h->E32.as<float>(),
                                         h->nE.as<float>(), h->stream);
  } else {
    CK(cudaMemcpyAsync(h->E32.p, vecs, n * sizeof(float),
                       where == 0 ? cudaMemcpyHostToDevice
                                  : cudaMemcpyDeviceToDevice,
                       h->stream));
    launches += launch_embed_norms(h->E32.as<float>(), V, d, h->nE.as<float>(),
                                   h->stream);
  }
  s = update_emax(h, V);
  if (s) return s;
  launches += 1;
  CK(cudaGetLastError());
  h->V = V;
  h->d = d;
  h->have_E = true;
  h->e16_fmt = -1;
  h->ehl_ready = false;
  h->ws_docs_ready = false;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  h->graph_epoch++;
  h->last_launches = launches;
  return WMD_OK;
}

// Host-side permutation of the documents by decreasing length (a counting
// sort on lengths), used by the solver to balance its persistent warps.
void length_order(const uint64_t* col_ptr, uint64_t N, std::vector<int32_t>& ord) {
  uint64_t maxlen = 0;
  for (uint64_t j = 0; j < N; ++j) maxlen = std::max(maxlen, col_ptr[j + 1] - col_ptr[j]);
  const uint64_t nb = std::min<uint64_t>(maxlen, 1u << 20) + 1;
  std::vector<uint64_t> cnt(nb + 1, 0);
  auto bucket = [&](uint64_t j) {
    const uint64_t l = col_ptr[j + 1] - col_ptr[j];
    return nb - 1 - std::min<uint64_t>(l, nb - 1);  // longest first
  };
  for (uint64_t j = 0; j < N; ++j) cnt[bucket(j) + 1]++;
  for (uint64_t b = 0; b < nb; ++b) cnt[b + 1] += cnt[b];
  ord.resize(N);
  for (uint64_t j = 0; j < N; ++j) ord[cnt[bucket(j)]++] = (int32_t)j;
}

// defer_check: return once the copies and the packing are enqueued; the
// caller synchronises later with finish(h) (which reports invalid indices or
// values) and may only enqueue work that tolerates unchecked word ids until
// then.
wmd_status set_targets_csc(wmd_handle* h, const wmd_csc_double_t* c,
                           bool defer_check = false) {
  if (!h || !c) return fail(WMD_ERR_INVALID_ARG, "set_targets: null argument");
  const uint64_t V = c->num_rows, N = c->num_cols, nnz = c->nnz;
  if (V == 0 || N == 0)
    return fail(WMD_ERR_INVALID_INPUT, "target matrix has no rows or columns");
  if (nnz == 0)  // the reference driver rejects an empty matrix (fused:431-435)
    return fail(WMD_ERR_INVALID_INPUT, "target matrix has no non-zeros");
  if (!c->col_ptr || !c->row_inds || !c->vals)
    return fail(WMD_ERR_INVALID_ARG, "target matrix has null arrays");
  if (N >= 0x7FFFFFFFull)
    return fail(WMD_ERR_UNSUPPORTED, "more than 2^31-1 target documents");
  if (c->col_ptr[N] != nnz || c->col_ptr[0] != 0)
    return fail(WMD_ERR_INVALID_INPUT, "column pointers do not span [0, nnz]");
  for (uint64_t j = 0; j < N; ++j)
    if (c->col_ptr[j + 1] < c->col_ptr[j])
      return fail(WMD_ERR_INVALID_INPUT, "column pointers decrease");
  wmd_status s = bind(h);
  if (s) return s;
  std::vector<int32_t>& ord = h->ord_host;  // outlives its async copy
  length_order(c->col_ptr, N, ord);
  CK(h->stage_cp.ensure((N + 1) * sizeof(uint64_t)));
  CK(h->stage_rows.ensure(nnz * sizeof(uint64_t)));
  CK(h->stage_vals.ensure(nnz * sizeof(double)));
  CK(h->col_ptr.ensure((N + 1) * sizeof(int64_t)));
  CK(h->ent.ensure(nnz * sizeof(uint2)));
  CK(h->order.ensure(N * sizeof(int32_t)));
  CK(cudaMemcpyAsync(h->stage_cp.p, c->col_ptr, (N + 1) * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->stage_rows.p, c->row_inds, nnz * sizeof(uint64_t),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->stage_vals.p, c->vals, nnz * sizeof(double),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->order.p, ord.data(), N * sizeof(int32_t),
                     cudaMemcpyHostToDevice, h->stream));
  s = clear_err(h);
  if (s) return s;
  const int launches = launch_pack_targets(
      h->stage_cp.as<uint64_t>(), h->stage_rows.as<uint64_t>(),
      h->stage_vals.as<double>(), V, N, nnz, h->col_ptr.as<int64_t>(),
      h->ent.as<uint2>(), h->err_dev.as<unsigned>(), h->stream);
  CK(cudaGetLastError());
  h->have_T = false;
  if (!defer_check) {
    s = finish(h);
    if (s) return s;
  }
  h->tV = V;
  h->N = N;
  h->nnz = nnz;
  h->have_T = true;
  h->wm_ready = false;
  h->ws_docs_ready = false;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  for (auto& row : h->tc_long)
    for (int64_t& x : row) x = -1;
  h->doc_len.resize(N);
  for (uint64_t j = 0; j < N; ++j) h->doc_len[j] = (uint32_t)(c->col_ptr[j + 1] - c->col_ptr[j]);
  h->graph_epoch++;
  h->last_launches = launches;
  return WMD_OK;
}

// Stable CSR (rows = words) -> CSC (columns = documents) transpose, the
// counting sort of sinkhorn_wmd_fused.cpp:493-506 keyed by document: within a
// document, entries come out in ascending word order (equal words keep their
// CSR order), which is the order the reference accumulates in on one thread.
wmd_status csr_to_csc_host(const wmd_csr_double_t* a, std::vector<uint64_t>& cp,
                           std::vector<uint64_t>& rows, std::vector<double>& vals) {
  const uint64_t V = a->num_rows, N = a->num_cols, nnz = a->nnz;
  if (!a->row_ptr || !a->col_inds || !a->vals)
    return fail(WMD_ERR_INVALID_ARG, "target matrix has null arrays");
  if (a->row_ptr[0] != 0 || a->row_ptr[V] != nnz)
    return fail(WMD_ERR_INVALID_INPUT, "row pointers do not span [0, nnz]");
  cp.assign(N + 1, 0);
  for (uint64_t w = 0; w < V; ++w) {
    if (a->row_ptr[w + 1] < a->row_ptr[w])
      return fail(WMD_ERR_INVALID_INPUT, "row pointers decrease");
  }
  for (uint64_t e = 0; e < nnz; ++e) {
    const uint64_t j = a->col_inds[e];
    if (j >= N) return fail(WMD_ERR_INVALID_INPUT, "document index >= num_cols");
    cp[j + 1]++;
  }
  for (uint64_t j = 0; j < N; ++j) cp[j + 1] += cp[j];
  std::vector<uint64_t> fill(cp.begin(), cp.end() - 1);
  rows.resize(nnz);
  vals.resize(nnz);
  for (uint64_t w = 0; w < V; ++w)
    for (uint64_t e = a->row_ptr[w]; e < a->row_ptr[w + 1]; ++e) {
      const uint64_t pos = fill[a->col_inds[e]]++;
      rows[pos] = w;
      vals[pos] = a->vals[e];
    }
  return WMD_OK;
}

// Documents of the target set longer than the tensor-core solve holds (they
// come first in the length order).
int64_t tc_long_count(wmd_handle* h, int ld16, int shape) {
  const int w = (ld16 / 128 - 1) & 3, k = shape - 3;
  if (h->tc_long[w][k] >= 0) return h->tc_long[w][k];
  const uint32_t cap = (uint32_t)tc_solve_capacity(ld16, 1 << k);
  int64_t c = 0;
  for (uint32_t l : h->doc_len) c += l > cap ? 1 : 0;
  h->tc_long[w][k] = c;
  return c;
}

// The block solve in launch shape `shape` (3-5: tensor cores with 1, 2 or 4
// CTAs per SM for the documents that fit, the build-time CUDA-core shape
// for the longer ones).
int launch_block_shape(wmd_handle* h, const void* K16, int ld16, float expo,
                       uint32_t vr, const SourceSel& sel, const Targets& t,
                       const SolveCtl& ctl, const float* u0, int64_t ldu,
                       double* out, int shape, cudaStream_t st) {
  if (shape >= 3 && shape <= 5)
    return launch_solve_tc(K16, ld16, expo, vr, sel, t, ctl, u0, ldu, out, st,
                           1 << (shape - 3), tc_long_count(h, ld16, shape));
  return launch_solve_block(K16, ld16, expo, vr, sel, t, ctl, u0, ldu, out, st, shape);
}
int launch_block_shape(wmd_handle* h, const void* K16, int ld16, float expo,
                       uint32_t vr, const SourceSel& sel, const Targets& t,
                       const SolveCtl& ctl, const float* u0, int64_t ldu,
                       double* out, int shape) {
  return launch_block_shape(h, K16, ld16, expo, vr, sel, t, ctl, u0, ldu, out, shape,
                            h->stream);
}

// Autotuner cache slot of a panel width (and whether the panel is beyond L2),
// and whether the shape for it is settled (pinned, tuning off, or tuned).
int block_shape_key(const wmd_handle* h, int ld16) {
  return ((ld16 / 128 - 1) & 3) * 2 + ((size_t)h->V * ld16 * 2 > (64u << 20) ? 1 : 0);
}
bool block_shape_known(const wmd_handle* h, int ld16) {
  return h->forced_shape != -2 || !h->autotune || h->blk_shape[block_shape_key(h, ld16)] != -2;
}

// Launch shape of the block solve for this panel: cached per (width, panel
// beyond L2); when not yet known and the call may synchronise, every
// candidate shape is timed on the real panel and target set (4 updates, CUDA
// events) and the fastest is kept.  Returns -1 (build-time default) when
// tuning is off or impossible (inside a graph capture).
int block_shape_for(wmd_handle* h, const void* K16, int ld16, float expo,
                    uint32_t vr, const SourceSel& sel, const Targets& t,
                    const SolveCtl& ctl, double* out, bool can_sync) {
  if (h->forced_shape != -2) return h->forced_shape;
  const int key = block_shape_key(h, ld16);
  if (h->blk_shape[key] != -2) return h->blk_shape[key];
  if (!h->autotune || !can_sync) return -1;
  SolveCtl c2 = ctl;
  c2.max_iter = 4;
  c2.tol = 0.f;
  c2.iters = nullptr;
  c2.u0 = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    return -1;
  }
  float best = 1e30f;
  int bi = -1;
  for (int sh = 0; sh < block_shape_count(); ++sh) {
    if (launch_block_shape(h, K16, ld16, expo, vr, sel, t, c2, nullptr, 0, out, sh) < 0)
      continue;  // shape unavailable (shared-memory budget)
    cudaEventRecord(a, h->stream);
    launch_block_shape(h, K16, ld16, expo, vr, sel, t, c2, nullptr, 0, out, sh);
    cudaEventRecord(b, h->stream);
    float ms = 0.f;
    if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess &&
        ms < best) {
      best = ms;
      bi = sh;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  h->blk_shape[key] = bi;
  return bi;
}

// Launch shape of the plain warp solve for sources of up to `cap` words,
// cached per lane layout; when not yet known and the call may synchronise,
// each candidate (warps per CTA x CTAs per SM) is timed on the real panel and
// target set (the query's update count, at most 15; CUDA events) and the
// fastest is kept.  -1: the
// build-time default (tuning off, inside a capture, or not a plain solve).
int warp_shape_for(wmd_handle* h, const float* K, int ld, float expo, uint32_t cap,
                   const SourceSel& sel, const Targets& t, const SolveCtl& ctl,
                   double* out, bool can_sync) {
  if (ctl.omega != 1.f || expo == 0.f) return -1;
  int k = 0;
  while (k < 5 && (32u << k) < cap) ++k;
  if (h->warp_shape[k] != -2) return h->warp_shape[k];
  if (!h->autotune || !can_sync) return -1;
  // The query's own update count (at most 15): the shapes rank differently
  // for the per-launch part (row gathers, final half-step) and the
  // per-update part, so a short tuning launch can pick the wrong one.
  SolveCtl c2 = ctl;
  c2.max_iter = std::min(std::max(ctl.max_iter, 1), 15);
  c2.tol = 0.f;
  c2.iters = nullptr;
  c2.u0 = nullptr;
  c2.mrow = nullptr;
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    return -1;
  }
  // The candidates differ by a few percent of a launch, near the event
  // clock's resolution for one launch: each is timed over kRuns groups of
  // kPer launches, the groups of the candidates interleaved.
  constexpr int kMaxShapes = 8, kRuns = 3, kPer = 2;
  const int ns = std::min(solve_shape_count(), kMaxShapes);
  float tot[kMaxShapes];
  bool ok[kMaxShapes];
  for (int sh = 0; sh < ns; ++sh) {
    tot[sh] = 0.f;
    ok[sh] = launch_solve(K, nullptr, ld, expo, cap, sel, t, c2, out, h->stream, sh) >= 0;
  }
  for (int run = 0; run < kRuns; ++run)
    for (int sh = 0; sh < ns; ++sh) {
      if (!ok[sh]) continue;
      cudaEventRecord(a, h->stream);
      for (int i = 0; i < kPer; ++i)
        launch_solve(K, nullptr, ld, expo, cap, sel, t, c2, out, h->stream, sh);
      cudaEventRecord(b, h->stream);
      float ms = 0.f;
      if (cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
        tot[sh] += ms;
      else
        ok[sh] = false;
    }
  float best = 1e30f;
  int bi = -1;
  for (int sh = 0; sh < ns; ++sh)
    if (ok[sh] && tot[sh] < best) {
      best = tot[sh];
      bi = sh;
    }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  h->warp_shape[k] = bi;
  return bi;
}

// Warm start: target centroids and the per-document first-layer terms of the
// current model (recomputed after the targets, embeddings or model change).
wmd_status ws_prepare_docs(wmd_handle* h) {
  if (h->ws_docs_ready) return WMD_OK;
  const WsLayout L = ws_layout((int)h->d);
  CK(h->ws_C.ensure((size_t)h->N * h->d * sizeof(float)));
  CK(h->ws_Bdoc.ensure((size_t)h->N * kWsH * sizeof(float)));
  launch_centroids(h->E32.as<float>(), (int)h->d, h->col_ptr.as<int64_t>(),
                   h->ent.as<uint2>(), (int64_t)h->N, h->ws_C.as<float>(), h->stream);
  launch_ws_doc_bias(L, h->ws_folded.as<float>(), h->ws_C.as<float>(), (int64_t)h->N,
                     h->ws_Bdoc.as<float>(), h->stream);
  CK(cudaGetLastError());
  h->ws_docs_ready = true;
  return WMD_OK;
}

// Word-major CSR of the resident target set (stable: documents ascending
// within a word), from the device's document-major entries; once per target
// set, synchronising.
wmd_status build_word_major(wmd_handle* h) {
  const uint64_t N = h->N, nnz = h->nnz, V = h->tV;
  std::vector<int64_t> cp(N + 1);
  std::vector<uint2> ent(nnz);
  CK(cudaMemcpyAsync(cp.data(), h->col_ptr.p, (N + 1) * 8, cudaMemcpyDeviceToHost, h->stream));
  if (nnz)
    CK(cudaMemcpyAsync(ent.data(), h->ent.p, nnz * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  std::vector<int64_t> rp(V + 1, 0);
  for (uint64_t e = 0; e < nnz; ++e) rp[ent[e].x + 1]++;
  for (uint64_t w = 0; w < V; ++w) rp[w + 1] += rp[w];
  std::vector<int64_t> pos(rp.begin(), rp.end() - 1);
  std::vector<uint2> went(std::max<uint64_t>(nnz, 1));
  for (uint64_t j = 0; j < N; ++j)
    for (int64_t e = cp[j]; e < cp[j + 1]; ++e)
      went[pos[ent[e].x]++] = make_uint2((unsigned)j, ent[e].y);
  CK(h->wm_rp.ensure((V + 1) * 8));
  CK(h->wm_ent.ensure(std::max<uint64_t>(nnz, 1) * 8));
  CK(cudaMemcpyAsync(h->wm_rp.p, rp.data(), (V + 1) * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->wm_ent.p, went.data(), std::max<uint64_t>(nnz, 1) * 8,
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));  // the host vectors go out of scope
  h->wm_ready = true;
  h->graph_epoch++;
  return WMD_OK;
}

// One query on device-resident r.  cap bounds v_r.  expo: K = exp(expo * M).
wmd_status query_device(wmd_handle* h, const double* r_dev, uint32_t cap,
                        float expo, int max_iter, double* out_dev) {
  const uint64_t V = h->V, d = h->d;
  const bool word_major = h->solve_order == 1;
  if (word_major) {
    if (h->tol > 0.f || h->omega != 1.f || h->ws_on || expo == 0.f)
      return fail(WMD_ERR_UNSUPPORTED, "the word-major order runs the fixed update "
                                       "count from the cold start, unrelaxed, lambda != 0");
    if (!h->wm_ready) {
      wmd_status sw = build_word_major(h);
      if (sw) return sw;
    }
  }
  const int nchunks = select_num_chunks(V);
  const int ld = (int)(((cap ? cap : 1) + 3u) & ~3u);
  CK(h->sel_ids.ensure((size_t)std::max<uint32_t>(cap, 1) * sizeof(uint32_t)));
  CK(h->sel_rinv.ensure((size_t)std::max<uint32_t>(cap, 1) * sizeof(float)));
  CK(h->sel_S.ensure((size_t)std::max<uint32_t>(cap, 1) * d * sizeof(float)));
  CK(h->sel_nS.ensure((size_t)std::max<uint32_t>(cap, 1) * sizeof(float)));
  CK(h->sel_vr.ensure(sizeof(uint32_t)));
  CK(h->sel_chunks.ensure((size_t)nchunks * sizeof(uint32_t)));
  CK(h->K.ensure((size_t)V * ld * sizeof(float)));
  // K.*M is stored only for expo = 0; otherwise the solve derives it from K.
  const bool need_km = expo == 0.f;
  if (need_km) CK(h->KM.ensure((size_t)V * ld * sizeof(float)));
  float* KMp = need_km ? h->KM.as<float>() : nullptr;
  // The row-scaled form (lambda * M beyond FP32's range) keeps the FP32
  // panel: BF16 rounding of K' is amplified there.
  const int ld16 = h->prec == WMD_SOLVE_BF16 && !need_km && !word_major &&
                           !row_scaled(h, expo)
                       ? block_panel_width(cap) : 0;
  if (ld16) CK(h->K16.ensure((size_t)V * ld16 * 2));
  if (word_major) {
    CK(h->wm_u.ensure((size_t)std::max<uint64_t>(h->N, 1) * ld * sizeof(float)));
    CK(h->wm_x.ensure((size_t)std::max<uint64_t>(h->N, 1) * ld * sizeof(float)));
  }
  SourceSel sel;
  sel.ids = h->sel_ids.as<uint32_t>();
  sel.rinv = h->sel_rinv.as<float>();
  sel.S = h->sel_S.as<float>();
  sel.nS = h->sel_nS.as<float>();
  sel.vr = h->sel_vr.as<uint32_t>();
  sel.chunk_counts = h->sel_chunks.as<uint32_t>();
  sel.cap = cap;
  Targets t;
  t.col_ptr = h->col_ptr.as<int64_t>();
  t.ent = h->ent.as<uint2>();
  t.order = h->order.as<int32_t>();
  t.N = (int64_t)h->N;
  t.nnz = (int64_t)h->nnz;
  if (cap > 1024)
    return fail(WMD_ERR_UNSUPPORTED, "more than 1024 non-zero source words");
  const bool tcm = h->mode == WMD_CDIST_BF16 || h->mode == WMD_CDIST_FP16;
  const bool bf16 = h->mode == WMD_CDIST_BF16;
  // Split-FP16 form; where it cannot tile, the split-TF32 form; widths
  // neither tiles use the FP32 CUDA-core panel.
  const bool h2 = h->mode == WMD_CDIST_F16X3 && tc_tile_n_h2(cap, d) != 0;
  const bool x3 = !h2 && (h->mode == WMD_CDIST_TF32X3 || h->mode == WMD_CDIST_F16X3) &&
                  tc_tile_n_x3(cap, d) != 0;
  const int dp = tc_padded_width(d);
  const size_t rs = tc_split_row_bytes(d);
  int launches = 0;
  if (h2) {
    if (!h->ehl_ready) {  // split rows of the embeddings, built once
      CK(h->Ehl.ensure((size_t)V * rs));
      launches += launch_to_split16(h->E32.as<float>(), V, d, h->Ehl.p, h->stream);
      h->ehl_ready = true;
    }
    CK(h->sel_S16.ensure((size_t)std::max<uint32_t>(cap, 1) * rs));
  }
  if (tcm) {
    if (tc_tile_n(cap, d) == 0)
      return fail(WMD_ERR_UNSUPPORTED, "embedding width too large for the tensor-core panel");
    const int fmt = bf16 ? 1 : 2;
    if (h->e16_fmt != fmt) {  // 16-bit copy of the embeddings, built once
      CK(h->E16.ensure((size_t)V * dp * 2));
      launches += launch_to16(h->E32.as<float>(), V, d, h->E16.p, bf16, h->stream);
      h->e16_fmt = fmt;
    }
    CK(h->sel_S16.ensure((size_t)std::max<uint32_t>(cap, 1) * dp * 2));
  }
  // Near-pair list for the exact fix-up of cancellation-prone entries.
  const unsigned near_cap = (unsigned)std::min<uint64_t>(
      (uint64_t)V * std::max<uint32_t>(cap, 1), 1u << 20);
  CK(h->near_pairs.ensure((size_t)near_cap * sizeof(uint2)));
  CK(h->near_count.ensure(sizeof(unsigned)));
  CK(h->iters.ensure((size_t)std::max<uint64_t>(h->N, 1) * sizeof(int)));
  if (h->omega != 1.f)
    CK(h->vstate.ensure((size_t)std::max<uint64_t>(h->nnz, 1) * sizeof(float)));
  NearList near;
  near.pairs = h->near_pairs.as<uint2>();
  near.count = h->near_count.as<unsigned>();
  near.cap = near_cap;
  near.E32 = h->E32.as<float>();
  near.S32 = sel.S;
  near.d = (int)d;
  // Row-scaled panel when lambda * M can underflow FP32 (panel_rescale.cu).
  float* mrow = nullptr;
  const int mdl = (int)max_doc_len(h);
  if (row_scaled(h, expo)) {
    CK(h->mrow.ensure((size_t)V * sizeof(float)));
    CK(h->exact_list.ensure(exact_f64_list_cap() * sizeof(int32_t)));
    CK(h->exact_count.ensure(sizeof(unsigned)));
    mrow = h->mrow.as<float>();
  }
  // Learned warm start (needs lambda != 0: its features read M = ln K / expo).
  const bool ws = h->ws_on && h->ws_d == (int)d && expo != 0.f;
  if (ws) {
    wmd_status sw = ws_prepare_docs(h);
    if (sw) return sw;
    CK(h->ws_Asrc.ensure((size_t)std::max<uint32_t>(cap, 1) * kWsH * sizeof(float)));
    CK(h->ws_u0.ensure((size_t)std::max<uint64_t>(h->N, 1) * ld * sizeof(float)));
    CK(h->ws_stats.ensure((size_t)std::max<uint64_t>(h->N, 1) * std::max<uint32_t>(cap, 1) *
                          3 * sizeof(float)));
  }
  // Everything below is stream work only (no allocation, no host sync), so
  // it can be captured into a CUDA graph and replayed.
  auto record = [&](int i, bool capturing) -> cudaError_t {
    if (!h->timing) return cudaSuccess;
    return capturing ? cudaEventRecordWithFlags(h->ev[i], h->stream,
                                                cudaEventRecordExternal)
                     : cudaEventRecord(h->ev[i], h->stream);
  };
  auto enqueue = [&](bool capturing, int* nlaunch) -> wmd_status {
    int n = 0;
    CK(record(0, capturing));
    // (the split form's source rows are whole split rows: rs / 2 halves)
    n += launch_select(r_dev, V, h->E32.as<float>(), h->nE.as<float>(), d, sel,
                       h->err_dev.as<unsigned>(), h->stream,
                       tcm ? h->E16.p : h2 ? h->Ehl.p : nullptr,
                       tcm || h2 ? h->sel_S16.p : nullptr, h2 ? (int)(rs / 2) : dp,
                       near.count);  // the selection also zeroes the near-pair count
    CK(record(1, capturing));
    if (mrow) CK(cudaMemsetAsync(mrow, 0x7f, (size_t)V * sizeof(float), h->stream));
    if (tcm || x3 || h2) {
      const int lc = launch_cdist_tc(h2 ? TC_F16X3 : x3 ? TC_TF32X3 : bf16 ? TC_BF16 : TC_FP16,
                                     h2 ? h->Ehl.p : h->E16.p, h->sel_S16.p,
                                     h->E32.as<float>(), h->nE.as<float>(), V, d,
                                     sel, expo, h->K.as<float>(), KMp, ld, near,
                                     h->err_dev.as<unsigned>(), h->sms, h->stream, mrow);
      if (lc < 0)
        return fail(WMD_ERR_UNSUPPORTED, "tensor-core cost panel unavailable "
                                         "(tensor map encoding failed)");
      n += lc;
    } else {
      n += launch_cdist_fp32(h->E32.as<float>(), h->nE.as<float>(), V, d, sel,
                             expo, h->K.as<float>(), KMp, ld, near, h->stream, mrow);
    }
    n += launch_near_fixup(near, expo, h->K.as<float>(), KMp, ld, V,
                           h->nE.as<float>(), sel.nS, sel.vr, h->sms, h->stream,
                           mrow != nullptr);
    if (mrow)
      n += launch_panel_rescale(h->K.as<float>(), ld, V, sel.vr, mrow, expo, h->sms,
                                h->stream);
    SolveCtl ctl;
    ctl.mrow = mrow;
    ctl.max_iter = max_iter;
    ctl.tol = h->tol;
    ctl.iters = h->iters.as<int>();
    ctl.omega = h->tol > 0.f ? h->omega : 1.f;  // relaxation needs stopping
    ctl.vstate = ctl.omega != 1.f ? h->vstate.as<float>() : nullptr;
    if (ws) {
      n += launch_ws_init(ws_layout((int)d), h->ws_folded.as<float>(),
                          h->ws_params.as<float>(), sel.S, sel.rinv, (int)cap,
                          h->K.as<float>(), ld, expo, t, h->ws_Bdoc.as<float>(),
                          h->ws_Asrc.as<float>(), h->ws_u0.as<float>(), ld,
                          h->err_dev.as<unsigned>(), h->sms, h->stream, mrow,
                          h->ws_stats.as<float>());
      ctl.u0 = h->ws_u0.as<float>();
      ctl.ldu = ld;
    }
    CK(record(2, capturing));
    if (word_major) {
      WordMajor wm;
      wm.row_ptr = h->wm_rp.as<int64_t>();
      wm.ent = h->wm_ent.as<uint2>();
      wm.V = (int64_t)V;
      wm.nnz = (int64_t)h->nnz;
      wm.mrow = mrow;
      const int lw = launch_solve_word(h->K.as<float>(), ld, expo, cap, sel, wm,
                                       (int64_t)h->N, max_iter, h->wm_u.as<float>(),
                                       h->wm_x.as<float>(), h->sms, out_dev, h->stream);
      if (lw < 0) return fail(WMD_ERR_UNSUPPORTED, "more than 1024 source words");
      n += lw;
    } else if (ld16) {
      n += launch_panel_to_bf16(h->K.as<float>(), ld, h->K16.p, ld16, V, sel.vr,
                                h->sms, h->stream);
      const int shape = block_shape_for(h, h->K16.p, ld16, expo, cap, sel, t, ctl,
                                        out_dev, !capturing);
      const int ls = launch_block_shape(h, h->K16.p, ld16, expo, cap, sel, t, ctl,
                                        ctl.u0, ctl.ldu, out_dev, shape);
      if (ls < 0) return fail(WMD_ERR_UNSUPPORTED, "block solve unavailable");
      n += ls;
    } else {
      const int shape = KMp ? -1 : warp_shape_for(h, h->K.as<float>(), ld, expo, cap, sel,
                                                  t, ctl, out_dev, !capturing);
      n += launch_solve(h->K.as<float>(), KMp, ld, expo, cap, sel, t, ctl,
                        out_dev, h->stream, shape);
    }
    if (mrow) {  // documents the row-scaled FP32 panel cannot carry, in FP64
      const int le = launch_exact_f64(h->E32.as<float>(), d, sel, t, expo, ctl, mdl,
                                      h->exact_list.as<int32_t>(),
                                      h->exact_count.as<unsigned>(), h->sms, out_dev,
                                      h->stream);
      if (le < 0) return fail(WMD_ERR_UNSUPPORTED, "documents too long for the FP64 re-solve");
      n += le;
    }
    CK(record(3, capturing));
    CK(cudaGetLastError());
    *nlaunch = n;
    return WMD_OK;
  };

  // Graph replay: the first call with a configuration runs eagerly (it also
  // warms per-device launch caches), the second is captured and
  // instantiated, later ones replay the instantiated graph.
  QueryKey key;
  key.r = r_dev;
  key.out = out_dev;
  key.cap = cap;
  key.expo = expo;
  key.max_iter = max_iter;
  key.mode = (int)h->mode;
  key.timing = h->timing;
  key.epoch = h->graph_epoch;
  key.tol = h->tol;
  key.omega = h->omega;
  key.prec = (int)h->prec + (ws ? 2 : 0);
  {
    const DevBuf* used[25] = {&h->E32, &h->nE, &h->E16, &h->sel_ids, &h->sel_rinv,
                              &h->sel_S, &h->sel_nS, &h->sel_S16, &h->K, &h->KM,
                              &h->near_pairs, &h->sel_chunks, &h->iters, &h->K16,
                              &h->ws_Asrc, &h->ws_u0, &h->vstate, &h->mrow,
                              &h->ws_stats, &h->exact_list, &h->exact_count,
                              &h->wm_u, &h->wm_x, &h->wm_ent, &h->Ehl};
    for (int i = 0; i < 25; ++i) key.bufs[i] = used[i]->p;
    key.prec += word_major ? 16 : 0;
  }
  if (!h->use_graphs) {
    int n = 0;
    wmd_status st = enqueue(false, &n);
    h->last_launches = launches + n;
    return st;
  }
  if (h->graph_exec && h->graph_key == key) {
    CK(cudaGraphLaunch(h->graph_exec, h->stream));
    h->last_launches = launches + h->graph_launches;
    return WMD_OK;
  }
  if (!(h->seen_key == key)) {
    h->seen_key = key;
    int n = 0;
    wmd_status st = enqueue(false, &n);
    h->last_launches = launches + n;
    return st;
  }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
  }
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int n = 0;
  wmd_status st = enqueue(true, &n);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
  if (st != WMD_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  CK(ce);
  const cudaError_t ie = cudaGraphInstantiate(&h->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  CK(ie);
  h->graph_key = key;
  h->graph_launches = n;
  CK(cudaGraphLaunch(h->graph_exec, h->stream));
  h->last_launches = launches + n;
  return WMD_OK;
}

// Query from a dense HOST histogram: copy, count the non-zeros on the GPU,
// size the panels for exactly that many source words, solve, copy back.
wmd_status query_host(wmd_handle* h, const double* r, float expo, int max_iter,
                      double* wmd_out, bool r_on_device = false) {
  if (!h->have_E || !h->have_T)
    return fail(WMD_ERR_INVALID_ARG, "embeddings and targets must be set first");
  if (h->tV != h->V)
    return fail(WMD_ERR_INVALID_ARG, "target rows != vocabulary size");
  if (max_iter < 0) return fail(WMD_ERR_INVALID_ARG, "max_iter < 0");
  const uint64_t V = h->V;
  const int nchunks = select_num_chunks(V);
  CK(h->r_dev.ensure(V * sizeof(double)));
  CK(h->sel_chunks.ensure((size_t)nchunks * sizeof(uint32_t)));
  CK(h->out_dev.ensure(h->N * sizeof(double)));
  if (h->chunks_host_cap < (size_t)nchunks) {
    if (h->chunks_host) cudaFreeHost(h->chunks_host);
    h->chunks_host = nullptr;
    h->chunks_host_cap = 0;
    CK(cudaMallocHost(&h->chunks_host, (size_t)nchunks * sizeof(uint32_t)));
    h->chunks_host_cap = nchunks;
  }
  wmd_status s = clear_err(h);
  if (s) return s;
  if (!r_on_device)
    CK(cudaMemcpyAsync(h->r_dev.p, r, V * sizeof(double), cudaMemcpyHostToDevice,
                       h->stream));
  // Count pass alone first: v_r sizes every later buffer.
  uint32_t* counts = h->sel_chunks.as<uint32_t>();
  const int lc = launch_select_count(h->r_dev.as<double>(), V, counts,
                                     h->err_dev.as<unsigned>(), h->stream);
  CK(cudaMemcpyAsync(h->chunks_host, counts,
                     (size_t)nchunks * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                     h->stream));
  s = finish(h);
  if (s) return s;
  uint64_t vr = 0;
  for (int c = 0; c < nchunks; ++c) vr += h->chunks_host[c];
  s = query_device(h, h->r_dev.as<double>(), (uint32_t)vr, expo, max_iter,
                   h->out_dev.as<double>());
  if (s) return s;
  h->last_launches += lc;
  if (wmd_out)
    CK(cudaMemcpyAsync(wmd_out, h->out_dev.p, h->N * sizeof(double),
                       cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

// k nearest documents of the scores in scores_dev (device, n): ascending WMD,
// ties by document index, NaN last.  Asynchronous on the handle's stream.
wmd_status topk_device(wmd_handle* h, const double* scores_dev, uint64_t n,
                       uint32_t k, uint32_t* idx_dev, double* val_dev) {
  if (k == 0 || k > 1024) return fail(WMD_ERR_INVALID_ARG, "k must be in [1, 1024]");
  if (n == 0 || n > 0xFFFFFFFFull) return fail(WMD_ERR_INVALID_ARG, "bad score count");
  CK(h->topk_scratch.ensure(topk_scratch_bytes(n, (int)k)));
  h->last_launches = launch_topk(scores_dev, n, (int)k, h->topk_scratch.p, idx_dev,
                                 val_dev, h->stream);
  CK(cudaGetLastError());
  return WMD_OK;
}

// Launch shape of a stacked solve: each of n candidates is run once (its
// first use) and then timed twice with CUDA events on the handle's stream;
// the one with the smallest time is returned (0 when none could be timed).  `launch(shape)` returns
// < 0 when a shape is unavailable.
template <class F>
int tune_group_shape(wmd_handle* h, int n, F&& launch) {
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    if (a) cudaEventDestroy(a);
    return 0;
  }
  float best = 1e30f;
  int bi = 0;
  for (int sh = 0; sh < n; ++sh) {
    if (launch(sh) < 0) continue;
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(a, h->stream);
      launch(sh);
      cudaEventRecord(b, h->stream);
      float ms = 0.f;
      if (cudaEventSynchronize(b) == cudaSuccess &&
          cudaEventElapsedTime(&ms, a, b) == cudaSuccess && ms < best) {
        best = ms;
        bi = sh;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return bi;
}

// Many sparse source documents against the resident target set.  Source s
// holds words src_ids[src_ptr[s] .. src_ptr[s+1]) (strictly ascending, < V)
// with weights src_w (> 0): the reference's select order (fused:45-63)
// already applied.  All sources are uploaded once; per source a gather, the
// cost panel, the near-pair fix-up and the solve run back to back on the
// handle's stream, re-using the single-source working buffers.
// Stacked batch: the sources of one width class run as groups whose panels
// fit h->group_budget, each group in a fixed number of launches (batch.cu):
// gather of the stacked source rows, one cost-panel launch writing every
// source's panel, the near-pair fix-up, (BF16 classes) the BF16 panels, and
// one persistent solve over all (source, document) pairs.  ids32 / rinv /
// vrs are the validated host arrays of query_batch, already uploaded into
// b_ids / b_rinv / b_vr.  form: the tensor-core cost-panel form.
wmd_status query_batch_stacked(wmd_handle* h, uint64_t S, const uint64_t* src_ptr,
                               const std::vector<uint32_t>& ids32,
                               const std::vector<uint32_t>& vrs, int form, float expo,
                               int max_iter, int* launches_out) {
  const uint64_t V = h->V, d = h->d, N = h->N, nnz = h->nnz;
  const bool bf16p = h->prec == WMD_SOLVE_BF16;
  const bool x3 = form == TC_TF32X3;
  const bool tcm = !x3;
  const int dp = tc_padded_width(d);
  const bool relax = h->tol > 0.f && h->omega != 1.f;
  // width class: a BF16 panel width (block solve) or a lane layout (warp solve)
  auto ld16_of = [&](uint32_t vr) { return bf16p ? block_panel_width(vr) : 0; };
  auto cls_of = [&](uint32_t vr) -> int {
    const int l16 = ld16_of(vr);
    if (l16) return 100 + l16 / 128;
    int lpw = 1;
    while (32 * lpw < (int)std::max<uint32_t>(vr, 1)) lpw <<= 1;
    return lpw;
  };
  std::vector<int> classes;
  for (uint64_t s = 0; s < S; ++s) {
    const int c = cls_of(vrs[s]);
    if (std::find(classes.begin(), classes.end(), c) == classes.end()) classes.push_back(c);
  }
  std::sort(classes.begin(), classes.end());
  Targets t;
  t.col_ptr = h->col_ptr.as<int64_t>();
  t.ent = h->ent.as<uint2>();
  t.order = h->order.as<int32_t>();
  t.N = (int64_t)N;
  t.nnz = (int64_t)nnz;
  int launches = 0, groups = 0;
  for (int cls : classes) {
    std::vector<uint64_t> members;
    for (uint64_t s = 0; s < S; ++s)
      if (cls_of(vrs[s]) == cls) members.push_back(s);
    const int l16 = cls > 100 ? 128 * (cls - 100) : 0;
    size_t m0 = 0;
    while (m0 < members.size()) {
      // the next group: as many members as the budget holds (at least one)
      size_t m1 = m0;
      uint64_t bytes = 0;
      while (m1 < members.size()) {
        const uint32_t vr = vrs[members[m1]];
        const uint64_t ld = ((vr ? vr : 1) + 3u) & ~3u;
        const uint64_t b = V * ld * 4 + (l16 ? V * (uint64_t)l16 * 2 : 0) +
                           (relax ? std::max<uint64_t>(nnz, 1) * 4 : 0);
        if (m1 > m0 && bytes + b > h->group_budget) break;
        bytes += b;
        ++m1;
      }
      const int ng = (int)(m1 - m0);
      uint32_t vmax = 1;
      for (size_t m = m0; m < m1; ++m) vmax = std::max(vmax, vrs[members[m]]);
      const int NT = x3 ? tc_tile_n_x3(vmax, d) : tc_tile_n(vmax, d);
      if (NT == 0) return fail(WMD_ERR_UNSUPPORTED, "cost panel cannot tile this width");
      // host tables: stacked rows, tiles, per-source descriptors
      std::vector<int32_t> rowword, rowsrc;
      std::vector<int4> tiles;
      std::vector<GroupSrc> src(ng);
      uint64_t off32 = 0, off16 = 0, offv = 0;
      for (int k = 0; k < ng; ++k) {
        const uint64_t s = members[m0 + k];
        const uint32_t vr = vrs[s];
        const int ld = (int)(((vr ? vr : 1) + 3u) & ~3u);
        const int nt = (ld + NT - 1) / NT;
        GroupSrc& g = src[k];
        g.vr = (int)vr;
        g.ld = ld;
        g.row0 = (int)rowword.size();
        g.rinv = h->b_rinv.as<float>() + src_ptr[s];
        g.vr_dev = h->b_vr.as<uint32_t>() + s;
        g.out = h->b_out.as<double>() + s * N;
        g.iters = h->b_iters.as<int>() + s * N;
        g.K = reinterpret_cast<float*>(off32);    // offsets, rebased below
        g.K16 = l16 ? reinterpret_cast<void*>(off16) : nullptr;
        g.vstate = relax ? reinterpret_cast<float*>(offv) : nullptr;
        off32 += V * (uint64_t)ld * 4;
        off16 += l16 ? V * (uint64_t)l16 * 2 : 0;
        offv += relax ? std::max<uint64_t>(nnz, 1) * 4 : 0;
        for (int i = 0; i < nt * NT; ++i) {
          rowword.push_back(i < (int)vr ? (int32_t)ids32[src_ptr[s] + i] : -1);
          rowsrc.push_back(k);
        }
        for (int i = 0; i < nt; ++i) tiles.push_back(make_int4(k, g.row0 + i * NT, i * NT, 0));
      }
      const int rows = (int)rowword.size();
      CK(h->g_pool.ensure(std::max<uint64_t>(off32, 256)));
      if (l16) CK(h->g_pool16.ensure(std::max<uint64_t>(off16, 256)));
      if (relax) CK(h->g_vst.ensure(std::max<uint64_t>(offv, 256)));
      for (GroupSrc& g : src) {
        g.K = reinterpret_cast<float*>(h->g_pool.as<unsigned char>() +
                                       reinterpret_cast<uintptr_t>(g.K));
        if (l16)
          g.K16 = h->g_pool16.as<unsigned char>() + reinterpret_cast<uintptr_t>(g.K16);
        if (relax)
          g.vstate = reinterpret_cast<float*>(h->g_vst.as<unsigned char>() +
                                              reinterpret_cast<uintptr_t>(g.vstate));
      }
      CK(h->g_S.ensure((size_t)rows * d * 4));
      CK(h->g_nS.ensure((size_t)rows * 4));
      if (tcm) CK(h->g_S16.ensure((size_t)rows * dp * 2));
      CK(h->g_rowword.ensure((size_t)rows * 4));
      CK(h->g_rowsrc.ensure((size_t)rows * 4));
      CK(h->g_tiles.ensure(tiles.size() * sizeof(int4)));
      CK(h->g_src.ensure(src.size() * sizeof(GroupSrc)));
      const unsigned near_cap =
          (unsigned)std::min<uint64_t>((uint64_t)V * rows, (uint64_t)rows * 64 + 4096);
      CK(h->near_pairs.ensure((size_t)near_cap * sizeof(uint2)));
      CK(h->near_count.ensure(sizeof(unsigned)));
      // pageable sources: each copy has been staged when the call returns
      CK(cudaMemcpyAsync(h->g_rowword.p, rowword.data(), (size_t)rows * 4,
                         cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(h->g_rowsrc.p, rowsrc.data(), (size_t)rows * 4,
                         cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(h->g_tiles.p, tiles.data(), tiles.size() * sizeof(int4),
                         cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemcpyAsync(h->g_src.p, src.data(), src.size() * sizeof(GroupSrc),
                         cudaMemcpyHostToDevice, h->stream));
      CK(cudaMemsetAsync(h->near_count.p, 0, sizeof(unsigned), h->stream));
      launches += launch_group_gather(h->g_rowword.as<int32_t>(), rows, h->E32.as<float>(),
                                      h->nE.as<float>(), d, h->g_S.as<float>(),
                                      h->g_nS.as<float>(), tcm ? h->E16.p : nullptr,
                                      tcm ? h->g_S16.p : nullptr, dp, h->sms, h->stream);
      SourceSel sel;
      sel.S = h->g_S.as<float>();
      sel.nS = h->g_nS.as<float>();
      sel.cap = (uint32_t)rows;
      NearList near;
      near.pairs = h->near_pairs.as<uint2>();
      near.count = h->near_count.as<unsigned>();
      near.cap = near_cap;
      near.E32 = h->E32.as<float>();
      near.S32 = sel.S;
      near.d = (int)d;
      StackedPanels sp;
      sp.tiles = h->g_tiles.as<int4>();
      sp.src = h->g_src.as<GroupSrc>();
      sp.ntiles = (int)tiles.size();
      sp.nt = NT;
      const int lc = launch_cdist_tc(form, h->E16.p, h->g_S16.p, h->E32.as<float>(),
                                     h->nE.as<float>(), V, d, sel, expo, nullptr, nullptr,
                                     0, near, h->err_dev.as<unsigned>(), h->sms, h->stream,
                                     nullptr, &sp);
      if (lc < 0) return fail(WMD_ERR_UNSUPPORTED, "stacked cost panel unavailable");
      launches += lc;
      launches += launch_near_fixup_group(near, expo, h->g_rowsrc.as<int32_t>(),
                                          sp.src, ng, V, h->nE.as<float>(),
                                          h->g_nS.as<float>(), h->sms, h->stream);
      SolveCtl ctl;
      ctl.max_iter = max_iter;
      ctl.tol = h->tol;
      ctl.omega = relax ? h->omega : 1.f;
      ctl.vstate = nullptr;  // per source, in src[]
      int ls;
      if (l16) {
        launches += launch_panel_to_bf16_group(sp.src, ng, V, l16, h->sms, h->stream);
        int& shp = h->grp_shape[l16 / 128 - 1];
        if (shp == -2) {
          // autotune the stacked block solve's launch shape on this group
          // (4 updates of every pair per candidate, CUDA events)
          SolveCtl c2 = ctl;
          c2.max_iter = 4;
          c2.tol = 0.f;
          c2.omega = 1.f;
          shp = tune_group_shape(h, 3, [&](int sh) {
            return launch_block_group(sp.src, ng, l16, expo, t, c2, sh, h->stream);
          });
        }
        ls = launch_block_group(sp.src, ng, l16, expo, t, ctl, shp, h->stream);
      } else {
        int k = 0;
        while (k < 5 && (32u << k) < vmax) ++k;
        int& shp = h->wgrp_shape[k];
        if (shp == -2 && ctl.omega == 1.f) {
          // the same for the stacked warp solve (unrelaxed; the relaxed
          // solve keeps the build-time shape)
          SolveCtl c2 = ctl;
          c2.max_iter = 4;
          c2.tol = 0.f;
          shp = tune_group_shape(h, solve_shape_count(), [&](int sh) {
            return launch_solve_group(vmax, sp.src, ng, expo, t, c2, h->stream, sh);
          });
        }
        ls = launch_solve_group(vmax, sp.src, ng, expo, t, ctl, h->stream,
                                ctl.omega == 1.f ? shp : -1);
      }
      if (ls < 0) return fail(WMD_ERR_UNSUPPORTED, "stacked solve unavailable");
      launches += ls;
      ++groups;
      m0 = m1;
    }
  }
  h->last_groups = groups;
  *launches_out = launches;
  return WMD_OK;
}

wmd_status query_batch(wmd_handle* h, const uint64_t* src_ptr,
                       const uint64_t* src_ids, const double* src_w, uint64_t S,
                       float expo, int max_iter, double* wmd_out, int* iters_out) {
  if (!h->have_E || !h->have_T)
    return fail(WMD_ERR_INVALID_ARG, "embeddings and targets must be set first");
  if (h->solve_order != 0)
    return fail(WMD_ERR_UNSUPPORTED, "batched queries run document-major only");
  if (h->tV != h->V)
    return fail(WMD_ERR_INVALID_ARG, "target rows != vocabulary size");
  if (!src_ptr || S == 0 || !wmd_out) return fail(WMD_ERR_INVALID_ARG, "bad batch");
  if (max_iter < 0) return fail(WMD_ERR_INVALID_ARG, "max_iter < 0");
  if (src_ptr[0] != 0) return fail(WMD_ERR_INVALID_INPUT, "src_ptr[0] != 0");
  const uint64_t total = src_ptr[S];
  if (total && (!src_ids || !src_w)) return fail(WMD_ERR_INVALID_ARG, "null source arrays");
  const uint64_t V = h->V, d = h->d, N = h->N;
  std::vector<uint32_t> ids32(std::max<uint64_t>(total, 1));
  std::vector<float> rinv(std::max<uint64_t>(total, 1));
  std::vector<uint32_t> vrs(S);
  uint32_t vr_max = 1;
  for (uint64_t s = 0; s < S; ++s) {
    if (src_ptr[s + 1] < src_ptr[s])
      return fail(WMD_ERR_INVALID_INPUT, "source pointers decrease");
    const uint64_t n = src_ptr[s + 1] - src_ptr[s];
    if (n > 1024) return fail(WMD_ERR_UNSUPPORTED, "a source has more than 1024 words");
    vrs[s] = (uint32_t)n;
    vr_max = std::max<uint32_t>(vr_max, (uint32_t)n);
    for (uint64_t e = src_ptr[s]; e < src_ptr[s + 1]; ++e) {
      if (src_ids[e] >= V) return fail(WMD_ERR_INVALID_INPUT, "source word id >= V");
      if (e > src_ptr[s] && src_ids[e] <= src_ids[e - 1])
        return fail(WMD_ERR_INVALID_INPUT, "source word ids not strictly ascending");
      if (!(src_w[e] > 0.0) || !std::isfinite(src_w[e]))
        return fail(WMD_ERR_INVALID_INPUT, "source weight <= 0 or not finite");
      ids32[e] = (uint32_t)src_ids[e];
      rinv[e] = (float)(1.0 / src_w[e]);
    }
  }
  const bool tcm = h->mode == WMD_CDIST_BF16 || h->mode == WMD_CDIST_FP16;
  const bool bf16 = h->mode == WMD_CDIST_BF16;
  // The split-FP16 mode runs its batches on the split-TF32 form (the same
  // FP32 accuracy class).
  const bool x3 = (h->mode == WMD_CDIST_TF32X3 || h->mode == WMD_CDIST_F16X3) &&
                  tc_tile_n_x3(vr_max, d) != 0;
  const int dp = tc_padded_width(d);
  if (tcm && tc_tile_n(vr_max, d) == 0)
    return fail(WMD_ERR_UNSUPPORTED, "embedding width too large for the tensor-core panel");
  const int ld_max = (int)((vr_max + 3u) & ~3u);
  CK(h->b_ids.ensure(ids32.size() * sizeof(uint32_t)));
  CK(h->b_rinv.ensure(rinv.size() * sizeof(float)));
  CK(h->b_vr.ensure(S * sizeof(uint32_t)));
  CK(h->b_out.ensure(S * N * sizeof(double)));
  CK(h->b_iters.ensure(S * N * sizeof(int)));
  if (h->omega != 1.f)
    CK(h->vstate.ensure((size_t)std::max<uint64_t>(h->nnz, 1) * sizeof(float)));
  CK(h->sel_S.ensure((size_t)vr_max * d * sizeof(float)));
  CK(h->sel_nS.ensure((size_t)vr_max * sizeof(float)));
  CK(h->K.ensure((size_t)V * ld_max * sizeof(float)));
  const bool need_km = expo == 0.f;
  if (need_km) CK(h->KM.ensure((size_t)V * ld_max * sizeof(float)));
  float* KMp = need_km ? h->KM.as<float>() : nullptr;
  int ld16_max = 0;
  if (h->prec == WMD_SOLVE_BF16 && !need_km)
    for (uint64_t s = 0; s < S; ++s) ld16_max = std::max(ld16_max, block_panel_width(vrs[s]));
  if (ld16_max) CK(h->K16.ensure((size_t)V * ld16_max * 2));
  const bool scaled = row_scaled(h, expo);  // panel_rescale.cu
  const int mdl = (int)max_doc_len(h);
  if (scaled) {
    CK(h->mrow.ensure((size_t)V * sizeof(float)));
    CK(h->exact_list.ensure(exact_f64_list_cap() * sizeof(int32_t)));
    CK(h->exact_count.ensure(sizeof(unsigned)));
  }
  const bool ws = h->ws_on && h->ws_d == (int)d && expo != 0.f;
  if (ws) {
    wmd_status sw = ws_prepare_docs(h);
    if (sw) return sw;
    CK(h->ws_Asrc.ensure((size_t)vr_max * kWsH * sizeof(float)));
    CK(h->ws_u0.ensure((size_t)std::max<uint64_t>(N, 1) * ld_max * sizeof(float)));
    CK(h->ws_stats.ensure((size_t)std::max<uint64_t>(N, 1) * vr_max * 3 * sizeof(float)));
  }
  const unsigned near_cap = (unsigned)std::min<uint64_t>((uint64_t)V * vr_max, 1u << 20);
  CK(h->near_pairs.ensure((size_t)near_cap * sizeof(uint2)));
  CK(h->near_count.ensure(sizeof(unsigned)));
  // Two pipeline slots when there is more than one source: slot 1 mirrors
  // slot 0's per-source scratch on its own stream.
  const bool overlap = S > 1;
  if (overlap) {
    wmd_handle::BatchSlot& b1 = h->slot1;
    if (!h->stream2) CK(cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->join)
      if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(b1.sel_S.ensure((size_t)vr_max * d * sizeof(float)));
    CK(b1.sel_nS.ensure((size_t)vr_max * sizeof(float)));
    CK(b1.K.ensure((size_t)V * ld_max * sizeof(float)));
    if (need_km) CK(b1.KM.ensure((size_t)V * ld_max * sizeof(float)));
    if (ld16_max) CK(b1.K16.ensure((size_t)V * ld16_max * 2));
    if (h->omega != 1.f)
      CK(b1.vstate.ensure((size_t)std::max<uint64_t>(h->nnz, 1) * sizeof(float)));
    if (ws) {
      CK(b1.ws_Asrc.ensure((size_t)vr_max * kWsH * sizeof(float)));
      CK(b1.ws_u0.ensure((size_t)std::max<uint64_t>(N, 1) * ld_max * sizeof(float)));
      CK(b1.ws_stats.ensure((size_t)std::max<uint64_t>(N, 1) * vr_max * 3 * sizeof(float)));
    }
    CK(b1.near_pairs.ensure((size_t)near_cap * sizeof(uint2)));
    CK(b1.near_count.ensure(sizeof(unsigned)));
    if (scaled) {
      CK(b1.mrow.ensure((size_t)V * sizeof(float)));
      CK(b1.exact_list.ensure(exact_f64_list_cap() * sizeof(int32_t)));
      CK(b1.exact_count.ensure(sizeof(unsigned)));
    }
    if (tcm) CK(b1.sel_S16.ensure((size_t)vr_max * dp * 2));
  }
  int launches = 0;
  if (tcm) {
    const int fmt = bf16 ? 1 : 2;
    if (h->e16_fmt != fmt) {
      CK(h->E16.ensure((size_t)V * dp * 2));
      launches += launch_to16(h->E32.as<float>(), V, d, h->E16.p, bf16, h->stream);
      h->e16_fmt = fmt;
    }
    CK(h->sel_S16.ensure((size_t)vr_max * dp * 2));
  }
  wmd_status st = clear_err(h);
  if (st) return st;
  CK(cudaMemcpyAsync(h->b_ids.p, ids32.data(), ids32.size() * sizeof(uint32_t),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->b_rinv.p, rinv.data(), rinv.size() * sizeof(float),
                     cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->b_vr.p, vrs.data(), S * sizeof(uint32_t),
                     cudaMemcpyHostToDevice, h->stream));
  Targets t;
  t.col_ptr = h->col_ptr.as<int64_t>();
  t.ent = h->ent.as<uint2>();
  t.order = h->order.as<int32_t>();
  t.N = (int64_t)N;
  t.nnz = (int64_t)h->nnz;
  if (h->timing)
    for (int i = 0; i < 3; ++i) CK(cudaEventRecord(h->ev[i], h->stream));
  // Stacked groups (batch.cu): several sources, tensor-core cost panel, cold
  // start, lambda != 0, panels within FP32 range.
  if (h->stacked && S > 1 && expo != 0.f && !scaled && !ws && (tcm || x3)) {
    int lg = 0;
    wmd_status sg = query_batch_stacked(h, S, src_ptr, ids32, vrs,
                                        x3 ? TC_TF32X3 : bf16 ? TC_BF16 : TC_FP16, expo,
                                        max_iter, &lg);
    if (sg) return sg;
    if (h->timing) CK(cudaEventRecord(h->ev[3], h->stream));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(wmd_out, h->b_out.p, S * N * sizeof(double),
                       cudaMemcpyDeviceToHost, h->stream));
    if (iters_out)
      CK(cudaMemcpyAsync(iters_out, h->b_iters.p, S * N * sizeof(int),
                         cudaMemcpyDeviceToHost, h->stream));
    h->last_launches = launches + lg;
    return finish(h);
  }
  h->last_groups = 0;
  if (overlap) {  // slot 1 starts after the uploads above
    CK(cudaEventRecord(h->join[0], h->stream));
    CK(cudaStreamWaitEvent(h->stream2, h->join[0], 0));
  }
  for (uint64_t s = 0; s < S; ++s) {
    const uint64_t off = src_ptr[s];
    const uint32_t vr = vrs[s];
    const int ld = (int)(((vr ? vr : 1) + 3u) & ~3u);
    // this source's pipeline slot: stream and scratch
    const bool in1 = overlap && (s & 1);
    cudaStream_t sst = in1 ? h->stream2 : h->stream;
    DevBuf& bS = in1 ? h->slot1.sel_S : h->sel_S;
    DevBuf& bnS = in1 ? h->slot1.sel_nS : h->sel_nS;
    DevBuf& bS16 = in1 ? h->slot1.sel_S16 : h->sel_S16;
    DevBuf& bNP = in1 ? h->slot1.near_pairs : h->near_pairs;
    DevBuf& bNC = in1 ? h->slot1.near_count : h->near_count;
    DevBuf& bK = in1 ? h->slot1.K : h->K;
    DevBuf& bK16 = in1 ? h->slot1.K16 : h->K16;
    DevBuf& bVS = in1 ? h->slot1.vstate : h->vstate;
    DevBuf& bAs = in1 ? h->slot1.ws_Asrc : h->ws_Asrc;
    DevBuf& bU0 = in1 ? h->slot1.ws_u0 : h->ws_u0;
    DevBuf& bSt = in1 ? h->slot1.ws_stats : h->ws_stats;
    float* KMs = need_km ? (in1 ? h->slot1.KM : h->KM).as<float>() : nullptr;
    float* mrow = scaled ? (in1 ? h->slot1.mrow : h->mrow).as<float>() : nullptr;
    SourceSel sel;
    sel.ids = h->b_ids.as<uint32_t>() + off;
    sel.rinv = h->b_rinv.as<float>() + off;
    sel.S = bS.as<float>();
    sel.nS = bnS.as<float>();
    sel.vr = h->b_vr.as<uint32_t>() + s;
    sel.cap = vr;
    NearList near;
    near.pairs = bNP.as<uint2>();
    near.count = bNC.as<unsigned>();
    near.cap = near_cap;
    near.E32 = h->E32.as<float>();
    near.S32 = sel.S;
    near.d = (int)d;
    launches += launch_gather_sources(sel.ids, (int)vr, h->E32.as<float>(),
                                      h->nE.as<float>(), d, sel.S, sel.nS,
                                      tcm ? h->E16.p : nullptr,
                                      tcm ? bS16.p : nullptr, dp, sst);
    CK(cudaMemsetAsync(near.count, 0, sizeof(unsigned), sst));
    if (mrow) CK(cudaMemsetAsync(mrow, 0x7f, (size_t)V * sizeof(float), sst));
    if (tcm || x3) {
      const int lc = launch_cdist_tc(x3 ? TC_TF32X3 : bf16 ? TC_BF16 : TC_FP16,
                                     h->E16.p, bS16.p, h->E32.as<float>(),
                                     h->nE.as<float>(), V, d, sel, expo,
                                     bK.as<float>(), KMs, ld, near,
                                     h->err_dev.as<unsigned>(), h->sms, sst, mrow);
      if (lc < 0) {
        if (overlap) cudaStreamSynchronize(h->stream2);
        return fail(WMD_ERR_UNSUPPORTED, "tensor-core cost panel unavailable");
      }
      launches += lc;
    } else {
      launches += launch_cdist_fp32(h->E32.as<float>(), h->nE.as<float>(), V, d,
                                    sel, expo, bK.as<float>(), KMs, ld, near, sst, mrow);
    }
    launches += launch_near_fixup(near, expo, bK.as<float>(), KMs, ld, V,
                                  h->nE.as<float>(), sel.nS, sel.vr, h->sms, sst,
                                  mrow != nullptr);
    if (mrow)
      launches += launch_panel_rescale(bK.as<float>(), ld, V, sel.vr, mrow, expo,
                                       h->sms, sst);
    SolveCtl ctl;
    ctl.mrow = mrow;
    ctl.max_iter = max_iter;
    ctl.tol = h->tol;
    ctl.iters = h->b_iters.as<int>() + s * N;
    ctl.omega = h->tol > 0.f ? h->omega : 1.f;  // relaxation needs stopping
    ctl.vstate = ctl.omega != 1.f ? bVS.as<float>() : nullptr;
    if (ws && vr > 0) {
      launches += launch_ws_init(ws_layout((int)d), h->ws_folded.as<float>(),
                                 h->ws_params.as<float>(), sel.S, sel.rinv, (int)vr,
                                 bK.as<float>(), ld, expo, t, h->ws_Bdoc.as<float>(),
                                 bAs.as<float>(), bU0.as<float>(), ld,
                                 h->err_dev.as<unsigned>(), h->sms, sst, mrow,
                                 bSt.as<float>());
      ctl.u0 = bU0.as<float>();
      ctl.ldu = ld;
    }
    const int ld16 = h->prec == WMD_SOLVE_BF16 && !KMs && !mrow ? block_panel_width(vr) : 0;
    int ls;
    if (ld16) {
      launches += launch_panel_to_bf16(bK.as<float>(), ld, bK16.p, ld16, V, sel.vr,
                                       h->sms, sst);
      if (overlap && !block_shape_known(h, ld16)) {
        // the autotuner times its candidates on the handle's stream: nothing
        // else may run meanwhile, and this slot's panel must be complete
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaStreamSynchronize(h->stream2));
      }
      const int shape = block_shape_for(h, bK16.p, ld16, expo, vr, sel, t, ctl,
                                        h->b_out.as<double>() + s * N, true);
      ls = launch_block_shape(h, bK16.p, ld16, expo, vr, sel, t, ctl, ctl.u0, ctl.ldu,
                              h->b_out.as<double>() + s * N, shape, sst);
    } else {
      ls = launch_solve(bK.as<float>(), KMs, ld, expo, vr, sel, t, ctl,
                        h->b_out.as<double>() + s * N, sst);
    }
    if (ls < 0) {
      if (overlap) cudaStreamSynchronize(h->stream2);
      return fail(WMD_ERR_UNSUPPORTED, "a source has more than 1024 words");
    }
    launches += ls;
    if (mrow) {  // documents the row-scaled FP32 panel cannot carry, in FP64
      DevBuf& bL = in1 ? h->slot1.exact_list : h->exact_list;
      DevBuf& bC = in1 ? h->slot1.exact_count : h->exact_count;
      const int le = launch_exact_f64(h->E32.as<float>(), d, sel, t, expo, ctl, mdl,
                                      bL.as<int32_t>(), bC.as<unsigned>(), h->sms,
                                      h->b_out.as<double>() + s * N, sst);
      if (le < 0) {
        if (overlap) cudaStreamSynchronize(h->stream2);
        return fail(WMD_ERR_UNSUPPORTED, "documents too long for the FP64 re-solve");
      }
      launches += le;
    }
  }
  if (overlap) {  // the results wait for both slots
    CK(cudaEventRecord(h->join[1], h->stream2));
    CK(cudaStreamWaitEvent(h->stream, h->join[1], 0));
  }
  if (h->timing) CK(cudaEventRecord(h->ev[3], h->stream));
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(wmd_out, h->b_out.p, S * N * sizeof(double),
                     cudaMemcpyDeviceToHost, h->stream));
  if (iters_out)
    CK(cudaMemcpyAsync(iters_out, h->b_iters.p, S * N * sizeof(int),
                       cudaMemcpyDeviceToHost, h->stream));
  h->last_launches = launches;
  return finish(h);
}

// Device view of [p, p + bytes) when the whole range lies in one pinned,
// device-mapped host allocation (the runtime reports host memory and the
// driver's allocation range covers the span); null otherwise.
typedef CUresult (*PtrAttrFn)(void*, CUpointer_attribute, CUdeviceptr);
PtrAttrFn ptr_attr_fn() {
  static PtrAttrFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PtrAttrFn>(p);
  }
  return fn;
}

const void* mapped_host_range(const void* p, size_t bytes) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || !a.devicePointer) return nullptr;
  PtrAttrFn f = ptr_attr_fn();
  if (!f) return nullptr;
  const CUdeviceptr dp = (CUdeviceptr)(uintptr_t)a.devicePointer;
  CUdeviceptr start = 0;
  size_t size = 0;
  if (f(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, dp) != CUDA_SUCCESS ||
      f(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, dp) != CUDA_SUCCESS)
    return nullptr;
  if (dp < start || dp - start > size || bytes > size - (size_t)(dp - start))
    return nullptr;
  return a.devicePointer;
}

// Pinned staging of the drop-in calls' host-narrowed rows: a ring of slots
// of about 8 MB (at least one row of d floats each).
constexpr int kStageSlots = 4;
inline size_t kStageSlotBytes(uint64_t d) {
  const size_t row = (size_t)d * sizeof(float);
  return std::max<size_t>(row, ((size_t)8 << 20) / row * row);
}

// Drop-in embeddings, split two ways so that the host threads and the host
// bus work at the same time:
//   * the rows of the words below wh = host_share * V (all of them when the
//     embeddings are not device-mapped) are converted FP64 -> FP32 by the
//     host threads into pinned memory, chunk by chunk, each chunk copied to
//     the device on the second stream while the next one is converted (4
//     bytes per entry on the bus; every word of the prefix, needed or not:
//     the low ids are the frequent words, nearly all of them needed);
//   * above wh the GPU flags the words a query can touch (the target words of
//     the resident target set and the source words r != 0) and reads their
//     rows in FP64 straight from the caller's device-mapped memory (8 bytes
//     per entry), meanwhile; every other row is zeroed.
// Both conversions round FP64 to FP32 to nearest and the norms are summed in
// one order, so the results are bit-identical whatever the split.  The
// handle's E then holds zeros for unneeded words above wh, so it is only
// valid for this target set and this r, which is how the drop-in calls use
// their private handle.  Leaves r uploaded in r_dev.
wmd_status set_embeddings_split(wmd_handle* h, const double* vecs, const double* vmap,
                                const double* r, uint64_t V, uint64_t d, double host_share,
                                uint64_t* host_rows, uint64_t* dev_rows) {
  if (V > 0xFFFFFFFFull)
    return fail(WMD_ERR_UNSUPPORTED, "vocabulary larger than 2^32 words");
  if (d > 65536) return fail(WMD_ERR_UNSUPPORTED, "embedding width above 65536");
  if (!h->have_T || h->tV != V)
    return fail(WMD_ERR_INVALID_ARG, "targets must be set first");
  uint64_t wh = vmap ? (uint64_t)(host_share * (double)V + 0.5) : V;
  if (wh > V) wh = V;
  const size_t n = (size_t)V * d;
  CK(h->E32.ensure(n * sizeof(float)));
  CK(h->nE.ensure((size_t)V * sizeof(float)));
  CK(h->r_dev.ensure(V * sizeof(double)));
  CK(h->need.ensure((size_t)V));
  CK(h->need_count.ensure(sizeof(unsigned long long)));
  CK(h->rows32.ensure(std::max<size_t>(wh, 1) * d * sizeof(float)));
  if (wh > 0) {
    // (a call that failed part-way may have left copies from the staging
    // slots in flight: they end before the slots are written again)
    if (h->stream2) CK(cudaStreamSynchronize(h->stream2));
    CK(h->hstage.ensure(kStageSlots * kStageSlotBytes(d)));
    if (!h->stream2) CK(cudaStreamCreateWithFlags(&h->stream2, cudaStreamNonBlocking));
    if (!h->ev_split) CK(cudaEventCreateWithFlags(&h->ev_split, cudaEventDisableTiming));
    for (cudaEvent_t& e : h->ev_slot)
      if (!e) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  CK(cudaMemcpyAsync(h->r_dev.p, r, V * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  // The GPU's share: starts now.
  int launches = launch_gather_rows_split(vmap, h->ent.as<uint2>(), h->nnz,
                                          h->r_dev.as<double>(), h->need.as<unsigned char>(),
                                          V, d, wh, nullptr, 0, h->E32.as<float>(),
                                          h->nE.as<float>(),
                                          h->need_count.as<unsigned long long>(), h->stream);
  // The host's share, in chunks of about 8 MB of FP32 (at least 8 chunks when
  // there are enough rows), each copied on the second stream while the next
  // one is converted; the chunks go through a ring of kStageSlots pinned
  // slots, a slot reused once its copy is done, so the pinned memory stays
  // kStageSlots x 8 MB whatever the vocabulary.
  if (wh > 0) {
    const uint64_t per_chunk = std::max<uint64_t>(
        1, std::min<uint64_t>(kStageSlotBytes(d) / (d * 4), (wh + 7) / 8));
    uint64_t k = 0;
    for (uint64_t i0 = 0; i0 < wh; i0 += per_chunk, ++k) {
      const uint64_t i1 = std::min(wh, i0 + per_chunk);
      const int slot = (int)(k % kStageSlots);
      if (k >= (uint64_t)kStageSlots) CK(cudaEventSynchronize(h->ev_slot[slot]));
      float* rows = reinterpret_cast<float*>(static_cast<char*>(h->hstage.p) +
                                             (size_t)slot * kStageSlotBytes(d));
      const double* src = vecs + i0 * d;
      const int64_t n = (int64_t)((i1 - i0) * d);
#pragma omp parallel for schedule(static)
      for (int64_t e = 0; e < n; ++e) rows[e] = (float)src[e];
      CK(cudaMemcpyAsync(h->rows32.as<float>() + i0 * d, rows, (size_t)n * sizeof(float),
                         cudaMemcpyHostToDevice, h->stream2));
      CK(cudaEventRecord(h->ev_slot[slot], h->stream2));
    }
    CK(cudaEventRecord(h->ev_split, h->stream2));
    CK(cudaStreamWaitEvent(h->stream, h->ev_split, 0));
    launches += launch_gather_rows_split(vmap, h->ent.as<uint2>(), h->nnz,
                                         h->r_dev.as<double>(), h->need.as<unsigned char>(),
                                         V, d, wh, h->rows32.as<float>(), 1,
                                         h->E32.as<float>(), h->nE.as<float>(),
                                         h->need_count.as<unsigned long long>(), h->stream);
  }
  CK(cudaGetLastError());
  wmd_status se = update_emax(h, V);
  if (se) return se;
  launches += 1;
  h->V = V;
  h->d = d;
  h->have_E = true;
  h->e16_fmt = -1;
  h->ehl_ready = false;
  h->ws_docs_ready = false;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  h->graph_epoch++;
  h->last_launches = launches;
  *host_rows = wh;
  *dev_rows = 0;  // known once the stream has run: dropin_csc reads need_count
  return WMD_OK;
}

// Share of the vocabulary (a prefix of the word ids) whose rows the host
// threads narrow in a drop-in call when the GPU can read the others itself
// (measured on the B200 box's host, single-source workload).
constexpr double kDropinHostShare = 0.5;

// Per-host-thread default handle for the drop-in calls.
struct TlHandle {
  wmd_handle* h = nullptr;
  ~TlHandle() {
    if (h) wmd_destroy(h);
  }
};
thread_local TlHandle tl_handle;

wmd_status default_handle(wmd_handle** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (tl_handle.h && tl_handle.h->device != dev) {
    wmd_destroy(tl_handle.h);
    tl_handle.h = nullptr;
  }
  if (!tl_handle.h) {
    wmd_status s = wmd_create(&tl_handle.h, dev);
    if (s) return s;
    // The drop-in calls build their cost panel on the tensor cores in the
    // FP32-accurate split-TF32 form (FP32 rows read in place, three TF32
    // products); widths it cannot tile (d % 4 != 0) take the FP32 CUDA-core
    // panel.  Both hold the plain path's 1e-5 against the reference.
    tl_handle.h->mode = WMD_CDIST_TF32X3;
    // Every drop-in call brings a new target set and embeddings, so nothing
    // that pays off over repeated queries is kept: the launch shapes are the
    // build-time defaults (the autotuner would re-time its candidates on
    // every call) and the kernels are launched directly (a captured graph
    // would be re-captured and instantiated on every call).
    tl_handle.h->autotune = false;
    tl_handle.h->use_graphs = false;
  }
  *out = tl_handle.h;
  return WMD_OK;
}

wmd_status dropin_csc(const double* r, const double* vecs, double* WMD,
                      float expo, int max_iter, uint64_t V, uint64_t N,
                      uint64_t d, const wmd_csc_double_t* c) {
  if (!r || !vecs || !WMD || !c)
    return fail(WMD_ERR_INVALID_ARG, "null argument");
  if (V == 0 || N == 0 || d == 0)
    return fail(WMD_ERR_INVALID_INPUT, "zero vocabulary, document count or width");
  if (c->num_rows != V || c->num_cols != N)
    return fail(WMD_ERR_INVALID_ARG, "matrix shape does not match V x num_docs");
  if (max_iter < 0) return fail(WMD_ERR_INVALID_ARG, "max_iter < 0");
  wmd_handle* h = nullptr;
  wmd_status s = default_handle(&h);
  if (s) return s;
  const uint64_t csc_bytes = (N + 1) * 8 + c->nnz * 16 + N * 4;  // + order
  // Embedding rows.  With the embeddings in pinned, device-mapped memory the
  // host threads narrow the rows of a prefix of the vocabulary to FP32 while
  // the GPU reads the needed rows above it in FP64 (the prefix, as a share of
  // V: WMD_DROPIN_HOST_SHARE in [0, 1], by default kDropinHostShare, none
  // with fewer than 4 host threads); pageable embeddings are narrowed on the
  // host whole, or copied whole when there are fewer than 4 host threads or
  // the share is 0.
  const double* vmap = static_cast<const double*>(
      mapped_host_range(vecs, (size_t)V * d * sizeof(double)));
  double share = omp_get_max_threads() >= 4 ? kDropinHostShare : 0.0;
  if (const char* env = getenv("WMD_DROPIN_HOST_SHARE")) {
    const double x = atof(env);
    share = x < 0.0 ? 0.0 : x > 1.0 ? 1.0 : x;
  }
  const bool split = vmap || share > 0.0;
  int le = 0, lt = 0;
  uint64_t nh = 0, nd = 0;
  if (split) {
    // The targets' copies and packing, the GPU's row reads and the host's
    // conversion all overlap; the targets' checks are read afterwards.
    s = set_targets_csc(h, c, true);
    if (s) return s;
    lt = h->last_launches;
    s = set_embeddings_split(h, vecs, vmap, r, V, d, share, &nh, &nd);
    if (s) return s;
    le = h->last_launches;
    s = finish(h);
    if (s) {
      h->have_T = false;
      return s;
    }
  } else {
    s = set_embeddings(h, vecs, V, d, 0, true);
    if (s) return s;
    le = h->last_launches;
    s = set_targets_csc(h, c);
    if (s) return s;
    lt = h->last_launches;
  }
  s = query_host(h, r, expo, max_iter, WMD, split);
  if (s) return s;
  h->last_launches += le + lt;
  if (split) {  // rows the GPU read over the bus (query_host synchronised)
    unsigned long long cnt = 0;
    CK(cudaMemcpy(&cnt, h->need_count.p, sizeof(cnt), cudaMemcpyDeviceToHost));
    nd = cnt;
  }
  // bus bytes: CSC + r + the host-narrowed prefix (FP32) + the rows the GPU
  // read (FP64), or the whole FP64 matrix
  h->dropin_h2d = split ? csc_bytes + V * 8 + nh * d * 4 + nd * d * 8
                        : csc_bytes + V * 8 + V * d * 8;
  h->dropin_host_rows = nh;
  h->dropin_dev_rows = nd;
  return WMD_OK;
}

wmd_status dropin_csr(const double* r, const double* vecs, double* WMD,
                      float expo, int max_iter, uint64_t V, uint64_t N,
                      uint64_t d, const wmd_csr_double_t* a) {
  if (!a) return fail(WMD_ERR_INVALID_ARG, "null matrix");
  if (a->num_rows != V || a->num_cols != N)
    return fail(WMD_ERR_INVALID_ARG, "matrix shape does not match V x num_docs");
  if (a->nnz == 0)
    return fail(WMD_ERR_INVALID_INPUT, "target matrix has no non-zeros");
  std::vector<uint64_t> cp, rows;
  std::vector<double> vals;
  wmd_status s = csr_to_csc_host(a, cp, rows, vals);
  if (s) return s;
  wmd_csc_double_t c;
  c.num_rows = V;
  c.num_cols = N;
  c.nnz = a->nnz;
  c.col_ptr = cp.data();
  c.row_inds = rows.data();
  c.vals = vals.data();
  return dropin_csc(r, vecs, WMD, expo, max_iter, V, N, d, &c);
}

}  // namespace

extern "C" {

int wmd_abi_version(void) { return WMD_B200_ABI_VERSION; }

const char* wmd_status_string(wmd_status s) {
  switch (s) {
    case WMD_OK: return "ok";
    case WMD_ERR_INVALID_ARG: return "invalid argument";
    case WMD_ERR_INVALID_INPUT: return "invalid input data";
    case WMD_ERR_OUT_OF_MEMORY: return "out of device memory";
    case WMD_ERR_CUDA: return "CUDA error";
    case WMD_ERR_NO_DEVICE: return "no CUDA device";
    case WMD_ERR_UNSUPPORTED: return "unsupported";
    case WMD_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
  }
  return "unknown status";
}

const char* wmd_last_error(void) { return g_last_error.c_str(); }

wmd_status wmd_create(wmd_handle** out, int device) {
  if (!out) return fail(WMD_ERR_INVALID_ARG, "wmd_create: null out");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(WMD_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= n)
    return fail(WMD_ERR_INVALID_ARG, "wmd_create: device out of range");
  wmd_handle* h = new wmd_handle();
  h->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = h->err_dev.ensure(sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(h->err_dev.p, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMallocHost(&h->err_host, sizeof(unsigned));
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&h->ev[i]);
  if (e != cudaSuccess) {
    wmd_destroy(h);
    return fail_cuda(e, "wmd_create");
  }
  *out = h;
  return WMD_OK;
}

wmd_status wmd_destroy(wmd_handle* h) {
  if (!h) return WMD_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (DevBuf* b : {&h->E32, &h->nE, &h->E64_stage, &h->E16, &h->Ehl, &h->col_ptr,
                    &h->ent, &h->order, &h->stage_cp, &h->stage_rows,
                    &h->stage_vals, &h->r_dev, &h->sel_ids, &h->sel_rinv,
                    &h->sel_S, &h->sel_nS, &h->sel_S16, &h->sel_vr,
                    &h->sel_chunks, &h->K, &h->KM, &h->out_dev, &h->err_dev,
                    &h->near_pairs, &h->near_count, &h->iters, &h->b_ids,
                    &h->b_rinv, &h->b_vr, &h->b_out, &h->b_iters,
                    &h->topk_scratch, &h->topk_idx, &h->topk_val, &h->K16,
                    &h->ws_params, &h->ws_folded, &h->ws_C, &h->ws_Bdoc,
                    &h->ws_Asrc, &h->ws_u0, &h->ws_X, &h->ws_y, &h->ws_gptr,
                    &h->edge_words, &h->edge_docs, &h->edge_w, &h->edge_temp})
    b->release();
  if (h->err_host) cudaFreeHost(h->err_host);
  if (h->chunks_host) cudaFreeHost(h->chunks_host);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  for (int i = 0; i < 4; ++i)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->ev_split) cudaEventDestroy(h->ev_split);
  for (cudaEvent_t e : h->ev_slot)
    if (e) cudaEventDestroy(e);
  if (h->stream2) {
    cudaStreamSynchronize(h->stream2);
    cudaStreamDestroy(h->stream2);
  }
  for (cudaEvent_t e : h->join)
    if (e) cudaEventDestroy(e);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return WMD_OK;
}

wmd_status wmd_set_embeddings_f64(wmd_handle* h, const double* vecs, uint64_t V,
                                  uint64_t d, int where) {
  return set_embeddings(h, vecs, V, d, where, true);
}

wmd_status wmd_set_embeddings_f32(wmd_handle* h, const float* vecs, uint64_t V,
                                  uint64_t d, int where) {
  return set_embeddings(h, vecs, V, d, where, false);
}

wmd_status wmd_set_embeddings_bf16(wmd_handle* h, const uint16_t* vecs, uint64_t V,
                                   uint64_t d, int where) {
  if (!h || !vecs || V == 0 || d == 0 || (where != 0 && where != 1))
    return fail(WMD_ERR_INVALID_ARG, "set_embeddings_bf16: bad argument");
  if (V > 0xFFFFFFFFull)
    return fail(WMD_ERR_UNSUPPORTED, "vocabulary larger than 2^32 words");
  if (d > 65536) return fail(WMD_ERR_UNSUPPORTED, "embedding width above 65536");
  wmd_status s = bind(h);
  if (s) return s;
  const size_t n = (size_t)V * d;
  const int dp = tc_padded_width(d);
  CK(h->E32.ensure(n * sizeof(float)));
  CK(h->nE.ensure((size_t)V * sizeof(float)));
  CK(h->E16.ensure((size_t)V * dp * 2));
  const void* src = vecs;
  if (where == 0) {  // host BF16: staged through the FP64 staging buffer
    CK(h->E64_stage.ensure(n * 2));
    CK(cudaMemcpyAsync(h->E64_stage.p, vecs, n * 2, cudaMemcpyHostToDevice, h->stream));
    src = h->E64_stage.p;
  }
  int launches = launch_embed_from_bf16(src, V, d, dp, h->E32.as<float>(), h->E16.p,
                                        h->stream);
  launches += launch_embed_norms(h->E32.as<float>(), V, d, h->nE.as<float>(), h->stream);
  s = update_emax(h, V);
  if (s) return s;
  CK(cudaGetLastError());
  h->V = V;
  h->d = d;
  h->have_E = true;
  h->e16_fmt = 1;  // E16 holds the BF16 embeddings themselves
  h->ehl_ready = false;
  h->ws_docs_ready = false;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  h->graph_epoch++;
  h->last_launches = launches + 1;
  return WMD_OK;
}

wmd_status wmd_set_targets_csc(wmd_handle* h, const wmd_csc_double_t* c) {
  return set_targets_csc(h, c);
}

wmd_status wmd_set_targets_csr(wmd_handle* h, const wmd_csr_double_t* a) {
  if (!h || !a) return fail(WMD_ERR_INVALID_ARG, "set_targets: null argument");
  if (a->num_rows == 0 || a->num_cols == 0 || a->nnz == 0)
    return fail(WMD_ERR_INVALID_INPUT, "empty target matrix");
  std::vector<uint64_t> cp, rows;
  std::vector<double> vals;
  wmd_status s = csr_to_csc_host(a, cp, rows, vals);
  if (s) return s;
  wmd_csc_double_t c;
  c.num_rows = a->num_rows;
  c.num_cols = a->num_cols;
  c.nnz = a->nnz;
  c.col_ptr = cp.data();
  c.row_inds = rows.data();
  c.vals = vals.data();
  return set_targets_csc(h, &c);
}

wmd_status wmd_set_cdist_mode(wmd_handle* h, wmd_cdist_mode mode) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (mode != WMD_CDIST_FP32 && mode != WMD_CDIST_BF16 && mode != WMD_CDIST_FP16 &&
      mode != WMD_CDIST_TF32X3 && mode != WMD_CDIST_F16X3)
    return fail(WMD_ERR_INVALID_ARG, "unknown cdist mode");
  h->mode = mode;
  return WMD_OK;
}

wmd_status wmd_set_relaxation(wmd_handle* h, double omega) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (!(omega > 0.0 && omega < 2.0))
    return fail(WMD_ERR_INVALID_ARG, "relaxation must be in (0, 2)");
  h->omega = (float)omega;
  return WMD_OK;
}

wmd_status wmd_set_autotune(wmd_handle* h, int enable) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  h->autotune = enable != 0;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  h->graph_epoch++;
  return WMD_OK;
}

wmd_status wmd_set_block_shape(wmd_handle* h, int shape) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (shape < -2 || shape >= block_shape_count())
    return fail(WMD_ERR_INVALID_ARG, "unknown block-solve shape");
  h->forced_shape = shape;
  h->graph_epoch++;
  return WMD_OK;
}

wmd_status wmd_autotune_choices(wmd_handle* h, int* shapes) {
  if (!h || !shapes) return fail(WMD_ERR_INVALID_ARG, "null argument");
  for (int i = 0; i < 8; ++i) shapes[i] = h->blk_shape[i];
  return WMD_OK;
}

const char* wmd_block_shape_name(int shape) { return block_shape_name(shape); }

wmd_status wmd_set_batch_mode(wmd_handle* h, int stacked, uint64_t group_budget_bytes) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (group_budget_bytes < (64ull << 20))
    return fail(WMD_ERR_INVALID_ARG, "group budget below 64 MiB");
  h->stacked = stacked != 0;
  h->group_budget = group_budget_bytes;
  return WMD_OK;
}

int wmd_last_batch_groups(wmd_handle* h) { return h ? h->last_groups : 0; }

wmd_status wmd_solve_shape_choices(wmd_handle* h, int* shapes) {
  if (!h || !shapes) return fail(WMD_ERR_INVALID_ARG, "null argument");
  for (int i = 0; i < 6; ++i) shapes[i] = h->warp_shape[i];
  return WMD_OK;
}

const char* wmd_solve_shape_name(int shape) { return solve_shape_name(shape); }

wmd_status wmd_group_shape_choices(wmd_handle* h, int* shapes) {
  if (!h || !shapes) return fail(WMD_ERR_INVALID_ARG, "null argument");
  for (int i = 0; i < 4; ++i) shapes[i] = h->grp_shape[i];
  for (int i = 0; i < 6; ++i) shapes[4 + i] = h->wgrp_shape[i];
  return WMD_OK;
}

wmd_status wmd_set_solve_order(wmd_handle* h, int order) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (order != 0 && order != 1) return fail(WMD_ERR_INVALID_ARG, "order must be 0 or 1");
  h->solve_order = order;
  h->graph_epoch++;
  return WMD_OK;
}

wmd_status wmd_set_solve_precision(wmd_handle* h, wmd_solve_precision prec) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (prec != WMD_SOLVE_FP32 && prec != WMD_SOLVE_BF16)
    return fail(WMD_ERR_INVALID_ARG, "unknown solve precision");
  h->prec = prec;
  return WMD_OK;
}

wmd_status wmd_query_dense(wmd_handle* h, const double* r, double lambda,
                           int max_iter, double* wmd_out) {
  if (!h || !r || !wmd_out) return fail(WMD_ERR_INVALID_ARG, "null argument");
  wmd_status s = bind(h);
  if (s) return s;
  return query_host(h, r, (float)(-lambda), max_iter, wmd_out);
}

wmd_status wmd_query_dense_device(wmd_handle* h, const double* r_dev,
                                  uint64_t vr_cap, double lambda, int max_iter,
                                  double* wmd_dev) {
  if (!h || !r_dev || !wmd_dev) return fail(WMD_ERR_INVALID_ARG, "null argument");
  if (!h->have_E || !h->have_T)
    return fail(WMD_ERR_INVALID_ARG, "embeddings and targets must be set first");
  if (h->tV != h->V)
    return fail(WMD_ERR_INVALID_ARG, "target rows != vocabulary size");
  if (max_iter < 0) return fail(WMD_ERR_INVALID_ARG, "max_iter < 0");
  if (vr_cap > 1024)
    return fail(WMD_ERR_UNSUPPORTED, "vr_cap above 1024");
  wmd_status s = bind(h);
  if (s) return s;
  return query_device(h, r_dev, (uint32_t)vr_cap, (float)(-lambda), max_iter,
                      wmd_dev);
}

wmd_status wmd_query_batch(wmd_handle* h, const uint64_t* src_ptr,
                           const uint64_t* src_ids, const double* src_w,
                           uint64_t num_sources, double lambda, int max_iter,
                           double* wmd_out, int* iters_out) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  wmd_status s = bind(h);
  if (s) return s;
  return query_batch(h, src_ptr, src_ids, src_w, num_sources, (float)(-lambda),
                     max_iter, wmd_out, iters_out);
}

wmd_status wmd_query_topk(wmd_handle* h, const double* r, double lambda,
                          int max_iter, uint32_t k, uint32_t* idx_out,
                          double* wmd_out) {
  if (!h || !r || !idx_out || !wmd_out) return fail(WMD_ERR_INVALID_ARG, "null argument");
  wmd_status s = bind(h);
  if (s) return s;
  if (k == 0 || k > 1024) return fail(WMD_ERR_INVALID_ARG, "k must be in [1, 1024]");
  s = query_host(h, r, (float)(-lambda), max_iter, nullptr);
  if (s) return s;
  const int lq = h->last_launches;
  CK(h->topk_idx.ensure(k * sizeof(uint32_t)));
  CK(h->topk_val.ensure(k * sizeof(double)));
  s = topk_device(h, h->out_dev.as<double>(), h->N, k, h->topk_idx.as<uint32_t>(),
                  h->topk_val.as<double>());
  if (s) return s;
  h->last_launches += lq;
  CK(cudaMemcpyAsync(idx_out, h->topk_idx.p, k * sizeof(uint32_t),
                     cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(wmd_out, h->topk_val.p, k * sizeof(double),
                     cudaMemcpyDeviceToHost, h->stream));
  return finish(h);
}

wmd_status wmd_topk_device(wmd_handle* h, const double* scores_dev, uint64_t n,
                           uint32_t k, uint32_t* idx_dev, double* val_dev) {
  if (!h || !scores_dev || !idx_dev || !val_dev)
    return fail(WMD_ERR_INVALID_ARG, "null argument");
  wmd_status s = bind(h);
  if (s) return s;
  return topk_device(h, scores_dev, n, k, idx_dev, val_dev);
}

wmd_status wmd_selftest_bounded_wait(wmd_handle* h, uint64_t limit_ns) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (limit_ns < 1000 || limit_ns > 2000000000ull)
    return fail(WMD_ERR_INVALID_ARG, "limit_ns outside [1e3, 2e9]");
  wmd_status s = bind(h);
  if (s) return s;
  h->last_launches = launch_wait_selftest(h->err_dev.as<unsigned>(), limit_ns, h->stream);
  CK(cudaGetLastError());
  set_last_error("");
  return WMD_OK;
}

wmd_status wmd_check(wmd_handle* h) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  wmd_status s = bind(h);
  if (s) return s;
  return finish(h);
}

void* wmd_stream(wmd_handle* h) { return h ? (void*)h->stream : nullptr; }

int wmd_last_launch_count(wmd_handle* h) { return h ? h->last_launches : 0; }

wmd_status wmd_set_tolerance(wmd_handle* h, double tol) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (!(tol >= 0.0)) return fail(WMD_ERR_INVALID_ARG, "tolerance must be >= 0");
  h->tol = (float)tol;
  return WMD_OK;
}

wmd_status wmd_last_iterations(wmd_handle* h, int* iters) {
  if (!h || !iters) return fail(WMD_ERR_INVALID_ARG, "null argument");
  if (!h->have_T || !h->iters.p) return fail(WMD_ERR_INVALID_ARG, "no query has run");
  wmd_status s = bind(h);
  if (s) return s;
  CK(cudaMemcpyAsync(iters, h->iters.p, h->N * sizeof(int), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return WMD_OK;
}

wmd_status wmd_set_timing(wmd_handle* h, int enable) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  h->timing = enable != 0;
  return WMD_OK;
}

wmd_status wmd_stage_times(wmd_handle* h, float* select_ms, float* cdist_ms,
                           float* solve_ms) {
  if (!h || !select_ms || !cdist_ms || !solve_ms)
    return fail(WMD_ERR_INVALID_ARG, "null argument");
  if (!h->timing) return fail(WMD_ERR_INVALID_ARG, "timing is not enabled");
  wmd_status s = bind(h);
  if (s) return s;
  CK(cudaEventSynchronize(h->ev[3]));
  CK(cudaEventElapsedTime(select_ms, h->ev[0], h->ev[1]));
  CK(cudaEventElapsedTime(cdist_ms, h->ev[1], h->ev[2]));
  CK(cudaEventElapsedTime(solve_ms, h->ev[2], h->ev[3]));
  return WMD_OK;
}

wmd_status wmd_sinkhorn_fused(const double* r, const double* vecs, double* WMD,
                              double lamda, int max_iter,
                              uint64_t data_vocab_size, uint64_t num_docs,
                              uint64_t word2vec_word_embedding_size,
                              const wmd_csr_double_t* c_csr) {
  return dropin_csr(r, vecs, WMD, (float)lamda, max_iter, data_vocab_size,
                    num_docs, word2vec_word_embedding_size, c_csr);
}

wmd_status wmd_sinkhorn_nonfused(const double* r, const double* vecs,
                                 double* WMD, double lamda, int max_iter,
                                 uint64_t data_vocab_size, uint64_t num_docs,
                                 uint64_t word2vec_word_embedding_size,
                                 const wmd_csr_double_t* c_csr) {
  return dropin_csr(r, vecs, WMD, (float)(-lamda), max_iter, data_vocab_size,
                    num_docs, word2vec_word_embedding_size, c_csr);
}

uint64_t wmd_dropin_h2d_bytes(void) { return tl_handle.h ? tl_handle.h->dropin_h2d : 0; }

wmd_status wmd_sinkhorn_fused_csc(const double* r, const double* vecs,
                                  double* WMD, double lamda, int max_iter,
                                  uint64_t data_vocab_size, uint64_t num_docs,
                                  uint64_t word2vec_word_embedding_size,
                                  const wmd_csc_double_t* c_csc) {
  return dropin_csc(r, vecs, WMD, (float)lamda, max_iter, data_vocab_size,
                    num_docs, word2vec_word_embedding_size, c_csc);
}

wmd_status wmd_sinkhorn_nonfused_csc(const double* r, const double* vecs,
                                     double* WMD, double lamda, int max_iter,
                                     uint64_t data_vocab_size,
                                     uint64_t num_docs,
                                     uint64_t word2vec_word_embedding_size,
                                     const wmd_csc_double_t* c_csc) {
  return dropin_csc(r, vecs, WMD, (float)(-lamda), max_iter, data_vocab_size,
                    num_docs, word2vec_word_embedding_size, c_csc);
}

/* ------------------------------------------------------------------------
 * Learned warm start.
 * ---------------------------------------------------------------------- */

uint64_t wmd_ws_param_count(uint64_t d) {
  if (d == 0 || d > 65536) return 0;
  return (uint64_t)ws_layout((int)d).count;
}

wmd_status wmd_ws_init_params(uint64_t d, uint64_t seed, float* params) {
  if (!params || d == 0 || d > 65536) return fail(WMD_ERR_INVALID_ARG, "bad argument");
  const WsLayout L = ws_layout((int)d);
  std::mt19937_64 rng(seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  std::fill(params, params + L.count, 0.f);
  for (int f = 0; f < L.F; ++f) params[L.scale + f] = 1.f;
  const float s1 = 1.f / std::sqrt((float)L.F), s2 = 1.f / std::sqrt((float)kWsH);
  for (size_t i = 0; i < (size_t)kWsH * L.F; ++i) params[L.W1 + i] = s1 * nd(rng);
  for (size_t i = 0; i < (size_t)kWsH * kWsH; ++i) params[L.W2 + i] = s2 * nd(rng);
  for (int i = 0; i < kWsH; ++i) params[L.w3 + i] = s2 * nd(rng);
  return WMD_OK;
}

wmd_status wmd_ws_build_training_set(wmd_handle* h, const uint64_t* src_ptr,
                                     const uint64_t* src_ids, const double* src_w,
                                     uint64_t S, double lambda,
                                     uint32_t docs_per_source, uint32_t words_per_doc,
                                     double label_tol, int label_max_iter,
                                     uint64_t seed, uint64_t* rows_out,
                                     uint64_t* groups_out, double* mean_label_iters) {
  if (!h || !src_ptr || S == 0 || docs_per_source == 0 || words_per_doc == 0 ||
      label_max_iter <= 0 || !(label_tol > 0.0) || lambda == 0.0)
    return fail(WMD_ERR_INVALID_ARG, "bad argument");
  if (!h->have_E || !h->have_T || h->tV != h->V)
    return fail(WMD_ERR_INVALID_ARG, "embeddings and targets must be set first");
  wmd_status st = bind(h);
  if (st) return st;
  const uint64_t V = h->V, d = h->d, N = h->N;
  const WsLayout L = ws_layout((int)d);
  const float expo = (float)(-lambda);
  std::vector<int32_t> nonempty;
  for (uint64_t j = 0; j < N; ++j)
    if (h->doc_len[j] > 0) nonempty.push_back((int32_t)j);
  if (nonempty.empty()) return fail(WMD_ERR_INVALID_INPUT, "no non-empty target document");
  const uint32_t D = std::min<uint64_t>(docs_per_source, nonempty.size());
  const int G = (int)words_per_doc;
  // Upper bound of the rows, then the buffers.
  uint64_t maxrows = 0, vr_max = 1;
  for (uint64_t s = 0; s < S; ++s) {
    if (src_ptr[s + 1] < src_ptr[s]) return fail(WMD_ERR_INVALID_INPUT, "source pointers decrease");
    const uint64_t vr = src_ptr[s + 1] - src_ptr[s];
    if (vr > 512) return fail(WMD_ERR_UNSUPPORTED, "training sources must have <= 512 words");
    for (uint64_t e = src_ptr[s]; e < src_ptr[s + 1]; ++e) {
      if (src_ids[e] >= V) return fail(WMD_ERR_INVALID_INPUT, "source word id >= V");
      if (e > src_ptr[s] && src_ids[e] <= src_ids[e - 1])
        return fail(WMD_ERR_INVALID_INPUT, "source word ids not strictly ascending");
      if (!(src_w[e] > 0.0) || !std::isfinite(src_w[e]))
        return fail(WMD_ERR_INVALID_INPUT, "source weight <= 0 or not finite");
    }
    maxrows += (uint64_t)D * std::min<uint64_t>(vr, (uint64_t)G);
    vr_max = std::max(vr_max, vr);
  }
  const int ld_max = (int)((vr_max + 3) & ~3ull);
  CK(h->ws_C.ensure((size_t)N * d * sizeof(float)));
  CK(h->ws_X.ensure((size_t)std::max<uint64_t>(maxrows, 1) * L.F * sizeof(float)));
  CK(h->ws_y.ensure((size_t)std::max<uint64_t>(maxrows, 1) * sizeof(float)));
  CK(h->K.ensure((size_t)V * ld_max * sizeof(float)));
  CK(h->sel_S.ensure((size_t)vr_max * d * sizeof(float)));
  CK(h->sel_nS.ensure((size_t)vr_max * sizeof(float)));
  const unsigned near_cap = (unsigned)std::min<uint64_t>((uint64_t)V * vr_max, 1u << 20);
  CK(h->near_pairs.ensure((size_t)near_cap * sizeof(uint2)));
  CK(h->near_count.ensure(sizeof(unsigned)));
  DevBuf ids_d, r64_d, rinv_d, docs_d, u_d, it_d, res_d, sel_d, row0_d, vrd;
  CK(ids_d.ensure(vr_max * 4));
  CK(r64_d.ensure(vr_max * 8));
  CK(rinv_d.ensure(vr_max * 4));
  CK(vrd.ensure(4));
  CK(docs_d.ensure((size_t)D * 4));
  CK(u_d.ensure((size_t)D * vr_max * 8));
  CK(it_d.ensure((size_t)D * 4));
  CK(res_d.ensure((size_t)D * 8));
  CK(sel_d.ensure((size_t)D * G * 4));
  CK(row0_d.ensure((size_t)D * 8));
  launch_centroids(h->E32.as<float>(), (int)d, h->col_ptr.as<int64_t>(),
                   h->ent.as<uint2>(), (int64_t)N, h->ws_C.as<float>(), h->stream);
  Targets t;
  t.col_ptr = h->col_ptr.as<int64_t>();
  t.ent = h->ent.as<uint2>();
  t.N = (int64_t)N;
  t.nnz = (int64_t)h->nnz;
  std::mt19937_64 rng(seed);
  std::vector<int64_t> gptr(1, 0);
  std::vector<uint32_t> gsrc, gdoc;
  std::vector<int32_t> rword;
  int64_t rows = 0;
  double it_sum = 0.0;
  uint64_t it_cnt = 0;
  std::vector<int32_t> docs(D), sel((size_t)D * G);
  std::vector<int> its(D);
  std::vector<double> res(D);
  std::vector<int64_t> row0(D);
  std::vector<uint32_t> ids32;
  std::vector<float> rinv;
  for (uint64_t s = 0; s < S; ++s) {
    const uint64_t off = src_ptr[s];
    const uint32_t vr = (uint32_t)(src_ptr[s + 1] - off);
    if (vr == 0) continue;
    const int ld = (int)((vr + 3) & ~3u);
    ids32.assign(vr, 0);
    rinv.assign(vr, 0.f);
    for (uint32_t i = 0; i < vr; ++i) {
      ids32[i] = (uint32_t)src_ids[off + i];
      rinv[i] = (float)(1.0 / src_w[off + i]);
    }
    CK(cudaMemcpyAsync(ids_d.p, ids32.data(), vr * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(r64_d.p, src_w + off, vr * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(rinv_d.p, rinv.data(), vr * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(vrd.p, &vr, 4, cudaMemcpyHostToDevice, h->stream));
    SourceSel sel_s;
    sel_s.ids = ids_d.as<uint32_t>();
    sel_s.rinv = rinv_d.as<float>();
    sel_s.S = h->sel_S.as<float>();
    sel_s.nS = h->sel_nS.as<float>();
    sel_s.vr = vrd.as<uint32_t>();
    sel_s.cap = vr;
    NearList near;
    near.pairs = h->near_pairs.as<uint2>();
    near.count = h->near_count.as<unsigned>();
    near.cap = near_cap;
    near.E32 = h->E32.as<float>();
    near.S32 = sel_s.S;
    near.d = (int)d;
    launch_gather_sources(sel_s.ids, (int)vr, h->E32.as<float>(), h->nE.as<float>(), d,
                          sel_s.S, sel_s.nS, nullptr, nullptr, 0, h->stream);
    CK(cudaMemsetAsync(near.count, 0, sizeof(unsigned), h->stream));
    // row-scaled panel when lambda * M can underflow FP32 (panel_rescale.cu);
    // the labels u are the same either way
    float* mrow = nullptr;
    if (row_scaled(h, expo)) {
      CK(h->mrow.ensure((size_t)V * sizeof(float)));
      mrow = h->mrow.as<float>();
      CK(cudaMemsetAsync(mrow, 0x7f, (size_t)V * sizeof(float), h->stream));
    }
    launch_cdist_fp32(h->E32.as<float>(), h->nE.as<float>(), V, d, sel_s, expo,
                      h->K.as<float>(), nullptr, ld, near, h->stream, mrow);
    launch_near_fixup(near, expo, h->K.as<float>(), nullptr, ld, V, h->nE.as<float>(),
                      sel_s.nS, sel_s.vr, h->sms, h->stream, mrow != nullptr);
    if (mrow)
      launch_panel_rescale(h->K.as<float>(), ld, V, sel_s.vr, mrow, expo, h->sms,
                           h->stream);
    // documents of this source: a seeded sample without replacement
    for (uint32_t q = 0; q < D; ++q) {
      const uint64_t k = q + rng() % (nonempty.size() - q);
      std::swap(nonempty[q], nonempty[k]);
      docs[q] = nonempty[q];
    }
    CK(cudaMemcpyAsync(docs_d.p, docs.data(), D * 4, cudaMemcpyHostToDevice, h->stream));
    if (launch_solve_f64(h->K.as<float>(), ld, (int)vr, r64_d.as<double>(),
                         t.col_ptr, t.ent, docs_d.as<int32_t>(), (int)D, label_tol,
                         label_max_iter, u_d.as<double>(), it_d.as<int>(),
                         res_d.as<double>(), h->stream) < 0)
      return fail(WMD_ERR_UNSUPPORTED, "label solve: too many source words");
    CK(cudaMemcpyAsync(its.data(), it_d.p, D * 4, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(res.data(), res_d.p, D * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const int g = std::min<int>(G, (int)vr);
    const uint32_t stride = vr / (uint32_t)g;
    for (uint32_t q = 0; q < D; ++q) {
      const bool keep = res[q] <= label_tol;
      row0[q] = keep ? rows : -1;
      const uint32_t rot = (uint32_t)(rng() % vr);
      for (int m = 0; m < G; ++m)
        sel[(size_t)q * G + m] = (keep && m < g) ? (int32_t)((rot + m * stride) % vr) : -1;
      if (keep) {
        rows += g;
        gptr.push_back(rows);
        gsrc.push_back((uint32_t)s);
        gdoc.push_back((uint32_t)docs[q]);
        for (int m = 0; m < g; ++m) rword.push_back(sel[(size_t)q * G + m]);
        it_sum += its[q];
        ++it_cnt;
      }
    }
    CK(cudaMemcpyAsync(sel_d.p, sel.data(), (size_t)D * G * 4, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(row0_d.p, row0.data(), (size_t)D * 8, cudaMemcpyHostToDevice, h->stream));
    launch_ws_rows(h->E32.as<float>(), (int)d, h->ws_C.as<float>(), h->K.as<float>(), ld,
                   expo, ids_d.as<uint32_t>(), r64_d.as<double>(), (int)vr, t.col_ptr,
                   t.ent, docs_d.as<int32_t>(), u_d.as<double>(), (int)D,
                   sel_d.as<int32_t>(), G, row0_d.as<int64_t>(), L.F,
                   h->ws_X.as<float>(), h->ws_y.as<float>(), h->stream, mrow);
    CK(cudaStreamSynchronize(h->stream));  // host vectors reused next source
    CK(cudaGetLastError());
  }
  if (rows == 0) return fail(WMD_ERR_INVALID_INPUT, "no labelled document converged");
  // Standardisation statistics (FP64 partial sums), then X in place.
  const int chunks = 256;
  DevBuf s1, s2;
  CK(s1.ensure((size_t)chunks * L.F * 8));
  CK(s2.ensure((size_t)chunks * L.F * 8));
  launch_ws_colstats(h->ws_X.as<float>(), rows, L.F, s1.as<double>(), s2.as<double>(),
                     chunks, h->stream);
  std::vector<double> a((size_t)chunks * L.F), b((size_t)chunks * L.F);
  CK(cudaMemcpyAsync(a.data(), s1.p, a.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(b.data(), s2.p, b.size() * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->ws_shift.assign(L.F, 0.f);
  h->ws_scale.assign(L.F, 1.f);
  for (int f = 0; f < L.F; ++f) {
    double m = 0.0, q = 0.0;
    for (int c = 0; c < chunks; ++c) {
      m += a[(size_t)c * L.F + f];
      q += b[(size_t)c * L.F + f];
    }
    m /= (double)rows;
    const double var = std::max(q / (double)rows - m * m, 0.0);
    h->ws_shift[f] = (float)m;
    h->ws_scale[f] = var > 1e-12 ? (float)(1.0 / std::sqrt(var)) : 1.f;
  }
  DevBuf sh, sc;
  CK(sh.ensure(L.F * 4));
  CK(sc.ensure(L.F * 4));
  CK(cudaMemcpyAsync(sh.p, h->ws_shift.data(), L.F * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(sc.p, h->ws_scale.data(), L.F * 4, cudaMemcpyHostToDevice, h->stream));
  launch_ws_standardize(h->ws_X.as<float>(), rows, L.F, sh.as<float>(), sc.as<float>(),
                        h->stream);
  h->ws_gptr_host = gptr;
  h->ws_gsrc = gsrc;
  h->ws_gdoc = gdoc;
  h->ws_rword = rword;
  CK(h->ws_gptr.ensure(gptr.size() * 8));
  CK(cudaMemcpyAsync(h->ws_gptr.p, gptr.data(), gptr.size() * 8, cudaMemcpyHostToDevice,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  h->ws_rows = rows;
  h->ws_d = (int)d;
  if (rows_out) *rows_out = (uint64_t)rows;
  if (groups_out) *groups_out = gptr.size() - 1;
  if (mean_label_iters) *mean_label_iters = it_cnt ? it_sum / (double)it_cnt : 0.0;
  return WMD_OK;
}

wmd_status wmd_ws_train(wmd_handle* h, float* params, int epochs,
                        uint64_t batch_groups, float lr, uint64_t seed,
                        double* loss_out) {
  if (!h || !params || epochs <= 0 || batch_groups == 0 || !(lr > 0.f))
    return fail(WMD_ERR_INVALID_ARG, "bad argument");
  if (h->ws_rows == 0) return fail(WMD_ERR_INVALID_ARG, "no training set built");
  wmd_status st = bind(h);
  if (st) return st;
  const WsLayout L = ws_layout(h->ws_d);
  // The model's standardisation is the training set's.
  std::copy(h->ws_shift.begin(), h->ws_shift.end(), params + L.shift);
  std::copy(h->ws_scale.begin(), h->ws_scale.end(), params + L.scale);
  const int64_t ngroups = (int64_t)h->ws_gptr_host.size() - 1;
  int64_t maxg = 0;
  for (int64_t g = 0; g < ngroups; ++g)
    maxg = std::max(maxg, h->ws_gptr_host[g + 1] - h->ws_gptr_host[g]);
  const int64_t bmax = (int64_t)std::min<uint64_t>(batch_groups, ngroups) * maxg;
  DevBuf P, Gd, M1, M2, Xb, tb, bp, perm_d, scr, lossg;
  CK(P.ensure(L.count * 4));
  CK(Gd.ensure(L.count * 4));
  CK(M1.ensure(L.count * 4));
  CK(M2.ensure(L.count * 4));
  CK(Xb.ensure((size_t)bmax * L.F * 4));
  CK(tb.ensure((size_t)bmax * 4));
  CK(bp.ensure((size_t)(batch_groups + 1) * 8));
  CK(perm_d.ensure((size_t)ngroups * 8));
  CK(scr.ensure(ws_scratch_floats(bmax, L.F) * 4));
  CK(lossg.ensure((size_t)batch_groups * 8));
  CK(cudaMemcpyAsync(P.p, params, L.count * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(M1.p, 0, L.count * 4, h->stream));
  CK(cudaMemsetAsync(M2.p, 0, L.count * 4, h->stream));
  std::vector<int64_t> perm(ngroups), bptr;
  std::vector<double> lg(batch_groups);
  std::mt19937_64 rng(seed);
  int step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int64_t g = 0; g < ngroups; ++g) perm[g] = g;
    std::shuffle(perm.begin(), perm.end(), rng);
    CK(cudaMemcpyAsync(perm_d.p, perm.data(), ngroups * 8, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double loss = 0.0;
    for (int64_t g0 = 0; g0 < ngroups; g0 += (int64_t)batch_groups) {
      const int64_t ng = std::min<int64_t>((int64_t)batch_groups, ngroups - g0);
      bptr.assign(ng + 1, 0);
      for (int64_t q = 0; q < ng; ++q) {
        const int64_t g = perm[g0 + q];
        bptr[q + 1] = bptr[q] + (h->ws_gptr_host[g + 1] - h->ws_gptr_host[g]);
      }
      const int64_t rows = bptr[ng];
      CK(cudaMemcpyAsync(bp.p, bptr.data(), (ng + 1) * 8, cudaMemcpyHostToDevice, h->stream));
      launch_ws_gather(h->ws_X.as<float>(), h->ws_y.as<float>(), h->ws_gptr.as<int64_t>(),
                       perm_d.as<int64_t>(), bp.as<int64_t>(), g0, ng, L.F,
                       Xb.as<float>(), tb.as<float>(), h->stream);
      launch_ws_fwd_bwd(L, P.as<float>(), Xb.as<float>(), tb.as<float>(), bp.as<int64_t>(),
                        ng, rows, Gd.as<float>(), lossg.as<double>(), scr.as<float>(),
                        h->stream);
      launch_ws_adam(L, P.as<float>(), Gd.as<float>(), M1.as<float>(), M2.as<float>(), lr,
                     ++step, h->stream);
      CK(cudaMemcpyAsync(lg.data(), lossg.p, ng * 8, cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));  // bptr / lg reused next batch
      CK(cudaGetLastError());
      double bl = 0.0;
      for (int64_t q = 0; q < ng; ++q) bl += lg[q];
      loss += bl * (double)rows;
    }
    if (loss_out) loss_out[ep] = loss / (double)h->ws_rows;
  }
  CK(cudaMemcpyAsync(params, P.p, L.count * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return WMD_OK;
}

wmd_status wmd_ws_loss_grad(wmd_handle* h, uint64_t d, const float* X,
                            const float* t, const int64_t* gptr, uint64_t ngroups,
                            const float* params, double* loss, float* grad) {
  if (!h || !X || !t || !gptr || ngroups == 0 || !params || !loss || !grad || d == 0)
    return fail(WMD_ERR_INVALID_ARG, "bad argument");
  wmd_status st = bind(h);
  if (st) return st;
  const WsLayout L = ws_layout((int)d);
  const int64_t rows = gptr[ngroups];
  if (rows <= 0 || gptr[0] != 0) return fail(WMD_ERR_INVALID_ARG, "bad group pointers");
  DevBuf P, Gd, Xd, td, gp, scr, lossg;
  CK(P.ensure(L.count * 4));
  CK(Gd.ensure(L.count * 4));
  CK(Xd.ensure((size_t)rows * L.F * 4));
  CK(td.ensure((size_t)rows * 4));
  CK(gp.ensure((ngroups + 1) * 8));
  CK(scr.ensure(ws_scratch_floats(rows, L.F) * 4));
  CK(lossg.ensure(ngroups * 8));
  CK(cudaMemcpyAsync(P.p, params, L.count * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(Xd.p, X, (size_t)rows * L.F * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(td.p, t, (size_t)rows * 4, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(gp.p, gptr, (ngroups + 1) * 8, cudaMemcpyHostToDevice, h->stream));
  launch_ws_standardize(Xd.as<float>(), rows, L.F, P.as<float>() + L.shift,
                        P.as<float>() + L.scale, h->stream);
  launch_ws_fwd_bwd(L, P.as<float>(), Xd.as<float>(), td.as<float>(), gp.as<int64_t>(),
                    (int64_t)ngroups, rows, Gd.as<float>(), lossg.as<double>(),
                    scr.as<float>(), h->stream);
  std::vector<double> lg(ngroups);
  CK(cudaMemcpyAsync(grad, Gd.p, L.count * 4, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(lg.data(), lossg.p, ngroups * 8, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  double l = 0.0;
  for (uint64_t g = 0; g < ngroups; ++g) l += lg[g];
  *loss = l;
  return WMD_OK;
}

wmd_status wmd_ws_get_training_set(wmd_handle* h, float* X, float* y, int64_t* gptr,
                                   uint32_t* group_source, uint32_t* group_doc,
                                   int32_t* row_word) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  if (h->ws_rows == 0) return fail(WMD_ERR_INVALID_ARG, "no training set built");
  wmd_status st = bind(h);
  if (st) return st;
  const WsLayout L = ws_layout(h->ws_d);
  if (X) CK(cudaMemcpy(X, h->ws_X.p, (size_t)h->ws_rows * L.F * 4, cudaMemcpyDeviceToHost));
  if (y) CK(cudaMemcpy(y, h->ws_y.p, (size_t)h->ws_rows * 4, cudaMemcpyDeviceToHost));
  if (gptr) std::copy(h->ws_gptr_host.begin(), h->ws_gptr_host.end(), gptr);
  if (group_source) std::copy(h->ws_gsrc.begin(), h->ws_gsrc.end(), group_source);
  if (group_doc) std::copy(h->ws_gdoc.begin(), h->ws_gdoc.end(), group_doc);
  if (row_word) std::copy(h->ws_rword.begin(), h->ws_rword.end(), row_word);
  return WMD_OK;
}

wmd_status wmd_set_warm_start(wmd_handle* h, const float* params) {
  if (!h) return fail(WMD_ERR_INVALID_ARG, "null handle");
  wmd_status st = bind(h);
  if (st) return st;
  h->graph_epoch++;
  h->ws_docs_ready = false;
  if (!params) {
    h->ws_on = false;
    return WMD_OK;
  }
  if (!h->have_E) return fail(WMD_ERR_INVALID_ARG, "embeddings must be set first");
  const WsLayout L = ws_layout((int)h->d);
  CK(h->ws_params.ensure(L.count * 4));
  CK(h->ws_folded.ensure(ws_folded_floats(L) * 4));
  CK(cudaMemcpyAsync(h->ws_params.p, params, L.count * 4, cudaMemcpyHostToDevice,
                     h->stream));
  launch_ws_fold(L, h->ws_params.as<float>(), h->ws_folded.as<float>(), h->stream);
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaGetLastError());
  h->ws_d = (int)h->d;
  h->ws_on = true;
  return WMD_OK;
}

wmd_status wmd_ws_init_scalings(wmd_handle* h, const double* r, double lambda,
                                float* u0_out, uint64_t* vr_out) {
  if (!h || !r || !u0_out || !vr_out || lambda == 0.0)
    return fail(WMD_ERR_INVALID_ARG, "bad argument");
  if (!h->ws_on) return fail(WMD_ERR_INVALID_ARG, "no warm-start model set");
  wmd_status st = bind(h);
  if (st) return st;
  // A zero-iteration query runs selection, the cost panel and the
  // warm-start init; the scalings are then read back.
  const bool g = h->use_graphs;
  h->use_graphs = false;
  std::vector<double> scratch(h->N);
  st = query_host(h, r, (float)(-lambda), 0, scratch.data());
  h->use_graphs = g;
  if (st) return st;
  uint32_t vr = 0;
  CK(cudaMemcpy(&vr, h->sel_vr.p, 4, cudaMemcpyDeviceToHost));
  const int ld = (int)(((vr ? vr : 1) + 3u) & ~3u);
  *vr_out = vr;
  if (vr == 0) return WMD_OK;
  CK(cudaMemcpy2D(u0_out, vr * sizeof(float), h->ws_u0.p, ld * sizeof(float),
                  vr * sizeof(float), h->N, cudaMemcpyDeviceToHost));
  return WMD_OK;
}

/* ------------------------------------------------------------------------
 * Edge lists (the reference's mat.mtx entries) -> document-major CSC on the
 * GPU.
 * ---------------------------------------------------------------------- */
static wmd_status edges_to_stage(wmd_handle* h, const uint64_t* words,
                                 const uint64_t* docs, const double* w, uint64_t nnz,
                                 uint64_t V, uint64_t N) {
  if (!h || (nnz && (!words || !docs || !w)) || V == 0 || N == 0)
    return fail(WMD_ERR_INVALID_ARG, "bad argument");
  if (nnz == 0) return fail(WMD_ERR_INVALID_INPUT, "edge list is empty");
  if (N >= 0x7FFFFFFFull) return fail(WMD_ERR_UNSUPPORTED, "more than 2^31-1 documents");
  wmd_status st = bind(h);
  if (st) return st;
  const size_t tb = csc_build_temp_bytes(nnz, V, N);
  CK(h->edge_words.ensure(nnz * 8));
  CK(h->edge_docs.ensure(nnz * 8));
  CK(h->edge_w.ensure(nnz * 8));
  CK(h->edge_temp.ensure(tb));
  CK(h->stage_cp.ensure((N + 1) * 8));
  CK(h->stage_rows.ensure(nnz * 8));
  CK(h->stage_vals.ensure(nnz * 8));
  CK(cudaMemcpyAsync(h->edge_words.p, words, nnz * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->edge_docs.p, docs, nnz * 8, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->edge_w.p, w, nnz * 8, cudaMemcpyHostToDevice, h->stream));
  st = clear_err(h);
  if (st) return st;
  const int n = launch_csc_build(h->edge_words.as<uint64_t>(), h->edge_docs.as<uint64_t>(),
                                 h->edge_w.as<double>(), nnz, V, N, h->edge_temp.p, tb,
                                 h->stage_cp.as<uint64_t>(), h->stage_rows.as<uint64_t>(),
                                 h->stage_vals.as<double>(), h->err_dev.as<unsigned>(),
                                 h->stream);
  if (n < 0) return fail(WMD_ERR_UNSUPPORTED, "edge list too large for the GPU sort");
  CK(cudaGetLastError());
  h->last_launches = n;
  return finish(h);
}

wmd_status wmd_edges_to_csc(wmd_handle* h, const uint64_t* words, const uint64_t* docs,
                            const double* w, uint64_t nnz, uint64_t V, uint64_t N,
                            uint64_t* col_ptr_out, uint64_t* rows_out,
                            double* vals_out) {
  if (!col_ptr_out || !rows_out || !vals_out) return fail(WMD_ERR_INVALID_ARG, "null output");
  wmd_status st = edges_to_stage(h, words, docs, w, nnz, V, N);
  if (st) return st;
  CK(cudaMemcpy(col_ptr_out, h->stage_cp.p, (N + 1) * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(rows_out, h->stage_rows.p, nnz * 8, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(vals_out, h->stage_vals.p, nnz * 8, cudaMemcpyDeviceToHost));
  return WMD_OK;
}

wmd_status wmd_set_targets_edges(wmd_handle* h, const uint64_t* words,
                                 const uint64_t* docs, const double* w, uint64_t nnz,
                                 uint64_t V, uint64_t N) {
  wmd_status st = edges_to_stage(h, words, docs, w, nnz, V, N);
  if (st) return st;
  std::vector<uint64_t> cp(N + 1);
  CK(cudaMemcpy(cp.data(), h->stage_cp.p, (N + 1) * 8, cudaMemcpyDeviceToHost));
  std::vector<int32_t> ord;
  length_order(cp.data(), N, ord);
  CK(h->col_ptr.ensure((N + 1) * sizeof(int64_t)));
  CK(h->ent.ensure(nnz * sizeof(uint2)));
  CK(h->order.ensure(N * sizeof(int32_t)));
  CK(cudaMemcpyAsync(h->order.p, ord.data(), N * sizeof(int32_t), cudaMemcpyHostToDevice,
                     h->stream));
  st = clear_err(h);
  if (st) return st;
  const int launches = launch_pack_targets(
      h->stage_cp.as<uint64_t>(), h->stage_rows.as<uint64_t>(), h->stage_vals.as<double>(),
      V, N, nnz, h->col_ptr.as<int64_t>(), h->ent.as<uint2>(), h->err_dev.as<unsigned>(),
      h->stream);
  CK(cudaGetLastError());
  h->have_T = false;
  st = finish(h);
  if (st) return st;
  h->tV = V;
  h->N = N;
  h->nnz = nnz;
  h->have_T = true;
  h->wm_ready = false;
  h->ws_docs_ready = false;
  for (int& x : h->blk_shape) x = -2;
  for (int& x : h->warp_shape) x = -2;
  for (auto& row : h->tc_long)
    for (int64_t& x : row) x = -1;
  h->doc_len.resize(N);
  for (uint64_t j = 0; j < N; ++j) h->doc_len[j] = (uint32_t)(cp[j + 1] - cp[j]);
  h->graph_epoch++;
  h->last_launches += launches;
  return WMD_OK;
}

}  // extern "C"
