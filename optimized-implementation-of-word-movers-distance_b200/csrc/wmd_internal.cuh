// Internal interfaces between the kernels and the C-ABI layer.
//
// Device data layout (all row-major, all resident in HBM):
//   E32   [V][d]    float   embeddings (converted once from the caller's FP64)
//   nE    [V]       float   squared row norms of E32
//   E16   [V][dp]   bf16/f16 tensor-core copy of E32, dp = d rounded up to 64
//   S     [cap][d]  float   embeddings of the selected source words
//   nS    [cap]     float   their squared norms
//   K     [V][ld]   float   exp(expo * M) for every (vocabulary word, source word)
//   KM    [V][ld]   float   K * M, only when expo = 0 (otherwise the solve
//                           recovers K*M from K as K ln(K) / expo)
//   col_ptr [N+1]   int64   target columns (documents)
//   ent   [nnz]     uint2   {word id, float bits of the normalised count}
// ld = number of source words rounded up to a multiple of 4, so that every
// panel row starts on a 16-byte boundary and is one contiguous gather.
#pragma once
#include <cuda_runtime.h>
#include <utility>
#include <stdint.h>

namespace wmd {

// Programmatic dependent launch (build-time option, off by default).  With
// WMD_PDL >= 1 the kernels of a query after the first (selection write, cost
// panel, near-pair fix-up, solve) are launched with
// cudaLaunchAttributeProgrammaticStreamSerialization, so each one's launch
// and set-up (shared-memory layout, barrier initialisation, tensor-memory
// allocation) may overlap the end of the kernel before it; grid_dep_wait()
// then blocks until that kernel has completed and its writes are visible.
// Every kernel launched this way calls it before its first access to
// anything an earlier kernel of the stream writes, and before its first write
// to anything an earlier kernel reads; launched without the attribute it
// returns at once.  Measured on the B200 (single-source query, 100 timed
// steps, two runs each on one box): 0.163 / 0.165 ms per step with ordinary
// launches, 0.166 / 0.166 with the attribute, 0.170 / 0.171 with the early
// triggers as well (the next kernel's early CTAs take SM resources from the
// kernel before it), hence the default.
// Build-time knob: 0 = ordinary launches, 1 = the attribute (each kernel's
// launch overlaps the end of the one before), 2 = also the early triggers
// below.
#ifndef WMD_PDL
#define WMD_PDL 0
#endif
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}
// Lets the next kernel of the stream (if launched with the attribute) start
// its CTAs now: called at the start of the query's selection, cost-panel and
// fix-up kernels, when every CTA of the grid is resident, so the early CTAs
// of the next kernel can only take resources this grid no longer waits for.
__device__ __forceinline__ void grid_dep_launch() {
#if WMD_PDL >= 2
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
#endif
}

template <class... P, class... A>
inline cudaError_t launch_pdl(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = WMD_PDL >= 1 ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// Device-side validation bits, OR-ed into one word per handle.
enum : unsigned {
  ERR_ROW_RANGE = 1u,  // word id >= V
  ERR_COLPTR = 2u,     // column pointers decrease, do not start at 0 or pass nnz
  ERR_NEG_R = 4u,      // source weight < 0 (the reference driver rejects it)
  ERR_BAD_VAL = 8u,    // target value <= 0 or not finite
  ERR_VR_CAP = 16u,    // more selected source words than the panel capacity
  ERR_TIMEOUT = 32u,   // a bounded device-side wait gave up (kernel aborted)
  ERR_DOC_RANGE = 64u, // document id >= N (edge-list input)
};

constexpr int kSelectThreads = 256;
constexpr int kSelectPerThread = 4;
constexpr int kSelectChunk = kSelectThreads * kSelectPerThread;

// Near-pair threshold: pairs whose GEMM-form squared distance falls below
// this are recomputed exactly (the GEMM form cancels for close pairs).
__host__ __device__ __forceinline__ float near_threshold(float na, float nb) {
  return fmaxf(0.25f, (na + nb) * (1.f / 30.f));
}

// Exact FP32 |a - b|^2 computed by a whole warp (lanes split the d
// coordinates, shuffle-reduced); every lane gets the result.  Must be called
// by all 32 lanes.
__device__ __forceinline__ float warp_sqdist(const float* __restrict__ a,
                                             const float* __restrict__ b,
                                             int d, int lane) {
  float s = 0.f;
  for (int k = lane; k < d; k += 32) {
    const float t = a[k] - b[k];
    s = fmaf(t, t, s);
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  return s;
}

// Cancellation-prone (vocabulary word, source word) pairs found by a cost-panel
// epilogue, recomputed exactly by near_fixup_kernel.  When more than `cap`
// pairs turn up, that kernel scans the whole panel instead (correct, only
// slower).
struct NearList {
  uint2* pairs = nullptr;     // [cap] {word id, source index}
  unsigned* count = nullptr;  // must be zero before the cost panel runs
  unsigned cap = 0;
  const float* E32 = nullptr;
  const float* S32 = nullptr;
  int d = 0;
};

__device__ __forceinline__ void near_pair(const NearList& nl, uint64_t w, int i) {
  const unsigned pos = atomicAdd(nl.count, 1u);
  if (pos < nl.cap) nl.pairs[pos] = make_uint2((unsigned)w, (unsigned)i);
}

struct SourceSel {
  uint32_t* ids = nullptr;     // [cap]
  float* rinv = nullptr;       // [cap]  1 / r_i
  float* S = nullptr;          // [cap][d]
  float* nS = nullptr;         // [cap]
  uint32_t* vr = nullptr;      // [1]    number of selected words
  uint32_t* chunk_counts = nullptr;  // [ceil(V / kSelectChunk)]
  uint32_t cap = 0;
};

struct Targets {
  const int64_t* col_ptr = nullptr;
  const uint2* ent = nullptr;
  const int32_t* order = nullptr;  // columns by decreasing length (or null)
  int64_t N = 0;
  int64_t nnz = 0;
};

// Message returned by wmd_last_error() on the calling host thread.
void set_last_error(const char* msg);

inline int select_num_chunks(uint64_t V) {
  return (int)((V + kSelectChunk - 1) / kSelectChunk);
}

// Embeddings: FP64 or FP32 source -> E32 + nE.  Returns launches issued.
int launch_embed_convert_f64(const double* src, uint64_t V, uint64_t d,
                             float* E32, float* nE, cudaStream_t st);
int launch_embed_norms(const float* E32, uint64_t V, uint64_t d, float* nE,
                       cudaStream_t st);
// BF16 embeddings [V][d] (raw bit patterns) -> E32 (exact) and E16 [V][dp].
int launch_embed_from_bf16(const void* src, uint64_t V, uint64_t d, int dp, float* E32,
                           void* E16, cudaStream_t st);
// Drop-in rows split between the host and the bus: words below wh from
// rows32 (narrowed on the host; phase 1), above it the rows of the words a
// query can touch (target words in `ent`, source words r_dev != 0; flags in
// `need`, V bytes of scratch) read from device-mapped host memory, the others
// zeroed (phase 0; *nrows receives the rows read over the bus).  E32 and nE
// come out as launch_embed_convert_f64 writes them for the whole matrix.
int launch_gather_rows_split(const double* src_mapped, const uint2* ent, uint64_t nnz,
                             const double* r_dev, unsigned char* need, uint64_t V,
                             uint64_t d, uint64_t wh, const float* rows32, int phase,
                             float* E32, float* nE, unsigned long long* nrows,
                             cudaStream_t st);

// Targets: validated packing of a CSC triple into (col_ptr, ent).
int launch_pack_targets(const uint64_t* col_ptr_in, const uint64_t* rows_in,
                        const double* vals_in, uint64_t V, uint64_t N,
                        uint64_t nnz, int64_t* col_ptr, uint2* ent,
                        unsigned* err, cudaStream_t st);

// Count pass of the selection alone (per-chunk non-zero counts).
int launch_select_count(const double* r, uint64_t V, uint32_t* chunk_counts,
                        unsigned* err, cudaStream_t st);

// Source selection r != 0 (ascending id) + gather of the source rows (and,
// when S16 is given, of their 16-bit copies [cap][dp] from E16 [V][dp]).
// zero_word, when given, is set to 0 by the first kernel (the near-pair
// counter of the cost panel that follows).
int launch_select(const double* r, uint64_t V, const float* E32,
                  const float* nE, uint64_t d, const SourceSel& s,
                  unsigned* err, cudaStream_t st, const void* E16 = nullptr,
                  void* S16 = nullptr, int dp = 0, unsigned* zero_word = nullptr);

// Top-k nearest documents (topk.cu): stable ascending order of the FP64
// scores, ties by index, NaN last.  1 <= k <= 1024.
size_t topk_scratch_bytes(uint64_t n, int k);
int launch_topk(const double* scores, uint64_t n, int k, void* scratch,
                uint32_t* out_idx, double* out_val, cudaStream_t st);

// Batched queries: gather the rows of one source from its uploaded ids.
int launch_gather_sources(const uint32_t* ids, int count, const float* E32,
                          const float* nE, uint64_t d, float* S, float* nS,
                          const void* E16, void* S16, int dp, cudaStream_t st);

// FP32 CUDA-core cost panel: K = exp(expo * M), and KM = K * M when KM is
// not null; M from the GEMM form with near pairs recomputed directly.
// mrow (row-scaled form, expo != 0): the panel receives M and mrow [V] (set
// to FLT_MAX bits 0x7f7f7f7f beforehand) the row minima; see panel_rescale.cu.
int launch_cdist_fp32(const float* E32, const float* nE, uint64_t V, uint64_t d,
                      const SourceSel& s, float expo, float* K, float* KM,
                      int ld, const NearList& near, cudaStream_t st,
                      float* mrow = nullptr);

// Tensor-core cost panel (cdist_tc.cu).  Forms: 16-bit operands (E16/S16
// rows are dp = d rounded up to 8 elements), or the FP32-accurate split-TF32
// form that reads E32/S directly (E16/S16 unused; needs d % 4 == 0).
// Returns launches, or -1 if unsupported (tensor maps or shared-memory
// budget).
// TC_F16X3: the split-FP16 form; E16 / S16 then hold split rows of
// tc_split_row_bytes(d) bytes each (launch_to_split16): FP16 high part,
// scaled FP16 low part, the row's 1/scale.
enum TcForm { TC_FP16 = 0, TC_BF16 = 1, TC_TF32X3 = 2, TC_F16X3 = 3 };
struct GroupSrc;
// A stacked batch group's cost panel (batch.cu): N-tile y of the launch is
// tiles[y] = {source, first stacked source row, first panel column, 0}, the
// sources' panels in src[] (device arrays), nt source rows per tile.
struct StackedPanels {
  const int4* tiles = nullptr;
  const GroupSrc* src = nullptr;
  int ntiles = 0, nt = 0;
};
int tc_padded_width(uint64_t d);
int tc_tile_n(uint32_t cap, uint64_t d);
int tc_tile_n_x3(uint32_t cap, uint64_t d);  // 0 = form unsupported
int tc_tile_n_h2(uint32_t cap, uint64_t d);  // 0 = form unsupported
size_t tc_split_row_bytes(uint64_t d);       // 4 * dp + 16
int launch_to_split16(const float* E32, uint64_t rows, uint64_t d, void* Esplit,
                      cudaStream_t st);
int launch_to16(const float* E32, uint64_t rows, uint64_t d, void* E16,
                bool bf16, cudaStream_t st);
int launch_cdist_tc(int form, const void* E16, const void* S16,
                    const float* E32, const float* nE, uint64_t V, uint64_t d,
                    const SourceSel& s, float expo, float* K, float* KM, int ld,
                    const NearList& near, unsigned* err, int num_sms,
                    cudaStream_t st, float* mrow = nullptr,
                    const StackedPanels* grp = nullptr);

// Exact FP32 recompute of the listed near pairs (after either cost panel);
// pairs beyond the list capacity are recomputed by a full-panel scan.
// scaled: the row-scaled form (the panel holds M; exact M is written).
int launch_near_fixup(const NearList& near, float expo, float* K, float* KM,
                      int ld, uint64_t V, const float* nE, const float* nS,
                      const uint32_t* vr, int num_sms, cudaStream_t st,
                      bool scaled = false);

// Row-scaled panel (panel_rescale.cu): M -> K' = exp(expo (M - mrow[w])) in
// place, zero past v_r.  max_norm: the largest squared row norm of E as float
// bits into *out (device), which decides whether the row-scaled form is used.
int launch_panel_rescale(float* K, int ld, uint64_t V, const uint32_t* vr,
                         const float* mrow, float expo, int num_sms, cudaStream_t st);
int launch_max_norm(const float* nE, uint64_t V, unsigned* out, cudaStream_t st);
// lambda * M can pass this in a panel row only when the row-scaled form is on.
constexpr float kScaleLimit = 80.f;
// On a row-scaled panel, a final scaling u_i above this marks a document
// whose K entries for source word i sit at the FP32 floor; it is re-solved
// in FP64 with the non-finite ones.
constexpr float kScaledUMax = 1e30f;

// FP64 re-solve (exact_f64.cu) of the documents whose FP32 result on a
// row-scaled panel is not finite: lists them (at most exact_f64_list_cap())
// and solves them again with M recomputed from E32 and the selected rows.
// Returns launches, -1 if max_doc_len is too long for its shared memory.
size_t exact_f64_list_cap();
struct SolveCtl;
int launch_exact_f64(const float* E32, uint64_t d, const SourceSel& s, const Targets& t,
                     float expo, const SolveCtl& ctl, int max_doc_len, int32_t* list,
                     unsigned* count, int num_sms, double* out, cudaStream_t st);

// Iteration control of the solve.  tol <= 0: exactly max_iter x-updates, as
// the reference (sinkhorn_wmd_fused.cpp:246).  tol > 0: a document stops
// after the first update whose marginal residual sum_i |u_i (K v)_i - r_i|
// (measured with the scalings entering that update) is <= tol, or after
// max_iter updates.  iters (optional, [N]) receives each document's count.
// u0 (optional, [N][ldu]): initial scaling per document (warm start); the
// first update is then evaluated from both u0 and the cold start and the one
// with the smaller marginal residual is kept.
// omega: over-relaxation of both half-steps, v <- v^(1-omega) * v_hat^omega
// and u <- u^(1-omega) * u_hat^omega with v_hat = c / (K^T u) and u_hat the
// plain u update (omega = 1: the reference's iteration).  The fixed point is
// the same; for 1 < omega < 2 slowly converging documents need far fewer
// updates (overrelaxed Sinkhorn-Knopp: Thibault, Chizat, Dossal and
// Papadakis, 2017; Lehmann, von Renesse, Sambale and Uschmajew, 2021).  A
// word's previous v lives in vstate[entry] (required when omega != 1, [nnz]);
// the residual then adds the c-side marginal sum_k |v_k (K u)_k - c_k|, and a
// per-document guard halves omega - 1 (restarting v exactly) when the
// residual exceeds kRelaxGuard times the best one seen, and restarts the
// document from the cold start unrelaxed (omega = 1 from then on) when the
// residual is not finite.  Relaxation needs per-document stopping (tol > 0):
// the caller passes omega = 1 for a fixed update count.
// mrow: row minima of M of a row-scaled panel (panel_rescale.cu), or null;
// the final sum then adds c_w * mrow[w] per document word.
struct SolveCtl {
  int max_iter = 15;
  float tol = 0.f;
  int* iters = nullptr;
  const float* u0 = nullptr;
  int64_t ldu = 0;
  float omega = 1.f;
  float* vstate = nullptr;
  const float* mrow = nullptr;
};

constexpr float kRelaxGuard = 100.f;

// The relaxed update of one scaling entry (see SolveCtl::omega).
__device__ __forceinline__ float relaxed_update(float u_old, float u_hat, float omega) {
  if (omega == 1.f) return u_hat;
  return u_old * exp2f(omega * __log2f(u_hat / u_old));
}

// v of one target word under over-relaxation: v_hat = c / s relaxed against
// the word's previous v (kept in *slot); exactly v_hat on a document's first
// pass or after a guard reset.  Adds |v s - c| to resv.  Padding words
// (c = 0) give 0 and touch nothing.
__device__ __forceinline__ float relaxed_v(float c, float s, float* slot, bool first,
                                           float omega, float& resv) {
  if (c == 0.f) return 0.f;
  const float vh = __fdividef(c, s);
  const float v = first ? vh : relaxed_update(*slot, vh, omega);
  *slot = v;
  resv += fabsf(v * s - c);
  return v;
}
// The same with the previous v already loaded (vold, ignored when first):
// kernels prefetch it with the word's row, off the s -> v critical path.
__device__ __forceinline__ float relaxed_v_pre(float c, float s, float vold, float* slot,
                                               bool first, float omega, float& resv) {
  if (c == 0.f) return 0.f;
  const float vh = __fdividef(c, s);
  const float v = first ? vh : relaxed_update(vold, vh, omega);
  *slot = v;
  resv += fabsf(v * s - c);
  return v;
}

// Per-document over-relaxation guard (uniform over the threads of a
// document).  Returns true when it reset: omega stepped halfway to 1, v to
// restart exactly; *reset_u when the residual was not finite.
struct RelaxGuard {
  float omega, best;
  bool vfirst;
  __device__ __forceinline__ void init(float om) {
    omega = om;
    best = __int_as_float(0x7f800000);
    vfirst = true;
  }
  __device__ __forceinline__ bool step(float res, int it, bool* reset_u) {
    *reset_u = false;
    vfirst = false;
    if (omega == 1.f) return false;
    if (!isfinite(res)) {  // diverged: cold start, plain iteration
      omega = 1.f;
      vfirst = true;
      *reset_u = true;
      return true;
    }
    if (it > 2 && res > kRelaxGuard * best) {
      omega = 1.f + 0.5f * (omega - 1.f);
      if (omega < 1.01f) omega = 1.f;
      best = __int_as_float(0x7f800000);
      vfirst = true;
      return true;
    }
    best = fminf(best, res);
    return false;
  }
};

// One source of a stacked batch group (batch.cu): its panels, weights and
// outputs, and its place in the stacked source rows.
struct GroupSrc {
  float* K = nullptr;          // FP32 panel [V][ld]
  void* K16 = nullptr;         // BF16 panel [V][ld16] (block solve) or null
  float* mrow = nullptr;       // row minima (row-scaled panel) or null
  const float* rinv = nullptr; // [vr] 1 / r_i
  const uint32_t* vr_dev = nullptr;  // [1] v_r on the device
  double* out = nullptr;       // [N] scores
  int* iters = nullptr;        // [N] update counts or null
  float* vstate = nullptr;     // [nnz] previous v (over-relaxed) or null
  int vr = 0, ld = 0, row0 = 0, pad = 0;
};

// Stacked batch group: one persistent warp-solve launch over all (source,
// document) pairs of nsrc sources with v_r <= vr_max (grp: device array).
// shape: launch shape of the unrelaxed solve (0 .. solve_shape_count() - 1,
// as for launch_solve), -1 the build-time default.
int launch_solve_group(uint32_t vr_max, const GroupSrc* grp, int nsrc, float expo,
                       const Targets& t, const SolveCtl& ctl, cudaStream_t st,
                       int shape = -1);

// Stacked batch groups (batch.cu): stacked source rows (rowword: embedding
// row per stacked row, -1 = zeros), near-pair fix-up with pairs {word,
// stacked row} (rowsrc: source of each stacked row), FP32 -> BF16 panels.
int launch_group_gather(const int32_t* rowword, int rows, const float* E32,
                        const float* nE, uint64_t d, float* S, float* nS,
                        const void* E16, void* S16, int dp, int num_sms, cudaStream_t st);
int launch_near_fixup_group(const NearList& near, float expo, const int32_t* rowsrc,
                            const GroupSrc* grp, int nsrc, uint64_t V, const float* nE,
                            const float* nS, int num_sms, cudaStream_t st);
int launch_panel_to_bf16_group(const GroupSrc* grp, int nsrc, uint64_t V, int ld16,
                               int num_sms, cudaStream_t st);

// Stacked batch group on BF16 panels of width ld16 (64 < v_r <= 512): one
// persistent CTA-per-document launch over all (source, document) pairs.
// shape: 0 = 4 warps x 4 CTAs/SM, 1 = 8 x 2, 2 = 16 x 1.
int launch_block_group(const GroupSrc* grp, int nsrc, int ld16, float expo,
                       const Targets& t, const SolveCtl& ctl, int shape, cudaStream_t st);

// Fused Sinkhorn iterations + final half-step + FP64 reduction, one warp per
// target document.  Returns launches issued (-1 on unsupported vr_cap).
// KM may be null unless expo == 0.
// shape: an autotuner candidate of the plain warp solve (0 .. 2, see
// solve_shape_name) or -1 for the build-time default.
int launch_solve(const float* K, const float* KM, int ld, float expo,
                 uint32_t vr_cap, const SourceSel& s, const Targets& t,
                 const SolveCtl& ctl, double* out, cudaStream_t st, int shape = -1);
int solve_shape_count();
const char* solve_shape_name(int shape);

// Word-major solve (solve_word.cu): the reference's traversal order, each K
// row read once per pass, u gathered and x scattered (atomics) per entry.
// Fixed update count, cold start, unrelaxed.  ent: {document, float bits of
// c} in word-major order, row_ptr [V+1].  u, x: scratch [N][ld].
struct WordMajor {
  const int64_t* row_ptr = nullptr;
  const uint2* ent = nullptr;
  int64_t V = 0, nnz = 0;
  const float* mrow = nullptr;  // row-scaled panel, or null
};
int launch_solve_word(const float* K, int ld, float expo, uint32_t vr_cap,
                      const SourceSel& s, const WordMajor& wm, int64_t N, int max_iter,
                      float* u, float* x, int num_sms, double* out, cudaStream_t st);

// Wide-source solve (solve_block.cu): one CTA per document over a BF16 panel
// [V][ld16], ld16 = block_panel_width(v_r) (0: not applicable).  u0, when
// not null, is an initial scaling [N][ldu] (warm start, cold fallback).
int block_panel_width(uint32_t vr_cap);
int launch_panel_to_bf16(const float* K, int ld, void* K16, int ld16, uint64_t V,
                         const uint32_t* vr, int num_sms, cudaStream_t st);
// shape: index of a launch shape (0 .. block_shape_count()-1) or -1 for the
// build-time default of the panel width.
int launch_solve_block(const void* K16, int ld16, float expo, uint32_t vr_cap,
                       const SourceSel& s, const Targets& t, const SolveCtl& ctl,
                       const float* u0, int64_t ldu, double* out, cudaStream_t st,
                       int shape = -1);
int block_shape_count();
const char* block_shape_name(int shape);
// Tensor-core form of the block solve (solve_tc.cu): documents up to
// tc_solve_capacity(ld16) rows on the tensor cores; order[0 .. n_long), the
// longer ones, on the CUDA-core block kernel.
// cps: CTAs sharing an SM (the row capacity shrinks with it).
int tc_solve_capacity(int ld16, int cps);
int launch_solve_tc(const void* K16, int ld16, float expo, uint32_t vr_cap,
                    const SourceSel& s, const Targets& t, const SolveCtl& ctl,
                    const float* u0, int64_t ldu, double* out, cudaStream_t st,
                    int cps, int64_t n_long);

// Learned warm start (warmstart.cu: training, ws_infer.cu: inference).
// Parameter vector layout (FP32), for embedding width d:
//   shift [F], scale [F], W1 [256][F], b1 [256], W2 [256][256], b2 [256],
//   w3 [256], b3 [1] (+3 pad);  F = 2d + 5 rounded up to 16.
constexpr int kWsH = 256;
struct WsLayout {
  int d = 0, F = 0;
  size_t shift = 0, scale = 0, W1 = 0, b1 = 0, W2 = 0, b2 = 0, w3 = 0, b3 = 0,
         count = 0;
};
WsLayout ws_layout(int d);
int launch_centroids(const float* E32, int d, const int64_t* col_ptr,
                     const uint2* ent, int64_t N, float* C, cudaStream_t st);
int launch_solve_f64(const float* K, int ld, int vr, const double* r,
                     const int64_t* col_ptr, const uint2* ent, const int32_t* docs,
                     int ndocs, double tol, int cap, double* u_out, int* it_out,
                     double* res_out, cudaStream_t st);
int launch_ws_rows(const float* E32, int d, const float* C, const float* K, int ld,
                   float expo, const uint32_t* src_ids, const double* r, int vr,
                   const int64_t* col_ptr, const uint2* ent, const int32_t* docs,
                   const double* u, int ndocs, const int32_t* sel, int G,
                   const int64_t* row0, int F, float* X, float* y, cudaStream_t st,
                   const float* mrow = nullptr);
int launch_ws_colstats(const float* X, int64_t P, int F, double* s1, double* s2,
                       int chunks, cudaStream_t st);
int launch_ws_standardize(float* X, int64_t P, int F, const float* shift,
                          const float* scale, cudaStream_t st);
size_t ws_scratch_floats(int64_t P, int F);
int launch_ws_fwd_bwd(const WsLayout& L, const float* params, const float* X,
                      const float* t, const int64_t* gptr, int64_t ngroups,
                      int64_t P, float* grad, double* loss_g, float* scratch,
                      cudaStream_t st);
int launch_ws_adam(const WsLayout& L, float* params, const float* grad, float* m1,
                   float* m2, float lr, int step, cudaStream_t st);
int launch_ws_gather(const float* X, const float* t, const int64_t* gptr,
                     const int64_t* perm, const int64_t* bptr, int64_t g0, int64_t ng,
                     int F, float* Xb, float* tb, cudaStream_t st);
size_t ws_folded_floats(const WsLayout& L);
int launch_ws_fold(const WsLayout& L, const float* params, float* folded,
                   cudaStream_t st);
int launch_ws_doc_bias(const WsLayout& L, const float* folded, const float* C,
                       int64_t N, float* Bdoc, cudaStream_t st);
int launch_ws_init(const WsLayout& L, const float* folded, const float* params,
                   const float* S, const float* rinv, int vr, const float* K, int ld,
                   float expo, const Targets& t, const float* Bdoc, float* Asrc,
                   float* u0, int64_t ldu, unsigned* err, int num_sms,
                   cudaStream_t st, const float* mrow = nullptr,
                   float* stats = nullptr);
// stats: scratch [N][vr][3] for the per-pair M statistics (computed
// document-major first); null: the fused kernel walks the panel per pair.

// Self-test of the bounded device-side wait (selftest.cu): a wait that can
// only end through its limit; sets ERR_TIMEOUT in *err.
int launch_wait_selftest(unsigned* err, unsigned long long limit_ns, cudaStream_t st);

// GPU CSC build from an edge list (csc_build.cu).  The result equals the
// host's stable counting sorts word-major (file order within a word,
// sinkhorn_wmd_fused.cpp:493-506) then document-major: entries sorted by
// (document, word, edge index).
size_t csc_build_temp_bytes(uint64_t nnz, uint64_t V, uint64_t N);
int launch_csc_build(const uint64_t* words, const uint64_t* docs, const double* w,
                     uint64_t nnz, uint64_t V, uint64_t N, void* temp,
                     size_t temp_bytes, uint64_t* col_ptr, uint64_t* rows,
                     double* vals, unsigned* err, cudaStream_t st);

}  // namespace wmd
