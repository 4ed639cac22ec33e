/*
 * wmd_b200.h — C ABI of the B200 Sinkhorn Word Mover's Distance engine.
 *
 * Reference interface being replaced (IntelLabs/Optimized-Implementation-of-
 * Word-Movers-Distance):
 *
 *   void sinkhorn_wmd(const double* r, const double* vecs, REAL* WMD,
 *                     const REAL lamda, const int max_iter,
 *                     const u64 data_vocab_size, const u64 num_docs,
 *                     const u64 word2vec_word_embedding_size);
 *       sinkhorn_wmd_fused.cpp:112-114, sinkhorn_wmd_nonfused.cpp:114-116
 *
 * whose target-document matrix is the global `puma_csr_double_t c_csr`
 * (sinkhorn_wmd_fused.cpp:13, sinkhorn_wmd_nonfused.cpp:15).  The drop-in
 * entry points below take the same arguments in the same order and meaning,
 * plus that matrix as a trailing pointer.  All pointers of the drop-in calls
 * are HOST pointers; the library copies to the GPU, solves there and copies
 * WMD back before returning.
 *
 * Errors: where the reference asserts or exit(0)s (sinkhorn_wmd_fused.cpp:
 * 131-153, 431-435, 474-478, 570-574), every call here returns a wmd_status
 * and leaves a message for wmd_last_error().
 *
 * Threading: the drop-in calls are reentrant (each uses a per-thread default
 * handle).  A wmd_handle must not be used by two host threads at once.
 */
#ifndef WMD_B200_H
#define WMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WMD_B200_ABI_VERSION 1

typedef enum wmd_status {
  WMD_OK = 0,
  WMD_ERR_INVALID_ARG = 1,   /* bad pointer, size or option */
  WMD_ERR_INVALID_INPUT = 2, /* data the reference driver rejects: r < 0,
                                c value <= 0, word/doc index out of range,
                                non-monotone column pointers */
  WMD_ERR_OUT_OF_MEMORY = 3,
  WMD_ERR_CUDA = 4,          /* CUDA runtime error; see wmd_last_error() */
  WMD_ERR_NO_DEVICE = 5,
  WMD_ERR_UNSUPPORTED = 6,   /* option not available on this device/build */
  WMD_ERR_DEVICE_TIMEOUT = 7 /* a bounded device-side wait gave up; the
                                kernel returned early, results are invalid,
                                the CUDA context stays usable */
} wmd_status;

/* Word-major target matrix; field-for-field the reference's
 * puma_csr_double_t (common.h:38-46).  num_rows = vocabulary size V,
 * num_cols = number of target documents N. */
typedef struct wmd_csr_double_t {
  uint64_t num_rows;
  uint64_t num_cols;
  uint64_t nnz;
  uint64_t* row_ptr;  /* [num_rows + 1] */
  uint64_t* col_inds; /* [nnz] document ids */
  double* vals;       /* [nnz] normalised counts */
} wmd_csr_double_t;

/* Document-major target matrix; field-for-field the reference's
 * puma_csc_double_t (common.h:49-57). */
typedef struct wmd_csc_double_t {
  uint64_t num_rows;
  uint64_t num_cols;
  uint64_t nnz;
  uint64_t* col_ptr;  /* [num_cols + 1] */
  uint64_t* row_inds; /* [nnz] word ids */
  double* vals;       /* [nnz] */
} wmd_csc_double_t;

/* ---------------------------------------------------------------------------
 * Drop-in solves (host buffers).
 * ------------------------------------------------------------------------ */

/* Replaces the fused sinkhorn_wmd (sinkhorn_wmd_fused.cpp:112-412).
 * K = exp(lamda * M) exactly as sinkhorn_wmd_fused.cpp:217 computes it, so
 * the usual regulariser lambda = 10 is passed as lamda = -10.  WMD receives
 * num_docs values.  c_csr->num_rows must equal data_vocab_size and
 * c_csr->num_cols must equal num_docs. */
wmd_status wmd_sinkhorn_fused(const double* r, const double* vecs, double* WMD,
                              double lamda, int max_iter,
                              uint64_t data_vocab_size, uint64_t num_docs,
                              uint64_t word2vec_word_embedding_size,
                              const wmd_csr_double_t* c_csr);

/* Replaces the nonfused sinkhorn_wmd (sinkhorn_wmd_nonfused.cpp:114-318).
 * K = exp(-lamda * M) as sinkhorn_wmd_nonfused.cpp:172-173 computes it, so
 * lambda = 10 is passed as lamda = +10.  Same math and results otherwise. */
wmd_status wmd_sinkhorn_nonfused(const double* r, const double* vecs,
                                 double* WMD, double lamda, int max_iter,
                                 uint64_t data_vocab_size, uint64_t num_docs,
                                 uint64_t word2vec_word_embedding_size,
                                 const wmd_csr_double_t* c_csr);

/* As wmd_sinkhorn_fused / wmd_sinkhorn_nonfused with the target matrix in
 * the document-major layout the GPU iterates in (no transpose needed).
 * Replaces the same reference functions. */
wmd_status wmd_sinkhorn_fused_csc(const double* r, const double* vecs,
                                  double* WMD, double lamda, int max_iter,
                                  uint64_t data_vocab_size, uint64_t num_docs,
                                  uint64_t word2vec_word_embedding_size,
                                  const wmd_csc_double_t* c_csc);
wmd_status wmd_sinkhorn_nonfused_csc(const double* r, const double* vecs,
                                     double* WMD, double lamda, int max_iter,
                                     uint64_t data_vocab_size,
                                     uint64_t num_docs,
                                     uint64_t word2vec_word_embedding_size,
                                     const wmd_csc_double_t* c_csc);

/* Host -> device bytes moved by the calling thread's last successful drop-in
 * call above (target matrix, r, embedding rows).  When `vecs` lies in one
 * pinned, device-mapped host allocation (cudaHostAlloc / cudaMallocHost /
 * cudaHostRegister), the host threads narrow the rows of a prefix of the
 * vocabulary (half of it by default; the environment variable
 * WMD_DROPIN_HOST_SHARE, 0 to 1, sets the share) to FP32 and copy them while
 * the GPU reads, above the prefix, only the rows of the words that occur in
 * the target matrix or in r, in FP64 directly from host memory.  Pageable
 * embeddings are narrowed on the host whole (copied whole with a share of 0
 * or fewer than 4 host threads).  Results are the same on every path.  No
 * reference counterpart (a measurement aid). */
uint64_t wmd_dropin_h2d_bytes(void);

/* ---------------------------------------------------------------------------
 * Handle API: embeddings and target set stay resident on the GPU across
 * queries (the serving form of the same solve).  No reference counterpart:
 * the reference re-reads its inputs on every run (sinkhorn_wmd_fused.cpp:
 * 415-598).  lambda here is the positive regulariser: K = exp(-lambda * M).
 * ------------------------------------------------------------------------ */

typedef struct wmd_handle wmd_handle;

/* Cost-matrix (cdist) precision. */
typedef enum wmd_cdist_mode {
  WMD_CDIST_FP32 = 0, /* FP32 CUDA-core GEMM form, near pairs recomputed */
  WMD_CDIST_BF16 = 1, /* tcgen05 tensor cores, BF16 operands, FP32 accum */
  WMD_CDIST_FP16 = 2, /* tcgen05 tensor cores, FP16 operands, FP32 accum */
  /* tcgen05 tensor cores on the FP32 embeddings: each operand split into a
   * TF32 high part and its FP32 remainder, three products (hi*hi + hi*lo +
   * lo*hi) accumulated in FP32: FP32-accurate, near pairs recomputed as in
   * WMD_CDIST_FP32.  Widths d that are not a multiple of 4 (or too wide for
   * the tile) use the FP32 CUDA-core panel instead. */
  WMD_CDIST_TF32X3 = 3,
  /* tcgen05 tensor cores on a resident split-FP16 copy of the embeddings
   * (built from the FP32 embeddings on first use, 4*d + 16 bytes per word):
   * each row scaled by a power of two, an FP16 high part and its remainder
   * scaled by 2^11 in FP16, three products (hi*hi + 2^-11 (hi*lo + lo*hi))
   * accumulated in FP32: FP32-accurate like WMD_CDIST_TF32X3, read by TMA
   * with no in-kernel conversion.  Single-source queries (wmd_query_dense*)
   * only; batches and widths the tile cannot hold run the WMD_CDIST_TF32X3
   * form. */
  WMD_CDIST_F16X3 = 4
} wmd_cdist_mode;

wmd_status wmd_create(wmd_handle** out, int device);
wmd_status wmd_destroy(wmd_handle* h);

/* Embeddings: V x d row-major.  `where` is 0 for host memory, 1 for device
 * memory on the handle's GPU. */
wmd_status wmd_set_embeddings_f64(wmd_handle* h, const double* vecs, uint64_t V,
                                  uint64_t d, int where);
wmd_status wmd_set_embeddings_f32(wmd_handle* h, const float* vecs, uint64_t V,
                                  uint64_t d, int where);

/* Embeddings given in BF16 ([V][d] raw BF16 bit patterns, host (where = 0)
 * or device (where = 1) memory), no reference counterpart (the reference's
 * vecs are FP64).  The engine keeps the BF16 rows as the tensor-core copy the
 * BF16 cost panel reads (wmd_set_cdist_mode(h, WMD_CDIST_BF16)) and their
 * exact FP32 values for the near-pair recompute and the other forms. */
wmd_status wmd_set_embeddings_bf16(wmd_handle* h, const uint16_t* vecs, uint64_t V,
                                   uint64_t d, int where);

/* Target documents (host memory).  Validated on the GPU. */
wmd_status wmd_set_targets_csc(wmd_handle* h, const wmd_csc_double_t* c);
wmd_status wmd_set_targets_csr(wmd_handle* h, const wmd_csr_double_t* c);

wmd_status wmd_set_cdist_mode(wmd_handle* h, wmd_cdist_mode mode);

/* Storage of the K panel the Sinkhorn iterations read.  FP32 (default) is
 * the form held to 1e-5 against the reference.  BF16 applies to sources with
 * 64 < v_r <= 512 and lambda != 0: the panel is rounded to BF16 and solved by
 * the CTA-per-document kernel that keeps each document's rows in shared
 * memory (iterations still in FP32, final reduction in FP64).  Other sources
 * use the FP32 path in either setting. */
typedef enum wmd_solve_precision {
  WMD_SOLVE_FP32 = 0,
  WMD_SOLVE_BF16 = 1
} wmd_solve_precision;
wmd_status wmd_set_solve_precision(wmd_handle* h, wmd_solve_precision prec);

/* Traversal order of the iterations.  0 (default): document-major, a
 * document's u and x on chip for all passes (solve.cu, solve_block.cu).
 * 1: word-major, the reference's own order (sinkhorn_wmd_fused.cpp:249-292:
 * nnz-balanced chunks of the word-major CSR, each K row read once per pass,
 * u gathered and x scattered with atomics per entry); the fixed update count
 * from the cold start only (no tolerance, relaxation or warm start, lambda
 * != 0), single-source queries only.  Results agree with order 0 within the
 * plain path's tolerance (atomic summation order). */
wmd_status wmd_set_solve_order(wmd_handle* h, int order);

/* Batched queries (wmd_query_batch), no reference counterpart.  stacked != 0
 * (the default): sources of one width class (lane layout of the warp solve,
 * or BF16 panel width of the CTA-per-document solve) run in groups whose
 * panels fit group_budget_bytes of device memory (default 32 GiB), each group
 * in a fixed number of launches whatever its size: one gather of all the
 * group's source rows, one tensor-core cost-panel launch writing every
 * source's panel, one near-pair fix-up, (BF16) one panel conversion, and one
 * persistent solve launch over all (source, document) pairs.  Used with a
 * tensor-core cost panel, lambda != 0, the cold start and panels in FP32
 * range; otherwise (and with stacked = 0) sources run one after another on
 * two pipeline slots.  Results are the same either way (same kernels' math). */
wmd_status wmd_set_batch_mode(wmd_handle* h, int stacked, uint64_t group_budget_bytes);

/* Number of stacked groups the last wmd_query_batch ran (0: per source). */
int wmd_last_batch_groups(wmd_handle* h);

/* Launch shapes the autotuner chose for the plain warp solve, per lane
 * layout (v_r <= 32, 64, 128, 256, 512, 1024): a candidate index (see
 * wmd_solve_shape_name), -1 for the build-time default, -2 not tuned yet.
 * Chosen on the first query of each layout after targets or embeddings are
 * set (each candidate timed on the real panel at the query's update count,
 * at most 15, in three interleaved groups of two launches: a one-time cost
 * of 21 solves, about 2.4 ms at V = 1e5, N = 5000, v_r = 32), unless tuning
 * is off (wmd_set_autotune).  No reference counterpart. */
wmd_status wmd_solve_shape_choices(wmd_handle* h, int* shapes);
const char* wmd_solve_shape_name(int shape);

/* Launch shapes chosen for the stacked batch solves (each timed on the first
 * group of its class, 4 updates): shapes[0..3] the stacked block solve per
 * BF16 panel width 128, 256, 384, 512 (names: wmd_block_shape_name, 0-2),
 * shapes[4..9] the stacked warp solve per lane layout v_r <= 32 .. 1024
 * (names: wmd_solve_shape_name); -2 = not tuned yet.  No reference
 * counterpart. */
wmd_status wmd_group_shape_choices(wmd_handle* h, int* shapes);

/* Launch-shape autotuner of the BF16 block solve (on by default): the first
 * solve of each panel width (and panel size class: within / beyond 64 MiB)
 * times every candidate shape on the handle's real data and keeps the
 * fastest.  wmd_autotune_choices fills shapes[8] (index (width/128 - 1) * 2 +
 * beyond; -2 = not tuned yet, -1 = build-time default); the name of a shape
 * comes from wmd_block_shape_name. */
wmd_status wmd_set_autotune(wmd_handle* h, int enable);

/* Over-relaxed iteration, 0 < omega < 2 (default 1: the reference's
 * iteration exactly): both half-steps are relaxed, v <- v^(1-omega) *
 * v_hat^omega and u <- u^(1-omega) * u_hat^omega, each target word keeping
 * its previous v.  Same fixed point; with per-document stopping
 * (wmd_set_tolerance, whose residual then also counts the target-side
 * marginal) 1 < omega < 2 reaches the tolerance in far fewer updates on
 * slowly converging documents (overrelaxed Sinkhorn-Knopp: Thibault et al.
 * 2017; Lehmann et al. 2021).  A per-document guard steps omega halfway back
 * to 1 whenever the residual grows 100-fold over its best, and restarts the
 * document unrelaxed from the cold start if it stops being finite.  Applies
 * only with per-document stopping (tolerance > 0): a fixed update count runs
 * the reference's iteration.  Ignored for lambda = 0.  No reference
 * counterpart. */
wmd_status wmd_set_relaxation(wmd_handle* h, double omega);
wmd_status wmd_autotune_choices(wmd_handle* h, int* shapes);
const char* wmd_block_shape_name(int shape);
/* Pin the block solve to one shape (0..5; 3-5 = the tensor-core form with
 * 1, 2 or 4 CTAs per SM, whose longest documents run on the CUDA cores),
 * -1 = the build-time default, -2 = back to the autotuner. */
wmd_status wmd_set_block_shape(wmd_handle* h, int shape);

/* One source document as a dense host histogram r[V] (the reference's form,
 * zeros skipped as sinkhorn_wmd_fused.cpp:45-63 does).  wmd_out: host, N. */
wmd_status wmd_query_dense(wmd_handle* h, const double* r, double lambda,
                           int max_iter, double* wmd_out);

/* Device-resident variant: r_dev is a device pointer to V doubles, wmd_dev a
 * device pointer to N doubles.  Runs asynchronously on the handle's stream
 * (wmd_stream()); vr_cap bounds the number of non-zeros of r_dev (panels are
 * sized for it; more non-zeros raise WMD_ERR_INVALID_INPUT at the next
 * wmd_check()). */
wmd_status wmd_query_dense_device(wmd_handle* h, const double* r_dev,
                                  uint64_t vr_cap, double lambda, int max_iter,
                                  double* wmd_dev);

/* k nearest target documents (1 <= k <= 1024): the query of wmd_query_dense
 * followed by a GPU ranking of its N scores — ascending WMD, ties broken by
 * document index, NaN (empty documents) last, i.e. exactly
 * numpy.argsort(scores, kind="stable")[:k].  idx_out / wmd_out: host, k.
 * No reference counterpart (the reference writes the unsorted scores,
 * main.py:140-143). */
wmd_status wmd_query_topk(wmd_handle* h, const double* r, double lambda,
                          int max_iter, uint32_t k, uint32_t* idx_out,
                          double* wmd_out);

/* The same ranking of any device-resident score vector (n <= 2^32 - 1),
 * asynchronous on the handle's stream; idx_dev / val_dev: device, k. */
wmd_status wmd_topk_device(wmd_handle* h, const double* scores_dev, uint64_t n,
                           uint32_t k, uint32_t* idx_dev, double* val_dev);

/* Many source documents in one call (the batched serving form; no reference
 * counterpart, the reference solves one source per run).  Source s has the
 * words src_ids[src_ptr[s] .. src_ptr[s+1]) — strictly ascending ids < V, as
 * the reference's selection yields them (sinkhorn_wmd_fused.cpp:45-63) — with
 * weights src_w (> 0).  At most 1024 words per source.  wmd_out (host,
 * num_sources x N row-major) receives every source's scores against the
 * resident target set; iters_out (host, optional, same shape) the
 * per-document iteration counts. */
wmd_status wmd_query_batch(wmd_handle* h, const uint64_t* src_ptr,
                           const uint64_t* src_ids, const double* src_w,
                           uint64_t num_sources, double lambda, int max_iter,
                           double* wmd_out, int* iters_out);

/* Per-document convergence stopping.  tol = 0 (default): every document runs
 * exactly max_iter x-updates, as the reference does (sinkhorn_wmd_fused.cpp:
 * 246).  tol > 0: a document stops after the first update whose marginal
 * residual sum_i |u_i (K v)_i - r_i| (with the scalings entering the update)
 * is <= tol, max_iter becoming a cap.  No reference counterpart (the
 * reference fixes the iteration count, main.py:11-12). */
wmd_status wmd_set_tolerance(wmd_handle* h, double tol);

/* Number of x-updates each document of the last query took (host, N). */
wmd_status wmd_last_iterations(wmd_handle* h, int* iters);

/* Synchronises the handle's stream and reports device-side validation
 * failures of the calls issued since the previous check
 * (WMD_ERR_INVALID_INPUT), or WMD_ERR_DEVICE_TIMEOUT when a bounded
 * device-side wait gave up. */
wmd_status wmd_check(wmd_handle* h);

/* Failure-path self-test, no reference counterpart (the reference has no
 * device waits).  Launches, on the handle's stream, one thread that waits on
 * a device barrier nothing ever completes, through the same bounded wait the
 * tensor-core kernels use, with a limit of limit_ns (1e3 .. 2e9) instead of
 * their 2 s.  The wait gives up, flags the handle's error word and returns;
 * the next wmd_check() reports WMD_ERR_DEVICE_TIMEOUT and the handle stays
 * usable.  Hangs nothing and faults nothing. */
wmd_status wmd_selftest_bounded_wait(wmd_handle* h, uint64_t limit_ns);

/* Roofline probes, no reference counterpart: the measured L2 read bandwidth
 * (16-byte loads over an L2-resident buffer of l2_bytes, 1 MiB .. 96 MiB,
 * GB/s) and FP32 FMA rate (packed FMAs on registers, TFLOP/s) of `device`,
 * timed with CUDA events.  The denominators of the iteration kernels'
 * roofline, which neither HBM nor the tensor cores bound.  Allocates its own
 * buffers; not part of any solve. */
wmd_status wmd_probe_roofline(int device, uint64_t l2_bytes, double* l2_read_gbs,
                              double* fp32_tflops);

/* The handle's CUDA stream (a cudaStream_t), for event timing. */
void* wmd_stream(wmd_handle* h);

/* Number of kernels the last query launched. */
int wmd_last_launch_count(wmd_handle* h);

/* Stage timing.  While enabled, every query records CUDA events on the
 * handle's stream around its three stages; wmd_stage_times waits for the
 * last query and returns the select, cost-panel (cdist) and solve durations
 * in milliseconds.  No reference counterpart (the reference times only the
 * whole call, sinkhorn_wmd_fused.cpp:607-615). */
wmd_status wmd_set_timing(wmd_handle* h, int enable);
wmd_status wmd_stage_times(wmd_handle* h, float* select_ms, float* cdist_ms,
                           float* solve_ms);

/* ---------------------------------------------------------------------------
 * Allocation-free solve.  No counterpart in the reference.
 *
 * For callers that may not allocate device memory: code running inside a
 * framework or inference server that owns all device memory through its own
 * pool and hands a plugin only its input and output buffers, or a
 * latency-critical loop that cannot afford the device-wide synchronisation
 * cudaMalloc / cudaFree imply.  This call allocates nothing (no cudaMalloc,
 * cudaFree or allocating library routine); its working buffers live in a
 * fixed 64 MiB scratch array compiled into the library, which every GPU that
 * loads the library holds until the process exits.
 *
 * All pointers are DEVICE pointers on the current device: r_dev [V] (the
 * dense source histogram), vecs_dev [V][d] FP32 row-major, 16-byte aligned,
 * the target matrix as CSC (col_ptr_dev [N+1], row_inds_dev [nnz], vals_dev
 * [nnz], the fields of wmd_csc_double_t) and the output wmd_dev [N].  vr_cap
 * bounds the number of non-zeros of r (<= 1024).  lambda is the positive
 * regulariser, K = exp(-lambda * M).  Runs the same kernels as the other
 * entry points (FP32 cost panel) on `stream` (a cudaStream_t, NULL for the
 * default stream) and returns after synchronising it.
 *
 * Limit: the problem must fit the scratch, V*round_up(vr_cap,4)*4 (twice
 * that for lambda = 0, where the K.*M panel is stored too) + V*4 + nnz*8 +
 * (N+1)*8 + vr_cap*(d+3)*4 bytes (plus about 33 KB of counters, near-pair
 * list and alignment padding) <= 64 MiB; larger problems return
 * WMD_ERR_INVALID_ARG.  vecs_dev must be 16-byte aligned when d % 4 == 0
 * (WMD_ERR_INVALID_ARG otherwise).
 *
 * The first call on each device resolves the scratch array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture begins.  The address is cached for the life of
 * the device's primary context (do not call this again on a device after
 * cudaDeviceReset).  Every call on a device shares the one scratch array, so
 * calls that overlap on the GPU (other streams or host threads on the same
 * device) race: serialise them.
 */
wmd_status wmd_sinkhorn_noalloc(const double* r_dev, const float* vecs_dev,
                                uint64_t V, uint64_t d,
                                const uint64_t* col_ptr_dev,
                                const uint64_t* row_inds_dev,
                                const double* vals_dev, uint64_t N,
                                uint64_t nnz, uint64_t vr_cap, double lambda,
                                int max_iter, double* wmd_dev, void* stream);

/* ---------------------------------------------------------------------------
 * Diagnostics.
 * ------------------------------------------------------------------------ */
const char* wmd_status_string(wmd_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char* wmd_last_error(void);
int wmd_abi_version(void);

/* ---------------------------------------------------------------------------
 * Learned warm start.  No reference counterpart (the reference always starts
 * from u = v_r, sinkhorn_wmd_fused.cpp:188-191).  A 3-layer MLP (256 GELU,
 * 256 GELU, 1) predicts log u_i per (source word i, target document) from
 * the source word's embedding, r_i, log r_i, the document's weighted
 * embedding centroid and min / mean / max of M(i, w) over the document's
 * words; queries then start from exp(prediction), and each document falls
 * back to the cold start when the prediction's first-update marginal
 * residual is worse.  Parameters are one FP32 vector of
 * wmd_ws_param_count(d) floats: shift[F], scale[F], W1[256][F], b1[256],
 * W2[256][256], b2[256], w3[256], b3 (+3 pad), F = 2d + 5 rounded up to 16.
 * ------------------------------------------------------------------------ */
uint64_t wmd_ws_param_count(uint64_t d);
/* Seeded initial parameters (shift 0, scale 1, W ~ N(0, 1/fan_in), b = 0). */
wmd_status wmd_ws_init_params(uint64_t d, uint64_t seed, float* params);
/* Labels: for each source (same form as wmd_query_batch), `docs_per_source`
 * documents of the handle's target set are drawn (seeded, without
 * replacement) and solved to convergence in FP64 (marginal residual <=
 * label_tol within label_max_iter updates); for each converged pair
 * min(words_per_doc, v_r) source words become training rows (features,
 * log u).  The rows stay on the GPU, standardised, for wmd_ws_train. */
wmd_status wmd_ws_build_training_set(wmd_handle* h, const uint64_t* src_ptr,
                                     const uint64_t* src_ids, const double* src_w,
                                     uint64_t num_sources, double lambda,
                                     uint32_t docs_per_source, uint32_t words_per_doc,
                                     double label_tol, int label_max_iter,
                                     uint64_t seed, uint64_t* rows_out,
                                     uint64_t* groups_out, double* mean_label_iters);
/* Adam on the group-centred squared error of log u (each (source, document)
 * pair's mean offset is free: u and a u give the same transport plan).
 * params: in = initial values, out = trained (shift/scale set from the
 * training set).  loss_out: per-epoch mean loss (may be null). */
wmd_status wmd_ws_train(wmd_handle* h, float* params, int epochs,
                        uint64_t batch_groups, float lr, uint64_t seed,
                        double* loss_out);
/* Loss and gradient of every parameter over given raw feature rows X
 * [rows][F] (host), targets t [rows], groups gptr [ngroups + 1]: the
 * training kernels on caller data (for gradient checks). */
wmd_status wmd_ws_loss_grad(wmd_handle* h, uint64_t d, const float* X,
                            const float* t, const int64_t* gptr, uint64_t ngroups,
                            const float* params, double* loss, float* grad);
/* Read back the training set built last (any pointer may be NULL): the
 * standardised rows X [rows][F], labels y [rows] (log u), group pointers
 * [groups + 1], per group the source index and target document, per row the
 * source word's index within its source. */
wmd_status wmd_ws_get_training_set(wmd_handle* h, float* X, float* y, int64_t* gptr,
                                   uint32_t* group_source, uint32_t* group_doc,
                                   int32_t* row_word);
/* Use a model for subsequent queries (params = NULL: back to the cold start). */
wmd_status wmd_set_warm_start(wmd_handle* h, const float* params);
/* The initial scalings the model gives a dense source r: u0_out [N][v_r]
 * (host, FP32), v_r written to vr_out. */
wmd_status wmd_ws_init_scalings(wmd_handle* h, const double* r, double lambda,
                                float* u0_out, uint64_t* vr_out);

/* ---------------------------------------------------------------------------
 * The reference's input files and edge lists.
 * ------------------------------------------------------------------------ */
/* mat.mtx (sinkhorn_wmd_fused.cpp:427-486): header "num_rows num_cols nnz",
 * then nnz triples "word doc weight", 1-based.  wmd_read_mtx writes 0-based
 * word and document ids and the weights in file order (arrays of nnz_cap >=
 * the header's nnz); invalid entries (id 0 or out of range, weight <= 0,
 * missing triples) return WMD_ERR_INVALID_INPUT, as the reference exits. */
wmd_status wmd_mtx_header(const char* path, uint64_t* num_rows, uint64_t* num_cols,
                          uint64_t* nnz);
wmd_status wmd_read_mtx(const char* path, uint64_t nnz_cap, uint64_t* words,
                        uint64_t* docs, double* weights, uint64_t* nnz_out);
/* vecs.out (:511-549): V lines of d space-separated values -> vecs[V*d]. */
wmd_status wmd_read_vecs(const char* path, uint64_t V, uint64_t d, double* vecs);
/* r.out (:552-586): V whitespace-separated values >= 0 -> r[V]. */
wmd_status wmd_read_r(const char* path, uint64_t V, double* r);
/* Edge list (0-based, any order) -> document-major CSC built on the GPU:
 * entries sorted by (document, word, edge index), i.e. exactly the
 * reference's stable counting sort into CSR (:493-506) followed by a stable
 * transpose.  wmd_edges_to_csc returns it to host arrays (col_ptr[N+1],
 * rows[nnz], vals[nnz]); wmd_set_targets_edges makes it the handle's
 * target set. */
wmd_status wmd_edges_to_csc(wmd_handle* h, const uint64_t* words, const uint64_t* docs,
                            const double* w, uint64_t nnz, uint64_t V, uint64_t N,
                            uint64_t* col_ptr_out, uint64_t* rows_out,
                            double* vals_out);
wmd_status wmd_set_targets_edges(wmd_handle* h, const uint64_t* words,
                                 const uint64_t* docs, const double* w, uint64_t nnz,
                                 uint64_t V, uint64_t N);

#ifdef __cplusplus
}
#endif
#endif /* WMD_B200_H */
