// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// In-process harness around the reference's own CPU solver.  The reference
// translation unit is compiled where it lies (the include path is given by
// oracle/Makefile, which points at the reference checkout); nothing of it is
// copied into this repository.  One shared object is built per variant:
//
//   -DREF_VARIANT_FUSED     includes sinkhorn_wmd_fused.cpp
//   -DREF_VARIANT_NONFUSED  includes sinkhorn_wmd_nonfused.cpp
//
// The reference passes its target matrix and selection buffers through
// globals (sinkhorn_wmd_fused.cpp:6-18, sinkhorn_wmd_nonfused.cpp:15-23) and
// frees the caller-allocated v_sel / r_sel at the end of every solve
// (sinkhorn_wmd_fused.cpp:407-408).  ref_sinkhorn() below fills those globals,
// re-allocates the two buffers before every call and resets v_r, so the solver
// can be called any number of times from one process.
//
// The embedding width is the compile-time constant 300 (common.h:25).  Narrower
// embeddings (the d=3 sample of the reference's data/ directory) are run by
// zero-padding every row to 300 columns: the padded terms add exactly 0.0 to the
// squared distance (sinkhorn_wmd_fused.cpp:35-43), so results are bit-identical.

#define main wmd_reference_main
#if defined(REF_VARIANT_FUSED)
#include "sinkhorn_wmd_fused.cpp"
#elif defined(REF_VARIANT_NONFUSED)
#include "sinkhorn_wmd_nonfused.cpp"
#else
#error "define REF_VARIANT_FUSED or REF_VARIANT_NONFUSED"
#endif
#undef main

#include <stdint.h>

extern "C" {

// Returns v_r (number of selected source words) or a negative code:
//   -1: d differs from the reference's compile-time embedding width
//   -2: allocation failure
int ref_sinkhorn(const double* r, const double* vecs_in, double* wmd_out,
                 double lamda_arg, int max_iter_arg, uint64_t V, uint64_t N,
                 uint64_t d, const uint64_t* row_ptr, const uint64_t* col_inds,
                 const double* vals, uint64_t nnz, int nthreads) {
  if (d != (uint64_t)word2vec_word_embedding_size) return -1;
  c_csr.num_rows = V;
  c_csr.num_cols = N;
  c_csr.nnz = nnz;
  c_csr.row_ptr = (u64*)row_ptr;
  c_csr.col_inds = (u64*)col_inds;
  c_csr.vals = (double*)vals;
  if (posix_memalign((void**)&r_sel, ALN, (V + 1) * sizeof(double)) != 0) return -2;
  if (posix_memalign((void**)&v_sel, ALN, (V * d + 1) * sizeof(double)) != 0) {
    free(r_sel);
    return -2;
  }
  v_r = 0;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#if defined(REF_VARIANT_FUSED)
  // The fused driver reads the team size into this global before the call
  // (sinkhorn_wmd_fused.cpp:600-603).
#pragma omp parallel
  {
#pragma omp single
    nmtp_threads = (u64)omp_get_num_threads();
  }
#endif
  sinkhorn_wmd(r, vecs_in, wmd_out, lamda_arg, max_iter_arg, V, N, d);
  // r_sel and v_sel were released by the solver itself.
  r_sel = nullptr;
  v_sel = nullptr;
  return (int)v_r;
}

int ref_embedding_width(void) { return word2vec_word_embedding_size; }

}  // extern "C"
