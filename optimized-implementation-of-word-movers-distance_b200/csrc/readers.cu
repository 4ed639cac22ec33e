// Readers for the reference's on-disk inputs (host code).
//
// Formats, as the reference's driver reads them (sinkhorn_wmd_fused.cpp):
//   mat.mtx   first three whitespace-separated integers num_rows (words),
//             num_cols (documents), nnz; then nnz triples "word doc weight"
//             with 1-based word and document ids (:427-486).  A triple with
//             an id of 0 or beyond its dimension, or a weight <= 0, is
//             invalid input; so is a file with fewer than nnz triples.
//   vecs.out  one line per word, its d embedding values separated by spaces
//             (:511-549); fewer lines than words, or a line without exactly
//             d values, is invalid input.
//   r.out     the source histogram, one value per word, whitespace-separated
//             (:552-586); a negative value or a count other than the number
//             of words is invalid input.
// The whole file is read into memory once and parsed with strtoull/strtod
// (the reference streams it through iostreams); values parse to the same
// doubles.
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>

#include "wmd_b200.h"
#include "wmd_internal.cuh"

namespace {

wmd_status rfail(wmd_status s, const std::string& m) {
  wmd::set_last_error(m.c_str());
  return s;
}

bool slurp(const char* path, std::string& out) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  out.clear();
  char buf[1 << 16];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
  fclose(f);
  return true;
}

struct Cursor {
  const char* p;
  const char* end;
  void skip_ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  bool u64(uint64_t& v) {
    skip_ws();
    if (p >= end || *p == '-') return false;
    char* e = nullptr;
    errno = 0;
    const unsigned long long x = strtoull(p, &e, 10);
    if (e == p || errno) return false;
    p = e;
    v = x;
    return true;
  }
  bool f64(double& v) {
    skip_ws();
    if (p >= end) return false;
    char* e = nullptr;
    const double x = strtod(p, &e);
    if (e == p) return false;
    p = e;
    v = x;
    return true;
  }
};

}  // namespace

extern "C" {

wmd_status wmd_mtx_header(const char* path, uint64_t* num_rows, uint64_t* num_cols,
                          uint64_t* nnz) {
  if (!path || !num_rows || !num_cols || !nnz)
    return rfail(WMD_ERR_INVALID_ARG, "null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return rfail(WMD_ERR_INVALID_ARG, std::string("cannot open ") + path);
  char buf[4096];
  const size_t n = fread(buf, 1, sizeof buf - 1, f);
  fclose(f);
  buf[n] = 0;
  Cursor c{buf, buf + n};
  uint64_t V = 0, N = 0, Z = 0;
  if (!c.u64(V) || !c.u64(N) || !c.u64(Z) || V == 0 || N == 0 || Z == 0)
    return rfail(WMD_ERR_INVALID_INPUT, "matrix header invalid");
  *num_rows = V;
  *num_cols = N;
  *nnz = Z;
  return WMD_OK;
}

wmd_status wmd_read_mtx(const char* path, uint64_t nnz_cap, uint64_t* words,
                        uint64_t* docs, double* weights, uint64_t* nnz_out) {
  if (!path || !words || !docs || !weights || !nnz_out)
    return rfail(WMD_ERR_INVALID_ARG, "null argument");
  std::string s;
  if (!slurp(path, s)) return rfail(WMD_ERR_INVALID_ARG, std::string("cannot open ") + path);
  Cursor c{s.data(), s.data() + s.size()};
  uint64_t V = 0, N = 0, Z = 0;
  if (!c.u64(V) || !c.u64(N) || !c.u64(Z) || V == 0 || N == 0 || Z == 0)
    return rfail(WMD_ERR_INVALID_INPUT, "matrix header invalid");
  if (Z > nnz_cap) return rfail(WMD_ERR_INVALID_ARG, "nnz_cap smaller than the header's nnz");
  for (uint64_t e = 0; e < Z; ++e) {
    uint64_t a = 0, b = 0;
    double w = 0.0;
    if (!c.u64(a) || !c.u64(b) || !c.f64(w))
      return rfail(WMD_ERR_INVALID_INPUT, "matrix has fewer entries than its header says");
    if (a == 0 || b == 0 || !(w > 0.0) || a > V || b > N)
      return rfail(WMD_ERR_INVALID_INPUT, "matrix contains invalid input");
    words[e] = a - 1;
    docs[e] = b - 1;
    weights[e] = w;
  }
  *nnz_out = Z;
  return WMD_OK;
}

wmd_status wmd_read_vecs(const char* path, uint64_t V, uint64_t d, double* vecs) {
  if (!path || !vecs || V == 0 || d == 0) return rfail(WMD_ERR_INVALID_ARG, "bad argument");
  std::string s;
  if (!slurp(path, s)) return rfail(WMD_ERR_INVALID_ARG, std::string("cannot open ") + path);
  const char* p = s.data();
  const char* end = p + s.size();
  for (uint64_t j = 0; j < V; ++j) {
    if (p >= end) return rfail(WMD_ERR_INVALID_INPUT, "fewer embedding lines than words");
    const char* eol = p;
    while (eol < end && *eol != '\n') ++eol;
    Cursor c{p, eol};
    uint64_t l = 0;
    double x;
    while (true) {
      c.skip_ws();
      if (c.p >= eol) break;
      if (!c.f64(x) || l >= d)
        return rfail(WMD_ERR_INVALID_INPUT, "embedding line " + std::to_string(j + 1) +
                                                " does not hold exactly d values");
      vecs[j * d + l++] = x;
    }
    if (l != d)
      return rfail(WMD_ERR_INVALID_INPUT, "embedding line " + std::to_string(j + 1) +
                                              " does not hold exactly d values");
    p = eol < end ? eol + 1 : end;
  }
  return WMD_OK;
}

wmd_status wmd_read_r(const char* path, uint64_t V, double* r) {
  if (!path || !r || V == 0) return rfail(WMD_ERR_INVALID_ARG, "bad argument");
  std::string s;
  if (!slurp(path, s)) return rfail(WMD_ERR_INVALID_ARG, std::string("cannot open ") + path);
  Cursor c{s.data(), s.data() + s.size()};
  uint64_t i = 0;
  double x;
  while (true) {
    c.skip_ws();
    if (c.p >= c.end) break;
    if (!c.f64(x)) return rfail(WMD_ERR_INVALID_INPUT, "source histogram: unparsable value");
    if (x < 0.0) return rfail(WMD_ERR_INVALID_INPUT, "source contains invalid input");
    if (i >= V) return rfail(WMD_ERR_INVALID_INPUT, "source histogram longer than V");
    r[i++] = x;
  }
  if (i != V) return rfail(WMD_ERR_INVALID_INPUT, "source histogram shorter than V");
  return WMD_OK;
}

}  // extern "C"
