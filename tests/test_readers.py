"""The reference's file formats (mat.mtx, vecs.out, r.out) and the GPU CSC
build of an edge list.

CPU: the readers against files written in the reference's formats from the
golden d=3 sample (and invalid files the reference's driver rejects).
GPU: the edge-list CSC build bit-exact against the oracle's stable counting
sorts (word-major CSR as sinkhorn_wmd_fused.cpp:493-506, then the stable
transpose), and a query through files + GPU build equal to the golden
reference outputs."""
import numpy as np
import pytest

from conftest import rel_err


def _write_sample(tmp_path, s):
    rows, cols, w = (np.array(a) for a in s["edges"])
    mtx = tmp_path / "sample.mtx"
    with open(mtx, "w") as f:
        f.write(f"{s['V']} {s['N']} {rows.size}\n")
        for a, b, x in zip(rows, cols, w):
            f.write(f"{int(a) + 1} {int(b) + 1} {float(x)!r}\n")
    vecs = tmp_path / "vecs.out"
    with open(vecs, "w") as f:
        for row in s["vecs"]:
            f.write(" ".join(repr(float(x)) for x in row) + "\n")
    r = tmp_path / "r.out"
    with open(r, "w") as f:
        f.write("\n".join(repr(float(x)) for x in s["r"]) + "\n")
    return mtx, vecs, r


def test_readers_roundtrip_sample(wmd, golden, tmp_path):
    s = golden["sample_d3"]
    mtx, vecs, r = _write_sample(tmp_path, s)
    V, N, words, docs, w = wmd.read_mtx(mtx)
    rows, cols, ww = (np.array(a) for a in s["edges"])
    assert (V, N) == (s["V"], s["N"])
    np.testing.assert_array_equal(words, rows)
    np.testing.assert_array_equal(docs, cols)
    np.testing.assert_array_equal(w, ww)
    np.testing.assert_array_equal(wmd.read_vecs(vecs, V, 3), np.array(s["vecs"]))
    np.testing.assert_array_equal(wmd.read_r(r, V), np.array(s["r"]))


@pytest.mark.parametrize("body,what", [
    ("3 2 2\n1 1 0.5\n2 3 0.5\n", "document id beyond num_cols"),
    ("3 2 2\n1 1 0.5\n4 1 0.5\n", "word id beyond num_rows"),
    ("3 2 2\n0 1 0.5\n1 1 0.5\n", "id 0 (ids are 1-based)"),
    ("3 2 2\n1 1 0\n2 1 0.5\n", "weight <= 0"),
    ("3 2 3\n1 1 0.5\n2 1 0.5\n", "fewer triples than nnz"),
    ("0 2 1\n1 1 0.5\n", "empty dimension"),
])
def test_mtx_invalid_inputs(wmd, tmp_path, body, what):
    f = tmp_path / "bad.mtx"
    f.write_text(body)
    with pytest.raises(wmd.WMDError) as e:
        wmd.read_mtx(f)
    assert e.value.name == "WMD_ERR_INVALID_INPUT", what


def test_vecs_and_r_invalid_inputs(wmd, tmp_path):
    f = tmp_path / "v.out"
    f.write_text("1 2 3\n4 5\n")
    with pytest.raises(wmd.WMDError):
        wmd.read_vecs(f, 2, 3)
    f.write_text("1 2 3\n")
    with pytest.raises(wmd.WMDError):
        wmd.read_vecs(f, 2, 3)  # fewer lines than words
    g = tmp_path / "r.out"
    g.write_text("0.5 -0.1 0.6\n")
    with pytest.raises(wmd.WMDError):
        wmd.read_r(g, 3)
    g.write_text("0.5 0.5\n")
    with pytest.raises(wmd.WMDError):
        wmd.read_r(g, 3)
    g.write_text("0.5\n0.25\n0.25")  # no trailing newline is fine here
    np.testing.assert_array_equal(wmd.read_r(g, 3), [0.5, 0.25, 0.25])


def _edges(rng, V, N, nnz):
    words = rng.integers(0, V, nnz).astype(np.uint64)
    docs = rng.integers(0, N, nnz).astype(np.uint64)
    # repeated (word, document) pairs in varying file order
    dup = rng.integers(0, nnz, nnz // 10)
    words[dup[: dup.size // 2]] = words[dup[dup.size // 2:][: dup.size // 2]]
    docs[dup[: dup.size // 2]] = docs[dup[dup.size // 2:][: dup.size // 2]]
    w = rng.uniform(0.01, 1.0, nnz)
    return words, docs, w


@pytest.mark.gpu
@pytest.mark.parametrize("V,N,nnz", [(3000, 500, 20000), (100000, 70000, 400000),
                                     (7, 3, 40), (1, 1, 5)])
def test_gpu_csc_build_bit_exact(wmd, oracle_mod, V, N, nnz):
    rng = np.random.default_rng(V + N)
    words, docs, w = _edges(rng, V, N, nnz)
    eng = wmd.Engine()
    cp, rows, vals = eng.edges_to_csc(words, docs, w, V, N)
    rp, ci, cv = oracle_mod.counting_sort(V, words, docs, w)
    cp2, rows2, vals2 = oracle_mod.csc_from_csr(V, N, rp, ci, cv)
    np.testing.assert_array_equal(cp, cp2)
    np.testing.assert_array_equal(rows, rows2)
    np.testing.assert_array_equal(vals, vals2)  # bitwise (same doubles moved)
    eng.close()


@pytest.mark.gpu
def test_gpu_csc_build_rejects_invalid_edges(wmd):
    eng = wmd.Engine()
    words = np.array([0, 1, 5], np.uint64)
    docs = np.array([0, 1, 1], np.uint64)
    for bad_words, bad_docs, bad_w in ((words, docs, np.array([1.0, 1.0, 1.0])),
                                       (words[:2], np.array([0, 2], np.uint64), np.ones(2)),
                                       (words[:2], docs[:2], np.array([1.0, -1.0]))):
        with pytest.raises(wmd.WMDError) as e:
            eng.edges_to_csc(bad_words, bad_docs, bad_w, 5, 2)
        assert e.value.name == "WMD_ERR_INVALID_INPUT"
    cp, rows, vals = eng.edges_to_csc(words[:2], docs[:2], np.ones(2), 5, 2)
    np.testing.assert_array_equal(cp, [0, 1, 2])
    eng.close()


@pytest.mark.gpu
def test_files_to_query_matches_reference_outputs(wmd, golden, tmp_path):
    s = golden["sample_d3"]
    mtx, vecs_f, r_f = _write_sample(tmp_path, s)
    V, N, words, docs, w = wmd.read_mtx(mtx)
    vecs = wmd.read_vecs(vecs_f, V, 3)
    r = wmd.read_r(r_f, V)
    eng = wmd.Engine()
    eng.set_embeddings(vecs)
    eng.set_targets_edges(words, docs, w, V, N)
    for key, lam in (("fused_lam1", 1.0), ("fused_lam10", 10.0)):
        got = eng.query(r, lam, s["max_iter"])
        ref = np.array(s["outputs"][key])
        np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
        assert rel_err(got, ref).max() <= 1e-5
    eng.close()
