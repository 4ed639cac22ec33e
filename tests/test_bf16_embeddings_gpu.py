"""GPU: embeddings given in BF16 (wmd_set_embeddings_bf16).  The engine keeps
the BF16 rows for the BF16 tensor-core cost panel and their exact FP32 values
for everything else, so the scores are those of the BF16-valued embeddings:
checked against the FP64 oracle run on the same values."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode,tol", [("fp32", 1e-5), ("tf32x3", 1e-5), ("bf16", 1e-4)])
def test_bf16_embeddings_vs_oracle(wmd, synth, oracle_mod, mode, tol):
    import torch
    p = synth.case(3000, 300, 200, 40, 8, 160, 50, 71)
    e16 = torch.from_numpy(p.vecs).to(torch.bfloat16)
    vals = e16.to(torch.float64).numpy()  # the BF16 values exactly
    ref = oracle_mod.sinkhorn(p.r, vals, p.col_ptr, p.row_inds, p.vals, p.lam, p.max_iter)
    eng = wmd.Engine(0)
    eng.set_embeddings_bf16(e16)
    eng.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng.set_cdist_mode(mode)
    got = eng.query(p.r, p.lam, p.max_iter)
    # the same from device memory, and against FP32 input of the same values
    eng2 = wmd.Engine(0)
    eng2.set_embeddings_bf16(e16.cuda())
    eng2.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng2.set_cdist_mode(mode)
    got2 = eng2.query(p.r, p.lam, p.max_iter)
    eng3 = wmd.Engine(0)
    eng3.set_embeddings(vals.astype(np.float32))
    eng3.set_targets(p.col_ptr, p.row_inds, p.vals)
    eng3.set_cdist_mode(mode)
    got3 = eng3.query(p.r, p.lam, p.max_iter)
    for e in (eng, eng2, eng3):
        e.close()
    assert rel_err(got, ref).max() <= tol
    np.testing.assert_array_equal(got, got2)
    np.testing.assert_array_equal(got, got3)
