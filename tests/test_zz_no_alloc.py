"""lbg_fold_static: the fold for callers that may not allocate device memory when they fold (an
embedding runtime that owns all device memory through its own arena, or one that replays its
steps where allocator calls are not allowed). Its scratch is in static device arrays, so it is
checked here against the allocating entry point lbg_fold, twice in a row on the same scratch.

This file is collected last (test_zz_*) and passes both alone in a fresh process and after the
rest of the suite: the entry point sets its device up on first use either way."""
import numpy as np
import pytest

from rounds import MATRIX_SEED, WITNESS_SEED, product_params

pytestmark = pytest.mark.gpu


# the first three and the 4096-position shape split their columns over CTAs that add into the static
# sums; the 8192-position shapes fold in one pass, the last at the 1024-column limit
@pytest.mark.parametrize("shape", [(12, 4, [3889, 2917, 4861], 0), (13, 5, [2917, 9721], 0), (17, 10, [9721, 3889], 0),
                                   (19, 7, [3889, 9721], 0), (20, 7, [2917, 9721], 0), (23, 10, [3889, 9721], 0)],
                         ids=["3889", "2917", "1024-columns", "split-4096-positions", "one-pass-8192-positions",
                              "one-pass-1024-columns"])
def test_fold_static_matches_fold(shape):
    import torch

    import labinius_b200 as L
    from labinius_b200._native import LBG_ERR_INVALID, LBG_OK, lib

    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    prover = L.Prover(pp)
    verifier = L.Verifier(pp)
    c, op = prover.commit(w)
    t = L.Transcript(b"labinius/reference")
    point = verifier.derive_evaluation_point(t, c)
    ch = verifier.derive_folding_challenges(t, w.row_evaluate(point))
    want = prover.fold(op, ch).elements

    # device memory the caller owns
    d_w = torch.from_numpy(w.elements().view(np.int64)).cuda()
    d_ch = torch.from_numpy(np.ascontiguousarray(ch.challenges).view(np.uint8).copy()).cuda()
    d_v = torch.empty((params.len_ring(), 648), dtype=torch.int16, device="cuda")
    base, wl, cl, r = params.primes()[0], params.witness_log_len, params.column_log_len, params.columns()
    free_after = []
    for _ in range(2):
        d_v.fill_(0x5A5A)
        torch.cuda.synchronize()
        rc = lib().lbg_fold_static(base, wl, cl, d_w.data_ptr(), d_ch.data_ptr(), r, d_v.data_ptr(), None)
        assert rc == LBG_OK, lib().lbg_last_error()
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        assert np.array_equal(d_v.cpu().numpy(), want)
    # the second call took no device memory (the first may have loaded the module's static arrays)
    assert free_after[1] == free_after[0]

    # beyond the static maximum: rejected with a clear message, nothing launched
    rc = lib().lbg_fold_static(base, 20, 11, d_w.data_ptr(), d_ch.data_ptr(), 2048, d_v.data_ptr(), None)
    assert rc == LBG_ERR_INVALID
    assert b"at most 1024 columns" in lib().lbg_last_error()
