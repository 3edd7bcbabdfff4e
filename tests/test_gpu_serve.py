"""Serving with continuous batching: each request's result in the mix equals the same request run
alone through the single-instance path (native witnesses, and B128 traces opened through the
cross-field switch; mixed sizes, arrivals while other requests are on the GPU); admission respects
the arena size."""
import time

import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, product_params

pytestmark = pytest.mark.gpu


def alone(oracle, row_log, primes, req, r_hi):
    """The request's round on its own: Witness::random through the plain path, or a B128 trace
    through the switch (crates/pcs/examples/two_fields.rs:176-194)."""
    import labinius_b200 as L
    from labinius_b200 import switch

    cl = req.column_log_len
    params = product_params((row_log + cl, cl, primes, 0))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    prover, verifier = L.Prover(pp), L.Verifier(pp)
    t = L.Transcript(DOMAIN)
    proof = claim = None
    if req.kind == 1:
        n = params.witness_len()
        raw = oracle.blake3(b"labinius/b128-trace", 16 * n, key=req.seed)
        trace = np.frombuffer(raw, dtype=np.uint64).reshape(-1, 2)
        w = L.Witness.lifted(pp, trace)
        c, op = prover.commit(w)
        t.absorb_bytes(c.to_bytes())
        claim = oracle.switch_mle(trace, r_hi)
        proof, point = switch.prove(pp, w, r_hi, claim, t)
        mle = proof.opened
    else:
        w = L.Witness.random(pp, req.seed)
        c, op = prover.commit(w)
        point = verifier.derive_evaluation_point(t, c)
        mle = w.mle_evaluate(point)
    row = w.row_evaluate(point)
    ch = verifier.derive_folding_challenges(t, row)
    v = prover.fold(op, ch)
    return c.matrix, point, mle, row.values, ch.challenges, v.elements, proof, claim


@pytest.mark.parametrize("transcript,small", [("device", None), ("host", None), ("device", 2)],
                         ids=["device", "host", "size-classes"])
def test_results_in_the_mix_equal_results_alone(oracle, transcript, small):
    import labinius_b200 as L
    from labinius_b200.serve import Request, Server

    row_log, primes = 8, [3889, 9721]
    pp = L.PublicParameters.from_seed(product_params((row_log + 3, 3, primes, 0)), MATRIX_SEED)
    srv = Server(pp, capacity_columns=48, max_requests=8, slots=2, host_threads=4, transcript=transcript,
                 small_log_len=small)
    rng = np.random.default_rng(4)
    reqs = []
    for i in range(14):
        cl = int(rng.integers(1, 6))
        kind = int(i % 5 == 4) if transcript == "device" else 0  # the switch runs its transcript on the device
        reqs.append(srv.submit(Request(cl, bytes([0x40 + i]) * 32, kind=kind)))
        if i % 4 == 3:
            time.sleep(0.01)  # later arrivals join while earlier batches run
    too_big = srv.submit(Request(6, bytes(32)))  # 64 columns > 48
    for r in reqs:
        assert r.wait(120)
    srv.close()
    assert too_big.error is not None
    assert srv.batches >= 2
    for r in reqs:
        assert r.error is None, r.error
        m, point, mle, u, ch, v, proof, claim = alone(oracle, row_log, primes, r, srv.switch_point(r))
        res = r.result
        if r.kind == 1:
            assert np.array_equal(res.claim, claim)
            assert np.array_equal(res.switch.partials, proof.partials)
            assert np.array_equal(res.switch.rounds, proof.rounds)
            assert np.array_equal(res.switch.opened, proof.opened)
        assert np.array_equal(res.matrix, m)
        assert np.array_equal(res.p0, point.p0) and np.array_equal(res.p1, point.p1)
        assert np.array_equal(res.mle, mle) and np.array_equal(res.u, u)
        assert np.array_equal(res.challenges, ch)
        assert np.array_equal(res.v, v)


def test_arenas_are_sized_from_free_device_memory():
    """Without a capacity the arenas take hbm_fraction of the free device memory: the columns are
    a power of two whose arena fits the share and whose double does not (or the cap)."""
    import ctypes

    import labinius_b200 as L
    from labinius_b200._native import check, lib
    from labinius_b200.serve import arena_columns

    pp = L.PublicParameters.from_seed(product_params((11 + 3, 3, [3889, 9721], 0)), MATRIX_SEED)
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    check(lib().lbg_device_memory(pp._h, ctypes.byref(free), ctypes.byref(total)))
    assert 0 < free.value <= total.value
    cols = arena_columns(pp, 0.01, 2, 16)
    share = 0.01 * free.value / 2
    assert cols & (cols - 1) == 0
    assert lib().lbg_batch_arena_bytes(pp._h, cols, 16) <= share or cols == 1
    assert cols == 1 << 16 or lib().lbg_batch_arena_bytes(pp._h, 2 * cols, 16) > share
