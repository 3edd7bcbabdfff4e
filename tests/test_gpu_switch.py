"""The cross-field switch prover on the device (crates/pcs/src/switch.rs): its proof equals the
oracle's restatement (partials, every round's message, the opened value, the point) for word and
bit claims; the oracle's verifier accepts it; the opened value is the lifted witness's MLE at the
returned point (the reference's own round-trip property, switch.rs tests); the transcript ends
in the same state; a wrong claim still yields a proof the verifier rejects."""
import numpy as np
import pytest

from rounds import MATRIX_SEED

pytestmark = pytest.mark.gpu


def setup(wl, cl, seed):
    import labinius_b200 as L

    rng = np.random.default_rng(seed)
    params = L.Params.new(wl, cl, [L.Modulus.Q9721_FS_S])
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    n = params.witness_len()
    trace = rng.integers(0, 2 ** 63, (n, 2), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 2), dtype=np.uint64)
    w = L.Witness.lifted(pp, trace)
    r_hi = rng.integers(0, 2 ** 63, (wl, 2), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (wl, 2), dtype=np.uint64)
    r_lo = rng.integers(0, 2 ** 63, (7, 2), dtype=np.uint64)
    return L, params, pp, trace, w, r_hi, r_lo


@pytest.mark.parametrize("wl,cl,bits", [(9, 2, False), (10, 3, True), (14, 5, False), (16, 6, True)])
def test_switch_matches_oracle(oracle, wl, cl, bits):
    from labinius_b200 import switch

    L, params, pp, trace, w, r_hi, r_lo = setup(wl, cl, wl + 7 * bits)
    lo = r_lo if bits else None
    claim = oracle.switch_mle(trace, r_hi, lo)
    t_gpu = L.Transcript(b"switch/test")
    proof, point = (switch.prove_bits(pp, w, r_lo, r_hi, claim, t_gpu) if bits
                    else switch.prove(pp, w, r_hi, claim, t_gpu))
    t_orc = oracle.Transcript(b"switch/test")
    partials, rounds, opened, r_pp = oracle.switch_prove(trace, r_hi, claim, t_orc, r_lo=lo)
    assert np.array_equal(proof.partials, partials)
    assert np.array_equal(proof.rounds, rounds)
    assert np.array_equal(proof.opened, opened)
    assert np.array_equal(point.p0, r_pp[cl:][::-1]) and np.array_equal(point.p1, r_pp[:cl][::-1])
    assert t_gpu.fill(b"after", 32) == t_orc.fill(b"after", 32)
    ok, _ = oracle.switch_verify(r_hi, claim, proof.partials, proof.rounds, proof.opened,
                                 oracle.Transcript(b"switch/test"), r_lo=lo)
    assert ok
    assert np.array_equal(w.mle_evaluate(point), proof.opened)


def test_switch_wrong_claim_is_rejected(oracle):
    from labinius_b200 import switch

    L, params, pp, trace, w, r_hi, r_lo = setup(10, 3, 1)
    claim = oracle.switch_mle(trace, r_hi)
    claim[1] ^= np.uint64(1 << 40)
    proof, _ = switch.prove(pp, w, r_hi, claim, L.Transcript(b"t"))
    ok, _ = oracle.switch_verify(r_hi, claim, proof.partials, proof.rounds, proof.opened, oracle.Transcript(b"t"))
    assert not ok


def rand_b128(rng, n):
    return rng.integers(0, 2 ** 63, (n, 2), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 2), dtype=np.uint64)


@pytest.mark.parametrize("dropped", [0, 9])
def test_switch_round_through_the_api_matches_oracle(oracle, dropped):
    """A B128 trace opened through the switch with the API, step by step as
    crates/pcs/examples/two_fields.rs:176-194 does: every output and the transcript's tail equal
    the oracle's round."""
    import labinius_b200 as L
    from labinius_b200 import switch
    from rounds import product_params

    wl, cl = 12, 3
    primes = [9721] if not dropped else [9721, 3889]
    params = product_params((wl, cl, primes, dropped))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    rng = np.random.default_rng(300 + dropped)
    trace, r_hi = rand_b128(rng, 1 << wl), rand_b128(rng, wl)
    w = L.Witness.lifted(pp, trace)
    prover, verifier = L.Prover(pp), L.Verifier(pp)
    c, op = prover.commit(w)
    t = L.Transcript(b"example/ghash")
    t.absorb_bytes(c.to_bytes())
    claim = oracle.switch_mle(trace, r_hi)
    proof, point = switch.prove(pp, w, r_hi, claim, t)
    row = w.row_evaluate(point)
    ch = verifier.derive_folding_challenges(t, row)
    v = prover.fold(op, ch)
    o = oracle.switch_round(oracle.Params(wl, cl, primes, dropped), MATRIX_SEED, trace, r_hi, domain=b"example/ghash")
    assert np.array_equal(proof.partials, o["partials"])
    assert np.array_equal(proof.rounds, o["rounds"])
    assert np.array_equal(proof.opened, o["opened"])
    assert np.array_equal(point.p0, o["p0"]) and np.array_equal(point.p1, o["p1"])
    assert np.array_equal(row.values, o["u"])
    assert np.array_equal(ch.challenges, o["challenges"])
    assert np.array_equal(v.elements, o["v"])
    assert t.fill(b"labinius/test-tail", 32) == o["transcript_tail"]
    assert np.array_equal(w.mle_evaluate(point), proof.opened)


@pytest.mark.parametrize("graphs,given", [(False, False), (True, True)], ids=["stream-stated", "graph-given"])
def test_batch_switch_instances_match_oracle(oracle, graphs, given):
    """A batch mixing Witness::random instances with B128 traces opened through the switch, in one
    device round: each switch instance equals the oracle's switch round of its trace (commitment,
    proof, claim, point, row values, challenges, folded witness), each plain instance the
    single-instance API round; a second round gives the same results."""
    import labinius_b200 as L
    from labinius_b200.batch import Batch
    from rounds import DOMAIN, product_params, product_round

    row_log, primes = 9, [9721]
    col_logs, kinds = [3, 2, 4, 3, 2], [1, 0, 1, 0, 1]
    params = product_params((row_log + col_logs[0], col_logs[0], primes, 0))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    b = Batch(pp, col_logs)
    seeds = [bytes([(0x30 + i) & 0xFF]) * 32 for i in range(len(col_logs))]
    b.witness_random(seeds, kinds)
    marked = [i for i, k in enumerate(kinds) if k]
    rng = np.random.default_rng(11)
    r_his = [rand_b128(rng, row_log + col_logs[i]) for i in marked]
    traces = [b.elements(i)[:, :2].copy() for i in marked]
    claims = [oracle.switch_mle(tr, r) for tr, r in zip(traces, r_his)] if given else None
    b.set_switch([k == 1 for k in kinds], r_his, claims)
    if graphs:
        b.use_graphs(True)
    first = b.round(DOMAIN)
    second = b.round(DOMAIN)
    for k, i in enumerate(marked):
        cl = col_logs[i]
        o = oracle.switch_round(oracle.Params(row_log + cl, cl, primes, 0), MATRIX_SEED, traces[k], r_his[k],
                                domain=DOMAIN)
        for r in (first[i], second[i]):
            assert np.array_equal(r.matrix, o["C"])
            assert np.array_equal(r.claim, o["claim"])
            assert np.array_equal(r.switch.partials, o["partials"])
            assert np.array_equal(r.switch.rounds, o["rounds"])
            assert np.array_equal(r.switch.opened, o["opened"])
            assert np.array_equal(r.p0, o["p0"]) and np.array_equal(r.p1, o["p1"])
            assert np.array_equal(r.u, o["u"])
            assert np.array_equal(r.mle, o["opened"])
            assert np.array_equal(r.challenges, o["challenges"])
            assert np.array_equal(r.v, o["v"])
    for i, kind in enumerate(kinds):
        if kind:
            continue
        cl = col_logs[i]
        single = product_round((row_log + cl, cl, primes, 0), witness_seed=seeds[i])
        for r in (first[i], second[i]):
            assert np.array_equal(r.matrix, single["commitment"].matrix)
            assert np.array_equal(r.u, single["u"])
            assert np.array_equal(r.challenges, single["challenges"])
            assert np.array_equal(r.v, single["v"])
