"""The verifier's checks on the device (crates/pcs/src/scheme/verifier.rs:148-231): the folded row
value equals the oracle's, the claim check and the Clear opening check accept an honest round and
give the oracle's verdict on tampered ones (v off by one, v out of range, a wrong folded row value,
a wrong folded commitment, a norm beyond the cap), for split and quadratic base primes."""
import numpy as np
import pytest

from rounds import product_round

pytestmark = pytest.mark.gpu


def oracle_params(oracle, shape):
    wl, cl, primes, dropped = shape
    return oracle.Params(wl, cl, primes, dropped)


def gpu_accepts(verifier, fc, v, point, fr):
    import labinius_b200 as L

    try:
        verifier.verify_folded_opening(L.FoldedCommitment(verifier.params.primes(), fc), L.FoldedWitness(v), point, fr)
        return True
    except L.VerificationError:
        return False


@pytest.mark.parametrize("shape", [(12, 4, [3889, 2917, 9721], 0), (11, 3, [2917, 19441], 0), (12, 5, [19441], 0)],
                         ids=["3889", "2917", "19441"])
def test_verifier_on_device_matches_oracle(oracle, shape):
    import labinius_b200 as L

    r = product_round(shape)
    pp = r["pp"]
    verifier = L.Verifier(pp)
    P = oracle_params(oracle, shape)
    key = pp.key()
    ch = L.FoldingChallenges(r["challenges"])
    fr = verifier.fold_row_evaluation(L.RowEvaluation(r["u"]), ch)
    assert np.array_equal(fr, oracle.fold_binary(r["u"], r["challenges"]))
    verifier.verify_evaluation(L.EvaluationPoint(r["p0"], r["p1"]), r["mle"], L.RowEvaluation(r["u"]))
    bad = r["mle"].copy()
    bad[0] ^= np.uint64(1)
    with pytest.raises(L.VerificationError):
        verifier.verify_evaluation(L.EvaluationPoint(r["p0"], r["p1"]), bad, L.RowEvaluation(r["u"]))

    point = L.EvaluationPoint(r["p0"], r["p1"])
    fc, v = r["folded_commitment"], r["v"]
    msg = L.OpeningMessage.clear(L.FoldedCommitment(pp.params.primes(), fc), L.FoldedWitness(v), fr)
    verifier.verify_opening(r["commitment"], ch, point, msg)  # honest: accepted
    assert oracle.verify_folded_opening(P, key, fc, v, r["p0"], fr)

    half = (shape[2][0] - 1) // 2
    rng = np.random.default_rng(5)
    cases = []
    v1 = v.copy(); v1[3, 17] += 1; cases.append(("v+1", fc, v1, fr))
    v2 = v.copy(); v2[0, 0] = half + 1; cases.append(("out of range", fc, v2, fr))
    v3 = v.copy(); v3[1, 5] = -half - 1; cases.append(("out of range below", fc, v3, fr))
    fr2 = fr.copy(); fr2[2] ^= np.uint64(4); cases.append(("row value", fc, v, fr2))
    fc2 = fc.copy(); fc2[1, 0, 7] += 1; cases.append(("folded commitment", fc2, v, fr))
    v4 = np.full_like(v, 0); v4[:, ::7] = rng.integers(-half, half + 1, v4[:, ::7].shape); cases.append(("norm", fc, v4, fr))
    v5 = v.copy(); v5[2, 9] = -32768; cases.append(("i16 minimum", fc, v5, fr))
    for name, f, vv, rr in cases:
        want = oracle.verify_folded_opening(P, key, f, vv, r["p0"], rr)
        assert not want, name
        assert gpu_accepts(verifier, f, vv, point, rr) == want, name


@pytest.mark.parametrize("shape", [(12, 4, [9721, 3889], 9), (12, 3, [3889, 2917, 4861], 10), (11, 3, [9721], 8)],
                         ids=["two-limbs", "three-limbs", "one-limb"])
def test_bit_dropped_opening_on_device_matches_oracle(oracle, shape):
    """The bit-dropped arm (crates/pcs/src/scheme/verifier.rs:232-276): on an honest round the
    device's residual (crates/pcs/src/bd/residual.rs:66-130) equals the oracle's to the bit and the
    check accepts; tampered rounds get the oracle's verdict."""
    import labinius_b200 as L

    r = product_round(shape)
    pp = r["pp"]
    verifier = L.Verifier(pp)
    P = oracle_params(oracle, shape)
    key = pp.key()
    c = r["commitment"]
    ch = L.FoldingChallenges(r["challenges"])
    point = L.EvaluationPoint(r["p0"], r["p1"])
    fr = verifier.fold_row_evaluation(L.RowEvaluation(r["u"]), ch)
    v = r["v"]
    ok, res = verifier.bd_residual(c, ch, L.FoldedWitness(v), point, fr)
    want = oracle.bd_residual(P, key, c.top, c.digits, r["challenges"], v)
    assert res == want and ok
    assert 0 < res <= oracle.bd_cap(P)
    verifier.verify_opening(c, ch, point, L.OpeningMessage.bit_dropped(L.FoldedWitness(v), fr))

    half = (shape[2][0] - 1) // 2
    cases = []
    v1 = v.copy(); v1[3, 17] += 1; cases.append(("v+1", c.top, c.digits, v1, fr))
    v2 = v.copy(); v2[0, 0] = half + 1; cases.append(("out of range", c.top, c.digits, v2, fr))
    fr2 = fr.copy(); fr2[0] ^= np.uint64(1); cases.append(("row value", c.top, c.digits, v, fr2))
    t2 = (c.top.astype(np.int64) + 5) % (1 << 6); cases.append(("top", t2.astype(np.uint16), c.digits, v, fr))
    if len(shape[2]) > 1:
        d2 = c.digits.copy(); d2[0, ::3] = (d2[0, ::3] + 1) % shape[2][1]; cases.append(("digits", c.top, d2, v, fr))
    for name, top, digits, vv, rr in cases:
        want = oracle.verify_folded_opening_bd(P, key, top, digits, r["challenges"], vv, r["p0"], rr)
        c2 = L.Commitment(c.primes, c.columns, top=top, digits=digits, params=c.params)
        got, res2 = verifier.bd_residual(c2, ch, L.FoldedWitness(vv), point, rr)
        assert got == want, name
        assert res2 == oracle.bd_residual(P, key, top, digits, r["challenges"], vv), name
        assert not want, name
