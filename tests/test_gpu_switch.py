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
