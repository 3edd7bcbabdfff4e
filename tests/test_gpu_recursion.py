"""The recursive opening's device half against the oracle: Opening::Recursive parameters are accepted,
the commitment's residues (recursion::limbs::residues, crates/pcs/src/recursion/limbs.rs:379-398, the
input of T_y) and the left expansion's vector (Prover::commit_left_expansion,
crates/pcs/src/scheme/prover.rs:95-115, the input of T_u) equal the oracle's, and the fold inside
prove_opening (prover.rs:137-150) is the plain fold. The LaBRADOR commitments and proof stay on
the host, so the library's transcript steps refuse the recursive round."""
import numpy as np
import pytest

import oracle as O
from rounds import MATRIX_SEED, WITNESS_SEED

pytestmark = pytest.mark.gpu

SHAPES = [(12, 4, [3889, 9721]), (15, 6, [3889, 2917, 9721]), (18, 8, [9721, 12637]), (22, 10, [3889, 2917, 4861])]


def recursive_params(wl, cl, primes):
    import labinius_b200 as L

    return L.Params.with_base(wl, cl, L.Modulus(primes[0]), [L.Modulus(q) for q in primes[1:]],
                              L.Opening.recursive())


@pytest.mark.parametrize("shape", SHAPES, ids=["basic-like", "quadratic", "suite-s", "suite-l"])
def test_residues_and_left_expansion_match_oracle(shape):
    import labinius_b200 as L
    from labinius_b200._native import NativeError

    wl, cl, primes = shape
    params = recursive_params(*shape)
    assert params.recursion()
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    res = op.residues()

    P = O.Params(wl, cl, primes)
    r = P.columns
    if wl <= 18:
        A = O.key_expand(P, O.key_seed(MATRIX_SEED))
        C = O.commit(P, A, O.witness_random(P.witness_len, WITNESS_SEED), threads=8)
        assert np.array_equal(c.matrix, C)
    # the residues are a function of the commitment matrix alone: the oracle's from the same matrix
    assert np.array_equal(res, O.recursion_residues(P, c.matrix))
    # a wider padding only adds zero polynomials
    wide = op.residues(O.recursion_polys(r) + 32)
    assert np.array_equal(wide[:, : res.shape[1]], res) and not wide[:, res.shape[1]:].any()

    # the left expansion of a row evaluation (the point is the transcript's business on the host)
    rng = np.random.default_rng(wl)
    p0 = rng.integers(0, 2 ** 63, (wl - cl, 3), dtype=np.uint64)
    p0[:, 2] &= np.uint64((1 << 34) - 1)
    row = w.row_evaluate(L.EvaluationPoint(p0, np.zeros((cl, 3), np.uint64)))
    u = prover.commit_left_expansion_vector(row)
    assert np.array_equal(u, O.left_expansion(row.values))
    assert np.array_equal(prover.commit_left_expansion_vector(row, O.recursion_polys(r) + 64)[: len(u)], u)

    # the fold of prove_opening is the plain fold
    ch = L.FoldingChallenges(np.zeros(r, L.CHALLENGE_DTYPE))
    ch.challenges["weight"] = 28
    ch.challenges["positions"][:, :28] = (np.arange(28) * 5 + 1).astype(np.uint8)
    ch.challenges["signs"] = rng.integers(0, 2 ** 32, r, dtype=np.uint64).astype(np.uint32)
    v = prover.fold(op, ch).elements
    if wl <= 15:
        want = O.fold(P, O.witness_random(P.witness_len, WITNESS_SEED), ch.challenges, threads=8)
        assert np.array_equal(v, want)
    else:
        clear = L.Params.with_base(wl, cl, L.Modulus(primes[0]), [L.Modulus(q) for q in primes[1:]])
        pc = L.PublicParameters.from_seed(clear, MATRIX_SEED)
        pr2 = L.Prover(pc)
        _, op2 = pr2.commit(L.Witness.random(pc, WITNESS_SEED))
        assert np.array_equal(v, pr2.fold(op2, ch).elements)

    # the transcript of the recursive round absorbs LaBRADOR's T_y and T_u: refused here
    with pytest.raises(NativeError):
        L.Verifier(pp).derive_evaluation_point(L.Transcript(b"labinius/reference"), c)


def test_recursive_entry_points_refuse_misuse():
    """Too few polynomials, a row evaluation of the wrong width and a bit-dropped commitment are
    refused with a message; nothing is launched and the prover stays usable."""
    import labinius_b200 as L
    from labinius_b200._native import LBG_ERR_INVALID, NativeError

    params = recursive_params(12, 4, [3889, 9721])
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    with pytest.raises(NativeError) as e:
        op.residues(3 * params.columns() - 1)
    assert e.value.code == LBG_ERR_INVALID
    row = L.RowEvaluation(np.zeros((params.columns() + 1, 3), np.uint64))
    with pytest.raises(NativeError):
        prover.commit_left_expansion_vector(row)
    with pytest.raises(NativeError):
        prover.commit_left_expansion_vector(L.RowEvaluation(np.zeros((params.columns(), 3), np.uint64)),
                                            3 * params.columns() - 1)
    assert np.array_equal(op.residues(), O.recursion_residues(O.Params(12, 4, [3889, 9721]), c.matrix))

    bd = L.Params.with_base(12, 4, L.Modulus(3889), [L.Modulus(2917), L.Modulus(4861)], L.Opening.bit_dropped(9))
    ppb = L.PublicParameters.from_seed(bd, MATRIX_SEED)
    pb = L.Prover(ppb)
    _, opb = pb.commit(L.Witness.random(ppb, WITNESS_SEED))
    with pytest.raises(NativeError):
        opb.residues()
