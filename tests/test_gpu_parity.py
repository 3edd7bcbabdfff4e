"""Bit-exact parity of every GPU entry point against the oracle, through the C ABI (labinius_b200).

Shapes are small enough for the oracle; edge cases follow the reference's tests: adversarial 0/1
ring elements (crates/pcs/tests/common/mod.rs:49-81), every one of the seven primes as base and as
extra limb, extreme challenges, columns and ring elements that do not fill a CTA tile."""
import numpy as np
import pytest

from rounds import MATRIX_SEED, WITNESS_SEED, product_params

pytestmark = pytest.mark.gpu

ALL = [3889, 2917, 4861, 9721, 12637, 17497, 19441]
CH = np.dtype([("positions", np.uint8, 32), ("signs", np.uint32), ("weight", np.uint32)])


def pack4(polys):
    """crates/pcs/src/f162.rs:57-69: four F162 per ring element, coefficient 4m+k = bit m of k."""
    out = np.zeros((len(polys) * 4, 3), np.uint64)
    for r, c in enumerate(polys):
        for m in range(162):
            for k in range(4):
                if c[4 * m + k]:
                    out[4 * r + k, m >> 6] |= np.uint64(1) << np.uint64(m & 63)
    return out


def adversarial_witness(n, seed=5):
    """Adversarial ring elements first (all-zero, all-one, alternating, block-structured,
    monomials at tree boundaries), then random bits."""
    rng = np.random.default_rng(seed)
    polys = [np.zeros(648, np.uint8), np.ones(648, np.uint8)]
    for phase in range(2):
        polys.append(np.array([(i % 2 == phase) for i in range(648)], np.uint8))
        polys.append(np.array([(i % 3 == phase) for i in range(648)], np.uint8))
    for b in range(4):
        p = np.zeros(648, np.uint8)
        p[162 * b:162 * (b + 1)] = 1
        polys.append(p)
    for d in [0, 1, 53, 54, 80, 81, 107, 108, 161, 162, 163, 323, 324, 325, 485, 486, 646, 647]:
        p = np.zeros(648, np.uint8)
        p[d] = 1
        polys.append(p)
    w = pack4(polys)
    rest = rng.integers(0, 2 ** 63, (n - len(w), 3), dtype=np.uint64) * np.uint64(2) + rng.integers(
        0, 2, (n - len(w), 3), dtype=np.uint64)
    rest[:, 2] &= np.uint64((1 << 34) - 1)
    return np.concatenate([w, rest])


def setup(shape, witness=None):
    import labinius_b200 as L

    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED) if witness is None else L.Witness.from_elements(pp, witness)
    return L, params, pp, w


def oracle_params(oracle, shape):
    wl, cl, primes, d = shape
    return oracle.Params(wl, cl, primes, d)


@pytest.mark.parametrize("shape", [(10, 2, ALL, 0), (13, 6, [3889, 9721], 0), (13, 1, [19441, 2917], 0)],
                         ids=["allprimes", "64cols", "2cols"])
def test_key_matches_oracle(oracle, shape):
    L, params, pp, _ = setup(shape)
    P = oracle_params(oracle, shape)
    want = oracle.key_expand(P, oracle.key_seed(MATRIX_SEED))
    assert np.array_equal(pp.key(), want)


def test_witness_random_matches_oracle(oracle):
    shape = (12, 3, [3889], 0)
    L, params, pp, w = setup(shape)
    assert np.array_equal(w.elements(), oracle.witness_random(params.witness_len(), WITNESS_SEED))


@pytest.mark.parametrize("base", ALL)
def test_commit_every_prime_adversarial(oracle, base):
    primes = [base] + [q for q in ALL if q != base]
    shape = (10, 2, primes, 0)
    wit = adversarial_witness(1 << 10, seed=base)
    L, params, pp, w = setup(shape, wit)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    want = oracle.commit(oracle_params(oracle, shape), pp.key(), wit)
    assert np.array_equal(c.matrix, want)
    prover.recycle(op)


@pytest.mark.parametrize("shape", [(13, 6, [3889, 2917, 4861], 0), (13, 3, [9721], 0), (11, 1, [4861, 12637], 0),
                                   (14, 4, [3889, 2917, 9721], 0)],
                         ids=["64cols", "8cols", "2cols", "xl-limbs"])
def test_commit_shapes(oracle, shape):
    L, params, pp, w = setup(shape)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    want = oracle.commit(oracle_params(oracle, shape), pp.key(), w.elements(), threads=8)
    assert np.array_equal(c.matrix, want)
    # a second commitment on the recycled workspace is the same
    prover.recycle(op)
    c2, _ = prover.commit(w)
    assert np.array_equal(c2.matrix, want)


@pytest.mark.parametrize("shape", [(12, 4, [3889, 2917, 4861], 9), (11, 3, [2917, 3889], 10),
                                   (12, 2, [4861, 9721, 19441], 7), (11, 3, [12637], 8)],
                         ids=["bd9", "quadbase", "3limb", "1limb"])
def test_bit_dropped_commit(oracle, shape):
    L, params, pp, w = setup(shape)
    prover = L.Prover(pp)
    c, _ = prover.commit(w)
    P = oracle_params(oracle, shape)
    C = oracle.commit(P, pp.key(), w.elements())
    top, digits = oracle.drop_bits(P, C)
    assert np.array_equal(c.top, top)
    assert np.array_equal(c.digits, digits)


def random_point(rng, n):
    p = rng.integers(0, 2 ** 63, (n, 3), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 3), dtype=np.uint64)
    p[:, 2] &= np.uint64((1 << 34) - 1)
    return p


@pytest.mark.parametrize("shape", [(12, 3, [3889], 0), (13, 5, [3889], 0), (11, 1, [3889], 0)])
def test_row_and_mle_evaluate(oracle, shape):
    from labinius_b200 import EvaluationPoint

    L, params, pp, w = setup(shape)
    rng = np.random.default_rng(7)
    for trial in range(2):
        p0 = random_point(rng, params.row_log_len())
        p1 = random_point(rng, params.column_log_len)
        if trial == 1:
            p0[:] = 0
            p0[:, 0] = 1  # eq concentrates on the last row
        pt = EvaluationPoint(p0, p1)
        elems = w.elements()
        u = oracle.row_evaluate(elems, p0)
        assert np.array_equal(w.row_evaluate(pt).values, u)
        assert np.array_equal(w.mle_evaluate(pt), oracle.claim(u, p1))


def sampled_challenges(oracle, r, seed):
    t = oracle.Transcript(b"labinius/test-challenges")
    t.absorb_u64(seed)
    return np.array([oracle.sample_short_challenge(t)[0] for _ in range(r)], dtype=CH)


def edge_challenges(r):
    """weight 0, all-negative weight 32, every position a boundary, and mixtures."""
    c = np.zeros(r, CH)
    for j in range(r):
        kind = j % 4
        if kind == 0:
            continue
        if kind == 1:
            c[j]["weight"] = 32
            c[j]["positions"][:] = np.arange(130, 162)
            c[j]["signs"] = 0xFFFFFFFF
        elif kind == 2:
            c[j]["weight"] = 6
            c[j]["positions"][:6] = [0, 1, 80, 81, 160, 161]
            c[j]["signs"] = 0b101010
        else:
            c[j]["weight"] = 28
            c[j]["positions"][:28] = np.arange(0, 162, 5)[:28]
            c[j]["signs"] = 0x0F0F0F0
    return c


@pytest.mark.parametrize("shape", [(12, 3, [3889, 9721], 0), (11, 4, [2917, 3889], 0), (12, 5, [19441], 0),
                                   (11, 2, [4861], 0), (11, 2, [12637], 0), (11, 2, [17497], 0), (11, 2, [9721], 0)],
                         ids=["3889", "2917", "19441", "4861", "12637", "17497", "9721"])
def test_fold_and_fold_commitment(oracle, shape):
    from labinius_b200 import FoldingChallenges

    L, params, pp, w = setup(shape)
    prover = L.Prover(pp)
    verifier = L.Verifier(pp)
    P = oracle_params(oracle, shape)
    elems = w.elements()
    for keep in [True, False]:  # the fold from the kept transform, and transforming the witness again
        prover.keep_transform(keep)
        for ch in [sampled_challenges(oracle, params.columns(), 3), edge_challenges(params.columns())]:
            c, op = prover.commit(w)
            v = prover.fold(op, FoldingChallenges(ch))
            assert np.array_equal(v.elements, oracle.fold(P, elems, ch, threads=8)), keep
            fc = verifier.fold_commitment(c, FoldingChallenges(ch))
            assert np.array_equal(fc.rows, oracle.fold_commitment(P, c.matrix, ch))


def test_verifier_identities_hold_for_gpu_outputs(oracle):
    """A v = sum_j c_j C_j on every limb and the binary check, on the GPU's own outputs
    (crates/pcs/src/scheme/verifier.rs:178-231)."""
    from rounds import product_round

    shape = (12, 4, [3889, 2917, 9721], 0)
    r = product_round(shape)
    P = oracle_params(oracle, shape)
    fr = oracle.fold_binary(r["u"], r["challenges"])
    assert oracle.verify_folded_opening(P, r["pp"].key(), r["folded_commitment"], r["v"], r["p0"], fr)
    assert np.array_equal(oracle.claim(r["u"], r["p1"]), r["mle"])


def test_errors_do_not_cross_the_boundary():
    import labinius_b200 as L
    from labinius_b200._native import NativeError

    shape = (11, 3, [3889], 0)
    _, params, pp, w = setup(shape)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    with pytest.raises(NativeError):
        prover.fold(op, L.FoldingChallenges(np.zeros(3, CH)))  # wrong count: consumed, rejected
    with pytest.raises(ValueError):
        w.row_evaluate(L.EvaluationPoint(np.zeros((3, 3), np.uint64), np.zeros((3, 3), np.uint64)))
    with pytest.raises(L.WitnessError):
        L.Witness.from_elements(pp, np.zeros((10, 3), np.uint64))
    with pytest.raises(L.ParamError):
        L.PublicParameters.from_seed(L.Params(11, 3, L.Modulus.Q3889_FS_S, [L.Modulus.Q3889_FS_S]), MATRIX_SEED)
    # the prover still works after the rejected calls
    c2, op2 = prover.commit(w)
    assert np.array_equal(c.matrix, c2.matrix)


@pytest.mark.parametrize("shape", [(20, 9, [3889, 2917, 4861], 0), (19, 8, [9721, 3889], 9), (14, 3, [2917], 0)],
                         ids=["512-columns", "256-columns-bd", "8-columns"])
def test_commit_from_host_memory_equals_upload_then_commit(shape):
    """lbg_commit_host (the upload pipelined against the commit by column groups) gives the
    commitment, the witness and, after the fold, the folded witness of Witness::from_elements +
    Prover::commit."""
    import labinius_b200 as L
    from rounds import MATRIX_SEED, product_params

    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    rng = np.random.default_rng(shape[0])
    e = rng.integers(0, 2 ** 63, (params.witness_len(), 3), dtype=np.uint64)
    e[:, 2] &= np.uint64((1 << 34) - 1)
    prover = L.Prover(pp)
    w1 = L.Witness.from_elements(pp, e)
    c1, op1 = prover.commit(w1)
    w2, c2, op2 = prover.commit_elements(e)
    assert np.array_equal(w2.elements(), e)
    if params.dropped_bits():
        assert np.array_equal(c1.top, c2.top) and np.array_equal(c1.digits, c2.digits)
    else:
        assert np.array_equal(c1.matrix, c2.matrix)
    ch = L.FoldingChallenges(np.zeros(params.columns(), L.CHALLENGE_DTYPE))
    ch.challenges["weight"] = 28
    ch.challenges["positions"][:, :28] = np.arange(0, 28 * 5, 5, dtype=np.uint8)
    v1 = prover.fold(op1, ch)
    v2 = prover.fold(op2, ch)
    assert np.array_equal(v1.elements, v2.elements)


def test_commits_from_host_memory_in_a_row_stay_apart():
    """Three lbg_commit_host calls in a row on one prover (the limbs' streams and chunk partials
    reused, openings still open) each equal Witness::from_elements + Prover::commit of their own
    witness; the folds of the three openings equal the device-witness folds."""
    import labinius_b200 as L
    from rounds import MATRIX_SEED, product_params

    params = product_params((20, 9, [3889, 2917, 4861], 0))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    prover = L.Prover(pp)
    rng = np.random.default_rng(77)
    ch = L.FoldingChallenges(np.zeros(params.columns(), L.CHALLENGE_DTYPE))
    ch.challenges["weight"] = 28
    ch.challenges["positions"][:, :28] = np.arange(0, 28 * 3, 3, dtype=np.uint8)
    runs = []
    for _ in range(3):
        e = rng.integers(0, 2 ** 63, (params.witness_len(), 3), dtype=np.uint64)
        e[:, 2] &= np.uint64((1 << 34) - 1)
        runs.append((e,) + prover.commit_elements(e))
    for e, w, c, op in runs:
        c1, op1 = prover.commit(L.Witness.from_elements(pp, e))
        assert np.array_equal(c.matrix, c1.matrix)
        assert np.array_equal(prover.fold(op, ch).elements, prover.fold(op1, ch).elements)


def test_commit_from_pageable_and_page_locked_memory_agree():
    """lbg_commit_host stages a pageable witness through its page-locked ring and copies a
    page-locked one directly; both give Witness::from_elements + Prover::commit's commitment and
    witness, three calls in a row alternating the two kinds of memory."""
    import torch

    import labinius_b200 as L
    from rounds import MATRIX_SEED, product_params

    params = product_params((20, 9, [3889, 2917, 4861], 0))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    prover = L.Prover(pp)
    rng = np.random.default_rng(5)
    for locked in (True, False, True):
        e = rng.integers(0, 2 ** 63, (params.witness_len(), 3), dtype=np.uint64)
        e[:, 2] &= np.uint64((1 << 34) - 1)
        if locked:
            t = torch.empty((params.witness_len(), 3), dtype=torch.int64, pin_memory=True)
            src = t.numpy().view(np.uint64)
            src[:] = e
        else:
            src = e
        w, c, op = prover.commit_elements(src)
        c1, op1 = prover.commit(L.Witness.from_elements(pp, e))
        assert np.array_equal(w.elements(), e)
        assert np.array_equal(c.matrix, c1.matrix)
        prover.recycle(op)
        prover.recycle(op1)


def test_handles_free_in_any_order():
    """Parameters freed before their prover, and a prover freed before its opening, stay valid until
    the last handle that uses them goes (a garbage collector finalizes a cycle in no fixed order):
    the opening still folds to the oracle's folded witness afterwards."""
    import ctypes

    import labinius_b200 as L
    import oracle as O
    from labinius_b200._native import LBG_OK, lib, ptr
    from rounds import MATRIX_SEED, WITNESS_SEED, product_params

    shape = (12, 4, [3889, 9721], 0)
    params = product_params(shape)
    N = lib()
    pp, pr, w, op = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    p = params.native()
    assert N.lbg_public_parameters_from_seed(ctypes.byref(p), ptr(np.frombuffer(MATRIX_SEED, np.uint8).copy()),
                                             ctypes.byref(pp)) == LBG_OK
    assert N.lbg_prover_new(pp, ctypes.byref(pr)) == LBG_OK
    assert N.lbg_witness_random(pp, ptr(np.frombuffer(WITNESS_SEED, np.uint8).copy()), ctypes.byref(w)) == LBG_OK
    assert N.lbg_commit(pr, w, None, None, None, ctypes.byref(op)) == LBG_OK
    N.lbg_public_parameters_free(pp)  # the prover still holds the parameters
    N.lbg_witness_free(w)             # the opening still holds the witness
    N.lbg_prover_free(pr)             # the opening still holds the prover
    ch = np.zeros(params.columns(), L.CHALLENGE_DTYPE)
    ch["weight"] = 28
    ch["positions"][:, :28] = (np.arange(28) * 5 + 2).astype(np.uint8)
    v = np.zeros((params.len_ring(), 648), np.int16)
    assert N.lbg_fold(pr, op, ptr(ch), len(ch), ptr(v)) == LBG_OK  # frees the opening, then the prover
    P = O.Params(*shape[:3])
    assert np.array_equal(v, O.fold(P, O.witness_random(P.witness_len, WITNESS_SEED), ch))


def test_fold_of_a_wide_prover_matches_oracle():
    """A prover of 8192 columns (more than the fold's per-column operands are kept for) folds through
    the kernel that weights each column's transform on the CUDA cores; a 512-column prover through
    the operand-folded kernel, with column splits capped at 512. Both equal the oracle's fold."""
    import labinius_b200 as L
    import oracle as O
    from rounds import MATRIX_SEED, WITNESS_SEED, product_params

    for shape in [(20, 13, [3889], 0), (16, 9, [9721, 3889], 0)]:
        params = product_params(shape)
        pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
        prover = L.Prover(pp)
        _, op = prover.commit(L.Witness.random(pp, WITNESS_SEED))
        rng = np.random.default_rng(shape[1])
        ch = L.FoldingChallenges(np.zeros(params.columns(), L.CHALLENGE_DTYPE))
        ch.challenges["weight"] = 28
        for j in range(params.columns()):
            ch.challenges["positions"][j, :28] = np.sort(rng.choice(162, 28, replace=False)).astype(np.uint8)
        ch.challenges["signs"] = rng.integers(0, 2 ** 32, params.columns(), dtype=np.uint64).astype(np.uint32)
        v = prover.fold(op, ch).elements
        P = O.Params(*shape[:3])
        want = O.fold(P, O.witness_random(P.witness_len, WITNESS_SEED), ch.challenges, threads=8)
        assert np.array_equal(v, want), shape
