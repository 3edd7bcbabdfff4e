"""Bit-exact parity at the sizes the bench measures, against the oracle.

The rounds are the reference's bench round (crates/bench/src/bin/labinius.rs:104-130) at the
configurations of crates/pcs/src/scheme/params.rs:91-128 and 207-210:

* Params::basic() (2^18, moduli [3889, 9721]) and suite s (2^18; Clear [9721, 12637], bit-dropped
  [3889, 2917, 4861] with 10 bits): the whole round against the oracle;
* suite m (2^20, [3889, 2917, 4861]; Clear and 9 dropped bits) and suite l (2^22, 512 columns, the
  headline configuration; Clear and 8 dropped bits): the whole round, every column and every ring
  element, against the oracle on all host threads;
* suite xl (2^24, 1024 columns): a sample of columns of the commitment and of ring elements of the
  folded witness, everything else of the round in full.

Compared: the key, the witness, the commitment matrix (or top bits and digits), the evaluation
point, the row values, the mle claim, the challenges, the folded witness, the folded commitment
(Clear) and the transcript after the round."""
import functools
import os

import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, WITNESS_SEED, product_round

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)


@functools.lru_cache(maxsize=2)
def oracle_commitment(wl, cl, primes):
    """The oracle's key, witness and commitment matrix of a shape (shared by its Clear and
    bit-dropped rounds, which commit to the same moduli)."""
    import oracle as O

    P = O.Params(wl, cl, list(primes), 0)
    A = O.key_expand(P, O.key_seed(MATRIX_SEED))
    w = O.witness_random(P.witness_len, WITNESS_SEED)
    C = O.commit(P, A, w, threads=THREADS)
    return A, w, C


def oracle_round(O, shape):
    """crates/bench/src/bin/labinius.rs:104-130 on the oracle, the commitment from the cache."""
    wl, cl, primes, dropped = shape
    P = O.Params(wl, cl, primes, dropped)
    A, w, C = oracle_commitment(wl, cl, tuple(primes))
    out = dict(A=A, witness=w, C=C)
    t = O.Transcript(DOMAIN)
    if dropped:
        top, digits = O.drop_bits(P, C)
        out.update(top=top, digits=digits)
        p0, p1 = O.derive_evaluation_point(P, MATRIX_SEED, t, top=top, digits=digits)
    else:
        p0, p1 = O.derive_evaluation_point(P, MATRIX_SEED, t, C=C)
    u = O.row_evaluate(w, p0)
    ch = O.derive_folding_challenges(P, t, u)
    out.update(p0=p0, p1=p1, u=u, mle=O.claim(u, p1), challenges=ch, v=O.fold(P, w, ch, threads=THREADS))
    if not dropped:
        out["folded_commitment"] = O.fold_commitment(P, C, ch)
    out["tail"] = t.fill(b"labinius/test-tail", 32)
    return out


def check_round(got, want, dropped):
    assert np.array_equal(got["pp"].key(), want["A"]), "key"
    assert np.array_equal(got["witness"].elements(), want["witness"]), "witness"
    if dropped:
        assert np.array_equal(got["commitment"].top, want["top"]), "top bits"
        assert np.array_equal(got["commitment"].digits, want["digits"]), "digits"
    else:
        assert np.array_equal(got["commitment"].matrix, want["C"]), "commitment"
    for k in ["p0", "p1", "u", "mle", "v"]:
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got["challenges"].view(np.uint8), want["challenges"].view(np.uint8)), "challenges"
    if not dropped:
        assert np.array_equal(got["folded_commitment"], want["folded_commitment"]), "folded commitment"
    assert got["tail"] == want["tail"], "transcript"


FULL = [
    ((18, 7, [3889, 9721], 0), "basic"),
    ((18, 7, [9721, 12637], 0), "s-clear"),
    ((18, 7, [3889, 2917, 4861], 10), "s-bd10"),
    ((20, 8, [3889, 2917, 4861], 0), "m-clear"),
    ((20, 8, [3889, 2917, 4861], 9), "m-bd9"),
    ((22, 9, [3889, 2917, 4861], 0), "l-clear"),
    ((22, 9, [3889, 2917, 4861], 8), "l-bd8"),
]


@pytest.mark.parametrize("shape", [s for s, _ in FULL], ids=[i for _, i in FULL])
def test_full_round_at_bench_size(oracle, shape):
    got = product_round(shape)
    want = oracle_round(oracle, shape)
    check_round(got, want, shape[3])


def column_ranges(cols):
    """Columns compared at xl: the first and last 16 and 16 from the middle."""
    return [(0, 16), (cols // 2 - 8, cols // 2 + 8), (cols - 16, cols)]


def ring_ranges(len_ring):
    """Ring elements of the folded witness compared at xl: both ends and the middle, 96 in all."""
    return [(0, 32), (len_ring // 2 - 16, len_ring // 2 + 16), (len_ring - 32, len_ring)]


@pytest.mark.parametrize("shape", [(24, 10, [3889, 2917, 9721], 0), (24, 10, [3889, 2917, 4861], 7)],
                         ids=["xl-clear", "xl-bd7"])
def test_xl_round_sampled(oracle, shape):
    O = oracle
    wl, cl, primes, dropped = shape
    P = O.Params(wl, cl, primes, dropped)
    got = product_round(shape)
    A = O.key_expand(P, O.key_seed(MATRIX_SEED))
    assert np.array_equal(got["pp"].key(), A), "key"
    w = O.witness_random(P.witness_len, WITNESS_SEED)
    assert np.array_equal(got["witness"].elements(), w), "witness"
    C = np.zeros((P.columns, 4, P.limbs, 162), np.int16)
    for c0, c1 in column_ranges(P.columns):
        part = O.commit(P, A, w, c0, c1, threads=THREADS)
        C[c0:c1] = part[c0:c1]
    t = O.Transcript(DOMAIN)
    if dropped:
        # drop_bits works column by column: the sampled columns' top bits and digits from the
        # oracle's commitment; the transcript from the device's (checked on those columns)
        top, digits = O.drop_bits(P, C)
        gt, gd = got["commitment"].top.reshape(P.columns, -1), got["commitment"].digits.reshape(P.limbs - 1, P.columns, -1)
        top, digits = top.reshape(P.columns, -1), digits.reshape(P.limbs - 1, P.columns, -1)
        for c0, c1 in column_ranges(P.columns):
            assert np.array_equal(gt[c0:c1], top[c0:c1]), f"top bits {c0}..{c1}"
            assert np.array_equal(gd[:, c0:c1], digits[:, c0:c1]), f"digits {c0}..{c1}"
        p0, p1 = O.derive_evaluation_point(P, MATRIX_SEED, t, top=got["commitment"].top, digits=got["commitment"].digits)
    else:
        for c0, c1 in column_ranges(P.columns):
            assert np.array_equal(got["commitment"].matrix[c0:c1], C[c0:c1]), f"commitment {c0}..{c1}"
        p0, p1 = O.derive_evaluation_point(P, MATRIX_SEED, t, C=got["commitment"].matrix)
    assert np.array_equal(got["p0"], p0) and np.array_equal(got["p1"], p1), "point"
    u = O.row_evaluate(w, p0)
    assert np.array_equal(got["u"], u), "row values"
    assert np.array_equal(got["mle"], O.claim(u, p1)), "mle"
    ch = O.derive_folding_challenges(P, t, u)
    assert np.array_equal(got["challenges"].view(np.uint8), ch.view(np.uint8)), "challenges"
    for i0, i1 in ring_ranges(P.len_ring):
        v = O.fold(P, w, ch, i0, i1, threads=THREADS)
        assert np.array_equal(got["v"][i0:i1], v[i0:i1]), f"folded witness {i0}..{i1}"
    if not dropped:
        assert np.array_equal(got["folded_commitment"], O.fold_commitment(P, got["commitment"].matrix, ch))
    assert got["tail"] == t.fill(b"labinius/test-tail", 32), "transcript"
