"""The oracle's restatement of the recursive opening's device half: the residues a recursive commitment
opens (crates/pcs/src/recursion/limbs.rs:379-398) and the left expansion's vector
(crates/pcs/src/scheme/prover.rs:95-115), pinned by the reference's own relational test
(crates/pcs/tests/recursion.rs:134-174: the residues re-transform to the commitment's columns)."""
import numpy as np
import pytest

import oracle as O
from rounds import MATRIX_SEED, WITNESS_SEED


@pytest.mark.parametrize("primes", [[3889, 9721], [3889, 2917, 9721]], ids=["split", "quadratic"])
def test_residues_re_transform_to_the_commitment(primes):
    # crates/pcs/tests/recursion.rs:137-174: Params::new(9, 2, [Q9721]) and Params::new(15, 6, [Q2917, Q9721])
    wl, cl = (9, 2) if len(primes) == 2 else (15, 6)
    P = O.Params(wl, cl, primes)
    A = O.key_expand(P, O.key_seed(MATRIX_SEED))
    C = O.commit(P, A, O.witness_random(P.witness_len, WITNESS_SEED))
    res = O.recursion_residues(P, C)
    r = P.columns
    assert res.shape == (len(primes) * 4, O.recursion_polys(r), 64)
    for limb, q in enumerate(primes):
        for j in range(r):
            a = np.zeros(648, np.int64)
            for m in range(4):
                # chunk::decode: chunk b's positions 0..53 are coefficients 54 b ..
                e = np.concatenate([res[limb * 4 + m, b * r + j, :54] for b in range(3)]).astype(np.int64)
                t = np.arange(162)
                a[4 * t + m] = np.where(t % 2 == 0, e, -e)
            back = O.components(q, O.ntt(q, np.mod(a, q)))
            for m in range(4):
                assert np.array_equal(back[m], C[j, m, limb]), (q, j, m)
    # positions 54..63 and the padding polynomials are zero; coefficients are centred
    assert not res[:, :, 54:].any() and not res[:, 3 * r:].any()
    for limb, q in enumerate(primes):
        assert np.abs(res[limb * 4:(limb + 1) * 4]).max() <= (q - 1) // 2


def test_left_expansion_chunks_the_lift():
    rng = np.random.default_rng(3)
    r = 40
    u = rng.integers(0, 2 ** 63, (r, 3), dtype=np.uint64)
    u[:, 2] &= np.uint64((1 << 34) - 1)
    out = O.left_expansion(u)
    assert out.shape == (O.recursion_polys(r), 64)
    for j in range(r):
        bits = np.concatenate([out[b * r + j, :54] for b in range(3)])
        want = [(int(u[j, p >> 6]) >> (p & 63)) & 1 for p in range(162)]
        assert list(bits) == want
    assert not out[:, 54:].any() and not out[3 * r:].any()
