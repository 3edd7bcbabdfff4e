"""The oracle's cross-field switch (crates/pcs/src/switch.rs, crates/pcs/src/fields/crossfield.rs),
pinned by the reference's own relational tests restated: the B128 product against a bit-serial
product written here; the partial evaluations against their bitwise definition
(crates/pcs/src/fields/crossfield.rs:645-660); the claim against the partials' weights
(crates/pcs/src/switch.rs:116-122) and against the trace's MLE by definition; and the switch's
round trip and rejections (crates/pcs/src/switch.rs:205-240): the verifier accepts and returns
the prover's point, the opened value is the lifted witness's MLE there, and a wrong claim or a
tampered opened value is rejected, for word and bit statements. Also the oracle's whole switch
round (crates/pcs/examples/two_fields.rs:176-221) verifies."""
import numpy as np
import pytest

MOD128 = (1 << 128) | 0x87


def b128_mul_ref(a: int, b: int) -> int:
    r = 0
    for i in range(128):
        if (b >> i) & 1:
            r ^= a << i
    for i in range(254, 127, -1):
        if (r >> i) & 1:
            r ^= MOD128 << (i - 128)
    return r


def to_int(x) -> int:
    return int(x[0]) | (int(x[1]) << 64)


def rand_b128(rng, n):
    return rng.integers(0, 2 ** 63, (n, 2), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 2), dtype=np.uint64)


def eq_ref(r):
    """eq_expand_b128 by definition: entry j is the product over k of r_k or 1 + r_k by bit
    l-1-k of j (crates/pcs/src/fields/crossfield.rs:78-98)."""
    l = len(r)
    out = []
    for j in range(1 << l):
        acc = 1
        for k in range(l):
            f = to_int(r[k]) if (j >> (l - 1 - k)) & 1 else to_int(r[k]) ^ 1
            acc = b128_mul_ref(acc, f)
        out.append(acc)
    return out


def test_b128_product_is_the_bit_serial_product(oracle):
    rng = np.random.default_rng(5)
    a, b = rand_b128(rng, 100), rand_b128(rng, 100)
    for x, y in zip(a, b):
        assert to_int(oracle.b128_mul(x, y)) == b128_mul_ref(to_int(x), to_int(y))
    assert to_int(oracle.b128_mul(np.array([2, 0], np.uint64), np.array([0, 1 << 63], np.uint64))) == 0x87


@pytest.mark.parametrize("l", [1, 3, 6])
def test_partials_and_claim_by_definition(oracle, l):
    rng = np.random.default_rng(40 + l)
    trace, r = rand_b128(rng, 1 << l), rand_b128(rng, l)
    eq = eq_ref(r)
    mle = 0
    for j in range(1 << l):
        mle ^= b128_mul_ref(to_int(trace[j]), eq[j])
    claim = oracle.switch_mle(trace, r)
    assert to_int(claim) == mle
    partials, rounds, opened, r_pp = oracle.switch_prove(trace, r, claim, oracle.Transcript(b"t"))
    for k in range(128):
        want = 0
        for j in range(1 << l):
            if (to_int(trace[j]) >> k) & 1:
                want ^= eq[j]
        assert to_int(partials[k]) == want
    # word-level weights: the k-th basis element x^k
    acc = 0
    for k in range(128):
        acc ^= b128_mul_ref(to_int(partials[k]), 1 << k)
    assert acc == mle


@pytest.mark.parametrize("l,cl,bits", [(8, 2, False), (8, 3, True), (11, 4, False)])
def test_switch_round_trip_and_rejection(oracle, l, cl, bits):
    rng = np.random.default_rng(l * 10 + bits)
    trace, r_hi = rand_b128(rng, 1 << l), rand_b128(rng, l)
    r_lo = rand_b128(rng, 7) if bits else None
    claim = oracle.switch_mle(trace, r_hi, r_lo)
    partials, rounds, opened, r_pp = oracle.switch_prove(trace, r_hi, claim, oracle.Transcript(b"t"), r_lo=r_lo)
    ok, r_v = oracle.switch_verify(r_hi, claim, partials, rounds, opened, oracle.Transcript(b"t"), r_lo=r_lo)
    assert ok and np.array_equal(r_v, r_pp)
    witness = np.zeros((1 << l, 3), np.uint64)
    witness[:, :2] = trace
    p0, p1 = r_pp[::-1][: l - cl], r_pp[:cl][::-1]
    assert np.array_equal(oracle.claim(oracle.row_evaluate(witness, p0), p1), opened)
    wrong = claim.copy()
    wrong[0] ^= np.uint64(1)
    assert not oracle.switch_verify(r_hi, wrong, partials, rounds, opened, oracle.Transcript(b"t"), r_lo=r_lo)[0]
    bad = opened.copy()
    bad[0] ^= np.uint64(1)
    assert not oracle.switch_verify(r_hi, claim, partials, rounds, bad, oracle.Transcript(b"t"), r_lo=r_lo)[0]
    if bits:  # a bit statement is not a word statement
        assert not oracle.switch_verify(r_hi, claim, partials, rounds, opened, oracle.Transcript(b"t"))[0]


@pytest.mark.parametrize("dropped", [0, 9])
def test_switch_round_verifies(oracle, dropped):
    """The oracle's ghash-style round: the switch verifies against the same transcript, its point
    is the round's, the opened value equals the claim of the row values, and (Clear) the folded
    opening passes the verifier's checks."""
    wl, cl = 12, 3
    params = oracle.Params(wl, cl, [9721] if not dropped else [9721, 3889], dropped)
    rng = np.random.default_rng(77 + dropped)
    trace, r_hi = rand_b128(rng, 1 << wl), rand_b128(rng, wl)
    seed = bytes([0x5A]) * 32
    out = oracle.switch_round(params, seed, trace, r_hi, domain=b"example/ghash")
    t = oracle.Transcript(b"example/ghash")
    if dropped:
        t.absorb_bytes(oracle.tagged_commitment(params, top=out["top"], digits=out["digits"]))
    else:
        t.absorb_bytes(oracle.tagged_commitment(params, C=out["C"]))
    ok, r_pp = oracle.switch_verify(r_hi, out["claim"], out["partials"], out["rounds"], out["opened"], t)
    assert ok
    assert np.array_equal(r_pp[::-1][: wl - cl], out["p0"]) and np.array_equal(r_pp[:cl][::-1], out["p1"])
    assert np.array_equal(out["mle"], out["opened"])
    ch = oracle.derive_folding_challenges(params, t, out["u"])
    assert np.array_equal(ch, out["challenges"])
    if not dropped:
        folded_row = oracle.fold_binary(out["u"], ch)
        assert oracle.verify_folded_opening(params, out["A"], out["folded_commitment"], out["v"], out["p0"], folded_row)
