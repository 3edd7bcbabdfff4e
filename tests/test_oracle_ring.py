"""The oracle's ring arithmetic against the definitions the reference's own tests use:
crates/pcs/tests/ntt.rs (scalar_matches_definition, decomposition_matches_the_definition,
product identities), crates/pcs/tests/scalar_reference.rs and crates/pcs/tests/fields.rs."""
import numpy as np
import pytest

PRIMES = [2917, 3889, 4861, 9721, 12637, 17497, 19441]
QUAD = {2917, 4861, 12637}


def component_eval(q, theta, y, k, v):
    """y_k(theta^v) by Horner: component k is sum_m y[4m+k] Y^m."""
    th = pow(theta, v, q)
    acc = 0
    for m in range(161, -1, -1):
        acc = (acc * th + int(y[4 * m + k])) % q
    return acc


def adversarial():
    """crates/pcs/tests/common/mod.rs:49-81"""
    v = [np.zeros(648, np.uint32), np.ones(648, np.uint32)]
    for phase in range(2):
        v.append(np.array([(i % 2 == phase) for i in range(648)], np.uint32))
        v.append(np.array([(i % 3 == phase) for i in range(648)], np.uint32))
    for b in range(4):
        p = np.zeros(648, np.uint32)
        p[162 * b:162 * (b + 1)] = 1
        v.append(p)
    for d in [0, 1, 53, 54, 80, 81, 107, 108, 161, 162, 163, 323, 324, 325, 485, 486, 646, 647]:
        p = np.zeros(648, np.uint32)
        p[d] = 1
        v.append(p)
    return v


def test_slot_tables(oracle):
    """crates/pcs/tests/scalar_reference.rs:18-40, crates/pcs/tests/ntt.rs:1830-1860."""
    T = oracle.slot_tables()
    se = T["slot_exp"]
    assert sorted(int(u) for u in se) == [u for u in range(1944) if u % 2 and u % 3]
    qse = T["quad_slot_exp"]
    assert sorted(int(u) for u in qse) == [u for u in range(972) if u % 2 and u % 3]
    pow3 = [int(v) for v in T["pow3_slot_exp"]]
    assert sorted(pow3) == [v for v in range(486) if v % 2 and v % 3]
    for s in range(162):
        jp, jm = T["quad_class_slot"][:, s]
        assert qse[jp] == pow3[s] and qse[jm] == pow3[s] + 486
        for t in range(4):
            assert se[T["slot_648"][t, s]] == pow3[s] + 486 * t


@pytest.mark.parametrize("q", PRIMES)
def test_ntt_is_evaluation(oracle, q):
    T = oracle.slot_tables()
    rng = np.random.default_rng(q)
    for a in [rng.integers(0, q, 648).astype(np.uint32)] + adversarial()[:6]:
        y = oracle.ntt(q, a)
        if q in QUAD:
            for j in range(0, 324, 7):
                assert (int(y[2 * j]), int(y[2 * j + 1])) == oracle.eval_quad_at(q, a, int(T["quad_slot_exp"][j]))
        else:
            for j in range(0, 648, 11):
                assert int(y[j]) == oracle.eval_at(q, a, int(T["slot_exp"][j]))
        assert (oracle.intt(q, y) == a % q).all()


@pytest.mark.parametrize("q", PRIMES)
def test_decomposition_is_the_definition(oracle, q):
    info = oracle.prime_info(q)
    T = oracle.slot_tables()
    rng = np.random.default_rng(23 + q)
    a = rng.integers(0, q, 648).astype(np.uint32)
    comp = oracle.components(q, oracle.ntt(q, a))
    for k in range(4):
        for s in range(0, 162, 5):
            want = component_eval(q, info["theta"], a, k, int(T["pow3_slot_exp"][s]))
            assert int(comp[k, s]) % q == want
    # recombination is the exact inverse
    assert (oracle.recombine(q, comp) == oracle.ntt(q, a)).all()


def test_f162_product(oracle):
    """crates/pcs/tests/fields.rs:113-150: the reference's product equals the bit-serial one and x
    has order 243."""
    rng = np.random.default_rng(22)
    for _ in range(300):
        a = rng.integers(0, 2 ** 63, 3, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, 3, dtype=np.uint64)
        b = rng.integers(0, 2 ** 63, 3, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, 3, dtype=np.uint64)
        a[2] &= np.uint64((1 << 34) - 1)
        b[2] &= np.uint64((1 << 34) - 1)
        assert (oracle.f162_mul(a, b) == oracle.f162_mul(a, b, serial=True)).all()
    x = np.array([2, 0, 0], np.uint64)
    acc = np.array([1, 0, 0], np.uint64)
    hits = []
    for k in range(1, 244):
        acc = oracle.f162_mul(acc, x)
        if (acc == [1, 0, 0]).all():
            hits.append(k)
    assert hits == [243]
