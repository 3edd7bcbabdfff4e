"""The oracle reproduces the committed golden rounds (CPU), and the B200 path reproduces them
bit for bit through the C ABI (GPU)."""
import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, WITNESS_SEED, fixtures, load, product_round

FIXTURES = fixtures()


def test_fixtures_present():
    assert len(FIXTURES) >= 5


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.split("round_")[-1][:-4])
def test_oracle_reproduces_fixture(oracle, path):
    import blake3

    g = load(path)
    wl, cl, primes, dropped = g["shape"]
    P = oracle.Params(wl, cl, primes, dropped)
    r = oracle.round_trip(P, MATRIX_SEED, WITNESS_SEED, domain=DOMAIN)
    assert blake3.blake3(np.ascontiguousarray(r["A"]).tobytes()).digest() == g["A_digest"].tobytes()
    for k in ["p0", "p1", "u", "mle", "v"]:
        assert np.array_equal(r[k], g[k]), k
    assert np.array_equal(r["challenges"].view(np.uint8).reshape(-1, 40), g["challenges"])
    assert r["transcript_tail"] == g["tail"].tobytes()
    if dropped:
        assert np.array_equal(r["top"], g["top"]) and np.array_equal(r["digits"], g["digits"])
        assert r["packed"] == g["packed"].tobytes()
    else:
        assert np.array_equal(r["C"], g["C"])
        assert np.array_equal(r["folded_commitment"], g["folded_commitment"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.split("round_")[-1][:-4])
def test_gpu_round_matches_fixture(path):
    g = load(path)
    wl, cl, primes, dropped = g["shape"]
    r = product_round(g["shape"])
    key = r["pp"].key()
    assert np.array_equal(key[:, 0, :], g["A_head"])
    c = r["commitment"]
    if dropped:
        assert np.array_equal(c.top, g["top"])
        assert np.array_equal(c.digits, g["digits"])
    else:
        assert np.array_equal(c.matrix, g["C"])
        assert np.array_equal(r["folded_commitment"], g["folded_commitment"])
    for k in ["p0", "p1", "u", "mle", "v"]:
        assert np.array_equal(r[k], g[k]), k
    assert np.array_equal(r["challenges"].view(np.uint8).reshape(-1, 40), g["challenges"])
    assert r["tail"] == g["tail"].tobytes()
