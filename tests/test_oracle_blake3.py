"""The oracle's BLAKE3 against the Python `blake3` package (hash, keyed, derive-key, XOF seek)."""
import blake3
import pytest


@pytest.mark.parametrize("n", [0, 1, 63, 64, 65, 1023, 1024, 1025, 2047, 2048, 2049, 4096, 5000, 17000])
def test_modes(oracle, n):
    d = bytes((i * 7 + 3) & 255 for i in range(n))
    assert oracle.blake3(d, 100) == blake3.blake3(d).digest(length=100)
    key = bytes(range(32))
    assert oracle.blake3(d, 70, seek=131, key=key) == blake3.blake3(d, key=key).digest(length=70, seek=131)
    ctx = "labinius 2026 challenge signs v1"
    assert oracle.blake3(d, 40, context=ctx.encode()) == blake3.blake3(d, derive_key_context=ctx).digest(length=40)


def test_key_seed(oracle):
    seed = bytes([0x5A]) * 32
    d = blake3.blake3(seed).digest()
    assert oracle.key_seed(seed) == int.from_bytes(d[:8], "little")


def test_witness_random_matches_keyed_xof(oracle):
    seed = bytes([0xC7]) * 32
    w = oracle.witness_random(1000, seed)
    raw = blake3.blake3(b"labinius/witness", key=seed).digest(length=24 * 1000)
    import numpy as np

    want = np.frombuffer(raw, dtype=np.uint64).reshape(-1, 3).copy()
    want[:, 2] &= (1 << 34) - 1
    assert (w == want).all()
