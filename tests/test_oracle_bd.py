"""The oracle's bit-dropped opening check (crates/pcs/src/scheme/verifier.rs:232-276,
crates/pcs/src/bd/residual.rs:66-130), pinned by the reference's own properties: an honest round's
residual is within bd::cap (crates/pcs/src/bd/mod.rs:72-80) and of the size its expected value
gives (the rounding errors of the dropped bits folded with the challenges), while a changed folded
witness, dropped commitment or folded row value is rejected."""
import numpy as np
import pytest


@pytest.mark.parametrize("shape", [(12, 4, [9721, 3889], 9), (11, 3, [3889, 2917, 4861], 10), (11, 3, [9721], 8)])
def test_honest_rounds_pass_and_tampered_fail(oracle, shape):
    wl, cl, primes, d = shape
    P = oracle.Params(wl, cl, primes, d)
    out = oracle.round_trip(P, bytes([0x5A]) * 32, witness_seed=bytes([7]) * 32)
    fr = oracle.fold_binary(out["u"], out["challenges"])
    args = (P, out["A"], out["top"], out["digits"], out["challenges"])
    res = oracle.bd_residual(*args, out["v"])
    cap = oracle.bd_cap(P)
    expected = cap / 4.0  # bd::expected_normsq: BD_CAP = 4 times it
    assert 0.5 * expected < res <= cap
    assert oracle.verify_folded_opening_bd(*args, out["v"], out["p0"], fr)
    v = out["v"].copy()
    v[0, 0] += 1
    assert not oracle.verify_folded_opening_bd(*args, v, out["p0"], fr)
    top = ((out["top"].astype(np.int64) + 3) % 8).astype(np.uint16)
    assert not oracle.verify_folded_opening_bd(P, out["A"], top, out["digits"], out["challenges"], out["v"],
                                               out["p0"], fr)
    fr2 = fr.copy()
    fr2[1] ^= np.uint64(1)
    assert not oracle.verify_folded_opening_bd(*args, out["v"], out["p0"], fr2)
