"""The library's host side (BLAKE3 transcript, short-challenge sampler, evaluation-point and
challenge derivation, pack_dropped) against the oracle and the golden rounds. CPU only: these
entry points never touch the device."""
import ctypes

import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, fixtures, load

CH = np.dtype([("positions", np.uint8, 32), ("signs", np.uint32), ("weight", np.uint32)])


def test_transcript_fill_matches_oracle(oracle):
    from labinius_b200 import Transcript

    for n in [0, 1, 100, 5000]:
        a, b = Transcript(b"labinius/test"), oracle.Transcript(b"labinius/test")
        blob = bytes((i * 13) & 255 for i in range(n))
        for t in (a, b):
            t.absorb_bytes(blob)
            t.absorb_u64(0xDEADBEEF12345678)
        assert a.fill(b"x", 77) == b.fill(b"x", 77)
        assert a.fill(b"x", 300) == b.fill(b"x", 300)  # the counter advanced alike
        c = a.clone()
        assert c.fill(b"y", 64) == a.fill(b"y", 64)


def test_sampler_matches_oracle(oracle):
    from labinius_b200 import Transcript, sample_short_challenge

    total = 0
    for i in range(150):
        a, b = Transcript(b"labinius/stats"), oracle.Transcript(b"labinius/stats")
        a.absorb_u64(i)
        b.absorb_u64(i)
        ca, na = sample_short_challenge(a)
        cb, nb = oracle.sample_short_challenge(b)
        assert na == nb
        assert ca.tobytes() == cb.tobytes()
        assert ca["weight"] == 28 and list(ca["positions"][:28]) == sorted(ca["positions"][:28])
        total += na
    assert 1.0 <= total / 150 < 50


def _params(native, shape):
    wl, cl, primes, dropped = shape
    p = native.lbg_params()
    p.witness_log_len, p.column_log_len, p.n_moduli = wl, cl, len(primes)
    for i, q in enumerate(primes):
        p.moduli[i] = q
    p.opening, p.dropped_bits = (1, dropped) if dropped else (0, 0)
    return p


@pytest.mark.parametrize("path", fixtures(), ids=lambda p: p.split("round_")[-1][:-4])
def test_point_and_challenges_match_fixture(native, path):
    g = load(path)
    wl, cl, primes, dropped = g["shape"]
    L = native.lib()
    p = _params(native, g["shape"])
    d = np.frombuffer(DOMAIN, np.uint8).copy()
    t = L.lbg_transcript_new(native.ptr(d), len(DOMAIN))
    seed = np.frombuffer(MATRIX_SEED, np.uint8).copy()
    p0 = np.zeros((wl - cl, 3), np.uint64)
    p1 = np.zeros((cl, 3), np.uint64)
    if dropped:
        top = np.ascontiguousarray(g["top"])
        dig = np.ascontiguousarray(g["digits"])
        native.check(L.lbg_params_derive_evaluation_point(ctypes.byref(p), native.ptr(seed), t, None, native.ptr(top),
                                                          native.ptr(dig), native.ptr(p0), native.ptr(p1)))
        n = L.lbg_params_pack_dropped(ctypes.byref(p), native.ptr(top), native.ptr(dig), None, 0)
        buf = np.zeros(n, np.uint8)
        L.lbg_params_pack_dropped(ctypes.byref(p), native.ptr(top), native.ptr(dig), native.ptr(buf), n)
        assert buf.tobytes() == g["packed"].tobytes()
    else:
        C = np.ascontiguousarray(g["C"])
        native.check(L.lbg_params_derive_evaluation_point(ctypes.byref(p), native.ptr(seed), t, native.ptr(C), None,
                                                          None, native.ptr(p0), native.ptr(p1)))
    assert np.array_equal(p0, g["p0"]) and np.array_equal(p1, g["p1"])
    ch = np.zeros(1 << cl, CH)
    native.check(L.lbg_params_derive_folding_challenges(ctypes.byref(p), t, native.ptr(np.ascontiguousarray(g["u"])),
                                                        native.ptr(ch)))
    assert ch.view(np.uint8).reshape(-1, 40).tobytes() == g["challenges"].tobytes()
    out = np.zeros(32, np.uint8)
    L.lbg_transcript_fill(t, b"labinius/test-tail", native.ptr(out), 32)
    assert out.tobytes() == g["tail"].tobytes()
    L.lbg_transcript_free(t)
