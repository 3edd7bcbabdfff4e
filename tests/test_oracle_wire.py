"""The oracle's wire coder for the folded witness (crates/pcs/src/wire/rans.rs), pinned by the
reference's own tests restated (crates/pcs/tests/wire.rs:173-395): honest folds round-trip under
every base modulus and beat two bytes a coefficient; the degenerate and adversarial messages
(empty, constant, the bounds, alternating, a ramp, uniform over the centred range so that the
escape symbol is used) and any i16 round-trip; the coded size stays within the zeroth-order
entropy bound at every element count; a truncated, lengthened or corrupted stream is refused."""
import math

import numpy as np
import pytest

M64 = (1 << 64) - 1
BASES = [2917, 3889, 4861, 9721, 12637, 17497, 19441]


def xorshift(state):
    state ^= (state << 13) & M64
    state ^= state >> 7
    state ^= (state << 17) & M64
    return state


def entropy_bytes(v):
    _, counts = np.unique(np.asarray(v).ravel(), return_counts=True)
    total = counts.sum()
    p = counts / total
    return float(-(counts * np.log2(p)).sum() / 8.0)


def round_trips(oracle, v, q=3889):
    data = oracle.wire_encode(v, q)
    st, back = oracle.wire_decode(data)
    assert st == 0
    assert np.array_equal(back, np.asarray(v, np.int16).reshape(-1, 648))
    return data


@pytest.mark.parametrize("base", BASES)
def test_an_honest_fold_round_trips(oracle, base):
    second = BASES[(BASES.index(base) + 1) % len(BASES)]
    for wl, cl in [(11, 3), (12, 2)]:
        P = oracle.Params(wl, cl, [base, second], 0)
        out = oracle.round_trip(P, bytes([0x5A]) * 32, witness_seed=bytes([base & 0xFF]) * 32)
        data = round_trips(oracle, out["v"], base)
        assert len(data) < out["v"].size * 2


def test_an_adversarial_fold_round_trips(oracle):
    assert len(oracle.wire_encode(np.zeros((0, 648), np.int16), 3889)) == 16
    st, back = oracle.wire_decode(oracle.wire_encode(np.zeros((0, 648), np.int16), 3889))
    assert st == 0 and back.size == 0
    for q in BASES:
        half = (q - 1) // 2
        cases = [
            [[0] * 648],
            [[half] * 648],
            [[-half] * 648],
            [[half if i % 2 == 0 else -half for i in range(648)]],
            [[(i % (2 * half + 1)) - half for i in range(648)], [half] * 648, [-half] * 648],
        ]
        state = 0x2545F4914F6CDD1D
        uniform = []
        for _ in range(16):
            row = []
            for _ in range(648):
                state = xorshift(state)
                row.append(state % (2 * half + 1) - half)
            uniform.append(row)
        cases.append(uniform)
        for v in cases:
            round_trips(oracle, np.array(v, np.int16), q)


def test_the_coder_takes_any_i16(oracle):
    state = 0x9E3779B97F4A7C15
    v = np.zeros((8, 648), np.int16)
    for e in range(8):
        for i in range(648):
            state = (state * 6364136223846793005 + 1) & M64
            v[e, i] = np.int64(state >> 32).astype(np.int32).astype(np.int16)
    v[0, 0], v[0, 1] = -32768, 32767
    round_trips(oracle, v)


def test_an_interleaved_fold_round_trips_at_every_length(oracle):
    state = 0x123456789ABCDEF1
    for count in [1, 2, 3, 5, 7, 8]:
        v = np.zeros((count, 648), np.int16)
        for e in range(count):
            for i in range(648):
                state = (state * 6364136223846793005 + 1442695040888963407) & M64
                v[e, i] = sum((state >> (10 * k)) & 0x3F for k in range(6)) - 189
        data = round_trips(oracle, v)
        assert len(data) <= entropy_bytes(v) * 1.02 + 4.0 * 64 + 200.0


def test_a_broken_stream_is_refused(oracle):
    P = oracle.Params(11, 3, [3889, 9721], 0)
    out = oracle.round_trip(P, bytes([0x5A]) * 32, witness_seed=bytes([3]) * 32)
    data = oracle.wire_encode(out["v"], 3889)
    for cut in [0, 1, 15, 16, 20, len(data) // 2, len(data) - 1]:
        assert oracle.wire_decode(data[:cut])[0] != 0, cut
    assert oracle.wire_decode(data + b"\x00\x00")[0] == 2
    assert oracle.wire_decode(b"\x02" + data[1:])[0] == 2


def test_a_stream_short_or_long_by_one_word_on_any_lane_is_refused(oracle):
    """Per lane k: a message whose only expensive symbols sit in lane k (every other coefficient
    0), so that lane alone renormalises; one word fewer or one more is refused."""
    for k in [0, 1, 31, 63]:
        v = np.zeros((2, 648), np.int16)
        flat = v.ravel()
        flat[k::64][:8] = [1000, -1000, 900, -900, 800, -800, 700, -700]
        data = round_trips(oracle, v)
        assert oracle.wire_decode(data[:-2])[0] != 0
        assert oracle.wire_decode(data + b"\x00\x00")[0] != 0


# ---------------------------------------------------------------------------------------------
# the bit-packed commitment and row evaluation (crates/pcs/src/wire/mod.rs:85-140, 226-300, 435-470)
# ---------------------------------------------------------------------------------------------
class _BitWriter:
    """crates/pcs/src/wire/mod.rs:85-139, restated literally (accumulator, bit count, bytes)."""

    def __init__(self):
        self.bytes, self.acc, self.n = bytearray(), 0, 0

    def put(self, value, bits):
        self.acc |= (value & ((1 << bits) - 1)) << self.n
        self.n += bits
        while self.n >= 8:
            self.bytes.append(self.acc & 0xFF)
            self.acc >>= 8
            self.n -= 8

    def finish(self):
        if self.n > 0:
            self.bytes.append(self.acc & 0xFF)
        return bytes(self.bytes)


def _small_commitment(oracle, primes, cl=2, wl=10):
    P = oracle.Params(wl, cl, primes, 0)
    A = oracle.key_expand(P, oracle.key_seed(bytes([0x5A]) * 32))
    w = oracle.witness_random(P.witness_len, bytes([0xC7]) * 32)
    return P, oracle.commit(P, A, w), w


@pytest.mark.parametrize("primes", [[3889], [3889, 2917, 4861], [19441, 2917], [12637, 9721, 17497]])
def test_pack_commitment_is_the_reference_bit_writer(oracle, primes):
    P, C, _ = _small_commitment(oracle, primes)
    w = _BitWriter()
    for elem in C.reshape(-1, P.limbs, 162):
        for k, q in enumerate(primes):
            for slot in elem[k]:
                w.put(int(slot) % q, oracle.residue_bits(q))
    want = w.finish()
    got = oracle.pack_commitment(P, C)
    assert got == want
    # the size of crates/pcs/src/wire/mod.rs:381-384
    assert len(got) == (4 * P.columns * 162 * sum(oracle.residue_bits(q) for q in primes) + 7) // 8
    st, back = oracle.unpack_commitment(P, got)
    assert st == 0 and np.array_equal(back, C)


def test_unpack_commitment_refuses_what_the_reference_refuses(oracle):
    P, C, _ = _small_commitment(oracle, [3889, 2917])
    b = oracle.pack_commitment(P, C)
    assert oracle.unpack_commitment(P, b[:-1])[0] == 2
    assert oracle.unpack_commitment(P, b + b"\0")[0] == 2
    # a residue equal to q is malformed (crates/pcs/src/wire/mod.rs:282-284): the first slot's 12 bits
    bad = bytearray(b)
    v = 3889
    bad[0] = v & 0xFF
    bad[1] = (bad[1] & 0xF0) | (v >> 8)
    assert oracle.unpack_commitment(P, bytes(bad))[0] == 2


def test_pack_f162_is_the_reference_bit_writer(oracle):
    rng = np.random.default_rng(11)
    for count in [1, 2, 3, 7, 8, 64, 129]:
        u = rng.integers(0, 2 ** 63, (count, 3), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (count, 3),
                                                                                              dtype=np.uint64)
        u[:, 2] &= np.uint64((1 << 34) - 1)
        w = _BitWriter()
        for x in u:
            w.put(int(x[0]) & 0xFFFFFFFF, 32)
            w.put(int(x[0]) >> 32, 32)
            w.put(int(x[1]) & 0xFFFFFFFF, 32)
            w.put(int(x[1]) >> 32, 32)
            w.put(int(x[2]) & 0xFFFFFFFF, 32)
            w.put(int(x[2]) >> 32, 2)
        got = oracle.pack_f162(u)
        assert got == w.finish()
        assert len(got) == (162 * count + 7) // 8
        st, back = oracle.unpack_f162(got, count)
        assert st == 0 and np.array_equal(back, u)
        assert oracle.unpack_f162(got[:-1], count)[0] == 2
