"""wire::encode of the folded witness on the device (crates/pcs/src/wire/rans.rs:18-105): the
bytes equal the oracle's restatement on honest folds under every base modulus (from host memory
and from where Prover::fold left the fold), and on the reference's degenerate and adversarial
messages (crates/pcs/tests/wire.rs:205-345: empty, constant, the bounds, alternating, a ramp,
uniform over the centred range so that the escape symbol is used, any i16, every tail length);
the oracle decodes them back."""
import numpy as np
import pytest

from rounds import product_round
from test_oracle_wire import BASES, M64, xorshift

pytestmark = pytest.mark.gpu


def same(oracle, v, q=3889):
    from labinius_b200 import wire

    got = wire.encode(np.asarray(v, np.int16).reshape(-1, 648), q)
    assert got == oracle.wire_encode(v, q)
    st, back = oracle.wire_decode(got)
    assert st == 0 and np.array_equal(back, np.asarray(v, np.int16).reshape(-1, 648))
    return got


@pytest.mark.parametrize("base", [3889, 2917, 19441])
def test_honest_folds_encode_as_the_oracle(oracle, base):
    import labinius_b200 as L
    from labinius_b200 import wire

    second = BASES[(BASES.index(base) + 1) % len(BASES)]
    r = product_round((12, 3, [base, second], 0))
    same(oracle, r["v"], base)
    prover = L.Prover(r["pp"])
    c, op = prover.commit(r["witness"])
    prover.fold(op, L.FoldingChallenges(r["challenges"]))
    assert wire.encode_folded(prover) == oracle.wire_encode(r["v"], base)


def test_adversarial_messages_encode_as_the_oracle(oracle):
    same(oracle, np.zeros((0, 648), np.int16))
    for q in BASES:
        half = (q - 1) // 2
        cases = [[[0] * 648], [[half] * 648], [[-half] * 648],
                 [[half if i % 2 == 0 else -half for i in range(648)]],
                 [[(i % (2 * half + 1)) - half for i in range(648)], [half] * 648, [-half] * 648]]
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
            same(oracle, np.array(v, np.int16), q)


def test_any_i16_and_every_tail_length_encode_as_the_oracle(oracle):
    state = 0x9E3779B97F4A7C15
    v = np.zeros((8, 648), np.int16)
    for e in range(8):
        for i in range(648):
            state = (state * 6364136223846793005 + 1) & M64
            v[e, i] = np.int64(state >> 32).astype(np.int32).astype(np.int16)
    v[0, 0], v[0, 1] = -32768, 32767
    same(oracle, v)
    state = 0x123456789ABCDEF1
    for count in [1, 2, 3, 5, 7, 8, 300]:
        v = np.zeros((count, 648), np.int16)
        for e in range(count):
            for i in range(648):
                state = (state * 6364136223846793005 + 1442695040888963407) & M64
                v[e, i] = sum((state >> (10 * k)) & 0x3F for k in range(6)) - 189
        same(oracle, v)
