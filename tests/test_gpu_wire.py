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


# ---------------------------------------------------------------------------------------------
# the bit-packed commitment and row evaluation, from device memory (crates/pcs/src/wire/mod.rs:
# 226-245, 386-397, 435-459)
# ---------------------------------------------------------------------------------------------
@pytest.mark.parametrize("shape", [(12, 3, [3889], 0), (12, 4, [3889, 2917, 4861], 0), (11, 2, [19441, 12637], 0),
                                   (13, 5, [17497, 2917, 9721], 0), (12, 4, [3889, 2917, 4861], 9),
                                   (11, 3, [2917], 8), (22, 9, [3889, 2917, 4861], 0)],
                         ids=["1limb", "3limbs", "large", "mixed", "bd9", "bd-1limb", "suite-l"])
def test_pack_commitment_from_the_device_equals_the_oracle(oracle, shape):
    import labinius_b200 as L
    from labinius_b200 import wire
    from rounds import MATRIX_SEED, WITNESS_SEED, product_params

    wl, cl, primes, dropped = shape
    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    prover = L.Prover(pp)
    c, op = prover.commit(w)
    got = wire.pack_commitment(op)
    P = oracle.Params(wl, cl, primes, dropped)
    if dropped:
        assert got == oracle.pack_dropped(P, c.top, c.digits)
    else:
        assert got == oracle.pack_commitment(P, c.matrix)
        st, back = oracle.unpack_commitment(P, got)
        assert st == 0 and np.array_equal(back, c.matrix)
    prover.recycle(op)


@pytest.mark.parametrize("shape", [(12, 3, [3889], 0), (14, 7, [9721], 0), (22, 9, [3889, 2917, 4861], 0)],
                         ids=["8cols", "128cols", "suite-l"])
def test_pack_row_evaluation_from_the_device_equals_the_oracle(oracle, shape):
    import labinius_b200 as L
    from labinius_b200 import EvaluationPoint, wire
    from rounds import MATRIX_SEED, WITNESS_SEED, product_params

    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    rng = np.random.default_rng(3)
    p0 = rng.integers(0, 2 ** 63, (params.row_log_len(), 3), dtype=np.uint64)
    p0[:, 2] &= np.uint64((1 << 34) - 1)
    p1 = rng.integers(0, 2 ** 63, (params.column_log_len, 3), dtype=np.uint64)
    p1[:, 2] &= np.uint64((1 << 34) - 1)
    pt = EvaluationPoint(p0, p1)
    row, got = wire.row_evaluate_packed(w, pt)
    assert np.array_equal(row.values, w.row_evaluate(pt).values)
    assert got == oracle.pack_f162(row.values)
    st, back = oracle.unpack_f162(got, params.columns())
    assert st == 0 and np.array_equal(back, row.values)
