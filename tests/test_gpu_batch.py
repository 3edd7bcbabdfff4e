"""Batched rounds: every instance's commitment, row values, claim and folded witness equal the
same instance run alone through the single-instance path (and hence the oracle), with and
without CUDA graphs and after autotuning; uneven sizes, bit-dropped mode, and the full round
(transcripts per instance) against the single-instance round."""
import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, product_params, product_round

pytestmark = pytest.mark.gpu


def seeds(count):
    return [bytes([(0x10 + i) & 0xFF]) * 32 for i in range(count)]


def make(row_log, primes, dropped, col_logs):
    import labinius_b200 as L
    from labinius_b200.batch import Batch

    params = product_params((row_log + col_logs[0], col_logs[0], primes, dropped))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    b = Batch(pp, col_logs)
    b.witness_random(seeds(len(col_logs)))
    return L, pp, b


@pytest.mark.parametrize("graphs,keep,transcript", [(False, False, "host"), (True, False, "host"),
                                                    (False, True, "device"), (True, True, "device")],
                         ids=["stream", "graph", "stream-kept", "graph-kept"])
def test_batch_round_equals_single_rounds(graphs, keep, transcript):
    col_logs = [3, 1, 5, 2, 4, 1]
    row_log, primes = 7, [3889, 9721]
    L, pp, b = make(row_log, primes, 0, col_logs)
    if keep:
        b.keep_transform(True)
    if graphs:
        b.use_graphs(True)
    rounds = b.round(DOMAIN, transcript=transcript)
    for i, cl in enumerate(col_logs):
        single = product_round((row_log + cl, cl, primes, 0), witness_seed=seeds(len(col_logs))[i])
        assert np.array_equal(rounds[i].matrix, single["commitment"].matrix), i
        for k in ["p0", "p1", "u", "mle", "v"]:
            assert np.array_equal(getattr(rounds[i], k), single[k]), (i, k)
        assert np.array_equal(rounds[i].challenges, single["challenges"]), i


def test_batch_bit_dropped_and_autotune():
    col_logs = [2, 4, 3, 5]
    row_log, primes = 8, [3889, 2917, 4861]
    L, pp, b = make(row_log, primes, 9, col_logs)
    before = b.round(DOMAIN)
    tuned = b.autotune()
    assert tuned["commit_chunks"] >= 1 and tuned["fold_columns_per_split"] >= 1
    b.use_graphs(True)
    after = b.round(DOMAIN)
    for i, cl in enumerate(col_logs):
        single = product_round((row_log + cl, cl, primes, 9), witness_seed=seeds(len(col_logs))[i])
        for r in (before[i], after[i]):
            assert np.array_equal(r.top, single["commitment"].top), i
            assert np.array_equal(r.digits, single["commitment"].digits), i
            assert np.array_equal(r.v, single["v"]), i
            assert np.array_equal(r.u, single["u"]), i


def test_batch_matches_oracle_on_uploaded_witnesses(oracle):
    """Uploaded (not generated) witnesses, including an all-ones instance, against the oracle."""
    import labinius_b200 as L
    from labinius_b200.batch import Batch

    col_logs = [1, 2, 3]
    row_log, primes = 7, [2917, 19441]
    params = product_params((row_log + 1, 1, primes, 0))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    b = Batch(pp, col_logs)
    rng = np.random.default_rng(9)
    wits = []
    for i, cl in enumerate(col_logs):
        n = (1 << cl) << row_log
        w = rng.integers(0, 2 ** 63, (n, 3), dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, (n, 3), dtype=np.uint64)
        if i == 0:
            w[:] = np.uint64(2 ** 64 - 1)
        w[:, 2] &= np.uint64((1 << 34) - 1)
        wits.append(w)
        b.witness_upload(i, w)
    rounds = b.commit()
    key = pp.key()
    for i, cl in enumerate(col_logs):
        P = oracle.Params(row_log + cl, cl, primes, 0)
        assert np.array_equal(rounds[i].matrix, oracle.commit(P, key, wits[i])), i
        assert np.array_equal(b.elements(i), wits[i])
