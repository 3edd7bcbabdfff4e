"""The round's transcript on the device (lbg_batch_round): the commitment and row-value absorbs,
the evaluation point and the folding challenges drawn by device kernels equal the host
transcript's, byte for byte, whatever the alignment of the absorbed strings against BLAKE3's
64-byte blocks and 1024-byte chunks (swept through the domain's length), for commitments from a
few chunks to thousands (deep subtree merges), in Clear and bit-dropped modes; and the device
round of a batch equals each instance's single-instance round."""
import numpy as np
import pytest

from rounds import DOMAIN, MATRIX_SEED, product_params, product_round

pytestmark = pytest.mark.gpu


def batch(row_log, primes, dropped, col_logs, seed0=0x31):
    import labinius_b200 as L
    from labinius_b200.batch import Batch

    params = product_params((row_log + col_logs[0], col_logs[0], primes, dropped))
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    b = Batch(pp, col_logs)
    b.witness_random([bytes([(seed0 + i) & 0xFF]) * 32 for i in range(len(col_logs))])
    return b


def same(a, b):
    for k in ["matrix", "top", "digits", "p0", "p1", "mle", "u", "challenges", "v"]:
        x, y = getattr(a, k), getattr(b, k)
        if x is None and y is None:
            continue
        assert np.array_equal(x, y), k


# Clear, 2 limbs: the commitment's bytes start at offset 150 + len(domain); 873..875 put the
# old length around 1023/1024/1025 (a chunk boundary), 1898 at 2048, 42 at a block boundary
@pytest.mark.parametrize("dlen", [0, 5, 42, 873, 874, 875, 1850, 1898])
def test_device_transcript_alignment_sweep(dlen):
    b = batch(7, [3889, 9721], 0, [1, 3, 2, 5])
    domain = bytes((7 * i + 3) & 0xFF for i in range(dlen))
    dev = b.round(domain, transcript="device")
    host = b.round(domain, transcript="host")
    for i in range(b.count):
        same(dev[i], host[i])


def test_device_transcript_deep_tree_and_graphs():
    """1024 columns x 2600 bytes = 2540 chunks in one absorb, beside small instances."""
    b = batch(7, [3889, 9721], 0, [10, 1, 4])
    host = b.round(DOMAIN, transcript="host")
    dev = b.round(DOMAIN, transcript="device")
    b.use_graphs(True)
    dev2 = b.round(DOMAIN, transcript="device")
    dev3 = b.round(b"another domain", transcript="device")
    host3 = b.round(b"another domain", transcript="host")
    for i in range(b.count):
        same(dev[i], host[i])
        same(dev2[i], host[i])
        same(dev3[i], host3[i])


def test_device_transcript_bit_dropped():
    b = batch(8, [3889, 2917, 4861], 9, [2, 4, 3])
    for domain in [DOMAIN, bytes(700)]:
        dev = b.round(domain, transcript="device")
        host = b.round(domain, transcript="host")
        for i in range(b.count):
            same(dev[i], host[i])


def test_device_round_equals_single_rounds():
    col_logs = [3, 1, 5, 2]
    row_log, primes = 7, [3889, 9721]
    b = batch(row_log, primes, 0, col_logs, seed0=0x10)
    rounds = b.round(DOMAIN, transcript="device")
    for i, cl in enumerate(col_logs):
        single = product_round((row_log + cl, cl, primes, 0), witness_seed=bytes([0x10 + i]) * 32)
        assert np.array_equal(rounds[i].matrix, single["commitment"].matrix), i
        for k in ["p0", "p1", "u", "mle", "v"]:
            assert np.array_equal(getattr(rounds[i], k), single[k]), (i, k)
        assert np.array_equal(rounds[i].challenges, single["challenges"]), i
