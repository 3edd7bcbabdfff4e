"""The 648-point transform kernels (the NTT microbenchmark's): forward equals the oracle's
restatement of crates/pcs/src/scalar.rs:35-84 slot for slot, the inverse equals its inverse
(:123-177), inverse(forward(x)) = x at the benchmark's size, every splitting prime; quadratic-leaf
primes are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPLIT = [3889, 9721, 17497, 19441]


@pytest.mark.parametrize("q", SPLIT)
def test_forward_and_inverse_match_oracle(oracle, q):
    import torch

    from labinius_b200 import ntt

    rng = np.random.default_rng(q)
    count = 37  # not a multiple of the kernel's ring elements per CTA
    a = rng.integers(0, q, (count, 648)).astype(np.int16)
    a[0] = 0
    a[1] = q - 1
    y = ntt.forward(q, torch.from_numpy(a).cuda()).cpu().numpy().astype(np.int64)
    for i in range(count):
        assert np.array_equal(y[i], oracle.ntt(q, a[i].astype(np.uint32)).astype(np.int64)), i
    s = rng.integers(0, q, (count, 648)).astype(np.int16)
    x = ntt.inverse(q, torch.from_numpy(s).cuda()).cpu().numpy().astype(np.int64)
    for i in range(count):
        assert np.array_equal(x[i], oracle.intt(q, s[i].astype(np.uint32)).astype(np.int64)), i


def test_round_trip_at_benchmark_size():
    import torch

    from labinius_b200 import ntt

    q, count = 3889, 1 << 18
    g = torch.Generator(device="cuda").manual_seed(7)
    a = torch.randint(0, q, (count, 648), dtype=torch.int16, device="cuda", generator=g)
    y = ntt.forward(q, a)
    assert int(y.max()) < q and int(y.min()) >= 0
    assert torch.equal(ntt.inverse(q, y), a)


def test_quadratic_primes_refused():
    import torch

    from labinius_b200 import ntt
    from labinius_b200._native import NativeError

    a = torch.zeros((4, 648), dtype=torch.int16, device="cuda")
    for q in [2917, 4861, 12637]:
        with pytest.raises(NativeError):
            ntt.forward(q, a)


def test_forward_of_unaligned_buffers_matches():
    """Buffers 4-byte but not 16-byte aligned take the non-persistent forward kernel; it agrees with
    the aligned path (37 ring elements, a partial group). Buffers not 4-byte aligned are refused."""
    import torch

    from labinius_b200 import ntt

    q, count = 9721, 37
    g = torch.Generator(device="cuda").manual_seed(11)
    a = torch.randint(0, q, (count, 648), dtype=torch.int16, device="cuda", generator=g)
    want = ntt.forward(q, a)
    src = torch.zeros(count * 648 + 8, dtype=torch.int16, device="cuda")
    dst = torch.zeros(count * 648 + 8, dtype=torch.int16, device="cuda")
    x = src[2:2 + count * 648].view(count, 648)
    x.copy_(a)
    y = dst[6:6 + count * 648].view(count, 648)
    assert x.data_ptr() % 16 != 0 and y.data_ptr() % 16 != 0 and (x.data_ptr() | y.data_ptr()) % 4 == 0
    ntt.forward(q, x, out=y)
    assert torch.equal(y, want)
    from labinius_b200._native import NativeError

    with pytest.raises(NativeError):
        ntt.forward(q, src[1:1 + count * 648].view(count, 648), out=y)
