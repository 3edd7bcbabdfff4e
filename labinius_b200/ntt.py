"""The reference's 648-point transform of ring elements (crates/pcs/src/scalar.rs:35-84 forward,
:123-177 inverse) on the device, for splitting primes: the kernels of the NTT microbenchmark,
over the C ABI's lbg_ntt648_forward / lbg_ntt648_inverse. Inputs and outputs are CUDA tensors
of [count, 648] 16-bit values in [0, q) (int16 or uint16; q < 2^15)."""
from ._native import check, lib


def _call(fn, q, x, out, stream):
    import torch

    if x.device.type != "cuda" or x.dtype not in (torch.int16, torch.uint16) or x.shape[-1] != 648:
        raise ValueError("expected a CUDA tensor of [count, 648] 16-bit values")
    x = x.contiguous()
    if out is None:
        out = torch.empty_like(x)
    s = torch.cuda.current_stream(x.device).cuda_stream if stream is None else stream
    with torch.cuda.device(x.device):
        check(fn(int(q), x.data_ptr(), out.data_ptr(), x.numel() // 648, s))
    return out


def forward(q, x, out=None, stream=None):
    """slots[j] = a(psi^SLOT_EXP[j]) of every ring element, in the reference's slot order."""
    return _call(lib().lbg_ntt648_forward, q, x, out, stream)


def inverse(q, x, out=None, stream=None):
    """Coefficients from slots: the exact inverse of forward."""
    return _call(lib().lbg_ntt648_inverse, q, x, out, stream)
