"""wire::encode of the folded witness (crates/pcs/src/wire/rans.rs:18-105) over the C ABI: interleaved
static rANS over 64 lanes against the message's own histogram, the lanes, the histogram and the
word placement on the device."""
import numpy as np

from ._native import check, lib, ptr


def _result(n: int, out: np.ndarray) -> bytes:
    if n < 0:
        check(int(n))
    return out[:n].tobytes()


def encode(folded, base_q: int) -> bytes:
    """The bytes of wire::encode(folded, base_q); folded is a FoldedWitness or int16 [elements][648]."""
    v = np.ascontiguousarray(getattr(folded, "elements", folded), dtype=np.int16).reshape(-1, 648)
    cap = int(lib().lbg_wire_encode_bound(len(v)))
    out = np.zeros(cap, np.uint8)
    n = lib().lbg_wire_encode(ptr(v) if v.size else None, len(v), int(base_q), ptr(out), cap)
    return _result(n, out)


def encode_folded(prover) -> bytes:
    """wire::encode of the prover's last folded witness, read where Prover::fold left it on the
    device, against the base modulus."""
    cap = int(lib().lbg_wire_encode_bound(prover.params.len_ring()))
    out = np.zeros(cap, np.uint8)
    n = lib().lbg_prover_encode_folded(prover._h, ptr(out), cap)
    return _result(n, out)
