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


def pack_commitment(opening) -> bytes:
    """wire::pack_commitment (crates/pcs/src/wire/mod.rs:226-245) of the commitment an opening holds,
    packed on the device where Prover::commit left it (the bit-dropped form is wire::pack_dropped)."""
    n = int(lib().lbg_opening_pack_commitment(opening._h, None, 0))
    if n < 0:
        check(n)
    out = np.zeros(max(n, 1), np.uint8)
    return _result(lib().lbg_opening_pack_commitment(opening._h, ptr(out), n), out)


def row_evaluate_packed(witness, point):
    """Witness::row_evaluate and wire::pack_row_evaluation (crates/pcs/src/wire/mod.rs:435-459), both on
    the device: (RowEvaluation, its bytes)."""
    from .scheme import RowEvaluation

    pp = witness.pp
    p0 = np.ascontiguousarray(point.p0, dtype=np.uint64)
    n = int(lib().lbg_row_evaluate_packed(pp._h, None, None, 0, None, None, 0))
    if n < 0:
        check(n)
    u = np.zeros((pp.params.columns(), 3), np.uint64)
    out = np.zeros(max(n, 1), np.uint8)
    m = lib().lbg_row_evaluate_packed(pp._h, witness._h, ptr(p0), len(p0), ptr(u), ptr(out), n)
    return RowEvaluation(u), _result(m, out)
