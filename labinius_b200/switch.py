"""The cross-field switch prover (crates/pcs/src/switch.rs) over the C ABI's lbg_switch_prove.

A B128 trace of 2^l words, committed as Witness.lifted, carries a claim in B128; the switch turns
it into the F162 claim the commitment opens, at the point its sumcheck ends on. The prover's
passes over the trace and its sumcheck run on the device; the transcript is the caller's.
"""
import ctypes
from dataclasses import dataclass

import numpy as np

from ._native import check, lib, ptr
from .scheme import EvaluationPoint, PublicParameters, Transcript, Witness

LOG_WORD = 7


@dataclass
class SwitchProof:
    """crates/pcs/src/switch.rs:19-27"""
    partials: np.ndarray  # uint64 [128][2] (B128)
    rounds: np.ndarray    # uint64 [l][2][3] (F162 pairs)
    opened: np.ndarray    # uint64 [3] (F162)


def _prove(pp: PublicParameters, witness: Witness, r_lo, r_hi, claim, transcript: Transcript):
    params = pp.params
    l = params.witness_log_len
    hi = np.ascontiguousarray(r_hi, dtype=np.uint64).reshape(-1, 2)
    lo = None if r_lo is None else np.ascontiguousarray(r_lo, dtype=np.uint64).reshape(-1, 2)
    if len(hi) != l:
        raise ValueError("the point does not match the parameters")
    if lo is not None and len(lo) != LOG_WORD:
        raise ValueError("the point does not pick a bit")
    c = np.ascontiguousarray(claim, dtype=np.uint64).reshape(2)
    partials = np.zeros((128, 2), np.uint64)
    rounds = np.zeros((l, 2, 3), np.uint64)
    opened = np.zeros(3, np.uint64)
    p0 = np.zeros((params.row_log_len(), 3), np.uint64)
    p1 = np.zeros((params.column_log_len, 3), np.uint64)
    check(lib().lbg_switch_prove(pp._h, witness._h, ptr(lo), 0 if lo is None else len(lo), ptr(hi), l, ptr(c),
                                 transcript._h, ptr(partials), ptr(rounds), ptr(opened), ptr(p0), ptr(p1)))
    return SwitchProof(partials, rounds, opened), EvaluationPoint(p0, p1)


def prove(pp: PublicParameters, witness: Witness, r, claim, transcript: Transcript):
    """switch::prove: mle(trace, r) == claim, the trace being the lifted witness's words."""
    return _prove(pp, witness, None, r, claim, transcript)


def prove_bits(pp: PublicParameters, witness: Witness, r_lo, r_hi, claim, transcript: Transcript):
    """switch::prove_bits: bit_mle(trace, r_lo, r_hi) == claim."""
    return _prove(pp, witness, r_lo, r_hi, claim, transcript)
