"""TEST INFRASTRUCTURE: Python bindings of the CPU oracle (``oracle/oracle.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this
module, and only to check the device's results or as the timed CPU baseline. The product
(``labinius_b200``) never imports it.

Parity unpinned: the reference (osdnk/labinius) ships no golden vectors for this path and cannot be
built here; the oracle is a restatement of its scalar definitions, cross-checked against the
reference's relational tests and, for BLAKE3, against the Python ``blake3`` package.
"""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None

CHALLENGE_DTYPE = np.dtype([("positions", np.uint8, 32), ("signs", np.uint32), ("weight", np.uint32)])
N = 648
N162 = 162


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        _lib = ctypes.CDLL(path)
        _setup(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _setup(L):
    vp, sz, u32, u64, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
    sig = {
        "orc_blake3": (None, [i32, vp, sz, vp, sz, u64, vp, sz]),
        "orc_prime_info": (None, [u32, vp]),
        "orc_slot_tables": (None, [vp, vp, vp, vp, vp]),
        "orc_ntt": (None, [u32, vp, vp]),
        "orc_intt": (None, [u32, vp, vp]),
        "orc_eval_at": (u32, [u32, vp, u32]),
        "orc_eval_quad_at": (None, [u32, vp, u32, vp]),
        "orc_components": (None, [u32, vp, vp]),
        "orc_recombine": (None, [u32, vp, vp]),
        "orc_f162_mul": (None, [vp, vp, vp]),
        "orc_f162_mul_serial": (None, [vp, vp, vp]),
        "orc_eq_table": (None, [vp, i32, vp]),
        "orc_key_seed": (u64, [vp]),
        "orc_key_expand": (None, [vp, i32, sz, u64, vp]),
        "orc_witness_random": (None, [sz, vp, vp]),
        "orc_commit": (None, [vp, vp, vp, sz, sz, vp, vp, i32]),
        "orc_row_evaluate": (None, [vp, sz, vp, i32, vp]),
        "orc_claim": (None, [vp, vp, i32, vp]),
        "orc_fold": (None, [vp, vp, vp, sz, sz, vp, i32, i32]),
        "orc_fold_commitment": (None, [vp, vp, vp, vp]),
        "orc_slot_table": (None, [u32, vp]),
        "orc_drop_bits": (None, [vp, vp, vp, vp]),
        "orc_recursion_residues": (None, [vp, vp, sz, vp]),
        "orc_left_expansion": (None, [vp, sz, sz, vp]),
        "orc_pack_dropped": (sz, [vp, vp, vp, vp, sz]),
        "orc_transcript_new": (vp, [vp, sz]),
        "orc_transcript_free": (None, [vp]),
        "orc_transcript_clone": (vp, [vp]),
        "orc_transcript_absorb_bytes": (None, [vp, vp, sz]),
        "orc_transcript_absorb_u64": (None, [vp, u64]),
        "orc_transcript_fill": (None, [vp, ctypes.c_char_p, vp, sz]),
        "orc_transcript_absorb_raw": (None, [vp, vp, sz]),
        "orc_switch_prove": (None, [vp, sz, vp, sz, vp, vp, vp, vp, vp, vp, vp]),
        "orc_switch_verify": (i32, [sz, vp, sz, vp, vp, vp, vp, vp, vp, vp]),
        "orc_switch_mle": (None, [vp, sz, vp, sz, vp, vp]),
        "orc_b128_mul": (None, [vp, vp, vp]),
        "orc_sample_short_challenge": (None, [vp, u32, ctypes.c_double, vp, vp]),
        "orc_within": (i32, [vp, ctypes.c_double]),
        "orc_derive_evaluation_point": (None, [vp, vp, vp, vp, vp, vp, vp]),
        "orc_derive_folding_challenges": (None, [vp, vp, vp, vp]),
        "orc_verify_folded_opening": (i32, [vp, vp, vp, vp, vp, vp]),
        "orc_bd_residual": (None, [vp, vp, vp, vp, vp, vp, vp]),
        "orc_wire_encode": (sz, [vp, sz, u32, vp, sz]),
        "orc_wire_decode": (i32, [vp, sz, vp, sz, vp]),
        "orc_verify_folded_opening_bd": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "orc_fold_binary": (None, [vp, vp, sz, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


# ------------------------------------------------------------------------------------------------
# parameters
# ------------------------------------------------------------------------------------------------
class Params:
    """The round shape of crates/pcs/src/scheme/params.rs:62-68: moduli with the base first."""

    def __init__(self, witness_log_len, column_log_len, primes, dropped_bits=0):
        self.witness_log_len = witness_log_len
        self.column_log_len = column_log_len
        self.primes = list(primes)
        self.dropped_bits = dropped_bits

    @property
    def limbs(self):
        return len(self.primes)

    @property
    def columns(self):
        return 1 << self.column_log_len

    @property
    def row_log_len(self):
        return self.witness_log_len - self.column_log_len

    @property
    def column_len(self):
        return 1 << self.row_log_len

    @property
    def len_ring(self):
        return self.column_len // 4

    @property
    def witness_len(self):
        return 1 << self.witness_log_len

    def arr(self):
        return np.array([self.witness_log_len, self.column_log_len, self.limbs, self.dropped_bits, *self.primes],
                        dtype=np.uint32)


# ------------------------------------------------------------------------------------------------
# primitives
# ------------------------------------------------------------------------------------------------
def blake3(data: bytes, n: int = 32, seek: int = 0, key: bytes = None, context: bytes = None) -> bytes:
    mode, k = 0, b""
    if key is not None:
        mode, k = 1, key
    elif context is not None:
        mode, k = 2, context
    kb = np.frombuffer(k, dtype=np.uint8).copy() if k else np.zeros(1, np.uint8)
    db = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, np.uint8)
    out = np.zeros(max(n, 1), dtype=np.uint8)
    lib().orc_blake3(mode, _p(kb), len(k), _p(db), len(data), seek, _p(out), n)
    return out[:n].tobytes()


def prime_info(q):
    out = np.zeros(5, dtype=np.uint64)
    lib().orc_prime_info(q, _p(out))
    return dict(quad=bool(out[0]), psi=int(out[1]), omega=int(out[2]), zeta6=int(out[3]), theta=int(out[4]))


def slot_tables():
    se = np.zeros(N, np.uint32)
    qse = np.zeros(324, np.uint32)
    pow3 = np.zeros(N162, np.uint32)
    s648 = np.zeros((4, N162), np.uint32)
    qcs = np.zeros((2, N162), np.uint32)
    lib().orc_slot_tables(_p(se), _p(qse), _p(pow3), _p(s648), _p(qcs))
    return dict(slot_exp=se, quad_slot_exp=qse, pow3_slot_exp=pow3, slot_648=s648, quad_class_slot=qcs)


def ntt(q, a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    out = np.zeros(N, np.uint32)
    lib().orc_ntt(q, _p(a), _p(out))
    return out


def intt(q, a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    out = np.zeros(N, np.uint32)
    lib().orc_intt(q, _p(a), _p(out))
    return out


def eval_at(q, a, u):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return int(lib().orc_eval_at(q, _p(a), u))


def eval_quad_at(q, a, u):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    r = np.zeros(2, np.uint32)
    lib().orc_eval_quad_at(q, _p(a), u, _p(r))
    return int(r[0]), int(r[1])


def components(q, y):
    y = np.ascontiguousarray(y, dtype=np.uint32)
    out = np.zeros((4, N162), np.int16)
    lib().orc_components(q, _p(y), _p(out))
    return out


def recombine(q, comp):
    comp = np.ascontiguousarray(comp, dtype=np.int16)
    y = np.zeros(N, np.uint32)
    lib().orc_recombine(q, _p(comp), _p(y))
    return y


def f162_mul(a, b, serial=False):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.zeros(3, np.uint64)
    (lib().orc_f162_mul_serial if serial else lib().orc_f162_mul)(_p(a), _p(b), _p(out))
    return out


def eq_table(ps):
    ps = np.ascontiguousarray(ps, dtype=np.uint64).reshape(-1, 3)
    out = np.zeros((1 << len(ps), 3), np.uint64)
    lib().orc_eq_table(_p(ps), len(ps), _p(out))
    return out


def key_seed(seed: bytes) -> int:
    s = np.frombuffer(seed, dtype=np.uint8).copy()
    return int(lib().orc_key_seed(_p(s)))


def key_expand(params: Params, seed64: int):
    primes = np.array(params.primes, dtype=np.uint32)
    A = np.zeros((params.limbs, params.len_ring, N), np.int16)
    lib().orc_key_expand(_p(primes), params.limbs, params.len_ring, seed64, _p(A))
    return A


def witness_random(n: int, seed: bytes):
    s = np.frombuffer(seed, dtype=np.uint8).copy()
    out = np.zeros((n, 3), np.uint64)
    lib().orc_witness_random(n, _p(s), _p(out))
    return out


def commit(params: Params, A, witness, c0=0, c1=None, threads=1, raw=False):
    c1 = params.columns if c1 is None else c1
    w = np.ascontiguousarray(witness, dtype=np.uint64)
    A = np.ascontiguousarray(A, dtype=np.int16)
    C = np.zeros((params.columns, 4, params.limbs, N162), np.int16)
    R = np.zeros((params.columns, params.limbs, N), np.uint32) if raw else None
    pa = params.arr()
    lib().orc_commit(_p(pa), _p(A), _p(w), c0, c1, _p(C), _p(R) if raw else None, threads)
    return (C, R) if raw else C


def row_evaluate(witness, p0):
    w = np.ascontiguousarray(witness, dtype=np.uint64)
    p0 = np.ascontiguousarray(p0, dtype=np.uint64).reshape(-1, 3)
    n = len(w)
    u = np.zeros((n >> len(p0), 3), np.uint64)
    lib().orc_row_evaluate(_p(w), n, _p(p0), len(p0), _p(u))
    return u


def claim(u, p1):
    u = np.ascontiguousarray(u, dtype=np.uint64)
    p1 = np.ascontiguousarray(p1, dtype=np.uint64).reshape(-1, 3)
    out = np.zeros(3, np.uint64)
    lib().orc_claim(_p(u), _p(p1), len(p1), _p(out))
    return out


def fold(params: Params, witness, challenges, i0=0, i1=None, threads=1, use_ntt=False):
    i1 = params.len_ring if i1 is None else i1
    w = np.ascontiguousarray(witness, dtype=np.uint64)
    ch = np.ascontiguousarray(challenges, dtype=CHALLENGE_DTYPE)
    v = np.zeros((params.len_ring, N), np.int16)
    pa = params.arr()
    lib().orc_fold(_p(pa), _p(w), _p(ch), i0, i1, _p(v), threads, int(use_ntt))
    return v


def fold_commitment(params: Params, C, challenges):
    C = np.ascontiguousarray(C, dtype=np.int16)
    ch = np.ascontiguousarray(challenges, dtype=CHALLENGE_DTYPE)
    out = np.zeros((4, params.limbs, N162), np.int16)
    pa = params.arr()
    lib().orc_fold_commitment(_p(pa), _p(C), _p(ch), _p(out))
    return out


def slot_table(q):
    out = np.zeros((N162, N162), np.int16)
    lib().orc_slot_table(q, _p(out))
    return out


def drop_bits(params: Params, C):
    C = np.ascontiguousarray(C, dtype=np.int16)
    count = params.columns * N
    top = np.zeros(count, np.uint16)
    digits = np.zeros((max(params.limbs - 1, 1), count), np.uint16)
    pa = params.arr()
    lib().orc_drop_bits(_p(pa), _p(C), _p(top), _p(digits))
    return top, digits[: params.limbs - 1]


def recursion_polys(columns: int) -> int:
    """Three chunks per column, padded to a multiple of 32 (crates/pcs/src/recursion/limbs.rs:388)."""
    return -(-3 * columns // 32) * 32


def recursion_residues(params: Params, C, polys=None):
    """recursion::limbs::residues (crates/pcs/src/recursion/limbs.rs:379-398): int16
    [limbs * 4][polys][64]."""
    C = np.ascontiguousarray(C, dtype=np.int16)
    polys = recursion_polys(params.columns) if polys is None else int(polys)
    out = np.zeros((params.limbs * 4, polys, 64), np.int16)
    lib().orc_recursion_residues(_p(params.arr()), _p(C), polys, _p(out))
    return out


def left_expansion(u, rank=None):
    """Prover::commit_left_expansion's vector u (crates/pcs/src/scheme/prover.rs:95-115): int16
    [rank][64]."""
    u = np.ascontiguousarray(u, dtype=np.uint64).reshape(-1, 3)
    rank = recursion_polys(len(u)) if rank is None else int(rank)
    out = np.zeros((rank, 64), np.int16)
    lib().orc_left_expansion(_p(u), len(u), rank, _p(out))
    return out


def pack_dropped(params: Params, top, digits):
    pa = params.arr()
    top = np.ascontiguousarray(top, dtype=np.uint16)
    digits = np.ascontiguousarray(digits, dtype=np.uint16) if params.limbs > 1 else np.zeros(1, np.uint16)
    n = lib().orc_pack_dropped(_p(pa), _p(top), _p(digits), None, 0)
    out = np.zeros(n, np.uint8)
    lib().orc_pack_dropped(_p(pa), _p(top), _p(digits), _p(out), n)
    return out.tobytes()


class Transcript:
    """crates/pcs/src/challenge.rs:66-161"""

    def __init__(self, domain: bytes = None, _handle=None):
        if _handle is not None:
            self.h = _handle
        else:
            d = np.frombuffer(domain, dtype=np.uint8).copy()
            self.h = lib().orc_transcript_new(_p(d), len(domain))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_transcript_free(self.h)
            self.h = None

    def clone(self):
        return Transcript(_handle=lib().orc_transcript_clone(self.h))

    def absorb_bytes(self, b: bytes):
        a = np.frombuffer(b, dtype=np.uint8).copy() if b else np.zeros(1, np.uint8)
        lib().orc_transcript_absorb_bytes(self.h, _p(a), len(b))

    def absorb_u64(self, x: int):
        lib().orc_transcript_absorb_u64(self.h, x)

    def fill(self, label: bytes, n: int) -> bytes:
        out = np.zeros(max(n, 1), np.uint8)
        lib().orc_transcript_fill(self.h, label, _p(out), n)
        return out[:n].tobytes()


def sample_short_challenge(t: Transcript, weight=28, bound=12.0):
    out = np.zeros(1, CHALLENGE_DTYPE)
    att = np.zeros(1, np.uint64)
    lib().orc_sample_short_challenge(t.h, weight, bound, _p(out), _p(att))
    return out[0], int(att[0])


def derive_evaluation_point(params: Params, matrix_seed: bytes, t: Transcript, C=None, top=None, digits=None):
    pa = params.arr()
    seed = np.frombuffer(matrix_seed, dtype=np.uint8).copy()
    n = params.row_log_len + params.column_log_len
    p = np.zeros((n, 3), np.uint64)
    Cc = np.ascontiguousarray(C, dtype=np.int16) if C is not None else None
    tp = np.ascontiguousarray(top, dtype=np.uint16) if top is not None else None
    dg = (np.ascontiguousarray(digits, dtype=np.uint16) if (digits is not None and params.limbs > 1)
          else np.zeros(1, np.uint16))
    lib().orc_derive_evaluation_point(_p(pa), _p(seed), t.h, _p(Cc) if Cc is not None else None,
                                      _p(tp) if tp is not None else None, _p(dg), _p(p))
    return p[: params.row_log_len], p[params.row_log_len:]


def derive_folding_challenges(params: Params, t: Transcript, u):
    pa = params.arr()
    u = np.ascontiguousarray(u, dtype=np.uint64)
    out = np.zeros(params.columns, CHALLENGE_DTYPE)
    lib().orc_derive_folding_challenges(_p(pa), t.h, _p(u), _p(out))
    return out


def verify_folded_opening(params: Params, A, folded_commitment, v, p0, folded_row_value):
    pa = params.arr()
    A = np.ascontiguousarray(A, dtype=np.int16)
    fc = np.ascontiguousarray(folded_commitment, dtype=np.int16)
    v = np.ascontiguousarray(v, dtype=np.int16)
    p0 = np.ascontiguousarray(p0, dtype=np.uint64)
    fr = np.ascontiguousarray(folded_row_value, dtype=np.uint64)
    return bool(lib().orc_verify_folded_opening(_p(pa), _p(A), _p(fc), _p(v), _p(p0), _p(fr)))


def _dropped_args(params: Params, top, digits):
    top = np.ascontiguousarray(top, dtype=np.uint16)
    digits = np.ascontiguousarray(digits, dtype=np.uint16)
    if digits.size == 0:
        digits = np.zeros(1, np.uint16)
    return top, digits


def bd_residual(params: Params, A, top, digits, challenges, v):
    """crates/pcs/src/bd/residual.rs:66-130: the squared norm (an int) of the bit-dropped residual."""
    top, digits = _dropped_args(params, top, digits)
    out = np.zeros(2, np.uint64)
    lib().orc_bd_residual(_p(params.arr()), _p(np.ascontiguousarray(A, dtype=np.int16)), _p(top), _p(digits),
                          _p(np.ascontiguousarray(challenges, dtype=CHALLENGE_DTYPE)),
                          _p(np.ascontiguousarray(v, dtype=np.int16)), _p(out))
    return int(out[0]) | (int(out[1]) << 64)


def bd_cap(params: Params):
    """crates/pcs/src/bd/mod.rs:72-75"""
    import math

    d = params.dropped_bits
    return math.ceil(4.0 * float(N * params.columns * 28) * (float((1 << (2 * d)) - 1) / 12.0))


def verify_folded_opening_bd(params: Params, A, top, digits, challenges, v, p0, folded_row_value):
    """crates/pcs/src/scheme/verifier.rs:232-276"""
    top, digits = _dropped_args(params, top, digits)
    return bool(lib().orc_verify_folded_opening_bd(
        _p(params.arr()), _p(np.ascontiguousarray(A, dtype=np.int16)), _p(top), _p(digits),
        _p(np.ascontiguousarray(challenges, dtype=CHALLENGE_DTYPE)), _p(np.ascontiguousarray(v, dtype=np.int16)),
        _p(np.ascontiguousarray(p0, dtype=np.uint64)), _p(np.ascontiguousarray(folded_row_value, dtype=np.uint64))))


def fold_binary(u, challenges):
    u = np.ascontiguousarray(u, dtype=np.uint64)
    ch = np.ascontiguousarray(challenges, dtype=CHALLENGE_DTYPE)
    out = np.zeros(3, np.uint64)
    lib().orc_fold_binary(_p(u), _p(ch), len(ch), _p(out))
    return out


def round_trip(params: Params, matrix_seed: bytes, witness_seed: bytes = None, witness=None,
               domain: bytes = b"labinius/reference", threads=1):
    """One reference round (crates/bench/src/bin/labinius.rs:104-130): commit, evaluation point,
    mle and row evaluation, folding challenges, fold, and (Clear mode) the folded commitment."""
    if witness is None:
        witness = witness_random(params.witness_len, witness_seed)
    A = key_expand(params, key_seed(matrix_seed))
    C = commit(params, A, witness, threads=threads)
    out = dict(A=A, witness=witness, C=C)
    t = Transcript(domain)
    if params.dropped_bits:
        top, digits = drop_bits(params, C)
        out.update(top=top, digits=digits, packed=pack_dropped(params, top, digits))
        p0, p1 = derive_evaluation_point(params, matrix_seed, t, top=top, digits=digits)
    else:
        p0, p1 = derive_evaluation_point(params, matrix_seed, t, C=C)
    u = row_evaluate(witness, p0)
    mle = claim(u, p1)
    ch = derive_folding_challenges(params, t, u)
    v = fold(params, witness, ch, threads=threads)
    out.update(p0=p0, p1=p1, u=u, mle=mle, challenges=ch, v=v)
    if not params.dropped_bits:
        out["folded_commitment"] = fold_commitment(params, C, ch)
    out["transcript_tail"] = t.fill(b"labinius/test-tail", 32)
    return out


# ---------------------------------------------------------------------------------------------
# the cross-field switch (crates/pcs/src/switch.rs)
# ---------------------------------------------------------------------------------------------
def _b128(a):
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 2)
    return a if len(a) else np.zeros((1, 2), np.uint64)


def b128_mul(a, b):
    out = np.zeros(2, np.uint64)
    lib().orc_b128_mul(_p(np.ascontiguousarray(a, np.uint64)), _p(np.ascontiguousarray(b, np.uint64)), _p(out))
    return out


def switch_mle(trace, r_hi, r_lo=None):
    """switch::mle (r_lo None) or switch::bit_mle: a B128 [2] claim."""
    tr = _b128(trace)
    hi = _b128(r_hi)
    lo = _b128(r_lo if r_lo is not None else np.zeros((0, 2), np.uint64))
    nlo = 0 if r_lo is None else len(r_lo)
    out = np.zeros(2, np.uint64)
    lib().orc_switch_mle(_p(tr), len(r_hi), _p(lo), nlo, _p(hi), _p(out))
    return out


def switch_prove(trace, r_hi, claim, t: Transcript, r_lo=None):
    """switch::prove / prove_bits: (partials [128][2], rounds [l][2][3], opened [3], r_pp [l][3])."""
    l = len(r_hi)
    nlo = 0 if r_lo is None else len(r_lo)
    lo = _b128(r_lo if r_lo is not None else np.zeros((0, 2), np.uint64))
    partials = np.zeros((128, 2), np.uint64)
    rounds = np.zeros((l, 2, 3), np.uint64)
    opened = np.zeros(3, np.uint64)
    r_pp = np.zeros((l, 3), np.uint64)
    lib().orc_switch_prove(_p(_b128(trace)), l, _p(lo), nlo, _p(_b128(r_hi)), _p(np.ascontiguousarray(claim, np.uint64)),
                           t.h, _p(partials), _p(rounds), _p(opened), _p(r_pp))
    return partials, rounds, opened, r_pp


def switch_verify(r_hi, claim, partials, rounds, opened, t: Transcript, r_lo=None):
    """switch::verify / verify_bits: (accepted, r_pp [l][3])."""
    l = len(r_hi)
    nlo = 0 if r_lo is None else len(r_lo)
    lo = _b128(r_lo if r_lo is not None else np.zeros((0, 2), np.uint64))
    r_pp = np.zeros((max(l, 1), 3), np.uint64)
    ok = lib().orc_switch_verify(l, _p(lo), nlo, _p(_b128(r_hi)), _p(np.ascontiguousarray(claim, np.uint64)),
                                 _p(np.ascontiguousarray(partials, np.uint64)),
                                 _p(np.ascontiguousarray(rounds, np.uint64)),
                                 _p(np.ascontiguousarray(opened, np.uint64)), t.h, _p(r_pp))
    return bool(ok), r_pp[:l]


def tagged_commitment(params: Params, C=None, top=None, digits=None) -> bytes:
    """Commitment::to_bytes, wire::pack_tagged_commitment (crates/pcs/src/wire/mod.rs:307-333)."""
    head = int(params.columns).to_bytes(4, "little")
    if params.dropped_bits:
        return b"\x02" + head + pack_dropped(params, top, digits)
    return b"\x00" + head + np.ascontiguousarray(C, dtype="<i2").tobytes()


def switch_round(params: Params, matrix_seed: bytes, trace, r_hi, claim_value=None,
                 domain: bytes = b"labinius/reference"):
    """A B128 trace committed as Witness::lifted and opened through the switch, the prover of
    crates/pcs/examples/two_fields.rs:176-194: commit, absorb the tagged commitment, switch::prove
    (the claim defaults to the trace's value at r_hi), row_evaluate at the switch's point,
    FoldingChallenges::derive, fold."""
    tr = np.ascontiguousarray(trace, dtype=np.uint64).reshape(-1, 2)
    witness = np.zeros((len(tr), 3), np.uint64)
    witness[:, :2] = tr  # F162::from_b128 (crates/pcs/src/fields/scalar.rs:72-74)
    A = key_expand(params, key_seed(matrix_seed))
    C = commit(params, A, witness)
    out = dict(A=A, witness=witness, C=C)
    t = Transcript(domain)
    if params.dropped_bits:
        top, digits = drop_bits(params, C)
        out.update(top=top, digits=digits)
        t.absorb_bytes(tagged_commitment(params, top=top, digits=digits))
    else:
        t.absorb_bytes(tagged_commitment(params, C=C))
    c = switch_mle(tr, r_hi) if claim_value is None else np.asarray(claim_value, np.uint64)
    partials, rounds, opened, r_pp = switch_prove(tr, r_hi, c, t)
    rows, cl = params.row_log_len, params.column_log_len
    p0 = np.ascontiguousarray(r_pp[::-1][:rows])  # EvaluationPoint::msb_first
    p1 = np.ascontiguousarray(r_pp[:cl][::-1])
    u = row_evaluate(witness, p0)
    mle = claim(u, p1)
    ch = derive_folding_challenges(params, t, u)
    v = fold(params, witness, ch)
    out.update(claim=c, partials=partials, rounds=rounds, opened=opened, p0=p0, p1=p1, u=u, mle=mle,
               challenges=ch, v=v)
    if not params.dropped_bits:
        out["folded_commitment"] = fold_commitment(params, C, ch)
    out["transcript_tail"] = t.fill(b"labinius/test-tail", 32)
    return out


def wire_encode(v, base_q: int) -> bytes:
    """wire::encode (crates/pcs/src/wire/rans.rs:18-105): v is int16 [elements][648]."""
    v = np.ascontiguousarray(v, dtype=np.int16).reshape(-1, N)
    n = lib().orc_wire_encode(_p(v), len(v), base_q, None, 0)
    out = np.zeros(max(n, 1), np.uint8)
    lib().orc_wire_encode(_p(v), len(v), base_q, _p(out), n)
    return out[:n].tobytes()


def wire_decode(data: bytes):
    """wire::decode (crates/pcs/src/wire/rans.rs:107-226): (status, v) with status 0 (ok),
    1 (truncated) or 2 (malformed)."""
    b = np.frombuffer(bytes(data), dtype=np.uint8).copy() if len(data) else np.zeros(1, np.uint8)
    count = ctypes.c_size_t(0)
    lib().orc_wire_decode(_p(b), len(data), None, 0, ctypes.byref(count))
    v = np.zeros((count.value, N), np.int16) if count.value <= (1 << 20) else np.zeros((0, N), np.int16)
    st = lib().orc_wire_decode(_p(b), len(data), _p(v) if v.size else None, v.size, ctypes.byref(count))
    return st, v



# ---------------------------------------------------------------------------------------------
# wire: the bit-packed commitment and row evaluation (crates/pcs/src/wire/mod.rs)
# ---------------------------------------------------------------------------------------------
def residue_bits(q: int) -> int:
    """crates/pcs/src/wire/mod.rs:77-79: bits of q - 1."""
    return int(q - 1).bit_length()


def pack_commitment(params: Params, C) -> bytes:
    """wire::pack_commitment (crates/pcs/src/wire/mod.rs:226-245) of a Clear commitment matrix
    C [columns][4][limbs][162]: element by element (column-major), limb by limb, slot by slot,
    slot mod q in residue_bits(q) bits."""
    C = np.asarray(C, dtype=np.int64).reshape(-1, params.limbs, N162)
    # one row of bits per element: limb 0's 162 slots, then limb 1's, ...; each slot's residue in
    # residue_bits(q) bits, least significant first (BitWriter::put, crates/pcs/src/wire/mod.rs:101-110)
    cols = []
    for k, q in enumerate(params.primes):
        v = (C[:, k, :] % q).astype(np.uint64).reshape(len(C), N162, 1)
        bits = residue_bits(q)
        cols.append(((v >> np.arange(bits, dtype=np.uint64)) & np.uint64(1)).astype(np.uint8).reshape(len(C), -1))
    stream = np.concatenate(cols, axis=1).reshape(-1)
    return np.packbits(stream, bitorder="little").tobytes()


def unpack_commitment(params: Params, data: bytes):
    """wire::unpack_commitment (crates/pcs/src/wire/mod.rs:248-300), Clear: (status, C) with status
    0 (ok) or 2 (malformed: wrong length or a value >= q)."""
    bits = [residue_bits(q) for q in params.primes]
    n = 4 * params.columns
    if len(data) != (n * N162 * sum(bits) + 7) // 8:
        return 2, None
    stream = np.unpackbits(np.frombuffer(bytes(data), dtype=np.uint8), bitorder="little")
    stream = stream[: n * N162 * sum(bits)].reshape(n, -1)
    C = np.zeros((n, params.limbs, N162), np.int16)
    off = 0
    for k, (q, b) in enumerate(zip(params.primes, bits)):
        blk = stream[:, off: off + N162 * b].reshape(n, N162, b).astype(np.uint64)
        vals = (blk << np.arange(b, dtype=np.uint64)).sum(axis=2)
        if (vals >= q).any():
            return 2, None
        half = (q - 1) // 2
        C[:, k, :] = np.where(vals > half, vals.astype(np.int64) - q, vals.astype(np.int64))
        off += N162 * b
    return 0, C.reshape(params.columns, 4, params.limbs, N162)


def pack_f162(u) -> bytes:
    """wire::pack_f162 / pack_row_evaluation (crates/pcs/src/wire/mod.rs:435-453): 162 bits per
    element (64 + 64 + 34), least significant first, back to back."""
    u = np.ascontiguousarray(u, dtype=np.uint64).reshape(-1, 3)
    parts = [((u[:, w:w + 1] >> np.arange(64 if w < 2 else 34, dtype=np.uint64)) & np.uint64(1)).astype(np.uint8)
             for w in range(3)]
    return np.packbits(np.concatenate(parts, axis=1).reshape(-1), bitorder="little").tobytes()


def unpack_f162(data: bytes, count: int):
    """wire::unpack_f162 (crates/pcs/src/wire/mod.rs:456-470): (status, u) with status 0 or 2 (the
    length is not ceil(162 count / 8))."""
    if len(data) != (count * 162 + 7) // 8:
        return 2, None
    stream = np.unpackbits(np.frombuffer(bytes(data), dtype=np.uint8), bitorder="little")[: count * 162]
    b = stream.reshape(count, 162).astype(np.uint64)
    u = np.zeros((count, 3), np.uint64)
    u[:, 0] = (b[:, :64] << np.arange(64, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    u[:, 1] = (b[:, 64:128] << np.arange(64, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    u[:, 2] = (b[:, 128:] << np.arange(34, dtype=np.uint64)).sum(axis=1, dtype=np.uint64)
    return 0, u
