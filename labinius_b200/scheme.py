"""The reference's scheme API (osdnk/labinius crates/pcs/src/scheme/) over the B200 C ABI.

Same names, argument meaning and error behaviour as the Rust API for the commit / evaluate / fold
round (crates/pcs/src/lib.rs:51-61); the compute runs in ``liblabinius_gpu.so`` on the GPU, the
transcript and the challenge sampler on the host inside the same library. Arrays are numpy:

* an F162 is 3 x uint64 (limbs little-endian, bits 128..161 in limb 2);
* a commitment matrix is int16 [columns][4][limbs][162];
* a folded witness is int16 [len_ring][648];
* challenges are a structured array of ``CHALLENGE_DTYPE`` (positions, signs, weight).

Errors: ``ParamError`` and ``WitnessError`` where the Rust constructors return them, ``ValueError``
where the Rust code panics on misuse (assert!), ``VerificationError`` on rejection.
"""
import ctypes
import enum
import struct
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _native as nat
from ._native import check, lib, ptr

CHALLENGE_DTYPE = np.dtype([("positions", np.uint8, 32), ("signs", np.uint32), ("weight", np.uint32)])
N = 648
N162 = 162
MIN_COLUMN_LOG_LEN = 7
DEFAULT_WEIGHT = 28
DEFAULT_BOUND = 12.0


class ParamError(ValueError):
    """crates/pcs/src/scheme/params.rs:20-50"""


class WitnessError(ValueError):
    """crates/pcs/src/scheme/witness.rs:10-23"""


class VerificationError(Exception):
    """crates/pcs/src/scheme/commitment.rs:447-459"""


class Modulus(enum.IntEnum):
    """crates/pcs/src/ring/mod.rs:85-135 (the value is the prime)."""

    Q2917_Q_S = 2917
    Q3889_FS_S = 3889
    Q4861_Q_S = 4861
    Q9721_FS_S = 9721
    Q12637_Q_S = 12637
    Q17497_FS_L = 17497
    Q19441_FS_L = 19441

    def prime(self) -> int:
        return int(self)

    def is_quadratic(self) -> bool:
        q = int(self)
        return (q - 1) % 972 == 0 and (q - 1) % 1944 != 0


@dataclass(frozen=True)
class Opening:
    """Opening::Clear | BitDropped { bits } | Recursive (crates/pcs/src/scheme/params.rs:70-77)."""

    kind: str = "clear"
    bits: int = 0

    @staticmethod
    def clear():
        return Opening("clear", 0)

    @staticmethod
    def bit_dropped(bits: int):
        return Opening("bit_dropped", bits)

    @staticmethod
    def recursive():
        return Opening("recursive", 0)


@dataclass(frozen=True)
class Suite:
    name: str
    witness_log_len: int
    column_log_len_clear: int
    column_log_len_recursive: int
    moduli: tuple
    moduli_bd: tuple
    dropped_bits: int


# crates/pcs/src/scheme/params.rs:91-128
SUITES = [
    Suite("sizes", 18, 7, 8, (Modulus.Q9721_FS_S, Modulus.Q12637_Q_S),
          (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S), 10),
    Suite("sizem", 20, 8, 9, (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S),
          (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S), 9),
    Suite("sizel", 22, 9, 10, (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S),
          (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S), 8),
    Suite("sizexl", 24, 10, 11, (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q9721_FS_S),
          (Modulus.Q3889_FS_S, Modulus.Q2917_Q_S, Modulus.Q4861_Q_S), 7),
]


def suite_from_flag(flag: str) -> Optional[Suite]:
    for s in SUITES:
        if s.name == "size" + flag:
            return s
    return None


@dataclass
class Params:
    """crates/pcs/src/scheme/params.rs:62-288"""

    witness_log_len: int
    column_log_len: int
    base: Modulus = Modulus.Q3889_FS_S
    extra_moduli: List[Modulus] = field(default_factory=list)
    opening: Opening = field(default_factory=Opening.clear)

    @staticmethod
    def new(witness_log_len, column_log_len, extra_moduli, opening=None):
        return Params.with_base(witness_log_len, column_log_len, Modulus.Q3889_FS_S, extra_moduli, opening)

    @staticmethod
    def with_base(witness_log_len, column_log_len, base, extra_moduli, opening=None):
        opening = opening or Opening.clear()
        base = Modulus(int(base))
        extra = [Modulus(int(m)) for m in extra_moduli]
        if column_log_len > witness_log_len:
            raise ParamError("ColumnsExceedWitness")
        if column_log_len < 1:
            raise ParamError("TooFewColumns")
        if witness_log_len - column_log_len < MIN_COLUMN_LOG_LEN:
            raise ParamError("ColumnTooShort")
        for i, m in enumerate(extra):
            if m == base:
                raise ParamError(f"BaseIsAlsoExtra({m.name})")
            if m in extra[:i]:
                raise ParamError(f"DuplicateModulus({m.name})")
        return Params(witness_log_len, column_log_len, base, extra, opening)

    @staticmethod
    def basic():
        return Params.new(18, 7, [Modulus.Q9721_FS_S], Opening.clear())

    @staticmethod
    def sized(suite: Suite, opening: Opening):
        cl = suite.column_log_len_recursive if opening.kind == "recursive" else suite.column_log_len_clear
        lst = suite.moduli_bd if opening.kind == "bit_dropped" else suite.moduli
        return Params.with_base(suite.witness_log_len, cl, lst[0], list(lst[1:]), opening)

    def dropping(self, dropped_bits: int):
        self.opening = Opening.clear() if dropped_bits == 0 else Opening.bit_dropped(dropped_bits)
        return self

    def recursion(self) -> bool:
        return self.opening.kind == "recursive"

    def dropped_bits(self) -> int:
        return self.opening.bits if self.opening.kind == "bit_dropped" else 0

    def witness_len(self) -> int:
        return 1 << self.witness_log_len

    def columns(self) -> int:
        return 1 << self.column_log_len

    def row_log_len(self) -> int:
        return self.witness_log_len - self.column_log_len

    def column_len(self) -> int:
        return 1 << self.row_log_len()

    def len_ring(self) -> int:
        return self.column_len() // 4

    def primes(self) -> List[int]:
        return [int(self.base)] + [int(m) for m in self.extra_moduli]

    def native(self) -> nat.lbg_params:
        p = nat.lbg_params()
        p.witness_log_len = self.witness_log_len
        p.column_log_len = self.column_log_len
        pr = self.primes()
        p.n_moduli = len(pr)
        for i, q in enumerate(pr):
            p.moduli[i] = q
        p.opening = {"clear": 0, "bit_dropped": 1, "recursive": 2}[self.opening.kind]
        p.dropped_bits = self.dropped_bits()
        return p


def _seed32(seed) -> np.ndarray:
    b = bytes(seed)
    if len(b) != 32:
        raise ValueError("a seed is 32 bytes")
    return np.frombuffer(b, dtype=np.uint8).copy()


class PublicParameters:
    """Params plus the device-resident key A (crates/pcs/src/scheme/params.rs:309-354)."""

    def __init__(self, params: Params, handle, matrix_seed: bytes):
        self.params = params
        self._h = handle
        self.matrix_seed = bytes(matrix_seed)

    @staticmethod
    def from_seed(params: Params, matrix_seed) -> "PublicParameters":
        p = params.native()
        h = ctypes.c_void_p()
        rc = lib().lbg_public_parameters_from_seed(ctypes.byref(p), ptr(_seed32(matrix_seed)), ctypes.byref(h))
        if rc == nat.LBG_ERR_PARAMS:
            raise ParamError(lib().lbg_last_error().decode())
        check(rc)
        return PublicParameters(params, h, matrix_seed)

    def key(self) -> np.ndarray:
        """CommitmentKey::row for every limb: int16 [limbs][len_ring][648]."""
        pr = self.params
        out = np.zeros((len(pr.primes()), pr.len_ring(), N), np.int16)
        check(lib().lbg_key_download(self._h, ptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_public_parameters_free(h)
            self._h = None


class Witness:
    """crates/pcs/src/scheme/witness.rs:25-117. Device-resident; `pp` names the key it lives with."""

    def __init__(self, pp: PublicParameters, handle):
        self.pp = pp
        self.params = pp.params
        self._h = handle

    @staticmethod
    def random(pp: PublicParameters, seed) -> "Witness":
        h = ctypes.c_void_p()
        check(lib().lbg_witness_random(pp._h, ptr(_seed32(seed)), ctypes.byref(h)))
        return Witness(pp, h)

    @staticmethod
    def from_elements(pp: PublicParameters, elements) -> "Witness":
        e = np.ascontiguousarray(elements, dtype=np.uint64).reshape(-1, 3)
        if len(e) != pp.params.witness_len():
            raise WitnessError("WrongLength")
        h = ctypes.c_void_p()
        check(lib().lbg_witness_from_host(pp._h, ptr(e), len(e), ctypes.byref(h)))
        return Witness(pp, h)

    @staticmethod
    def lifted(pp: PublicParameters, trace) -> "Witness":
        t = np.ascontiguousarray(trace, dtype=np.uint64).reshape(-1, 2)
        if len(t) != pp.params.witness_len():
            raise WitnessError("WrongLength")
        h = ctypes.c_void_p()
        check(lib().lbg_witness_lifted(pp._h, ptr(t), len(t), ctypes.byref(h)))
        return Witness(pp, h)

    def elements(self) -> np.ndarray:
        out = np.zeros((self.params.witness_len(), 3), np.uint64)
        check(lib().lbg_witness_download(self._h, ptr(out), len(out)))
        return out

    def _check(self, point):
        if (len(point.p0), len(point.p1)) != (self.params.row_log_len(), self.params.column_log_len):
            raise ValueError("the evaluation point does not match the witness")

    def row_evaluate(self, point) -> "RowEvaluation":
        self._check(point)
        p0 = np.ascontiguousarray(point.p0, dtype=np.uint64)
        u = np.zeros((self.params.columns(), 3), np.uint64)
        check(lib().lbg_row_evaluate(self.pp._h, self._h, ptr(p0), len(p0), ptr(u)))
        return RowEvaluation(u)

    def mle_evaluate(self, point) -> np.ndarray:
        self._check(point)
        p0 = np.ascontiguousarray(point.p0, dtype=np.uint64)
        p1 = np.ascontiguousarray(point.p1, dtype=np.uint64)
        out = np.zeros(3, np.uint64)
        check(lib().lbg_mle_evaluate(self.pp._h, self._h, ptr(p0), len(p0), ptr(p1), len(p1), ptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_witness_free(h)
            self._h = None


@dataclass
class EvaluationPoint:
    p0: np.ndarray  # [row_log_len][3]
    p1: np.ndarray  # [column_log_len][3]


@dataclass
class RowEvaluation:
    values: np.ndarray  # [columns][3]


@dataclass
class FoldingChallenges:
    challenges: np.ndarray  # CHALLENGE_DTYPE [columns]

    def __len__(self):
        return len(self.challenges)


@dataclass
class FoldedWitness:
    elements: np.ndarray  # int16 [len_ring][648]


@dataclass
class OpeningMessage:
    """OpeningMessage (crates/pcs/src/scheme/verifier.rs): what the prover sends for the opening
    check; the Clear and bit-dropped arms are checked here (the recursive arm is not rebuilt)."""
    kind: str
    folded_commitment: "FoldedCommitment" = None
    folded_witness: FoldedWitness = None
    folded_row_value: np.ndarray = None

    @staticmethod
    def clear(folded_commitment, folded_witness, folded_row_value) -> "OpeningMessage":
        return OpeningMessage("clear", folded_commitment, folded_witness, folded_row_value)

    @staticmethod
    def bit_dropped(folded_witness, folded_row_value) -> "OpeningMessage":
        return OpeningMessage("bit_dropped", None, folded_witness, folded_row_value)


@dataclass
class FoldedCommitment:
    primes: List[int]
    rows: np.ndarray  # int16 [4][limbs][162]


@dataclass
class Commitment:
    """crates/pcs/src/scheme/commitment.rs:20-118: the matrix, or the bit-dropped digits."""

    primes: List[int]
    columns: int
    matrix: Optional[np.ndarray] = None
    top: Optional[np.ndarray] = None
    digits: Optional[np.ndarray] = None
    params: Optional["Params"] = None

    def moduli(self):
        return self.primes

    def rows(self):
        return 4

    def to_bytes(self) -> bytes:
        """wire::pack_tagged_commitment (crates/pcs/src/wire/mod.rs:307-333): the form's tag, the
        column count as a little-endian u32, then the matrix's i16 slots column by column, or the
        packed bit-dropped commitment."""
        head = struct.pack("<I", self.columns)
        if self.matrix is not None:
            return b"\x00" + head + np.ascontiguousarray(self.matrix, dtype="<i2").tobytes()
        if self.params is None:
            raise ValueError("a bit-dropped commitment packs against its parameters")
        top = np.ascontiguousarray(self.top, dtype=np.uint16)
        digits = np.ascontiguousarray(self.digits, dtype=np.uint16)
        cp = self.params.native()
        size = lib().lbg_params_pack_dropped(ctypes.byref(cp), ptr(top), ptr(digits), None, 0)
        out = np.zeros(size, np.uint8)
        lib().lbg_params_pack_dropped(ctypes.byref(cp), ptr(top), ptr(digits), ptr(out), size)
        return b"\x02" + head + out.tobytes()


def recursion_polys(columns: int) -> int:
    """Polynomials of a residue or left-expansion vector: three chunks per column, padded to a
    multiple of 32 (crates/pcs/src/recursion/limbs.rs:388, recursion/mod.rs PAD)."""
    return -(-3 * columns // 32) * 32


class CommitmentOpening:
    """The device handle a commitment leaves for the fold (crates/pcs/src/scheme/commitment.rs:120-139)."""

    def __init__(self, prover, handle):
        self.prover = prover
        self._h = handle

    def _take(self):
        h, self._h = self._h, None
        if h is None:
            raise ValueError("this opening was already consumed")
        return h

    def residues(self, polys: Optional[int] = None) -> np.ndarray:
        """recursion::limbs::residues of the commitment (crates/pcs/src/recursion/limbs.rs:379-398),
        computed on the device: int16 [limbs * 4][polys][64], polys = 3 x columns rounded up to a
        multiple of 32 by default. With the recursion on, the host's LaBRADOR bridge commits these
        as T_y."""
        if self._h is None:
            raise ValueError("this opening was already consumed")
        pr = self.prover.params
        polys = recursion_polys(pr.columns()) if polys is None else int(polys)
        out = np.zeros((len(pr.primes()) * 4, polys, 64), np.int16)
        check(lib().lbg_opening_residues(self._h, polys, ptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_opening_free(h)
            self._h = None


class Prover:
    """crates/pcs/src/scheme/prover.rs:21-135"""

    def __init__(self, pp: PublicParameters):
        self.pp = pp
        self.params = pp.params
        h = ctypes.c_void_p()
        check(lib().lbg_prover_new(pp._h, ctypes.byref(h)))
        self._h = h

    @staticmethod
    def new(pp: PublicParameters) -> "Prover":
        return Prover(pp)

    def commit(self, witness: Witness):
        if witness.params != self.params:
            raise ValueError("the witness was built for other parameters")
        pr = self.params
        L, r = len(pr.primes()), pr.columns()
        op = ctypes.c_void_p()
        if pr.dropped_bits():
            top = np.zeros(r * N, np.uint16)
            digits = np.zeros((max(L - 1, 1), r * N), np.uint16)
            check(lib().lbg_commit(self._h, witness._h, None, ptr(top), ptr(digits), ctypes.byref(op)))
            c = Commitment(pr.primes(), r, top=top, digits=digits[: L - 1], params=pr)
        else:
            m = np.zeros((r, 4, L, N162), np.int16)
            check(lib().lbg_commit(self._h, witness._h, ptr(m), None, None, ctypes.byref(op)))
            c = Commitment(pr.primes(), r, matrix=m, params=pr)
        return c, CommitmentOpening(self, op)

    def commit_left_expansion_vector(self, row: "RowEvaluation", rank: Optional[int] = None) -> np.ndarray:
        """Prover::commit_left_expansion's vector u (crates/pcs/src/scheme/prover.rs:95-115), made on the
        device: int16 [rank][64], chunk b of lift(u_j) at polynomial b x columns + j. rank is the
        recursion setup's ranks[U] (default: 3 x columns rounded up to a multiple of 32);
        T_u = key_u.commit_blocks(u) is LaBRADOR's, on the host."""
        pr = self.params
        r = pr.columns()
        rank = recursion_polys(r) if rank is None else int(rank)
        vals = np.ascontiguousarray(row.values, dtype=np.uint64).reshape(-1, 3)
        out = np.zeros((rank, 64), np.int16)
        check(lib().lbg_left_expansion(self.pp._h, ptr(vals), len(vals), rank, ptr(out)))
        return out

    def commit_elements(self, elements):
        """Witness::from_elements then Prover::commit in one call, the upload of the elements
        (uint64 [n][3]) pipelined against the commit: page-locked memory is copied directly,
        pageable memory through the prover's page-locked staging ring. Returns (witness,
        commitment, opening)."""
        pr = self.params
        e = np.ascontiguousarray(elements, dtype=np.uint64).reshape(-1, 3)
        if len(e) != pr.witness_len():
            raise WitnessError("WrongLength")
        L, r = len(pr.primes()), pr.columns()
        op, wh = ctypes.c_void_p(), ctypes.c_void_p()
        if pr.dropped_bits():
            top = np.zeros(r * N, np.uint16)
            digits = np.zeros((max(L - 1, 1), r * N), np.uint16)
            check(lib().lbg_commit_host(self._h, ptr(e), len(e), None, ptr(top), ptr(digits), ctypes.byref(wh),
                                        ctypes.byref(op)))
            c = Commitment(pr.primes(), r, top=top, digits=digits[: L - 1], params=pr)
        else:
            m = np.zeros((r, 4, L, N162), np.int16)
            check(lib().lbg_commit_host(self._h, ptr(e), len(e), ptr(m), None, None, ctypes.byref(wh),
                                        ctypes.byref(op)))
            c = Commitment(pr.primes(), r, matrix=m, params=pr)
        return Witness(self.pp, wh), c, CommitmentOpening(self, op)

    def keep_transform(self, enable: bool = True):
        """Keep the base limb's transform from commit for the fold, or transform the witness again
        in the fold (the default); the results are the same."""
        check(lib().lbg_prover_set_kept_transform(self._h, int(enable)))

    def recycle(self, opening: CommitmentOpening):
        lib().lbg_opening_free(opening._take())

    def fold(self, opening: CommitmentOpening, challenges: FoldingChallenges) -> FoldedWitness:
        ch = np.ascontiguousarray(challenges.challenges, dtype=CHALLENGE_DTYPE)
        v = np.zeros((self.params.len_ring(), N), np.int16)
        check(lib().lbg_fold(self._h, opening._take(), ptr(ch), len(ch), ptr(v)))
        return FoldedWitness(v)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_prover_free(h)
            self._h = None


class Transcript:
    """crates/pcs/src/challenge.rs:59-161 (host side of the library)."""

    def __init__(self, domain: bytes = None, _handle=None):
        if _handle is not None:
            self._h = _handle
        else:
            d = np.frombuffer(bytes(domain), dtype=np.uint8).copy() if domain else np.zeros(1, np.uint8)
            self._h = lib().lbg_transcript_new(ptr(d), len(domain or b""))

    @staticmethod
    def new(domain: bytes) -> "Transcript":
        return Transcript(domain)

    def clone(self) -> "Transcript":
        return Transcript(_handle=lib().lbg_transcript_clone(self._h))

    def absorb_bytes(self, b: bytes):
        a = np.frombuffer(bytes(b), dtype=np.uint8).copy() if b else np.zeros(1, np.uint8)
        lib().lbg_transcript_absorb_bytes(self._h, ptr(a), len(b))

    def absorb_u64(self, x: int):
        lib().lbg_transcript_absorb_u64(self._h, x)

    def fill(self, label: bytes, n: int) -> bytes:
        out = np.zeros(max(n, 1), np.uint8)
        lib().lbg_transcript_fill(self._h, label, ptr(out), n)
        return out[:n].tobytes()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_transcript_free(h)
            self._h = None


def sample_short_challenge(t: Transcript, weight=DEFAULT_WEIGHT, bound=DEFAULT_BOUND):
    """crates/pcs/src/challenge.rs:517-533: (challenge, attempts)."""
    out = np.zeros(1, CHALLENGE_DTYPE)
    att = np.zeros(1, np.uint64)
    check(lib().lbg_sample_short_challenge(t._h, weight, bound, ptr(out), ptr(att)))
    return out[0], int(att[0])


def _f162_eq(a, b) -> bool:
    return bool(np.array_equal(np.asarray(a, np.uint64), np.asarray(b, np.uint64)))


class Verifier:
    """crates/pcs/src/scheme/verifier.rs:21-146"""

    def __init__(self, pp: PublicParameters):
        self.pp = pp
        self.params = pp.params

    @staticmethod
    def new(pp: PublicParameters) -> "Verifier":
        return Verifier(pp)

    def derive_evaluation_point(self, transcript: Transcript, commitment: Commitment) -> EvaluationPoint:
        pr = self.params
        p0 = np.zeros((pr.row_log_len(), 3), np.uint64)
        p1 = np.zeros((pr.column_log_len, 3), np.uint64)
        if pr.dropped_bits():
            d = commitment.digits if len(pr.primes()) > 1 else np.zeros(1, np.uint16)
            check(lib().lbg_derive_evaluation_point(self.pp._h, transcript._h, None, ptr(commitment.top),
                                                    ptr(np.ascontiguousarray(d, np.uint16)), ptr(p0), ptr(p1)))
        else:
            check(lib().lbg_derive_evaluation_point(self.pp._h, transcript._h,
                                                    ptr(np.ascontiguousarray(commitment.matrix, np.int16)),
                                                    None, None, ptr(p0), ptr(p1)))
        return EvaluationPoint(p0, p1)

    def derive_folding_challenges(self, transcript: Transcript, source: RowEvaluation) -> FoldingChallenges:
        out = np.zeros(self.params.columns(), CHALLENGE_DTYPE)
        u = np.ascontiguousarray(source.values, dtype=np.uint64)
        check(lib().lbg_derive_folding_challenges(self.pp._h, transcript._h, ptr(u), ptr(out)))
        return FoldingChallenges(out)

    def fold_commitment(self, commitment: Commitment, challenges: FoldingChallenges) -> FoldedCommitment:
        if len(challenges) != commitment.columns:
            raise ValueError("one challenge per column")
        if commitment.matrix is None:
            raise ValueError("a bit-dropped commitment is its digits, not the matrix")
        L = len(self.params.primes())
        out = np.zeros((4, L, N162), np.int16)
        ch = np.ascontiguousarray(challenges.challenges, dtype=CHALLENGE_DTYPE)
        check(lib().lbg_fold_commitment(self.pp._h, ptr(np.ascontiguousarray(commitment.matrix, np.int16)),
                                        commitment.columns, ptr(ch), len(ch), ptr(out)))
        return FoldedCommitment(self.params.primes(), out)

    def fold_row_evaluation(self, row_evaluation: RowEvaluation, challenges: FoldingChallenges) -> np.ndarray:
        """u' = sum_j (c_j mod 2) u_j (crates/pcs/src/scheme/verifier.rs:148-154), on the device."""
        u = np.ascontiguousarray(row_evaluation.values, dtype=np.uint64)
        ch = np.ascontiguousarray(challenges.challenges, dtype=CHALLENGE_DTYPE)
        if len(u) != self.params.columns() or len(ch) != len(u):
            raise ValueError("one challenge per column")
        out = np.zeros(3, np.uint64)
        check(lib().lbg_fold_row_evaluation(self.pp._h, ptr(u), ptr(ch), len(ch), ptr(out)))
        return out

    def verify_evaluation(self, point: EvaluationPoint, claimed_value, row_evaluation: RowEvaluation):
        """The claim check u . eq(p1) == t (crates/pcs/src/scheme/verifier.rs:157-174), on the device;
        raises VerificationError on rejection."""
        u = np.ascontiguousarray(row_evaluation.values, dtype=np.uint64)
        p1 = np.ascontiguousarray(point.p1, dtype=np.uint64)
        t = np.ascontiguousarray(claimed_value, dtype=np.uint64)
        ok = ctypes.c_int(0)
        check(lib().lbg_verify_evaluation(self.pp._h, ptr(p1), len(p1), ptr(t), ptr(u), len(u), ctypes.byref(ok)))
        if not ok.value:
            raise VerificationError("Rejected")

    def verify_folded_opening(self, folded_commitment: FoldedCommitment, folded_witness: FoldedWitness,
                              point: EvaluationPoint, folded_row_value):
        """The Clear opening check (crates/pcs/src/scheme/verifier.rs:178-231) on the device: v in
        range and within the norm cap, A v equal to the folded commitment on every modulus, and
        eq(p0) . (v mod 2) equal to u'. Raises VerificationError on rejection."""
        if list(folded_commitment.primes) != self.params.primes():
            raise VerificationError("Rejected")
        v = np.ascontiguousarray(folded_witness.elements, dtype=np.int16)
        if v.shape != (self.params.len_ring(), 648):
            raise VerificationError("Rejected")
        fc = np.ascontiguousarray(folded_commitment.rows, dtype=np.int16)
        p0 = np.ascontiguousarray(point.p0, dtype=np.uint64)
        fr = np.ascontiguousarray(folded_row_value, dtype=np.uint64)
        ok = ctypes.c_int(0)
        check(lib().lbg_verify_folded_opening(self.pp._h, ptr(fc), ptr(v), ptr(p0), len(p0), ptr(fr),
                                              ctypes.byref(ok)))
        if not ok.value:
            raise VerificationError("Rejected")

    def bd_residual(self, commitment: Commitment, challenges: FoldingChallenges, folded_witness: FoldedWitness,
                    point: EvaluationPoint, folded_row_value):
        """The bit-dropped opening check (crates/pcs/src/scheme/verifier.rs:232-276) on the device:
        returns (accepted, the squared norm of the residual, crates/pcs/src/bd/residual.rs:66-130)."""
        v = np.ascontiguousarray(folded_witness.elements, dtype=np.int16)
        if v.shape != (self.params.len_ring(), 648) or commitment.top is None:
            return False, None
        if list(commitment.primes) != self.params.primes():
            return False, None
        top = np.ascontiguousarray(commitment.top, dtype=np.uint16)
        digits = np.ascontiguousarray(commitment.digits, dtype=np.uint16)
        ch = np.ascontiguousarray(challenges.challenges, dtype=CHALLENGE_DTYPE)
        p0 = np.ascontiguousarray(point.p0, dtype=np.uint64)
        fr = np.ascontiguousarray(folded_row_value, dtype=np.uint64)
        ok = ctypes.c_int(0)
        res = np.zeros(2, np.uint64)
        check(lib().lbg_verify_folded_opening_bd(self.pp._h, ptr(top), ptr(digits) if digits.size else None, ptr(ch),
                                                 len(ch), ptr(v), ptr(p0), len(p0), ptr(fr), ctypes.byref(ok),
                                                 ptr(res)))
        return bool(ok.value), int(res[0]) | (int(res[1]) << 64)

    def verify_opening(self, commitment: Commitment, challenges: FoldingChallenges, point: EvaluationPoint,
                       message: "OpeningMessage"):
        """crates/pcs/src/scheme/verifier.rs:280-337: the check the parameters' opening mode names.
        Opening::Clear and BitDropped run on the device; the recursive arm is not rebuilt."""
        if self.params.opening.kind != message.kind:
            raise VerificationError("Rejected")
        if message.kind == "clear":
            self.verify_folded_opening(message.folded_commitment, message.folded_witness, point,
                                       message.folded_row_value)
        elif message.kind == "bit_dropped":
            if commitment.params is not None and commitment.params.dropped_bits() != self.params.dropped_bits():
                raise VerificationError("Rejected")
            ok, _ = self.bd_residual(commitment, challenges, message.folded_witness, point, message.folded_row_value)
            if not ok:
                raise VerificationError("Rejected")
        else:
            raise NotImplementedError(f"the {message.kind} opening check is not on the device")
