"""labinius_b200 — the labinius prover hot path (commit, evaluate, fold) on B200 (sm_100a).

The compute lives in ``liblabinius_gpu.so`` (CUDA kernels behind the C ABI of
include/labinius_gpu.h); this package is the Python mirror of the reference's scheme API over it.
"""
from .scheme import (  # noqa: F401
    CHALLENGE_DTYPE,
    SUITES,
    Commitment,
    CommitmentOpening,
    EvaluationPoint,
    FoldedCommitment,
    FoldedWitness,
    FoldingChallenges,
    Modulus,
    Opening,
    OpeningMessage,
    ParamError,
    Params,
    Prover,
    PublicParameters,
    RowEvaluation,
    Suite,
    Transcript,
    VerificationError,
    Verifier,
    Witness,
    WitnessError,
    sample_short_challenge,
    suite_from_flag,
)
