"""Generate the golden round fixtures (tests/golden/round_*.npz) from the CPU oracle.

Each fixture is one reference round (crates/bench/src/bin/labinius.rs:104-130) at a small shape:
commitment (matrix or bit-dropped digits), evaluation point, row evaluation, claim, folding
challenges, folded witness, folded commitment, and 32 bytes of the transcript after the round.
The oracle's BLAKE3-derived inputs (witness, key seed) are checked against the Python `blake3`
package before anything is written. Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import blake3
import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
MATRIX_SEED = bytes([0x5A]) * 32
WITNESS_SEED = bytes([0xC7]) * 32

# name: (witness_log_len, column_log_len, primes (base first), dropped_bits)
CONFIGS = {
    "small": (11, 3, [3889, 9721], 0),            # crates/pcs/tests/common/mod.rs:115-123
    "quadbase": (11, 3, [2917, 3889, 9721], 0),
    "bd9": (12, 4, [3889, 2917, 4861], 9),        # the bit-dropped limb list of suites m/l/xl
    "large": (11, 2, [12637, 17497, 19441], 0),
    "b4861": (11, 3, [4861, 9721], 0),
}


def digest(a) -> bytes:
    return blake3.blake3(np.ascontiguousarray(a).tobytes()).digest()


def make(name, cfg):
    wl, cl, primes, d = cfg
    P = O.Params(wl, cl, primes, d)
    w = O.witness_random(P.witness_len, WITNESS_SEED)
    raw = blake3.blake3(b"labinius/witness", key=WITNESS_SEED).digest(length=24 * P.witness_len)
    want = np.frombuffer(raw, dtype=np.uint64).reshape(-1, 3).copy()
    want[:, 2] &= (1 << 34) - 1
    assert (w == want).all(), "oracle witness disagrees with blake3"
    assert O.key_seed(MATRIX_SEED) == int.from_bytes(blake3.blake3(MATRIX_SEED).digest()[:8], "little")
    r = O.round_trip(P, MATRIX_SEED, witness=w)
    out = dict(params=np.array([wl, cl, d, *primes], np.int64), A_digest=np.frombuffer(digest(r["A"]), np.uint8),
               A_head=r["A"][:, 0, :].copy(), p0=r["p0"], p1=r["p1"], u=r["u"], mle=r["mle"],
               challenges=r["challenges"].view(np.uint8).reshape(len(r["challenges"]), 40), v=r["v"],
               tail=np.frombuffer(r["transcript_tail"], np.uint8))
    if d:
        out.update(top=r["top"], digits=r["digits"], packed=np.frombuffer(r["packed"], np.uint8))
    else:
        out.update(C=r["C"], folded_commitment=r["folded_commitment"])
    path = os.path.join(HERE, f"round_{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    O.build.build()
    for name, cfg in CONFIGS.items():
        make(name, cfg)
