"""Shared helpers of the parity tests: the golden fixtures and a reference round through the
product API (labinius_b200) for comparison with them."""
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MATRIX_SEED = bytes([0x5A]) * 32
WITNESS_SEED = bytes([0xC7]) * 32
DOMAIN = b"labinius/reference"
CHALLENGE_BYTES = 40


def fixtures():
    return sorted(glob.glob(os.path.join(HERE, "golden", "round_*.npz")))


def load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    wl, cl, dropped, *primes = [int(x) for x in d["params"]]
    d["shape"] = (wl, cl, primes, dropped)
    return d


def product_params(shape):
    from labinius_b200 import Modulus, Opening, Params

    wl, cl, primes, dropped = shape
    op = Opening.bit_dropped(dropped) if dropped else Opening.clear()
    return Params.with_base(wl, cl, Modulus(primes[0]), [Modulus(q) for q in primes[1:]], op)


def product_round(shape, matrix_seed=MATRIX_SEED, witness_seed=WITNESS_SEED, witness=None):
    """crates/bench/src/bin/labinius.rs:104-130 through the B200 path."""
    import labinius_b200 as L

    params = product_params(shape)
    pp = L.PublicParameters.from_seed(params, matrix_seed)
    w = L.Witness.random(pp, witness_seed) if witness is None else L.Witness.from_elements(pp, witness)
    prover = L.Prover(pp)
    verifier = L.Verifier(pp)
    commitment, opening = prover.commit(w)
    t = L.Transcript(DOMAIN)
    point = verifier.derive_evaluation_point(t, commitment)
    mle = w.mle_evaluate(point)
    row = w.row_evaluate(point)
    ch = verifier.derive_folding_challenges(t, row)
    v = prover.fold(opening, ch)
    out = dict(pp=pp, witness=w, commitment=commitment, p0=point.p0, p1=point.p1, u=row.values, mle=mle,
               challenges=ch.challenges, v=v.elements, tail=t.fill(b"labinius/test-tail", 32))
    if not params.dropped_bits():
        out["folded_commitment"] = verifier.fold_commitment(commitment, ch).rows
    return out
