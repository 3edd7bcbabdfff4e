"""Batched rounds over the C ABI's lbg_batch: many independent witnesses under one key.

Every instance shares the public parameters' column length, moduli and opening mode; instance i
has 2^column_log_lens[i] columns, i.e. it is a round of
``Params(row_log_len + column_log_lens[i], column_log_lens[i], same moduli)``. Each device stage
(commit, row evaluation, fold) is one launch over all instances; the host steps of the round
(evaluation point, folding challenges) run per instance in the library's host code.
"""
import ctypes
from dataclasses import dataclass
from typing import List

import numpy as np

from . import _native as nat
from ._native import check, lib, ptr
from .scheme import CHALLENGE_DTYPE, N, N162, Params, PublicParameters

_CH = CHALLENGE_DTYPE


def _pinned(shape, dtype):
    """A page-locked host array (torch's caching host allocator keeps the blocks for reuse), so the
    device-to-host copies of a round run at full link speed; falls back to pageable memory when
    no CUDA device is visible."""
    try:
        import torch

        if torch.cuda.is_available():
            n = int(np.prod(shape)) * np.dtype(dtype).itemsize
            return torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy().view(dtype).reshape(shape)
    except ImportError:
        pass
    return np.zeros(shape, dtype)


@dataclass
class InstanceRound:
    matrix: np.ndarray = None  # int16 [cols][4][limbs][162] (Clear)
    top: np.ndarray = None     # uint16 [cols*648] (bit-dropped)
    digits: np.ndarray = None  # uint16 [limbs-1][cols*648]
    p0: np.ndarray = None
    p1: np.ndarray = None
    u: np.ndarray = None
    mle: np.ndarray = None
    challenges: np.ndarray = None
    v: np.ndarray = None
    switch: object = None      # SwitchProof of a B128 instance opened through the switch
    claim: np.ndarray = None   # its B128 claim (uint64 [2])


class Batch:
    def __init__(self, pp: PublicParameters, column_log_lens=None, capacity=None):
        """A batch of the given instances, or (capacity=(max_columns, max_instances)) an empty arena
        that `assign` lays instances out in."""
        self.pp = pp
        self.row_log = pp.params.row_log_len()
        self.wdim = 1 << self.row_log
        self.len_ring = self.wdim // 4
        self.limbs = len(pp.params.primes())
        self.dropped = pp.params.dropped_bits()
        h = ctypes.c_void_p()
        if capacity is not None:
            check(lib().lbg_batch_new_capacity(pp._h, int(capacity[0]), int(capacity[1]), ctypes.byref(h)))
            self._h = h
            self.capacity = (int(capacity[0]), int(capacity[1]))
            self._layout([])
            if column_log_lens is not None:
                self.assign(column_log_lens)
            return
        arr = np.array([int(c) for c in column_log_lens], np.uint32)
        check(lib().lbg_batch_new(pp._h, ptr(arr), len(arr), ctypes.byref(h)))
        self._h = h
        self.capacity = (sum(1 << int(c) for c in column_log_lens), len(arr))
        self._layout(column_log_lens)

    def _layout(self, column_log_lens):
        self.column_log_lens = [int(c) for c in column_log_lens]
        self.count = len(self.column_log_lens)
        self.cols = [1 << c for c in self.column_log_lens]
        self.col_off = np.concatenate([[0], np.cumsum(self.cols)]).astype(np.int64)
        self.total_cols = int(self.col_off[-1])
        self.switch_flags = []

    def assign(self, column_log_lens):
        arr = np.array([int(c) for c in column_log_lens], np.uint32)
        check(lib().lbg_batch_assign(self._h, ptr(arr), len(arr)))
        self._layout(column_log_lens)

    def set_switch(self, flags=None, r_his=None, claims=None):
        """Mark instances as B128 traces (Witness::lifted, kind 1 of witness_random) that the device
        round opens through the cross-field switch, as crates/pcs/examples/two_fields.rs:176-194
        does: commit, absorb Commitment::to_bytes, switch::prove, row_evaluate at the switch's
        point, FoldingChallenges::derive, fold. r_his: one array of witness_log_len B128
        coordinates ([l][2] uint64) per marked instance, in order; claims: one B128 per marked
        instance, or None (each instance states its trace's value at its point). None unmarks."""
        if flags is None:
            check(lib().lbg_batch_set_switch(self._h, None, None, None))
            self.switch_flags = [0] * self.count
            return
        f = np.ascontiguousarray([1 if x else 0 for x in flags], np.uint8)
        if len(f) != self.count:
            raise ValueError("one flag per instance")
        marked = [i for i in range(self.count) if f[i]]
        if len(r_his) != len(marked):
            raise ValueError("one point per marked instance")
        for k, i in enumerate(marked):
            if np.asarray(r_his[k]).size != 2 * (self.row_log + self.column_log_lens[i]):
                raise ValueError("the point does not match the instance")
        r = np.ascontiguousarray(np.concatenate([np.asarray(x, np.uint64).reshape(-1) for x in r_his])
                                 if marked else np.zeros(2, np.uint64))
        c = None if claims is None else np.ascontiguousarray(np.asarray(claims, np.uint64).reshape(-1, 2))
        check(lib().lbg_batch_set_switch(self._h, ptr(f), ptr(r), ptr(c)))
        self.switch_flags = list(f)

    def params_of(self, i) -> Params:
        p = self.pp.params
        return Params(self.row_log + self.column_log_lens[i], self.column_log_lens[i], p.base, list(p.extra_moduli),
                      p.opening)

    def witness_random(self, seeds: List[bytes], kinds=None):
        """kinds[i] = 0: Witness::random(seeds[i]); 1: a B128 trace from seeds[i], lifted."""
        s = np.frombuffer(b"".join(bytes(x) for x in seeds), dtype=np.uint8).copy()
        assert len(s) == 32 * self.count
        k = None if kinds is None else np.ascontiguousarray(kinds, dtype=np.uint8)
        check(lib().lbg_batch_witness_generate(self._h, ptr(s), ptr(k)))

    def witness_upload(self, i, elements):
        e = np.ascontiguousarray(elements, dtype=np.uint64).reshape(-1, 3)
        check(lib().lbg_batch_witness_upload(self._h, i, ptr(e), len(e)))

    def elements(self, i) -> np.ndarray:
        out = np.zeros((self.cols[i] * self.wdim, 3), np.uint64)
        check(lib().lbg_batch_witness_download(self._h, i, ptr(out), len(out)))
        return out

    def use_graphs(self, enable=True):
        check(lib().lbg_batch_use_graphs(self._h, int(enable)))

    def set_sm_limit(self, ctas=0):
        """At most `ctas` CTAs (one per SM; 0: every SM) for the persistent commit and fold launches."""
        check(lib().lbg_batch_set_sm_limit(self._h, int(ctas)))

    def set_priority(self, high=True):
        """Run the batch's stream at the device's greatest priority (or the default)."""
        check(lib().lbg_batch_set_priority(self._h, int(high)))

    def keep_transform(self, enable=True):
        """The fold reads the commit's kept transform (on) or transforms the witness again (off)."""
        check(lib().lbg_batch_set_kept_transform(self._h, int(enable)))

    def autotune(self):
        c, f = ctypes.c_uint32(), ctypes.c_uint32()
        check(lib().lbg_batch_autotune(self._h, ctypes.byref(c), ctypes.byref(f)))
        w, k = ctypes.c_uint32(), ctypes.c_int()
        check(lib().lbg_batch_schedule(self._h, ctypes.byref(w), ctypes.byref(k)))
        return {"commit_chunks": c.value, "fold_columns_per_split": f.value, "commit_warps": w.value,
                "kept_transform": bool(k.value)}

    def commit(self) -> List[InstanceRound]:
        C, L = self.total_cols, self.limbs
        out = [InstanceRound() for _ in range(self.count)]
        if self.dropped:
            top = np.zeros(C * N, np.uint16)
            dig = np.zeros((max(L - 1, 1), C * N), np.uint16)
            check(lib().lbg_batch_commit(self._h, None, ptr(top), ptr(dig)))
            for i in range(self.count):
                a, b = self.col_off[i] * N, self.col_off[i + 1] * N
                out[i].top, out[i].digits = top[a:b].copy(), dig[: L - 1, a:b].copy()
        else:
            m = np.zeros((C, 4, L, N162), np.int16)
            check(lib().lbg_batch_commit(self._h, ptr(m), None, None))
            for i in range(self.count):
                out[i].matrix = m[self.col_off[i]:self.col_off[i + 1]].copy()
        return out

    def commit_device(self):
        """The commit stage with the results left on the device (for timing)."""
        check(lib().lbg_batch_commit(self._h, None, None, None))

    def row_evaluate(self, p0s) -> List[np.ndarray]:
        p0 = np.ascontiguousarray(np.stack([np.asarray(p, np.uint64) for p in p0s]))
        u = np.zeros((self.total_cols, 3), np.uint64)
        check(lib().lbg_batch_row_evaluate(self._h, ptr(p0), ptr(u)))
        return [u[self.col_off[i]:self.col_off[i + 1]].copy() for i in range(self.count)]

    def mle_evaluate(self, p0s, p1s) -> List[np.ndarray]:
        p0 = np.ascontiguousarray(np.stack([np.asarray(p, np.uint64) for p in p0s]))
        p1 = np.ascontiguousarray(np.concatenate([np.asarray(p, np.uint64).reshape(-1, 3) for p in p1s]))
        out = np.zeros((self.count, 3), np.uint64)
        check(lib().lbg_batch_mle_evaluate(self._h, ptr(p0), ptr(p1), ptr(out)))
        return [out[i].copy() for i in range(self.count)]

    def fold(self, challenges, read_back=True):
        ch = np.ascontiguousarray(np.concatenate([np.asarray(c, _CH) for c in challenges]), dtype=_CH)
        v = np.zeros((self.count, self.len_ring, N), np.int16) if read_back else None
        check(lib().lbg_batch_fold(self._h, ptr(ch), len(ch), ptr(v)))
        return [v[i] for i in range(self.count)] if read_back else None

    def _point(self, i, r, domain):
        """Host: a fresh transcript for instance i, the commitment absorbed, the evaluation point."""
        seed = np.frombuffer(self.pp.matrix_seed, np.uint8).copy()
        d = np.frombuffer(domain, np.uint8).copy()
        pn = self.params_of(i).native()
        t = lib().lbg_transcript_new(ptr(d), len(domain))
        r.p0 = np.zeros((self.row_log, 3), np.uint64)
        r.p1 = np.zeros((self.column_log_lens[i], 3), np.uint64)
        if self.dropped:
            dig = r.digits if self.limbs > 1 else np.zeros(1, np.uint16)
            check(lib().lbg_params_derive_evaluation_point(ctypes.byref(pn), ptr(seed), t, None, ptr(r.top),
                                                           ptr(np.ascontiguousarray(dig)), ptr(r.p0), ptr(r.p1)))
        else:
            check(lib().lbg_params_derive_evaluation_point(ctypes.byref(pn), ptr(seed), t, ptr(r.matrix), None,
                                                           None, ptr(r.p0), ptr(r.p1)))
        return t

    def _challenges(self, i, r, t):
        """Host: absorb instance i's row values and sample its folding challenges."""
        pn = self.params_of(i).native()
        r.challenges = np.zeros(self.cols[i], _CH)
        check(lib().lbg_params_derive_folding_challenges(ctypes.byref(pn), t, ptr(r.u), ptr(r.challenges)))
        lib().lbg_transcript_free(t)

    def round(self, domain=b"labinius/reference", pool=None, transcript="device", copy=True) -> List[InstanceRound]:
        """commit -> per instance: evaluation point -> row and mle evaluation -> per instance: folding
        challenges -> fold, each instance with a fresh Transcript(domain).

        transcript="device": the whole round in one pass on the device (the absorbs, the point and
        the challenge sampler are device kernels; lbg_batch_round). transcript="host": the
        transcript steps run in the library's host code between the device stages, on `pool` (a
        concurrent.futures executor; the calls release the GIL) or instance by instance.
        copy=False (device transcript) returns views into the batch's page-locked output buffers,
        valid until its next round."""
        if transcript == "device":
            return self._round_device(domain, copy)
        if any(getattr(self, "switch_flags", [])):
            raise ValueError("switch instances run their transcript on the device")
        rounds = self.commit()
        run = (lambda f, xs: list(pool.map(f, xs))) if pool is not None else (lambda f, xs: [f(x) for x in xs])
        ts = run(lambda i: self._point(i, rounds[i], domain), range(self.count))
        mles = self.mle_evaluate([r.p0 for r in rounds], [r.p1 for r in rounds])
        us = self.row_evaluate([r.p0 for r in rounds])
        for i, r in enumerate(rounds):
            r.mle, r.u = mles[i], us[i]
        run(lambda i: self._challenges(i, rounds[i], ts[i]), range(self.count))
        vs = self.fold([r.challenges for r in rounds])
        for i, r in enumerate(rounds):
            r.v = vs[i]
        return rounds

    def _outputs(self):
        """Page-locked output buffers sized for the arena, allocated once per batch."""
        if getattr(self, "_out", None) is None:
            Cm, Im, L = self.capacity[0], self.capacity[1], self.limbs
            o = {"p0": _pinned((Im * self.row_log * 3,), np.uint64), "p1": _pinned((Im * 32 * 3,), np.uint64),
                 "mle": _pinned((Im * 3,), np.uint64), "u": _pinned((Cm * 3,), np.uint64),
                 "ch": _pinned((Cm * _CH.itemsize,), np.uint8), "v": _pinned((Im * self.len_ring * N,), np.int16)}
            if self.dropped:
                o["top"] = _pinned((Cm * N,), np.uint16)
                o["dig"] = _pinned((max(L - 1, 1) * Cm * N,), np.uint16)
            else:
                o["m"] = _pinned((Cm * 4 * L * N162,), np.int16)
            self._out = o
        return self._out

    def _round_device(self, domain, copy=True) -> List[InstanceRound]:
        C, L, I = self.total_cols, self.limbs, self.count
        o = self._outputs()
        out = nat.lbg_batch_outputs()
        m = top = dig = None
        if self.dropped:
            top = o["top"][: C * N]
            dig = o["dig"][: max(L - 1, 1) * C * N].reshape(max(L - 1, 1), C * N)
            out.top, out.digits = ptr(top).value, ptr(dig).value
        else:
            m = o["m"][: C * 4 * L * N162].reshape(C, 4, L, N162)
            out.matrix = ptr(m).value
        p0 = o["p0"][: I * self.row_log * 3].reshape(I, self.row_log, 3)
        p1 = o["p1"][: sum(self.column_log_lens) * 3].reshape(-1, 3)
        mle = o["mle"][: I * 3].reshape(I, 3)
        u = o["u"][: C * 3].reshape(C, 3)
        ch = o["ch"][: C * _CH.itemsize].view(_CH)
        v = o["v"][: I * self.len_ring * N].reshape(I, self.len_ring, N)
        for name, a in (("p0", p0), ("p1", p1), ("mle", mle), ("u", u), ("challenges", ch), ("v", v)):
            setattr(out, name, ptr(a).value)
        d = np.frombuffer(bytes(domain), np.uint8).copy()
        check(lib().lbg_batch_round(self._h, ptr(d), len(d), ctypes.byref(out)))
        rounds = []
        po = 0
        for i in range(I):
            a, b = int(self.col_off[i]), int(self.col_off[i + 1])
            r = InstanceRound()
            if self.dropped:
                r.top, r.digits = top[a * N:b * N], dig[: L - 1, a * N:b * N]
            else:
                r.matrix = m[a:b]
            cl = self.column_log_lens[i]
            r.p0, r.p1 = p0[i], p1[po:po + cl]
            po += cl
            r.mle, r.u, r.challenges, r.v = mle[i], u[a:b], ch[a:b], v[i]
            if copy:
                for k, val in vars(r).items():
                    if val is not None:
                        setattr(r, k, np.array(val))
            rounds.append(r)
        self._attach_switch(rounds)
        return rounds

    def _attach_switch(self, rounds):
        from .switch import SwitchProof

        marked = [i for i, f in enumerate(getattr(self, "switch_flags", [])) if f]
        if not marked:
            return
        ls = [self.row_log + self.column_log_lens[i] for i in marked]
        partials = np.zeros((len(marked), 128, 2), np.uint64)
        rs = np.zeros((sum(ls), 2, 3), np.uint64)
        opened = np.zeros((len(marked), 3), np.uint64)
        claims = np.zeros((len(marked), 2), np.uint64)
        check(lib().lbg_batch_switch_outputs(self._h, ptr(partials), ptr(rs), ptr(opened), ptr(claims)))
        o = 0
        for k, i in enumerate(marked):
            rounds[i].switch = SwitchProof(partials[k], rs[o:o + ls[k]], opened[k])
            rounds[i].claim = claims[k]
            o += ls[k]

    def launch_count(self) -> int:
        return int(lib().lbg_batch_launch_count(self._h))

    def stream(self):
        return lib().lbg_batch_stream(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and nat is not None and getattr(nat, "_lib", None) is not None:
            nat._lib.lbg_batch_free(h)
            self._h = None
