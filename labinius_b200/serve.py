"""Serving: a request loop with continuous batching over device arenas.

A request is one commit + open round of its own witness under the server's key: any column
count 2^c with the key's column length, a witness drawn from the request's seed. Kind 0 is
Witness::random (crates/pcs/src/scheme/witness.rs:66-87), opened as the plain round does (commit,
evaluation point, mle and row evaluation, folding challenges, fold). Kind 1 is a B128 trace,
committed lifted (crates/pcs/src/scheme/witness.rs:45-52) and opened through the cross-field
switch at the request's point r (crates/pcs/examples/two_fields.rs:176-194: commit, the tagged
commitment absorbed, switch::prove of the trace's value at r, row evaluation at the switch's
point, folding challenges, fold); its result carries the switch proof and the claim.

Continuous batching: the server owns `slots` device arenas (lbg_batch, sized once). Each slot's
arena fits `hbm_fraction` of the device's free memory split over the slots (cudaMemGetInfo through
lbg_device_memory, and lbg_batch_arena_bytes per arena); a given `capacity_columns` (the most
columns one batch runs, a latency bound) caps it further. Admission is by arena room, i.e. by the
HBM each slot reserved, and by size class: with `small_log_len` set, requests of at most
2^small_log_len columns are small; slot 0 runs small requests only, the other slots run the large
ones and take small ones when no large request waits, so a small request never queues behind a
batch of large ones; the small slot's stream runs at the device's greatest priority, so its launches
take SMs ahead of a large batch's once those free up, and with `large_sm_limit` the large slots'
persistent commit and fold launches take at most that many SMs, so the small slot never waits for
one of them to end. Whenever a slot is free it admits, in arrival order within its class, every
queued request that fits, lays them out in the arena and runs their rounds together:
each device stage is one launch over all of them, and the transcripts (absorbs, evaluation point,
challenge sampling) run on the device too (lbg_batch_round), so a batch is one pass on the
slot's stream from witness generation to the folded witnesses. While one slot reads its results
back and lays out its next batch, the other slot's round runs on its own stream: requests that
arrive while others are on the GPU are admitted as soon as a slot and its memory free up, and
their work overlaps on the device. The parameters, the key and each slot's state stay resident.
With transcript="host" (kind 0 requests only) the transcript steps run in the library's host code
on a thread pool.
"""
import collections
import concurrent.futures
import hashlib
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .batch import Batch, InstanceRound
from .scheme import PublicParameters


@dataclass
class Request:
    column_log_len: int
    seed: bytes
    kind: int = 0               # 0: Witness::random(seed); 1: lifted B128 trace from seed, opened through the switch
    point: Optional[np.ndarray] = None  # kind 1: r, [witness_log_len][2] uint64 (default: drawn from the seed)
    arrival: float = 0.0        # seconds on the server's clock
    admitted: float = 0.0
    done: float = 0.0
    result: Optional[InstanceRound] = None
    error: Optional[str] = None
    _event: threading.Event = field(default_factory=threading.Event, repr=False)

    def wait(self, timeout=None):
        return self._event.wait(timeout)

    @property
    def latency(self):
        return self.done - self.arrival


def arena_columns(pp: PublicParameters, hbm_fraction: float, slots: int, max_requests: int,
                  max_columns: int = 1 << 16) -> int:
    """The columns each of `slots` arenas can hold in `hbm_fraction` of the device's free memory (a
    power of two, at most max_columns): free bytes from lbg_device_memory, bytes per arena from
    lbg_batch_arena_bytes."""
    import ctypes

    from ._native import check, lib

    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    check(lib().lbg_device_memory(pp._h, ctypes.byref(free), ctypes.byref(total)))
    budget = hbm_fraction * free.value / slots
    cols = 1
    while cols * 2 <= max_columns and lib().lbg_batch_arena_bytes(pp._h, cols * 2, max_requests) <= budget:
        cols *= 2
    return cols


class Server:
    def __init__(self, pp: PublicParameters, capacity_columns: Optional[int] = None, max_requests: int = 256,
                 slots: int = 2, host_threads: int = 16, domain: bytes = b"labinius/reference",
                 keep_results: bool = True, transcript: str = "device", hbm_fraction: float = 0.5,
                 small_log_len: Optional[int] = None, large_sm_limit: int = 0, small_slot_takes_large: bool = False):
        self.pp = pp
        self.memory_columns = arena_columns(pp, hbm_fraction, slots, max_requests)
        self.capacity = self.memory_columns if capacity_columns is None else min(capacity_columns, self.memory_columns)
        self.max_requests = max_requests
        self.domain = domain
        self.keep_results = keep_results
        self.transcript = transcript
        self.small_log_len = small_log_len if slots >= 2 else None
        self.small_slot_takes_large = small_slot_takes_large
        self.slots = [Batch(pp, capacity=(self.capacity, max_requests)) for _ in range(slots)]
        if self.small_log_len is not None:
            # the small requests' slot is scheduled ahead of the large ones' when both wait for SMs,
            # and the large ones' persistent launches leave SMs free for it (large_sm_limit CTAs)
            self.slots[0].set_priority(True)
            for b in self.slots[1:]:
                b.set_sm_limit(large_sm_limit)
        self.pool = concurrent.futures.ThreadPoolExecutor(host_threads)
        self.small = collections.deque()  # every request when no size classes are set
        self.large = collections.deque()
        self.cv = threading.Condition()
        self.stop = False
        self.t0 = time.perf_counter()
        self.batches = 0
        self.workers = [threading.Thread(target=self._work, args=(b, i), daemon=True) for i, b in enumerate(self.slots)]
        for w in self.workers:
            w.start()

    def clock(self):
        return time.perf_counter() - self.t0

    def switch_point(self, req: Request) -> np.ndarray:
        """The B128 point a kind-1 request is opened at: its own, or SHAKE256 of its seed."""
        l = self.pp.params.row_log_len() + req.column_log_len
        if req.point is not None:
            return np.ascontiguousarray(req.point, dtype=np.uint64).reshape(l, 2)
        raw = hashlib.shake_256(bytes(req.seed) + b"labinius/served-point").digest(16 * l)
        return np.frombuffer(raw, dtype="<u8").reshape(l, 2).copy()

    def submit(self, req: Request) -> Request:
        if (1 << req.column_log_len) > self.capacity:
            req.error = "request larger than a slot"
            req.done = self.clock()
            req._event.set()
            return req
        with self.cv:
            if not req.arrival:
                req.arrival = self.clock()
            if self.small_log_len is None or req.column_log_len <= self.small_log_len:
                self.small.append(req)
            else:
                self.large.append(req)
            self.cv.notify_all()
        return req

    def _queue_for(self, slot: int):
        """The queue slot `slot` serves next: slot 0 the small requests (with size classes; also the
        large ones when no small one waits and small_slot_takes_large is set), the others the large
        ones first, then the small ones."""
        if self.small_log_len is None:
            return self.small
        if slot == 0:
            # the small slot: small requests, and large ones too when it would idle otherwise
            return self.large if (self.small_slot_takes_large and not self.small and self.large) else self.small
        return self.large if self.large else self.small

    def _admit(self, q) -> List[Request]:
        """Arrival order, as many as fit the arena (columns) and its request table."""
        taken, cols = [], 0
        while q and len(taken) < self.max_requests:
            c = 1 << q[0].column_log_len
            if cols + c > self.capacity:
                break
            cols += c
            taken.append(q.popleft())
        return taken

    def _work(self, b: Batch, slot: int):
        while True:
            with self.cv:
                while not self._queue_for(slot) and not self.stop:
                    self.cv.wait()
                if self.stop and not self._queue_for(slot):
                    return
                reqs = self._admit(self._queue_for(slot))
            if not reqs:
                continue
            now = self.clock()
            for r in reqs:
                r.admitted = now
            try:
                b.assign([r.column_log_len for r in reqs])
                b.witness_random([r.seed for r in reqs], [r.kind for r in reqs])
                if any(r.kind == 1 for r in reqs):
                    b.set_switch([r.kind == 1 for r in reqs], [self.switch_point(r) for r in reqs if r.kind == 1])
                rounds = b.round(self.domain, pool=self.pool, transcript=self.transcript, copy=self.keep_results)
                self.batches += 1
                err = None
            except Exception as e:  # noqa: BLE001 - reported on every request of the batch
                rounds, err = None, str(e)
            end = self.clock()
            for i, r in enumerate(reqs):
                r.done = end
                r.error = err
                if rounds is not None and self.keep_results:
                    r.result = rounds[i]
                r._event.set()

    def close(self):
        with self.cv:
            self.stop = True
            self.cv.notify_all()
        for w in self.workers:
            w.join()
        self.pool.shutdown()
