"""bench.py's N > 1 path on CPU: two gloo ranks on 127.0.0.1, as torchrun starts them (RANK,
WORLD_SIZE, LOCAL_RANK, MASTER_ADDR, MASTER_PORT in the environment). Each rank commits its own
witness (weak scaling over independent objects, no data-path collective); the only collectives are
the barrier around the timed region and the max of the ranks' times, from which rank 0 reports the
whole job's elements per second. The reference arm runs on rank 0 alone; the other ranks exit 0
without work."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as td

    try:
        r, w, local = bench.dist()
        bench.init_group(w, "gloo")
        bench.barrier(w)
        ms_max = bench.allreduce_max(times[r], w)
        bench.barrier(w)
        # the reference arm: rank 0 alone; here rank 1 returns at once, without the oracle
        ref = bench.run_reference(None) if r != 0 else 0
        q.put((r, w, local, ms_max, bench.rank_witness_seed(r), bench.whole_job_value(w, 1 << 22, ms_max), ref))
    finally:
        if td.is_initialized():
            td.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_distinct_witnesses():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [3.25, 4.5]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[:3] for o in out] == [(0, 2, 0), (1, 2, 1)]
    assert [o[3] for o in out] == [4.5, 4.5]
    assert out[0][4] != out[1][4]
    assert out[0][5] == out[1][5] == 2 * (1 << 22) / 4.5e-3
    assert out[1][6] == 0
