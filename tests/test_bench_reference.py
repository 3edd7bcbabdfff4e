"""bench.py's reference arm on CPU: whole oracle steps (commit of every column, fold of every ring
element), the same `config` dict as the device arm's line, a one-thread figure beside the
all-threads one. Run at suite s (2^18) so it takes seconds."""
import argparse
import contextlib
import io
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_times_whole_steps():
    sys.path.insert(0, ROOT)
    import bench

    args = argparse.Namespace(config="s", steps=2, warmup=1, gpus=1)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        assert bench.run_reference(args) == 0
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    params = bench.suite_shape("s")
    assert line["impl"] == "reference"
    assert line["config"] == bench.bench_config("s", params, 1)
    assert line["steps"] == 2 and line["warmup"] == 1
    # value is the whole step's elements over the measured mean step time
    assert abs(line["value"] - params.witness_len() / (line["ms_per_step"] / 1000)) < 1e-6 * line["value"]
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == (os.cpu_count() or 1)
    assert "whole steps" in cb["sample"]
    assert cb["single_thread"]["cores"] == 1 and cb["single_thread"]["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_oracle_step_matches_its_own_pieces():
    """The timed oracle step is the oracle's commit and fold of the round (a tiny shape)."""
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    import oracle as O

    s = bench.OracleStep((10, 2, [3889, 2917]))
    C, v, _, _ = s.step(2)
    P = O.Params(10, 2, [3889, 2917], 0)
    want = O.round_trip(P, bench.MATRIX_SEED, bench.WITNESS_SEED, domain=bench.DOMAIN)
    assert np.array_equal(C, want["C"])
    assert np.array_equal(v, want["v"])
