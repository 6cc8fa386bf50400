"""The multi-GPU path of bench.py (replicas: one process per GPU, whole
queries per rank, no data exchange) on CPU: two gloo ranks agree on the
max-over-ranks time, and the job's rate counts every rank's queries over it."""
import importlib.util
import os
import pathlib
import socket

import pytest
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank, world, port, times_ms, steps, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rep = _bench().Replicas(dist, "cpu")
        rep.barrier()
        rate, ms = rep.job_rate(steps, times_ms[rank])
        out.put((rank, rep.world, rate, ms))
        rep.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("times_ms", [(10.0, 12.5), (7.0, 3.5)])
def test_two_gloo_ranks_time_by_the_slowest(times_ms):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    steps, world, port = 40, 2, _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times_ms, steps, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    slowest = max(times_ms)
    for rank, w, rate, ms in got:
        assert w == world
        assert ms == pytest.approx(slowest)
        assert rate == pytest.approx(steps * world / (slowest / 1e3))


def test_one_rank_needs_no_process_group():
    rep = _bench().Replicas(None, "cpu")
    rate, ms = rep.job_rate(10, 5.0)
    assert rep.world == 1 and ms == 5.0 and rate == pytest.approx(2000.0)


REF_RUNNER = ROOT / "oracle" / "_ref" / "ref_runner"


@pytest.mark.skipif(not REF_RUNNER.exists(), reason="reference engine not built (oracle/Makefile ref)")
def test_reference_arm_prints_the_bench_line():
    # `bench.py --impl reference` runs on host cores only: one JSON line with
    # the bench's keys, its own e2e and cpu_baseline.
    import json
    import subprocess
    import sys

    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scale", "0.02",
                        "--steps", "3", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 3 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["rows"] > 0
