"""The multi-rank path of bench.py on CPU: two gloo ranks.  Each rank times its own replica; the reported
time is the slowest rank's (max over ranks), the value the whole job's throughput; the reference arm does
its work on rank 0 only."""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [bench.max_over_ranks(t, world, "cpu") for t in (1.0 + rank, 5.0 - 2 * rank)]
        q.put((rank, ms, bench.whole_job_gdofs(world, 3_000_000, ms[0])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # rank times (1, 5) and (2, 3): every rank sees the maxima 2 and 5
    assert [r[1] for r in res] == [[2.0, 5.0], [2.0, 5.0]]
    # 2 replicas x 3e6 DoFs in 2 ms: 3 GDoF/s
    assert all(abs(r[2] - 3.0) < 1e-12 for r in res)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1.25, 1, "cpu") == 1.25


def test_reference_arm_does_nothing_on_other_ranks(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, gpus = 3, 3, 2
    assert bench.run_reference(Args(), rank=1) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the reference's own CPU apply, or the C oracle where it is not built) prints one
    JSON line with the keys the benchmark contract asks of the reference arm."""
    import json
    import subprocess
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "3"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["value"] == line["value"]
