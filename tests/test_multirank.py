"""The multi-GPU path of bench.py on CPU: world_size 2 over gloo.

Each rank fuses an independent map (no data-path collective); the reported
value is every rank's frames over the slowest rank's device time, and the
reference arm runs on rank 0 only.  These tests run the rank logic with the
gloo backend on 127.0.0.1."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    # rank r fused 10 (r + 1) frames in 100 (r + 1) ms of device time
    value, ms = bench.whole_job_rate(10.0 * (rank + 1), 100.0 * (rank + 1))
    mx = bench.reduce_over_ranks(float(rank), "max")
    sm = bench.reduce_over_ranks(float(rank + 1), "sum")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, value, ms, mx, sm))


@pytest.mark.timeout(180)
def test_whole_job_rate_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, value, ms, mx, sm in out:
        # 10 + 20 frames over the slowest rank's 200 ms
        assert ms == 200.0
        assert value == pytest.approx(30.0 / 0.2)
        assert mx == 1.0 and sm == 3.0


def test_single_process_rate_without_group():
    import bench
    value, ms = bench.whole_job_rate(970.0, 200.0)
    assert ms == 200.0 and value == pytest.approx(4850.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun every rank starts bench.py --impl reference; ranks other
    than 0 exit at once without work (no rendering, no reference maps)."""
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "make_sequence", lambda *a, **k: called.append(1))
    assert bench.run_reference(bench.parse_args(["--impl", "reference", "--gpus", "2"])) is None
    assert not called
