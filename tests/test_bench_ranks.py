"""The bench's multi-GPU plumbing on CPU: two ranks over gloo run the same Ranks code the GPU ranks run over NCCL
(the barrier around a timed region, the maximum over ranks of its time, the whole-job rate), and the reference arm
runs on rank 0 alone.  Registrations are independent replicas, so these are the only cross-rank steps."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    ranks = bench.Ranks("gloo", "cpu", timeout_s=60)
    ranks.barrier()
    seconds = 10. + 5. * rank                  # rank 1 is the slower one
    slowest = ranks.max(seconds)
    rate = bench.whole_job_rate(3, slowest, ranks.world)
    ranks.close()
    out.put((rank, ranks.world, slowest, rate))


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=5) for _ in range(world))
    for rank, w, slowest, rate in got:
        assert w == world
        assert slowest == 15.                   # every rank sees the slowest rank's time
        assert rate == 2 * 3 / 15. * 3600.      # all ranks' pairs over that time


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        assert k not in os.environ or os.environ[k] in ("0", "1")
    ranks = bench.Ranks("gloo", "cpu")
    assert ranks.world == 1 and ranks.max(7.5) == 7.5
    ranks.barrier()
    ranks.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun every rank starts bench.py --impl reference; rank 1 exits 0 without work or output."""
    sys.path.insert(0, ROOT)
    import bench
    called = []
    monkeypatch.setattr(bench, "reference_arm", lambda *a: called.append(a) or 0)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"])
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.main() == 0 and called == []
    monkeypatch.setenv("RANK", "0")
    assert bench.main() == 0 and len(called) == 1
