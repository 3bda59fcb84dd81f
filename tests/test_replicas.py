"""The multi-process plumbing of bench.py, run as two gloo ranks on the CPU.

On GPUs `bench.py --gpus N` runs N independent replicas of the single-GPU
step (one process per GPU under torchrun); the ranks share no data and only
meet at the barriers around the timed region and in the max / sum of the
timings.  These tests run that plumbing with the gloo backend: the whole-job
aggregate, the reference arm's rank > 0 behaviour, and a rank that leaves
without joining the collectives."""
import multiprocessing as mp
import os
import socket
import time

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank: int, world: int, port: int) -> None:
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})


def _replica(rank: int, world: int, port: int, q) -> None:
    _env(rank, world, port)
    import bench
    d = bench.Dist("gloo", timeout_s=30)
    try:
        d.barrier()
        # rank r timed 10 + 5 r ms for (r + 1) M cell-steps
        ms_max, value = bench.aggregate(d, 10.0 + 5.0 * rank, 1e6 * (rank + 1))
        ref = bench.run_reference(None, d) if rank != 0 else "skipped"
        d.barrier()
        q.put((rank, d.world, ms_max, value, ref))
    finally:
        d.close()


def _leaver(rank: int, world: int, port: int, q) -> None:
    _env(rank, world, port)
    import bench
    d = bench.Dist("gloo", timeout_s=5)
    if rank == 1:
        # leaves between steps: joined the group, never reaches the barrier
        os._exit(0)
    t0 = time.time()
    try:
        d.barrier()
        q.put((rank, "no error", time.time() - t0))
    except Exception as e:  # noqa: BLE001 - any error is the detection
        q.put((rank, type(e).__name__, time.time() - t0))
    # flush the queue's feeder thread before leaving without the group's
    # teardown (which would wait for the rank that left)
    q.close()
    q.join_thread()
    os._exit(0)


def _run(target, world: int = 2, wall: float = 60.0):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = []
    deadline = time.time() + wall
    try:
        while len(out) < world and time.time() < deadline:
            try:
                out.append(q.get(timeout=1.0))
            except Exception:  # queue.Empty
                if all(not p.is_alive() for p in procs) and q.empty():
                    break
    finally:
        for p in procs:
            p.join(timeout=max(1.0, deadline - time.time()))
            if p.is_alive():
                p.kill()
    return sorted(out, key=lambda r: r[0])


@pytest.mark.timeout(120)
def test_two_replicas_aggregate_over_gloo():
    """Whole-job value = all ranks' cell-steps over the slowest rank's time:
    3 M cell-steps in 15 ms = 200 Mcell-steps/s on both ranks; the
    reference arm does no work on rank 1."""
    res = _run(_replica)
    assert len(res) == 2, res
    for rank, world, ms_max, value, ref in res:
        assert world == 2
        assert ms_max == 15.0
        assert value == pytest.approx(3e6 / 0.015 / 1e6, rel=1e-12)
        if rank == 1:
            assert ref is None


@pytest.mark.timeout(120)
def test_rank_that_leaves_is_detected_by_the_other():
    """A rank that exits without reaching the barrier: the remaining rank's
    barrier ends with an error (peer gone or the 5 s group timeout) instead
    of waiting for good."""
    res = _run(_leaver, wall=90.0)
    assert len(res) == 1, res
    rank, outcome, secs = res[0]
    assert rank == 0
    assert outcome != "no error"
    assert secs < 60.0
