"""The multi-GPU bench path on the CPU: two replica processes over gloo
(127.0.0.1) take the timing barrier and the max over ranks as bench.py does
under torchrun; a rank that never joins ends the others' collective with an
error after the process-group timeout instead of a hang; the reference arm
runs on rank 0 only."""

import os
import socket
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)


def _replica(rank, world, port, q):
    _env(rank, world, port)
    import bench

    w, r, _ = bench.dist_setup()
    g = bench.Replicas(w, r, backend="gloo", timeout_s=30.0)
    g.barrier()
    elapsed = 1.0 + r  # per-rank seconds for 10 frames
    slowest = g.max(elapsed)
    rate = bench.whole_job_rate(w, 10, slowest)
    g.barrier()
    g.close()
    q.put((r, slowest, rate))


def _deserter(rank, world, port, q):
    _env(rank, world, port)
    import bench

    if rank == 1:
        q.put((rank, "left"))  # leaves between steps: never joins the group
        return
    t0 = time.monotonic()
    try:
        g = bench.Replicas(world, rank, backend="gloo", timeout_s=3.0)
        g.barrier()
        q.put((rank, "joined"))
    except Exception as e:  # the rendezvous or the collective times out
        q.put((rank, "error", type(e).__name__, time.monotonic() - t0))


def _run(target, world):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert not p.is_alive()
    out = []
    while not q.empty():
        out.append(q.get())
    return out, [p.exitcode for p in procs]


def test_two_replicas_take_the_max_over_ranks():
    out, codes = _run(_replica, 2)
    assert codes == [0, 0]
    assert sorted(o[0] for o in out) == [0, 1]
    for _, slowest, rate in out:
        assert slowest == 2.0          # the slowest rank's time
        assert rate == 2 * 10 / 2.0    # whole-job frames per second


def test_a_rank_that_never_joins_times_out_the_others():
    out, codes = _run(_deserter, 2)
    by_rank = {o[0]: o for o in out}
    assert by_rank[1][1] == "left"
    assert by_rank[0][1] == "error" and by_rank[0][3] < 60.0
    assert codes[1] == 0


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    g = bench.Replicas(1, 0)
    g.barrier()
    assert g.max(3.5) == 3.5
    g.close()
    assert bench.whole_job_rate(1, 200, 0.1) == pytest.approx(2000.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        steps, warmup, gpus = 1, 0, 2

    bench.run_reference(Args(), 2, 1)  # rank 1: no work, no output
    assert capsys.readouterr().out == ""
