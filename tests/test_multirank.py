"""The bench's multi-rank host logic (one process per GPU under torchrun) on two gloo ranks on
the CPU: the max over ranks of per-rank times that every rank receives, the whole-job rate of
the weak-scaling run, and the reference arm that only rank 0 runs."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, results):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from datetime import timedelta
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        r, w, l = bench.rank_env()
        mine = [10.0 + 5.0 * rank, 3.0 * (world - rank)]
        got = [bench.max_over_ranks(m, dist) for m in mine]  # same order on every rank
        dist.barrier()
        results[rank] = (r, w, l, got, bench.job_rate(1000.0, w, got[0]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_on_two_gloo_ranks():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        res = m.dict()
        ps = [ctx.Process(target=_rank_main, args=(r, 2, port, res)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
            assert p.exitcode == 0
        res = dict(res)
    assert sorted(res) == [0, 1]
    for rank, (r, w, l, got, rate) in res.items():
        assert (r, w, l) == (rank, 2, rank)
        assert got == [15.0, 6.0]  # max over ranks of (10, 15) and (6, 3)
        assert rate == pytest.approx(2 * 1000.0 / 15e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun every rank launches the reference arm; ranks other than 0 exit at once,
    without work or output."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    assert bench.run_reference(None) == 0
    assert capsys.readouterr().out == ""
