"""Replica plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1.

The path does not shard (one solver instance per GPU); the only collective is
the max over ranks of the timed region, and under torchrun only rank 0 prints.
"""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    got_ws, got_rank, _ = bench.dist_setup(ws)
    try:
        assert (got_ws, got_rank) == (ws, rank)
        assert dist.get_backend() == "gloo"
        bench.barrier(got_ws)
        # each replica's elapsed time differs; the reported time is the slowest
        t = bench.max_over_ranks(got_ws, 1.0 + rank)
        out[rank] = t
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ws = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    mp.start_processes(_rank_main, args=(ws, port, out), nprocs=ws, join=True, start_method="spawn")
    assert dict(out) == {0: 2.0, 1: 2.0}


def test_reference_arm_runs_on_rank0_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class A:
        steps, warmup, gpus = 1, 0, 2
    # rank 1 returns at once without work or output
    assert bench.run_reference(A, None, 2, 1) is None
    assert capsys.readouterr().out == ""


def test_legendre_flop_count():
    """The useful FP64 flops bench.py divides the GEMM times into: 2 NR (sum over
    m < NTCHOP of NRCHOP - m) NXCHOPDIM, i.e. 474 MFLOP per RTRAN-equivalent at
    192x128x256 (chops 128, 85, 85: sum 7310, NXCHOPDIM 169)."""
    sys.path.insert(0, ROOT)
    import bench
    from mlegs_b200.inputs import CONFIGS
    cfg = CONFIGS["etd_192x128x256"]
    assert (cfg.nr, cfg.nrchop, cfg.ntchop, cfg.nxchop) == (192, 128, 85, 85)
    assert bench.legendre_flops(cfg, 2 * cfg.nxchop - 1) == 2.0 * 192 * 7310 * 169
    # m past NRCHOP contributes nothing
    small = type("C", (), {"nr": 8, "nrchop": 3, "ntchop": 6})()
    assert bench.legendre_flops(small, 5) == 2.0 * 8 * (3 + 2 + 1) * 5


if __name__ == "__main__":
    sys.exit(pytest.main([__file__, "-q"]))
