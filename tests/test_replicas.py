"""The multi-GPU timing path on CPU: two gloo ranks, as bench.py --gpus 2
uses them (barrier, max over ranks, whole-job rate)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from pywrf_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        replicas.barrier()
        ms = [40.0, 55.0][rank]
        m = replicas.max_over_ranks(ms)
        out[rank] = (replicas.world(), m, replicas.job_rate(20, m, replicas.world()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_the_job_rate():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(_free_port(), out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1]
    w, m, rate = out[0]
    assert w == 2 and m == 55.0
    assert rate == pytest.approx(2 * 20 / 0.055)


def test_single_rank_needs_no_process_group():
    assert replicas.world() == 1
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.job_rate(10, 100.0, 1) == pytest.approx(100.0)
