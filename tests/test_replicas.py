"""Replica parallelism (one process per GPU) on CPU ranks over gloo.

The multi-GPU path of this library partitions independent instances across
ranks with no data-path collective; these tests run its host logic with two
ranks: the start barrier, the max-over-ranks step time, the whole-job rate,
per-rank seeds and the round-robin split of a fixed request set.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from gradient_domain_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    w, r, local = replicas.rank_env()
    replicas.init(w, backend="gloo", timeout_s=60)
    replicas.barrier(w)
    step_ms = 10.0 + 5.0 * r                   # rank 1 is the slower one
    job_ms = replicas.max_over_ranks(step_ms, w, "cpu")
    rate = replicas.aggregate_rate(1000.0, w, job_ms / 1e3)
    share = replicas.split_evenly(range(7), r, w)
    out.put((r, local, job_ms, rate, replicas.replica_seed(1, r), share))
    replicas.finish(w)


@pytest.mark.timeout(120)
def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=90) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, l0, ms0, rate0, seed0, share0), (r1, l1, ms1, rate1, seed1, share1) = got
    assert (r0, l0, r1, l1) == (0, 0, 1, 1)
    assert ms0 == ms1 == 15.0                  # the job takes as long as its slowest rank
    assert rate0 == rate1 == pytest.approx(2 * 1000.0 / 0.015)
    assert seed0 != seed1                      # replicas solve different instances
    assert sorted(share0 + share1) == list(range(7)) and not set(share0) & set(share1)


def test_single_rank_needs_no_process_group():
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.aggregate_rate(10.0, 1, 2.0) == 5.0
    assert replicas.split_evenly([1, 2, 3], 0, 1) == [1, 2, 3]
    assert not torch.distributed.is_initialized()
