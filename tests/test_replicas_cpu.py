"""The multi-GPU path without GPUs: two gloo ranks on CPU run the replica
collectives (max-over-ranks timing, the all-reduce of the running sums) and
must agree with one process that holds every replica's samples."""
import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from openferric_b200 import _abi as A
from openferric_b200.replicas import combine_sums, finish, max_over_ranks, replica_seed


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _samples(rank, n=5000):
    rng = np.random.default_rng(100 + rank)
    x = np.maximum(rng.normal(1.0, 2.0, n), 0.0)
    y = x + rng.normal(0.0, 0.5, n)
    return x, y


def _sums(x, y):
    return [x.sum(), (x * x).sum(), y.sum(), (x * y).sum(), (y * y).sum()]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = A.OfMcResult()
        x, y = _samples(rank)
        s = _sums(x, y)
        r.sum_x, r.sum_x2, r.sum_y, r.sum_xy, r.sum_y2 = s
        r.samples = len(x)
        plain = combine_sums(r, discount=0.95)
        cv = combine_sums(r, cv_kind=A.OF_CV_VANILLA_TERMINAL, cv_expected=1.2, discount=0.95)
        slow = max_over_ranks(10.0 + rank)
        out[rank] = (plain, cv, slow, replica_seed(2 ** 64 - 1, rank))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_combine_like_one_process():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    xs, ys = zip(*[_samples(r) for r in range(world)])
    x, y = np.concatenate(xs), np.concatenate(ys)
    ref_plain = finish(_sums(x, y), len(x), discount=0.95)
    ref_cv = finish(_sums(x, y), len(x), A.OF_CV_VANILLA_TERMINAL, 1.2, 0.95)
    for rank in range(world):
        plain, cv, slow, seed = out[rank]
        assert plain[2] == len(x) and cv[2] == len(x)
        assert plain[0] == pytest.approx(ref_plain[0], rel=1e-12) and plain[1] == pytest.approx(ref_plain[1], rel=1e-10)
        assert cv[0] == pytest.approx(ref_cv[0], rel=1e-12) and cv[1] == pytest.approx(ref_cv[1], rel=1e-9)
        assert slow == 11.0  # the slowest rank's time
        assert seed == (rank - 1) % 2 ** 64  # seed + rank wraps
    # the combined estimator is the mean over both replicas' samples
    assert ref_plain[0] == pytest.approx(0.95 * x.mean(), rel=1e-12)


def test_single_process_is_the_identity():
    assert max_over_ranks(3.5) == 3.5
    r = A.OfMcResult()
    x, y = _samples(0, 100)
    r.sum_x, r.sum_x2, r.sum_y, r.sum_xy, r.sum_y2 = _sums(x, y)
    r.samples = 100
    price, stderr, n = combine_sums(r)
    assert n == 100 and price == pytest.approx(x.mean()) and stderr == pytest.approx(x.std(ddof=1) / 10.0)
