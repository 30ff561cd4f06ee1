"""Sharding one read set over ranks (care_b200.shard), on CPU: two gloo
ranks each correct their anchor range -- with the oracle standing in for
the device -- and gather their record streams; the merged stream equals a
single run's records. Also the range partition itself."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import _oracle
from care_b200 import shard

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("paired", [False, True])
def test_shard_ranges_partition(paired):
    rng = np.random.default_rng(1)
    for _ in range(300):
        world = int(rng.integers(1, 9))
        n = int(rng.integers(0, 5000)) * (2 if paired else 1)
        got = [shard.shard_range(n, r, world, paired) for r in range(world)]
        pos = 0
        for first, count in got:
            assert first == pos and count >= 0
            if paired:
                assert first % 2 == 0 and count % 2 == 0
            pos += count
        assert pos == n
        assert max(c for _, c in got) - min(c for _, c in got) <= (2 if paired else 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, inp, args, out):
    sys.path.insert(0, HERE)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        o = _oracle.opts_from_args(args)
        probe = _oracle.OracleRun([inp], o, threads=1, first=0, count=0)
        n = probe.reads.contents.n
        probe.close()
        first, count = shard.shard_range(n, rank, world, bool(o.paired_end))
        run = _oracle.OracleRun([inp], o, threads=2, first=first, count=count)
        try:
            blob = run.records()
        finally:
            run.close()
        merged = shard.gather_records(blob)
        if rank == 0:
            with open(out, "wb") as f:
                f.write(merged)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["pe_q2_cand", "se_cand"])
def test_two_ranks_equal_one_run(golden, tmp_path, case):
    m = golden.cases[case]
    inp = golden.input(m["input"])
    full = _oracle.OracleRun([inp], _oracle.opts_from_args(m["args"]), threads=4)
    try:
        ref = full.records()
    finally:
        full.close()
    out = str(tmp_path / "merged.bin")
    mp.start_processes(_worker, args=(2, _free_port(), inp, m["args"], out), nprocs=2, start_method="spawn")
    merged = open(out, "rb").read()
    assert len(merged) == len(ref)
    assert shard.record_multiset(merged) == shard.record_multiset(ref)
    assert any(t == 1 for _, _, _, t, _ in shard.iter_records(ref))      # candidate corrections included


def _gather_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        blob = bytes(range(256)) * (rank * 3) + bytes([rank]) * (rank % 2)   # rank 0 contributes nothing
        merged = shard.gather_records(blob)
        with open(out % rank, "wb") as f:
            f.write(merged)
    finally:
        dist.destroy_process_group()


def test_gather_streams_of_unequal_and_empty_sizes(tmp_path):
    """The byte-tensor gather returns the streams in rank order on every
    rank, whatever their sizes (an empty one included)."""
    world = 3
    out = str(tmp_path / "g%d.bin")
    mp.start_processes(_gather_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    exp = b"".join(bytes(range(256)) * (r * 3) + bytes([r]) * (r % 2) for r in range(world))
    for r in range(world):
        assert open(out % r, "rb").read() == exp
