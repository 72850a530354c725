"""Multi-rank (replica) aggregation of bench.py on CPU: two gloo ranks with
different proof counts and device times; the whole-job value is the proofs of
all ranks over the slowest rank's time, and every rank sees the same result.
The rendezvous uses 127.0.0.1; no GPU and no data-path collective."""
import importlib.util
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    bench = _bench()
    w, r, _, pg = bench.dist_setup("gloo")
    assert (w, r) == (world, rank)
    bench.barrier(pg, None)
    proofs = [5.0, 7.0][rank]
    device_s = [2.0, 3.5][rank]
    value, t, total = bench.aggregate(pg, proofs, device_s, None)
    out[rank] = (value, t, total)
    bench.barrier(pg, None)
    pg.destroy_process_group()


def test_replica_aggregation_gloo():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        value, t, total = res[rank]
        assert t == 3.5 and total == 12.0
        assert abs(value - 12.0 / 3.5) < 1e-12


def test_single_rank_aggregation_is_identity():
    bench = _bench()
    value, t, total = bench.aggregate(None, 4.0, 2.0, None)
    assert (value, t, total) == (2.0, 2.0, 4.0)
