"""Sharding of independent systems over ranks (CPU; world size 2 over gloo)."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from thermofem_b200 import problems as P
from thermofem_b200 import shard


def _weights():
    return [P.transient3d_nnz(m) for m, _ in P.batched_transient_params(48, seed=1004)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_assign_covers_every_system_once_and_balances(world):
    w = _weights()
    parts = shard.assign(w, world)
    assert len(parts) == world
    flat = sorted(k for ks in parts for k in ks)
    assert flat == list(range(len(w)))
    assert all(ks == sorted(ks) for ks in parts)
    # LPT: the largest load is within 4/3 of the lower bound max(mean, largest)
    loads = [sum(w[k] for k in ks) for ks in parts]
    bound = max(sum(w) / world, max(w))
    assert max(loads) <= 4 / 3 * bound
    assert shard.assign(w, world) == parts  # deterministic


def test_assign_edge_cases():
    assert shard.assign([], 2) == [[], []]
    assert shard.assign([5], 3) == [[0], [], []]
    assert shard.assign([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.assign([1], 0)
    with pytest.raises(ValueError):
        shard.assign([-1], 1)


def test_gather_without_process_group():
    assert shard.gather_reports(["b", "a"], [1, 0], 2) == ["a", "b"]
    with pytest.raises(ValueError):
        shard.gather_reports(["a"], [0], 2)
    with pytest.raises(ValueError):
        shard.gather_reports(["a", "b"], [0, 0], 2)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        w = _weights()
        mine = shard.assign(w, world)[rank]
        reps = [{"system": k, "rank": rank, "nnz": w[k]} for k in mine]
        allr = shard.gather_reports(reps, mine, len(w))
        if rank == 0:
            with open(out, "w") as f:
                json.dump(allr, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_gather_reports_over_two_gloo_ranks(tmp_path):
    out = str(tmp_path / "reports.json")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    with open(out) as f:
        reps = json.load(f)
    w = _weights()
    parts = shard.assign(w, 2)
    assert [r["system"] for r in reps] == list(range(48))
    for k, r in enumerate(reps):
        assert r["rank"] == (0 if k in parts[0] else 1)
        assert r["nnz"] == w[k]


def _failing_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        # a rank that fails between steps, with nothing in flight
        raise RuntimeError("rank 1 failed before reporting")
    w = _weights()
    mine = shard.assign(w, world)[rank]
    try:
        shard.gather_reports([{"system": k} for k in mine], mine, len(w))
        outcome = "gathered"
    except Exception as e:  # the peer is gone: the collective ends with an error
        outcome = f"error: {type(e).__name__}"
    with open(out, "w") as f:
        f.write(outcome)
    dist.destroy_process_group()


def test_gather_fails_instead_of_hanging_when_a_rank_dies(tmp_path):
    out = str(tmp_path / "outcome.txt")
    pc = mp.start_processes(_failing_worker, args=(2, _free_port(), out), nprocs=2, join=False,
                            start_method="spawn")
    for p in pc.processes:  # each on its own: a failed rank must not take the other down
        p.join(timeout=120)
    codes = [p.exitcode for p in pc.processes]
    for p in pc.processes:
        if p.is_alive():
            p.kill()
    assert codes[1] not in (0, None)  # rank 1 failed
    assert codes[0] == 0  # rank 0 did not hang: its collective ended with an error
    with open(out) as f:
        assert f.read().startswith("error")
