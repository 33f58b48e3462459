"""Host logic of the multi-GPU paths, on CPU ranks over gloo.

The step shards only by independent runs: ``bench.py --gpus N`` runs N
replicas of the single-run workload, and the ensemble workload bin-packs its
runs over the ranks (``assign_runs``) with no data-path collective.  What is
left to check without GPUs is that every rank derives the same assignment,
that the assignment covers every run exactly once and is balanced, and that
the max-over-ranks timing reduction of ``bench.py`` works under gloo.
"""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_assign_runs_covers_and_balances(hqt):
    import numpy as np
    rng = np.random.default_rng(3)
    costs = [float(c) for c in rng.integers(1, 100, size=37)]
    for ws in (1, 2, 3, 4, 8):
        parts = hqt.assign_runs(costs, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # greedy longest-first: the heaviest rank exceeds the mean by less
        # than the largest single run
        assert max(loads) - sum(costs) / ws < max(costs) + 1e-9
    assert hqt.assign_runs(costs, 4) == hqt.assign_runs(costs, 4)
    with pytest.raises(ValueError):
        hqt.assign_runs(costs, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    import datetime
    import importlib
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ["WORLD_SIZE"] = str(ws)
    os.environ["RANK"] = str(rank)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        bench = importlib.import_module("bench")
        hqt = importlib.import_module(bench.PKG)
        runs = bench.ensemble_runs()
        costs = [r["nx"] * r["ny"] * r["nz"] for r in runs]
        mine = hqt.assign_runs(costs, ws)[rank]
        everyone = [None] * ws
        dist.all_gather_object(everyone, mine)
        t = bench.allreduce_max(10.0 + rank, ws)
        with open(out / f"rank{rank}.txt", "w") as f:
            f.write(repr((everyone, t)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2])
def test_ensemble_sharding_over_gloo_ranks(hqt, tmp_path, ws):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank, args=(ws, port, tmp_path), nprocs=ws, join=True,
                       start_method="spawn")
    results = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(ws)]
    everyone, t = results[0]
    assert all(res == results[0] for res in results)  # same view on every rank
    assert t == 10.0 + ws - 1                        # max over ranks
    flat = sorted(i for part in everyone for i in part)
    assert flat == list(range(32))
