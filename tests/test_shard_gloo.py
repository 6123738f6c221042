"""Multi-rank host logic on CPU: two gloo ranks (world_size 2, 127.0.0.1).

Each rank takes its shard of a batch (weak, strong and cost-balanced mixed
splits), decodes it with the C oracle standing in for its GPU, and the ranks
combine timings (max) and counts (sum) exactly as bench.py does over NCCL.
Rank 0 gathers every rank's results and checks they equal one unsharded run.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    import sys

    sys.path.insert(0, REPO)
    import datetime

    import torch
    import torch.distributed as dist

    from deeplearning_5g_ldpc_decoder_b200.shard import (balance_blocks, block_cost, max_over_ranks, strong_shard,
                                                         sum_over_ranks, weak_shard)
    from oracle.oracle import Oracle, dec_cfg, in_config, make_llrs

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc = Oracle()
        row = [1, 8, 22936, 0, 1280, 32767, -32767]
        cfg = (2, 488, 1, 1920, 0, 2, 0)
        total = 7
        llr, _ = make_llrs(orc, in_config(*cfg), total, noise_db=0.0, seed=5)
        start, count = strong_shard(total, rank, world)
        mine = []
        for i in range(start, start + count):
            st, bits, it, _ = orc.decode(llr[i], in_config(*cfg), dec_cfg(row))
            mine.append((i, st, it, bits.tobytes()))
        # a mixed batch: every rank computes the same balanced partition
        cfgs = [(1 + (k % 2), 0, 0, 0, 0, 0) for k in range(10)]
        zcs = [384, 64, 208, 16, 96, 384, 40, 112, 256, 2]
        parts = balance_blocks([block_cost(c, z) for c, z in zip(cfgs, zcs)], world)
        fake_ms = 3.0 + rank
        worst = max_over_ranks(fake_ms, dist)
        units = sum_over_ranks(count, dist)
        first, n = weak_shard(8192, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, {"rank": rank, "mine": mine, "parts": parts, "worst": worst,
                                          "units": units, "weak": (first, n)})
        if rank == 0:
            import pickle

            with open(os.path.join(outdir, "gathered.pkl"), "wb") as f:
                pickle.dump(gathered, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_combine(tmp_path, oracle):
    import pickle

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    gathered = pickle.load(open(tmp_path / "gathered.pkl", "rb"))
    assert [g["rank"] for g in gathered] == [0, 1]
    # every block decoded exactly once, results equal an unsharded run
    from oracle.oracle import dec_cfg, in_config, make_llrs

    cfg = (2, 488, 1, 1920, 0, 2, 0)
    llr, _ = make_llrs(oracle, in_config(*cfg), 7, noise_db=0.0, seed=5)
    got = sorted(x for g in gathered for x in g["mine"])
    assert [x[0] for x in got] == list(range(7))
    for i, st, it, bits in got:
        est, ebits, eit, _ = oracle.decode(llr[i], in_config(*cfg), dec_cfg([1, 8, 22936, 0, 1280, 32767, -32767]))
        assert (st, it, bits) == (est, eit, ebits.tobytes())
    # combined timing is the slowest rank's, units add up, weak shards tile the id space
    assert all(g["worst"] == 4.0 for g in gathered)
    assert all(g["units"] == 7 for g in gathered)
    assert [g["weak"] for g in gathered] == [(0, 8192), (8192, 8192)]
    # identical partitions on both ranks, covering every block once, balanced
    assert gathered[0]["parts"] == gathered[1]["parts"]
    flat = sorted(i for p in gathered[0]["parts"] for i in p)
    assert flat == list(range(10))


def test_shard_helpers_single_process():
    from deeplearning_5g_ldpc_decoder_b200.shard import balance_blocks, max_over_ranks, strong_shard, sum_over_ranks

    for total in (0, 1, 7, 8192, 32769):
        for world in (1, 2, 3, 8):
            spans = [strong_shard(total, r, world) for r in range(world)]
            assert spans[0][0] == 0
            assert all(spans[r][0] + spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            assert sum(c for _, c in spans) == total
            assert max(c for _, c in spans) - min(c for _, c in spans) <= 1
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, 500)
    parts = balance_blocks(costs, 4)
    loads = [int(sum(costs[i] for i in p)) for p in parts]
    assert max(loads) - min(loads) <= int(costs.max())
    assert max_over_ranks(2.5) == 2.5 and sum_over_ranks(3) == 3.0
    with pytest.raises(ValueError):
        strong_shard(10, 2, 2)


_PROBE = '''
import datetime, json, os, sys
sys.path.insert(0, {repo!r})
import torch.distributed as dist
from deeplearning_5g_ldpc_decoder_b200.shard import max_over_ranks, sum_over_ranks
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ms = max_over_ranks(10.0 + rank, dist)
units = sum_over_ranks(8192, dist)
dist.barrier()
if rank == 0:
    print(json.dumps({{"n_gpus": world, "ms_per_step": ms, "units": units, "argv": sys.argv[1:]}}), flush=True)
dist.destroy_process_group()
'''


def test_launch_ranks_starts_world_size_ranks(tmp_path):
    """`bench.py --gpus N` outside a launcher re-runs itself under
    torch.distributed.run through shard.launch_ranks: two gloo ranks on CPU
    start, combine a time (max) and a count (sum) like bench.py does, and rank 0
    prints one line with n_gpus 2."""
    import json
    import subprocess

    from deeplearning_5g_ldpc_decoder_b200.shard import torchrun_command

    script = tmp_path / "probe.py"
    script.write_text(_PROBE.format(repo=REPO))
    cmd = torchrun_command(2, str(script), ["--gpus", "2"], _free_port(), timeout_s=120)
    assert cmd[:3] == ["timeout", "-k", "60"] and "--nproc-per-node=2" in cmd
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=180)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec == {"n_gpus": 2, "ms_per_step": 11.0, "units": 16384.0, "argv": ["--gpus", "2"]}
