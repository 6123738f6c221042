"""Block error rates of the reference's own transmit -> channel -> decode chain
(c_ldpc_5g_encode -> tx_rx_process -> c_ldpc_5g_decode, the loop of
scripts/ldpc_c_sim_common.py:227-272), and Wilson score intervals.

TEST INFRASTRUCTURE ONLY (tests/test_gpu_bler.py).  The reference chain runs on
the host cores in spawned processes, one slice of blocks each; every process
seeds libc's rand() (the reference channel's generator) with its own seed."""

from __future__ import annotations

import math
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def payloads(n: int, A: int, seed: int) -> np.ndarray:
    """Seeded uniform payload bytes [n, A/8] (MSB first), shared by both chains."""
    return np.random.default_rng(seed).integers(0, 256, size=(n, A // 8), dtype=np.uint8)


def _chain_worker(job):
    cfg_t, row, noise_db, seed, lo, hi = job
    sys.path.insert(0, REPO)
    from oracle.oracle import RefLib, dec_cfg, in_config

    ref = RefLib()
    cfg, dcfg = in_config(*cfg_t), dec_cfg(row)
    pay = payloads(hi, cfg.A, seed)[lo:hi]
    ref.srand(1 + seed * 7919 + lo)
    errors = 0
    for p in pay:
        rm = ref.encode(p, cfg)
        llr = ref.channel(rm, cfg.E, cfg.Qm, noise_db)
        st, bits, _ = ref.decode(llr, cfg, dcfg)
        errors += int(st != 0 or not np.array_equal(bits[: cfg.A // 8], p))
    return errors


def reference_block_errors(cfg, row, noise_db: float, n: int, seed: int, procs: int = 0) -> int:
    """Block errors (CRC failure or wrong payload) of n blocks through the
    reference chain at AWGN power noise_db."""
    import multiprocessing as mp

    procs = max(1, min(procs or len(os.sched_getaffinity(0)) or 1, n))
    jobs = [(tuple(cfg), list(row), float(noise_db), seed, r * n // procs, (r + 1) * n // procs) for r in range(procs)]
    with mp.get_context("spawn").Pool(procs) as pool:
        return int(sum(pool.map(_chain_worker, jobs)))


def wilson(k: int, n: int, z: float = 1.959964) -> tuple:
    """Wilson score interval of a binomial proportion k/n (95 % by default)."""
    if n == 0:
        return (0.0, 1.0)
    p = k / n
    d = 1.0 + z * z / n
    c = (p + z * z / (2 * n)) / d
    h = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return (max(0.0, c - h), min(1.0, c + h))


def overlap(a: tuple, b: tuple) -> bool:
    return a[0] <= b[1] and b[0] <= a[1]
