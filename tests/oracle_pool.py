"""The oracle decoding many code blocks of different configurations alone, on
all host cores (spawned processes: the oracle keeps a static soft buffer, and a
pool forked after CUDA initialisation would hang).

TEST INFRASTRUCTURE ONLY."""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(job):
    folder, lo, hi, row = job
    sys.path.insert(0, REPO)
    from oracle.oracle import Oracle, dec_cfg, in_config

    tab = np.load(os.path.join(folder, "cfgs.npy"))
    arena = np.load(os.path.join(folder, "llr.npy"), mmap_mode="r")
    orc = Oracle()
    dcfg = dec_cfg(row)
    out = []
    for i in range(lo, hi):
        bgn, A, crc, E, rv, Qm, off = (int(v) for v in tab[i])
        st, bits, it, _ = orc.decode(np.ascontiguousarray(arena[off:off + E]), in_config(bgn, A, crc, E, rv, Qm, 0),
                                     dcfg)
        out.append((st, it, bits))
    return out


def oracle_decode_blocks(arena_h: np.ndarray, cfgs, llr_offsets, row, procs: int = 0):
    """(status, iterations, hard-bit arrays) of every block (bgn, A, crc, E, rv, Qm)
    whose E LLRs start at llr_offsets[i] of arena_h."""
    import multiprocessing as mp

    n = len(cfgs)
    procs = max(1, min(procs or len(os.sched_getaffinity(0)) or 1, n))
    folder = tempfile.mkdtemp(prefix="ldpc_oracle_pool_")
    try:
        np.save(os.path.join(folder, "cfgs.npy"),
                np.array([list(c[:6]) + [o] for c, o in zip(cfgs, llr_offsets)], dtype=np.int64))
        np.save(os.path.join(folder, "llr.npy"), arena_h)
        jobs = [(folder, k * n // procs, (k + 1) * n // procs, list(row)) for k in range(procs)]
        with mp.get_context("spawn").Pool(procs) as pool:
            parts = pool.map(_worker, jobs)
    finally:
        shutil.rmtree(folder, ignore_errors=True)
    res = [r for p in parts for r in p]
    return (np.array([r[0] for r in res], dtype=np.int32), np.array([r[1] for r in res], dtype=np.int32),
            [r[2] for r in res])
