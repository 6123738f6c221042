"""CUDA path vs the CPU oracle on seeded inputs: every lifting size of both
base graphs, every algorithm, edge cases (odd batches, zero iterations,
repetition, wide strides, saturation, custom tables)."""

import functools

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import ldpc_decode, set_degree_alpha, set_trained_weights
from golden_cases import lq_close
from oracle.oracle import dec_cfg, in_config, make_llrs

pytestmark = pytest.mark.gpu

LIFTING = sorted({2, 4, 8, 16, 32, 64, 128, 256, 3, 6, 12, 24, 48, 96, 192, 384, 5, 10, 20, 40, 80, 160, 320, 7, 14,
                  28, 56, 112, 224, 9, 18, 36, 72, 144, 288, 11, 22, 44, 88, 176, 352, 13, 26, 52, 104, 208, 15, 30,
                  60, 120, 240})
ROW1 = [1, 8, 22936, 0, 1280, 32767, -32767]


@functools.lru_cache(maxsize=None)
def config_for(oracle, bgn, zc):
    """Largest payload A (CRC24A) that lifts to exactly Zc, or None."""
    for crc in (1, 0):
        best = None
        for A in range(8, 8449, 8):
            rc, p = oracle.derive(in_config(bgn, A, crc, 960, 0, 2, 0))
            if rc == 0 and p.Zc == zc:
                best = (A, crc, p)
        if best:
            return best
    return None


def run_and_compare(oracle, cuda, cfg, row, llr, tag=""):
    res = ldpc_decode(torch.from_numpy(llr).to(cuda), cfg, row, return_app=True)
    torch.cuda.synchronize()
    bits, st, it, app = (res.hardbits.cpu().numpy(), res.status.cpu().numpy(), res.iterations.cpu().numpy(),
                         res.app.cpu().numpy())
    for i in range(llr.shape[0]):
        es, eb, ei, elq = oracle.decode(llr[i], in_config(*cfg), dec_cfg(row))
        assert st[i] == es, (tag, i)
        assert it[i] == ei, (tag, i)
        if ei > 0:
            assert np.array_equal(bits[i], eb), (tag, i)
        assert lq_close(app[i], elq, row[0], es == 0), (tag, i)
    return st, it


@pytest.mark.parametrize("bgn", [1, 2])
def test_every_lifting_size_algo1(oracle, cuda, bgn):
    covered = 0
    for zc in LIFTING:
        found = config_for(oracle, bgn, zc)
        if found is None:
            continue   # not reachable by any payload size (BG2 small Zc)
        A, crc, p = found
        E = ((p.B * 2 + 1) // 2) * 2
        cfg = (bgn, A, crc, E, zc % 4, 2, 0)
        llr, _ = make_llrs(oracle, in_config(*cfg), 3, noise_db=-1.0, seed=zc)
        run_and_compare(oracle, cuda, cfg, ROW1, llr, tag=f"bg{bgn} zc{zc}")
        covered += 1
    assert covered >= (51 if bgn == 1 else 45)


@pytest.mark.parametrize("algo", [0, 2, 3, 4])
def test_other_algorithms_across_sizes(oracle, cuda, algo):
    row = [algo, 6, 22936, 0, 1280, 32767 if algo else 20, -32767 if algo else -32768]
    for bgn, zc in [(1, 2), (1, 7), (1, 64), (1, 208), (1, 384), (2, 6), (2, 52), (2, 176), (2, 384)]:
        found = config_for(oracle, bgn, zc)
        if found is None:
            continue
        A, crc, p = found
        E = ((p.B * 5 // 3 + 3) // 4) * 4
        cfg = (bgn, A, crc, E, 1, 4, 0)
        llr, _ = make_llrs(oracle, in_config(*cfg), 3, noise_db=-4.0, seed=zc + algo)
        run_and_compare(oracle, cuda, cfg, row, llr, tag=f"algo{algo} bg{bgn} zc{zc}")


def test_c1_batch_1024_all_snrs(oracle, cuda):
    """BG2 Zc=64 (A=488, B=512, K=640, N=3200), E=1920, QPSK, algo 1, 10 iterations."""
    cfg = (2, 488, 1, 1920, 0, 2, 0)
    row = [1, 10, 22936, 0, 1280, 32767, -32767]
    for esn0 in (0.0, 1.0, 2.0, 3.0):
        llr, _ = make_llrs(oracle, in_config(*cfg), 256, noise_db=-esn0, seed=int(esn0 * 10))
        st, it = run_and_compare(oracle, cuda, cfg, row, llr, tag=f"c1 {esn0}")


def test_random_llrs_saturation_and_odd_settings(oracle, cuda):
    rng = np.random.default_rng(11)
    cases = [
        ((1, 8424, 1, 25344, 0, 8, 0), [1, 5, 22936, 0, 1280, 32767, -32767]),
        ((2, 488, 1, 1920, 0, 2, 0), [1, 6, 40000, 300, -500, 20000, -30000]),   # negative alpha as int16
        ((2, 488, 1, 1920, 1, 2, 0), [3, 6, 22936, 65000, 1280, 32767, -32768]),  # beta -536 as int16
        ((1, 1000, 2, 3000, 2, 4, 0), [1, 4, 32767, 0, 32767, -100, 100]),        # min_llr > max_llr
        ((2, 200, 0, 800, 0, 2, 0), [2, 5, 22936, 0, 1280, 32767, -32767]),
        ((1, 8424, 1, 30000, 1, 2, 0), [1, 3, 22936, 0, 1280, 32767, -32767]),    # E > N - F: repetition
        ((2, 1000, 1, 65000, 0, 2, 0), [1, 3, 22936, 0, 1280, 32767, -32767]),    # many repetitions, int16 wrap
        ((1, 480, 3, 2400, 3, 6, 0), [4, 5, 30000, 200, -3000, 5000, -7000]),
        ((2, 1200, 1, 4000, 2, 8, 0), [0, 4, 0, 0, 1280, 20, -32768]),
        # open-max arithmetic (max_llr 32767, beta 0) with negative alpha: scaled
        # minima down to -32767, and alpha -32768 as int16
        ((2, 488, 1, 1920, 0, 2, 0), [1, 6, 40000, 0, -500, 32767, -32767]),
        ((1, 8424, 1, 25344, 0, 8, 0), [1, 4, 32768, 0, 1280, 32767, -32768]),
        ((2, 488, 1, 1920, 1, 2, 0), [3, 6, 50000, 0, 1280, 32767, -32767]),
    ]
    for cfg, row in cases:
        E = cfg[3]
        llr = rng.integers(-32768, 32768, size=(5, E), dtype=np.int64).astype(np.int16)
        llr[1] = (rng.normal(size=E) * 3000).astype(np.int16)
        llr[2] = np.clip(rng.normal(size=E) * 400, -10000, 10000).astype(np.int16)
        run_and_compare(oracle, cuda, cfg, row, llr, tag=str((cfg, row)))


def test_zero_iterations_and_empty_batch(oracle, cuda):
    cfg = (2, 488, 1, 1920, 0, 2, 0)
    llr, _ = make_llrs(oracle, in_config(*cfg), 3, noise_db=0.0)
    res = ldpc_decode(torch.from_numpy(llr).to(cuda), cfg, [1, 0, 22936, 0, 1280, 32767, -32767], return_app=True)
    torch.cuda.synchronize()
    assert (res.status.cpu() == 1).all() and (res.iterations.cpu() == 0).all()
    assert not res.hardbits.cpu().numpy().any()          # untouched (zero-initialised) like the reference
    for i in range(3):
        assert np.array_equal(res.app[i].cpu().numpy(), oracle.rate_recover(in_config(*cfg), 1280, llr[i]))
    empty = ldpc_decode(torch.zeros((0, 1920), dtype=torch.int16, device=cuda), cfg, ROW1)
    assert empty.hardbits.shape[0] == 0


def test_strided_rows_and_batch_sizes(oracle, cuda):
    cfg = (1, 1320, 1, 4000, 2, 4, 0)
    llr, _ = make_llrs(oracle, in_config(*cfg), 7, noise_db=-2.0, seed=3)
    wide = np.zeros((7, 4096 + 13), dtype=np.int16)
    wide[:, :4000] = llr
    for n in (1, 2, 5, 7):
        run_and_compare(oracle, cuda, cfg, ROW1, wide[:n], tag=f"n={n}")


def test_custom_trained_and_degree_tables(oracle, cuda):
    rng = np.random.default_rng(4)
    cfg = (2, 488, 1, 1920, 0, 2, 0)
    llr, _ = make_llrs(oracle, in_config(*cfg), 5, noise_db=0.5, seed=9)
    alpha = rng.integers(18000, 30000, size=(3, 42)).astype(np.int16)
    beta = rng.integers(0, 200, size=(3, 42)).astype(np.int16)
    set_trained_weights(2, alpha, beta)
    oracle.set_trained(2, alpha, beta)
    try:
        run_and_compare(oracle, cuda, cfg, [2, 9, 0, 0, 1280, 32767, -32767], llr, tag="trained")
    finally:
        set_trained_weights(2, None)
        oracle.set_trained(2)
    tab = rng.integers(15000, 32000, size=19).astype(np.int16)
    set_degree_alpha(tab)
    oracle.set_degree_alpha(tab)
    try:
        run_and_compare(oracle, cuda, cfg, [3, 7, 0, 100, 1280, 32767, -32767], llr, tag="degree")
    finally:
        set_degree_alpha(None)
        oracle.set_degree_alpha(None)


def test_algo2_beyond_table_reuses_last_row(oracle, cuda):
    """The reference reads past its 32-iteration tables for max_iterations > 32;
    this library (and the oracle) reuse the last row instead."""
    cfg = (1, 1000, 1, 3000, 0, 2, 0)
    llr, _ = make_llrs(oracle, in_config(*cfg), 2, noise_db=6.0, seed=2)
    run_and_compare(oracle, cuda, cfg, [2, 40, 0, 0, 1280, 32767, -32767], llr, tag="algo2 40 it")


@pytest.mark.parametrize("algo", [1, 4])
def test_host_buffer_pipeline_matches_device_path(oracle, cuda, algo):
    """nrldpc_decode_batch_host copies and decodes in overlapped chunks (a
    quarter, a quarter and half a kernel wave, then whole waves, on four decode
    streams); results equal the device-pointer path for batches below, at and
    well above the chunking threshold, and a sample equals the oracle."""
    from deeplearning_5g_ldpc_decoder_b200 import ldpc_decode_host

    cfg = (2, 488, 1, 1920, 0, 2, 0)
    base, _ = make_llrs(oracle, in_config(*cfg), 64, noise_db=-1.0, seed=31)
    rng = np.random.default_rng(4)
    row = [algo, 8, 22936, 0, 1280, 32767, -32767]
    for n in (1, 7, 300, 4000, 13001):
        llr = base[rng.integers(0, 64, n)]
        llr = np.clip(llr.astype(np.int32) + rng.integers(-300, 300, llr.shape), -32767, 32767).astype(np.int16)
        bits, st, it = ldpc_decode_host(llr, cfg, row)
        ref = ldpc_decode(torch.from_numpy(llr).to(cuda), cfg, row)
        assert np.array_equal(st, ref.status.cpu().numpy()), n
        assert np.array_equal(it, ref.iterations.cpu().numpy()), n
        assert np.array_equal(bits, ref.hardbits.cpu().numpy()), n
        for i in rng.integers(0, n, 3):
            es, eb, ei, _ = oracle.decode(llr[i], in_config(*cfg), dec_cfg(row))
            assert (st[i], it[i]) == (es, ei) and np.array_equal(bits[i], eb)
