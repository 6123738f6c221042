"""Full-size workload (BG1, Zc=384, K=8448, E=25344, 256QAM-length, 8192 code
blocks in one launch): size-independent properties plus an exact oracle check
on a sample."""

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import ldpc_decode
from oracle.oracle import dec_cfg, in_config

pytestmark = pytest.mark.gpu

CFG = (1, 8424, 1, 25344, 0, 8, 0)
ROW = [1, 8, 22936, 0, 1280, 32767, -32767]
N_CW = 8192


def bpsk_llrs(rm_bits: np.ndarray, n: int, ebn0_db: float, seed: int) -> np.ndarray:
    """AWGN/BPSK int16 LLRs, round(128*LLR) clipped to +-10000, for n copies of
    the pool's rate-matched bit sequences (each copy with its own noise)."""
    rng = np.random.default_rng(seed)
    pool = rm_bits.shape[0]
    sigma = np.sqrt(0.5 / (10 ** (ebn0_db / 10)))
    out = np.empty((n, rm_bits.shape[1]), dtype=np.int16)
    for s in range(0, n, 512):
        e = min(n, s + 512)
        x = 1.0 - 2.0 * rm_bits[np.arange(s, e) % pool].astype(np.float32)
        y = x + sigma * rng.standard_normal(x.shape, dtype=np.float32)
        out[s:e] = np.clip(np.rint(128.0 * 2.0 * y / sigma ** 2), -10000, 10000).astype(np.int16)
    return out


@pytest.fixture(scope="module")
def workload(oracle):
    cfg = in_config(*CFG)
    rng = np.random.default_rng(2024)
    pool = 16
    pay = rng.integers(0, 256, size=(pool, 8424 // 8), dtype=np.uint8)
    rm = np.stack([np.unpackbits(oracle.encode(pay[i], cfg))[:25344] for i in range(pool)])
    cw = np.stack([oracle.encode_codeword(pay[i], cfg)[:8448] for i in range(pool)])
    llr = bpsk_llrs(rm, N_CW, ebn0_db=0.9, seed=1)
    return llr, cw, pool


def test_full_batch_round_trip_and_sample_parity(oracle, cuda, workload):
    llr, cw, pool = workload
    d = torch.from_numpy(llr).to(cuda)
    res = ldpc_decode(d, CFG, ROW, return_app=True)
    torch.cuda.synchronize()
    st = res.status.cpu().numpy()
    bits = res.hardbits.cpu().numpy()
    conv = np.nonzero(st == 0)[0]
    assert len(conv) > N_CW // 2
    # every code block that passed its CRC decoded to the transmitted payload||CRC
    want = np.stack([np.packbits(cw[i]) for i in range(pool)])
    assert np.array_equal(bits[conv], want[conv % pool])
    # exact agreement with the oracle on a sample, converged and not
    sample = list(conv[:8]) + list(np.nonzero(st != 0)[0][:8])
    app = res.app.cpu().numpy()
    its = res.iterations.cpu().numpy()
    for i in sample:
        es, eb, ei, elq = oracle.decode(llr[i], in_config(*CFG), dec_cfg(ROW))
        assert (st[i], its[i]) == (es, ei), i
        assert np.array_equal(bits[i], eb), i
        assert np.array_equal(app[i], elq), i
    # deterministic, and independent of which code block shares the int16x2 pair
    res2 = ldpc_decode(d, CFG, ROW)
    assert torch.equal(res2.hardbits, res.hardbits) and torch.equal(res2.iterations, res.iterations)
    for i in (0, 1, 4097, N_CW - 1):
        alone = ldpc_decode(d[i:i + 1].contiguous(), CFG, ROW, return_app=True)
        assert torch.equal(alone.app[0], res.app[i]) and torch.equal(alone.hardbits[0], res.hardbits[i])


def test_noise_only_runs_every_iteration(cuda):
    rng = np.random.default_rng(3)
    llr = np.clip(rng.normal(size=(1024, 25344)) * 700, -10000, 10000).astype(np.int16)
    res = ldpc_decode(torch.from_numpy(llr).to(cuda), CFG, ROW)
    torch.cuda.synchronize()
    assert (res.status.cpu() == 1).all()
    assert (res.iterations.cpu() == 8).all()


def _device_blocks(cuda, cfg, n, esn0_db, seed):
    from deeplearning_5g_ldpc_decoder_b200 import channel_llrs, ldpc_encode

    gen = torch.Generator(device=cuda).manual_seed(seed)
    pay = torch.randint(0, 256, (n, cfg[1] // 8), dtype=torch.uint8, device=cuda, generator=gen)
    llr = channel_llrs(ldpc_encode(pay, cfg), cfg[3], cfg[5], -esn0_db, seed=seed)
    return pay, llr


def test_high_rate_full_batch(oracle, cuda):
    """E = 9600 (rate 0.88, 256QAM) on 8192 blocks: passing blocks carry the sent
    payload, a sample of passing and failing blocks equals the oracle exactly."""
    cfg = (1, 8424, 1, 9600, 0, 8, 0)
    pay, llr = _device_blocks(cuda, cfg, N_CW, 24.5, 41)
    res = ldpc_decode(llr, cfg, ROW, return_app=True)
    st, bits = res.status.cpu().numpy(), res.hardbits.cpu().numpy()
    conv = np.nonzero(st == 0)[0]
    fail = np.nonzero(st != 0)[0]
    assert len(conv) > N_CW // 4
    assert np.array_equal(bits[conv, : 8424 // 8], pay.cpu().numpy()[conv])
    llr_h, app, its = llr.cpu().numpy(), res.app.cpu().numpy(), res.iterations.cpu().numpy()
    for i in list(conv[:4]) + list(fail[:4]):
        es, eb, ei, elq = oracle.decode(llr_h[i], in_config(*cfg), dec_cfg(ROW))
        assert (st[i], its[i]) == (es, ei) and np.array_equal(bits[i], eb) and np.array_equal(app[i], elq), i


def test_bp_full_size_blocks(oracle, cuda):
    """Algo 0 (float BP) on BG1 Zc=384 blocks at E = 25344: hard bits, status and
    iteration counts equal the oracle; beliefs within the BP tolerance."""
    from golden_cases import lq_close

    row = [0, 8, 22936, 0, 1280, 32767, -32767]
    pay, llr = _device_blocks(cuda, CFG, 1024, 10.5, 42)
    res = ldpc_decode(llr, CFG, row, return_app=True)
    st, bits = res.status.cpu().numpy(), res.hardbits.cpu().numpy()
    conv = np.nonzero(st == 0)[0]
    assert len(conv) > 256
    assert np.array_equal(bits[conv, : 8424 // 8], pay.cpu().numpy()[conv])
    llr_h, app, its = llr.cpu().numpy(), res.app.cpu().numpy(), res.iterations.cpu().numpy()
    for i in list(conv[:3]) + list(np.nonzero(st != 0)[0][:3]):
        es, eb, ei, elq = oracle.decode(llr_h[i], in_config(*CFG), dec_cfg(row))
        assert (st[i], its[i]) == (es, ei), i
        if ei > 0:
            assert np.array_equal(bits[i], eb), i
        assert lq_close(app[i], elq, 0, es == 0), i
