"""The per-stream work queue of the uniform decoders.

A launch of more than one kernel wave takes its code blocks from a device queue
(fixed point: every int16 half lane restarts on the next block as soon as its
block finishes; float: CTAs take work items).  A launch of one wave or less
uses fixed work items.  The same blocks must decode identically either way,
with blocks finishing at many different iterations (so half lanes refill at
different times) and with algo 2's iteration-dependent table (the two halves
of a lane pair then use different rows of it); a sample is checked against
the oracle.  Repeated launches on one stream, of different sizes, check that
each launch's last CTA rewinds the queue for the next.
"""

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import channel_llrs, ldpc_decode, ldpc_encode
from oracle.oracle import dec_cfg, in_config

pytestmark = pytest.mark.gpu

CFG = (2, 488, 1, 1920, 0, 2, 0)          # BG2, Zc=64, QPSK, rate 1/4
NOISE_DB = (-2.0, 0.0, 1.0, 2.0, 3.0)     # converges after 3 .. 10 iterations, or not at all


def _llrs(n, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    pay = torch.randint(0, 256, (n, CFG[1] // 8), dtype=torch.uint8, device="cuda", generator=gen)
    rm = ldpc_encode(pay, CFG)
    parts = [channel_llrs(rm, CFG[3], CFG[5], nd, seed=seed + k) for k, nd in enumerate(NOISE_DB)]
    k = torch.arange(n, device="cuda") % len(NOISE_DB)      # neighbouring blocks see different noise
    llr = torch.empty_like(parts[0])
    for j, part in enumerate(parts):
        llr[k == j] = part[k == j]
    return llr


@pytest.mark.parametrize("algo", [1, 2, 4])
def test_queue_and_fixed_items_decode_alike(oracle, cuda, algo):
    row = [algo, 10, 22936, 0, 1280, 32767, -32767]
    n = 12000                              # about 3.4 waves of the fixed-point kernel, 6.8 of the float one
    llr = _llrs(n, seed=40 + algo)
    full = ldpc_decode(llr, CFG, row)      # one launch: the queue
    chunk = 1000                           # under one wave: fixed work items
    parts = [ldpc_decode(llr[i:i + chunk], CFG, row) for i in range(0, n, chunk)]
    torch.cuda.synchronize()
    bits = torch.cat([p.hardbits for p in parts])
    status = torch.cat([p.status for p in parts])
    iters = torch.cat([p.iterations for p in parts])
    assert torch.equal(full.status, status)
    assert torch.equal(full.iterations, iters)
    assert torch.equal(full.hardbits, bits)
    it = iters.cpu().numpy()
    assert len(np.unique(it)) >= 6 and bool((status == 0).any()) and bool((status == 1).any())

    # a second, smaller queued launch on the same stream, then the first again
    again = ldpc_decode(llr[: 2 * n // 3], CFG, row)
    full2 = ldpc_decode(llr, CFG, row)
    torch.cuda.synchronize()
    assert torch.equal(again.hardbits, full.hardbits[: 2 * n // 3])
    assert torch.equal(full2.hardbits, full.hardbits) and torch.equal(full2.iterations, full.iterations)

    # a sample against the oracle
    host = llr.cpu().numpy()
    st, hb = full.status.cpu().numpy(), full.hardbits.cpu().numpy()
    icfg = in_config(*CFG)
    for i in range(0, n, 397):
        es, eb, ei, _ = oracle.decode(host[i], icfg, dec_cfg(row))
        assert (st[i], it[i]) == (es, ei), i
        assert np.array_equal(hb[i, : len(eb)], eb), i


@pytest.mark.parametrize("algo", [1, 2, 0, 4])
def test_queue_app_and_soft_buffers_alike(cuda, algo):
    """With final beliefs requested and HARQ soft buffers combined into, a
    queued launch (refilled half lanes, or queued work items for the float
    kernels) leaves the same beliefs and the same soft buffers as launches of
    fixed work items."""
    cfg = CFG[:6] + (1,)                   # HARQ_on: combine into the soft buffers
    row = [algo, 10, 22936, 0, 1280, 32767, -32767]
    n = 8000 if algo in (1, 2) else 4000  # over two waves of either kernel
    llr = _llrs(n, seed=70 + algo)
    gen = torch.Generator(device="cuda").manual_seed(5)
    harq0 = torch.randint(-200, 200, (n, 52 * 64), dtype=torch.int16, device="cuda", generator=gen)
    ha, hb = harq0.clone(), harq0.clone()
    full = ldpc_decode(llr, cfg, row, return_app=True, harq=ha)
    chunk = 500
    parts = [ldpc_decode(llr[i:i + chunk], cfg, row, return_app=True, harq=hb[i:i + chunk])
             for i in range(0, n, chunk)]
    torch.cuda.synchronize()
    assert torch.equal(ha, hb)
    assert not torch.equal(ha, harq0)
    assert torch.equal(full.hardbits, torch.cat([p.hardbits for p in parts]))
    assert torch.equal(full.iterations, torch.cat([p.iterations for p in parts]))
    app = torch.cat([p.app for p in parts])
    assert torch.equal(full.app, app)


@pytest.mark.parametrize("algo", [1, 4])
def test_queue_zero_iterations_alike(cuda, algo):
    """max_iterations == 0 (rate recovery only, status 1, bits untouched): a
    queued launch and fixed-item launches leave the same beliefs, soft buffers
    and outputs."""
    cfg = CFG[:6] + (1,)
    row = [algo, 0, 22936, 0, 1280, 32767, -32767]
    n = 8000
    llr = _llrs(n, seed=90 + algo)
    gen = torch.Generator(device="cuda").manual_seed(9)
    harq0 = torch.randint(-200, 200, (n, 52 * 64), dtype=torch.int16, device="cuda", generator=gen)
    ha, hb = harq0.clone(), harq0.clone()
    full = ldpc_decode(llr, cfg, row, return_app=True, harq=ha)
    parts = [ldpc_decode(llr[i:i + 500], cfg, row, return_app=True, harq=hb[i:i + 500]) for i in range(0, n, 500)]
    torch.cuda.synchronize()
    assert torch.equal(ha, hb) and not torch.equal(ha, harq0)
    assert bool((full.status == 1).all()) and bool((full.iterations == 0).all())
    assert not bool(full.hardbits.any())
    assert torch.equal(full.app, torch.cat([p.app for p in parts]))
