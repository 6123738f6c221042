"""Mixed-size persistent decode (CUDA graph, autotuner) vs the oracle decoding
every block on its own (config-3 style batch, smaller)."""

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200.mixed import MixedPlan, random_mixed_configs
from oracle.oracle import dec_cfg, in_config, make_llrs

pytestmark = pytest.mark.gpu


def _build(oracle, n, seed, noise_db, cfgs=None):
    cfgs = cfgs or random_mixed_configs(n, seed=seed)
    llrs = []
    for i, c in enumerate(cfgs):
        llr, _ = make_llrs(oracle, in_config(*c, 0), 1, noise_db=noise_db - 0.5 * (i % 4), seed=seed * 7919 + i)
        llrs.append(torch.from_numpy(llr[0]))
    return cfgs, llrs


@pytest.mark.parametrize("row", [[1, 10, 22936, 0, 1280, 32767, -32767], [3, 6, 22936, 0, 1280, 32767, -32767],
                                 [2, 7, 22936, 0, 1280, 32767, -32767]])
def test_mixed_batch_bit_exact_per_block(oracle, cuda, row):
    cfgs, llrs = _build(oracle, 300, seed=row[0], noise_db=-2.0)
    plan = MixedPlan(cfgs, row)
    arena = plan.pack_llrs(llrs)
    stream = torch.cuda.Stream(cuda)
    with torch.cuda.stream(stream):
        bits, status, iters = plan.decode(arena, use_graph=True)
        bits2, status2, iters2 = plan.decode(arena, use_graph=True)    # graph replay
    stream.synchronize()
    assert torch.equal(bits, bits2) and torch.equal(status, status2)
    st, it, b = status.cpu().numpy(), iters.cpu().numpy(), bits.cpu().numpy()
    conv = 0
    for i, c in enumerate(cfgs):
        es, eb, ei, _ = oracle.decode(llrs[i].numpy(), in_config(*c, 0), dec_cfg(row))
        assert (st[i], it[i]) == (es, ei), (i, c)
        got = b[plan.bits_offsets[i]: plan.bits_offsets[i] + plan.nbytes[i]]
        assert np.array_equal(got, eb), (i, c)
        conv += es == 0
    assert 0 < conv < len(cfgs)      # a mix of converging and failing blocks
    best, ms = plan.autotune(arena)
    assert 0 <= best < 4 and all(m > 0 for m in ms)
    bits3, status3, _ = plan.decode(arena, use_graph=False)
    torch.cuda.synchronize()
    assert torch.equal(bits3, bits) and torch.equal(status3, status)
    plan.close()


def test_mixed_lane_refill_bit_exact(oracle, cuda):
    """Many blocks of one lifting size per base graph (Zc = 16: 24 lane pairs per
    CTA, so each graph's queue refills every finished half lane several times),
    blocks converging at different iterations, and algo 2's iteration-dependent
    table: every block must still decode exactly as it does alone."""
    import ctypes

    from deeplearning_5g_ldpc_decoder_b200 import capi

    lib = capi.load_library()
    pool = random_mixed_configs(16000, seed=11, rvs=(0,))
    cfgs = []
    for c in pool:
        out = capi.LdpcConfig()
        assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(capi.make_in_config(*c, 0))) == 0
        if out.Zc == 16:
            cfgs.append(c)
    assert len(cfgs) >= 250
    cfgs, llrs = _build(oracle, len(cfgs), seed=5, noise_db=-10.0, cfgs=cfgs)
    row = [2, 9, 22936, 0, 1280, 32767, -32767]
    plan = MixedPlan(cfgs, row)
    arena = plan.pack_llrs(llrs)
    bits, status, iters = plan.decode(arena, use_graph=False)
    torch.cuda.synchronize()
    st, it, b = status.cpu().numpy(), iters.cpu().numpy(), bits.cpu().numpy()
    for i, c in enumerate(cfgs):
        es, eb, ei, _ = oracle.decode(llrs[i].numpy(), in_config(*c, 0), dec_cfg(row))
        assert (st[i], it[i]) == (es, ei), (i, c)
        assert np.array_equal(b[plan.bits_offsets[i]: plan.bits_offsets[i] + plan.nbytes[i]], eb), (i, c)
    assert len(set(it.tolist())) >= 5      # blocks finish at many different iterations
    plan.close()
