"""Mixed-size persistent decode (CUDA graph, autotuner) vs the oracle decoding
every block on its own (config-3 style batch, smaller)."""

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200.mixed import MixedPlan, random_mixed_configs
from oracle.oracle import dec_cfg, in_config, make_llrs

pytestmark = pytest.mark.gpu


def _build(oracle, n, seed, noise_db):
    cfgs = random_mixed_configs(n, seed=seed)
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
