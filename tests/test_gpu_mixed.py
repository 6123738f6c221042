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
    assert 0 <= best < 8 and len(ms) == 8 and all(m > 0 for m in ms)
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


def test_config3_full_batch_every_block_matches_oracle(cuda):
    """The mixed-size workload at its full size: 32768 code blocks, lifting
    sizes uniform over all 51, BG1 60 %, rate U[0.2, 0.92], Qm {2, 4, 6, 8},
    algo 1, 10 iterations, decoded in one persistent launch from a CUDA graph.
    Every block's status, iteration count and hard bits equal the oracle
    decoding that block alone (on all host cores)."""
    from deeplearning_5g_ldpc_decoder_b200 import channel_llrs, ldpc_encode
    from tests.oracle_pool import oracle_decode_blocks

    n = 32768
    cfgs = random_mixed_configs(n, seed=2024, rvs=(0,))
    gen = torch.Generator(device=cuda).manual_seed(7)
    llrs = []
    for i, (bgn, A, crc, E, rv, Qm) in enumerate(cfgs):
        pay = torch.randint(0, 256, (1, A // 8), dtype=torch.uint8, device=cuda, generator=gen)
        eta = (A + 24) / E * Qm
        snr = 10.0 * np.log10(2.0 ** eta - 1.0) + 3.0 + 0.5 * (i % 5)
        llrs.append(channel_llrs(ldpc_encode(pay, (bgn, A, crc, E, rv, Qm, 0)), E, Qm, -snr, seed=i)[0])
    row = [1, 10, 22936, 0, 1280, 32767, -32767]
    plan = MixedPlan(cfgs, row, device=cuda)
    arena = torch.cat(llrs)
    stream = torch.cuda.Stream(cuda)
    with torch.cuda.stream(stream):
        plan.decode(arena, use_graph=True)
        bits, status, iters = plan.decode(arena, use_graph=True)
    stream.synchronize()
    st, it, b = status.cpu().numpy(), iters.cpu().numpy(), bits.cpu().numpy()
    est, eit, ebits = oracle_decode_blocks(arena.cpu().numpy(), cfgs, plan.llr_offsets, row)
    bad_status = np.nonzero((st != est) | (it != eit))[0]
    bad_bits = [i for i in range(n)
                if eit[i] > 0 and not np.array_equal(b[plan.bits_offsets[i]: plan.bits_offsets[i] + plan.nbytes[i]],
                                                     ebits[i])]
    assert len(bad_status) == 0 and len(bad_bits) == 0, (bad_status[:10], bad_bits[:10])
    conv = int((est == 0).sum())
    assert 0.5 * n < conv < n and len(set(eit.tolist())) >= 5
    plan.close()


def test_right_sized_ctas_match_384_thread_ctas_and_oracle(oracle, cuda):
    """Lifting sizes where 384-thread CTAs leave threads idle (104 .. 240) go to
    256-thread CTAs (at most 240 active lifted rows, three per SM) under the
    right-sized candidates; the results must not depend on the CTA class: both
    equal the oracle block by block."""
    import ctypes

    from deeplearning_5g_ldpc_decoder_b200 import capi

    lib = capi.load_library()
    want_zc = {104, 112, 120, 208, 224, 240, 192, 384, 26, 13}
    pool = random_mixed_configs(20000, seed=41, rvs=(0,))
    cfgs, seen = [], {}
    for c in pool:
        out = capi.LdpcConfig()
        assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(capi.make_in_config(*c, 0))) == 0
        if out.Zc in want_zc and seen.get((c[0], out.Zc), 0) < 24:
            seen[(c[0], out.Zc)] = seen.get((c[0], out.Zc), 0) + 1
            cfgs.append(c)
    assert {z for _, z in seen} >= {208, 224, 240}
    cfgs, llrs = _build(oracle, len(cfgs), seed=9, noise_db=-6.0, cfgs=cfgs)
    row = [1, 8, 22936, 0, 1280, 32767, -32767]
    plan = MixedPlan(cfgs, row, device=cuda)
    arena = plan.pack_llrs(llrs)
    res = {}
    for cand in (0, 3, 4, 7):
        plan.select(cand)
        bits, status, iters = plan.decode(arena, use_graph=cand % 2 == 0)
        torch.cuda.synchronize()
        res[cand] = (bits.clone(), status.clone(), iters.clone())
    for cand in (3, 4, 7):
        assert all(torch.equal(a, b) for a, b in zip(res[0], res[cand])), cand
    b, st, it = (t.cpu().numpy() for t in res[0])     # (bits, status, iterations)
    for i, c in enumerate(cfgs):
        es, eb, ei, _ = oracle.decode(llrs[i].numpy(), in_config(*c, 0), dec_cfg(row))
        assert (st[i], it[i]) == (es, ei), (i, c)
        assert np.array_equal(b[plan.bits_offsets[i]: plan.bits_offsets[i] + plan.nbytes[i]], eb), (i, c)
    with pytest.raises(RuntimeError):
        plan.select(8)
    plan.close()
