"""GPU parity of the transport-block path: on-device segmentation, one mixed
decode of all code blocks, on-device transport-block CRC and payload gather,
and the serving loop.

Every code block is checked bit-exactly against the C oracle decoding the
same LLR slice with the code block's reference configuration; every
transport-block verdict against the oracle's segmentation and CRC
(oracle/tb_ref.py, pinned to py5gphy).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROW = [1, 10, 22936, 0, 1280, 32767, -32767]


def _traffic(rng, specs, device):
    """specs: (A0, R, Qm, snr_db) -> encoded first transmissions (rv 0: redundancy
    versions 1-3 alone carry few or no systematic bits, and a block whose
    information LLRs are all zero "decodes" to the all-zero word, whose CRC
    passes -- the reference behaves the same)."""
    from deeplearning_5g_ldpc_decoder_b200 import tb

    rows, pays, noise = [], [], []
    for A0, R, Qm, snr in specs:
        bgn = tb.select_bg(int(A0), R)
        A = tb.round_tbs(A0, bgn)
        G = tb.coded_bits(A, bgn, Qm, R)
        rows.append((A, G, Qm, 0, bgn, 0, 0))
        pays.append(rng.integers(0, 256, A // 8, dtype=np.uint8))
        noise.append(-snr)
    tbs, arena, out_bytes = tb.encode_transport_blocks(pays, tb.tb_array(rows), noise, seed=11, device=device)
    return tbs, arena, out_bytes, pays


def _expected(oracle, tbs, arena_h, i):
    """Per code block (status, bits, iterations) from the oracle, and the TB verdict."""
    from oracle import tb_ref
    from oracle.oracle import dec_cfg, in_config

    t = tbs[i]
    cbs, info = tb_ref.segment(int(t["A"]), int(t["G"]), int(t["Qm"]), int(t["bgn"]), int(t["rv"]))
    res = []
    for cfg, start in cbs:
        lo = int(t["llr_offset"]) + start
        st, bits, it, _ = oracle.decode(arena_h[lo:lo + cfg[3]], in_config(*cfg), dec_cfg(ROW))
        res.append((st, bits, it))
    ok = all(r[0] == 0 for r in res)
    if ok and info["C"] > 1:
        nb = cbs[0][0][1]
        tb_bits = np.concatenate([np.unpackbits(r[1])[:nb] for r in res])
        ok = tb_ref.crc_check(tb_bits, "24A")
    return res, (0 if ok else 1), info


def test_engine_matches_oracle_per_code_block_and_transport_block(cuda, oracle):
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine

    rng = np.random.default_rng(5)
    specs = []
    for k in range(28):
        A0 = float(np.exp(rng.uniform(np.log(200), np.log(60000))))
        Qm = int(rng.choice([2, 4, 6, 8]))
        R = float(rng.uniform(0.25, 0.85))
        snr = {2: 3.0, 4: 9.0, 6: 14.0, 8: 20.0}[Qm] + 10 * (R - 0.5) + (6.0 if k % 3 else -3.0)
        specs.append((A0, R, Qm, snr))
    specs += [(200, 0.3, 2, -5.0), (3824, 0.5, 2, 6.0), (8424, 0.8, 8, 30.0), (100000, 0.5, 4, 15.0)]
    tbs, arena, out_bytes, pays = _traffic(rng, specs, cuda)
    eng = TbEngine(max_tbs=64, max_cbs=512, decoder_row=ROW)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    status, iters = eng.decode(tbs, arena, out)
    torch.cuda.synchronize()
    p_bits, p_st, p_it, p_first = eng.views()
    n_cb_total = 0
    arena_h = arena.cpu().numpy()
    status_h, iters_h, out_h = status.cpu().numpy(), iters.cpu().numpy(), out.cpu().numpy()
    # device views of the code-block results
    first = _dev_array(p_first, len(tbs), torch.int32, cuda)
    seen_pass = seen_fail = 0
    for i in range(len(tbs)):
        res, tb_st, info = _expected(oracle, tbs, arena_h, i)
        C = info["C"]
        cb_st = _dev_array(p_st + 4 * int(first[i]), C, torch.int32, cuda)
        cb_it = _dev_array(p_it + 4 * int(first[i]), C, torch.int32, cuda)
        cb_bits = _dev_array(p_bits + 1056 * int(first[i]), C * 1056, torch.uint8, cuda).reshape(C, 1056)
        for r, (st, bits, it) in enumerate(res):
            assert cb_st[r] == st and cb_it[r] == it, (i, r)
            if it > 0:
                assert np.array_equal(cb_bits[r][: len(bits)], bits), (i, r)
        assert status_h[i] == tb_st, i
        assert iters_h[i] == max(r[2] for r in res)
        if tb_st == 0:
            A = int(tbs[i]["A"])
            o = int(tbs[i]["out_offset"])
            assert np.array_equal(out_h[o:o + A // 8], pays[i]), i
            seen_pass += 1
        else:
            seen_fail += 1
        n_cb_total += C
    assert seen_pass >= 10 and seen_fail >= 3 and n_cb_total > len(tbs)


class _DevBytes:
    """A device address range as a CUDA-array-interface object."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _dev_array(ptr, n, dtype, dev):
    """Copy n elements at a device address of the library into a numpy array."""
    out = torch.empty(n, dtype=dtype, device=dev)
    raw = torch.as_tensor(_DevBytes(ptr, n * out.element_size()), device=dev)
    out.view(torch.uint8).copy_(raw)
    return out.cpu().numpy()


def test_engine_flags_bad_and_oversize_batches(cuda):
    from deeplearning_5g_ldpc_decoder_b200 import tb
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine

    rng = np.random.default_rng(9)
    tbs, arena, out_bytes, _ = _traffic(rng, [(1000, 0.5, 2, 10.0), (20000, 0.5, 4, 20.0)], cuda)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    bad = tbs.copy()
    bad[0]["A"] = 1001            # not a multiple of 8: configuration error for this block only
    eng = TbEngine(max_tbs=8, max_cbs=64, decoder_row=ROW)
    st, _ = eng.decode(bad, arena, out)
    st = st.cpu().numpy()
    assert st[0] == -2 and st[1] == 0
    small = TbEngine(max_tbs=8, max_cbs=2, decoder_row=ROW)   # the 20000-bit block alone needs 3 code blocks
    assert tb.segment(int(tbs[1]["A"]), int(tbs[1]["G"]), 4, int(tbs[1]["bgn"])).C > 2
    st, _ = small.decode(tbs, arena, out)
    assert (st.cpu().numpy() == -4).all()


def test_serving_loop_matches_offline_decode(cuda):
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine, serve

    rng = np.random.default_rng(21)
    specs = []
    for k in range(160):
        A0 = float(np.exp(rng.uniform(np.log(200), np.log(200000))))
        Qm = int(rng.choice([2, 4, 6, 8]))
        R = float(rng.uniform(0.3, 0.8))
        snr = {2: 3.0, 4: 9.0, 6: 14.0, 8: 20.0}[Qm] + 10 * (R - 0.5) + rng.uniform(0, 6)
        specs.append((A0, R, Qm, snr))
    tbs, arena, out_bytes, pays = _traffic(rng, specs, cuda)
    eng = TbEngine(max_tbs=256, max_cbs=4096, decoder_row=ROW)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    ref_st, _ = eng.decode(tbs, arena, out)
    ref_st = ref_st.cpu().numpy()
    arrivals = np.cumsum(rng.exponential(1.0 / 4000.0, len(tbs)))     # Poisson, 4k blocks/s
    res = serve(eng, tbs, arrivals, arena, out, max_batch_tbs=64, pipeline_depth=2, timeout_s=60.0)
    assert res.stats["completed"] == len(tbs) and res.stats["dropped"] == 0
    assert np.array_equal(res.status, ref_st)
    assert np.all(np.isfinite(res.latency_s)) and np.all(res.latency_s > 0)
    assert res.latency_s.max() < 5.0
    assert res.stats["batches"] >= 2
    out_h = out.cpu().numpy()
    for i in np.nonzero(res.status == 0)[0]:
        o, A = int(tbs[i]["out_offset"]), int(tbs[i]["A"])
        assert np.array_equal(out_h[o:o + A // 8], pays[i])


def test_serving_admission_drops_over_budget(cuda):
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine, serve

    rng = np.random.default_rng(22)
    tbs, arena, out_bytes, _ = _traffic(rng, [(30000, 0.5, 4, 20.0)] * 40, cuda)
    eng = TbEngine(max_tbs=64, max_cbs=1024, decoder_row=ROW)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    budget = 2 * int(tbs[0]["G"]) * 3          # room for three blocks' LLRs
    res = serve(eng, tbs, np.zeros(len(tbs)), arena, out, llr_budget_bytes=budget, timeout_s=30.0)
    dropped = res.status == -5
    assert dropped.sum() == len(tbs) - 3 and res.stats["dropped"] == len(tbs) - 3
    assert np.all(res.status[~dropped] == 0)
    assert np.all(np.isnan(res.latency_s[dropped])) and np.all(np.isfinite(res.latency_s[~dropped]))
