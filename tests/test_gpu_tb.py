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


def test_limited_buffer_encoder_matches_oracle(cuda, oracle):
    """Device rate matching over a limited circular buffer equals the oracle's
    (itself pinned to py5gphy), every rv."""
    from oracle.oracle import in_config

    from deeplearning_5g_ldpc_decoder_b200.decoder import ldpc_encode

    rng = np.random.default_rng(31)
    for bgn, A, crc, E, Qm, ncb in [(1, 8424, 2, 12000, 8, 18000), (1, 3816, 2, 9000, 4, 10000),
                                    (2, 3816, 2, 8000, 4, 9000), (2, 1000, 1, 2400, 2, 2600)]:
        for rv in range(4):
            cfg = (bgn, A, crc, E, rv, Qm, 0)
            pay = rng.integers(0, 256, (3, A // 8), dtype=np.uint8)
            rm = ldpc_encode(torch.from_numpy(pay).to(cuda), cfg, ncb=ncb).cpu().numpy()
            for i in range(3):
                assert np.array_equal(rm[i], oracle.encode_ncb(pay[i], in_config(*cfg), ncb)), (cfg, ncb, i)


def _harq_expect(oracle, t, arena_h, soft):
    """Oracle soft buffers (combined into `soft`, a list per code block) and per
    code block decode results for one transmission of transport block t."""
    from oracle import tb_ref  # noqa: F401
    from oracle.oracle import dec_cfg, in_config

    from deeplearning_5g_ldpc_decoder_b200 import tb

    sg = tb.segment(int(t["A"]), int(t["G"]), int(t["Qm"]), int(t["bgn"]), int(t["rv"]), int(t["tbs_lbrm"]))
    res = []
    for r in range(sg.C):
        E = sg.E(r)
        cfg = (sg.cb_cfg[0], sg.cb_cfg[1], sg.cb_cfg[2], E, sg.cb_cfg[4], sg.cb_cfg[5],
               1 if (int(t["flags"]) & tb.HARQ_COMBINE) else 0)
        lo = int(t["llr_offset"]) + sg.llr_start(r)
        oracle.rate_recover_ncb(in_config(*cfg), sg.Ncb, 1280, arena_h[lo:lo + E], soft[r])
        res.append(oracle.decode_soft(soft[r], in_config(*cfg[:6], 0), dec_cfg(ROW)))
    return sg, res


def test_harq_retransmission_with_limited_buffer(cuda, oracle):
    """rv 0 then rv 2 of the same blocks with limited-buffer rate matching: the
    device soft buffers after each transmission equal the oracle's HARQ
    combining, every code block decodes as the oracle does from them, and more
    blocks pass after the retransmission."""
    from deeplearning_5g_ldpc_decoder_b200 import tb
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine

    rng = np.random.default_rng(44)
    specs = [(60000, 0.75, 4, 8.3), (20000, 0.8, 6, 14.0), (3000, 0.7, 2, 2.5), (100000, 0.7, 8, 18.5)]
    rows, pays = [], []
    harq_off = 0
    segs = []
    for A0, R, Qm, snr in specs:
        bgn = tb.select_bg(int(A0), R)
        A = tb.round_tbs(A0, bgn)
        G = tb.coded_bits(A, bgn, Qm, R)
        lbrm = int(A * 1.2)
        sg = tb.segment(A, G, Qm, bgn, 0, tbs_lbrm=lbrm)
        rows.append([A, G, Qm, 0, bgn, 0, 0, lbrm, tb.HARQ_STORE, harq_off])
        harq_off += sg.harq_elems
        pays.append(rng.integers(0, 256, A // 8, dtype=np.uint8))
        segs.append(sg)
    noise = [-s[3] for s in specs]
    harq = torch.zeros(harq_off, dtype=torch.int16, device=cuda)
    soft = [[np.zeros(68 * 384, dtype=np.int16) for _ in range(sg.C)] for sg in segs]
    eng = TbEngine(max_tbs=16, max_cbs=256, decoder_row=ROW)
    passed = []
    for tx, rv in enumerate((0, 2)):
        for r in rows:
            r[3] = rv
            r[8] = tb.HARQ_STORE | (tb.HARQ_COMBINE if tx else 0)
        tbs, arena, out_bytes = tb.encode_transport_blocks(pays, tb.tb_array([tuple(r) for r in rows]), noise,
                                                           seed=70 + tx, device=cuda)
        out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
        st, _ = eng.decode(tbs, arena, out, harq=harq)
        torch.cuda.synchronize()
        st = st.cpu().numpy()
        arena_h, harq_h = arena.cpu().numpy(), harq.cpu().numpy()
        p_bits, p_st, p_it, p_first = eng.views()
        first = _dev_array(p_first, len(tbs), torch.int32, cuda)
        for i, t in enumerate(tbs):
            sg, res = _harq_expect(oracle, t, arena_h, soft[i])
            L = 52 * sg.Zc if int(t["bgn"]) == 2 else 68 * sg.Zc
            cb_st = _dev_array(p_st + 4 * int(first[i]), sg.C, torch.int32, cuda)
            cb_it = _dev_array(p_it + 4 * int(first[i]), sg.C, torch.int32, cuda)
            for r in range(sg.C):
                base = int(t["harq_offset"]) + r * L
                assert np.array_equal(harq_h[base:base + L], soft[i][r][:L]), (tx, i, r)
                assert (cb_st[r], cb_it[r]) == (res[r][0], res[r][2]), (tx, i, r)
            if st[i] == 0:
                o = int(t["out_offset"])
                assert np.array_equal(out.cpu().numpy()[o:o + int(t["A"]) // 8], pays[i])
        passed.append(int((st == 0).sum()))
    assert passed[1] > passed[0]


def test_serving_depth8_every_code_block_decodes_as_alone(cuda, oracle):
    """Poisson arrivals through the serving loop with eight batches in flight:
    batches overlap on the device and their composition depends on timing.
    Every code block's status, iteration count and hard bits inside the serve
    run equal the oracle decoding that code block alone, and every transport
    block's verdict equals the oracle's."""
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine, serve

    rng = np.random.default_rng(61)
    specs = []
    for k in range(72):
        A0 = float(np.exp(rng.uniform(np.log(200), np.log(120000))))
        Qm = int(rng.choice([2, 4, 6, 8]))
        R = float(rng.uniform(0.3, 0.85))
        snr = {2: 3.0, 4: 9.0, 6: 14.0, 8: 20.0}[Qm] + 10 * (R - 0.5) + rng.uniform(-2.0, 5.0)
        specs.append((A0, R, Qm, snr))
    tbs, arena, out_bytes, pays = _traffic(rng, specs, cuda)
    eng = TbEngine(max_tbs=64, max_cbs=2048, decoder_row=ROW)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    arrivals = np.cumsum(rng.exponential(1.0 / 20000.0, len(tbs)))     # Poisson, 20k blocks/s
    res = serve(eng, tbs, arrivals, arena, out, max_batch_tbs=8, pipeline_depth=8, timeout_s=60.0, record=True)
    assert res.stats["completed"] == len(tbs) and res.stats["dropped"] == 0 and res.stats["expired"] == 0
    assert res.stats["batches"] >= 9          # more batches than slots: slots were reused while others ran
    arena_h = arena.cpu().numpy()
    n_cb = 0
    for i in range(len(tbs)):
        exp, tb_st, info = _expected(oracle, tbs, arena_h, i)
        f = int(res.cb_first[i])
        for r, (st, bits, it) in enumerate(exp):
            assert (res.cb_status[f + r], res.cb_iterations[f + r]) == (st, it), (i, r)
            if it > 0:
                assert np.array_equal(res.cb_bits[f + r][: len(bits)], bits), (i, r)
        assert res.status[i] == tb_st, i
        n_cb += len(exp)
    assert n_cb > 2 * len(tbs)
    assert 0 < (res.status == 0).sum() < len(tbs)


def test_serving_wait_bound_expires_queued_blocks(cuda):
    """With one batch in flight, one block per batch and everything arriving at
    once, blocks still queued after max_wait_s are dropped as expired (their
    budget freed, latency NaN); the ones served are decoded normally."""
    from deeplearning_5g_ldpc_decoder_b200.tb import TbEngine, serve

    rng = np.random.default_rng(23)
    tbs, arena, out_bytes, _ = _traffic(rng, [(60000, 0.5, 4, 20.0)] * 30, cuda)
    eng = TbEngine(max_tbs=4, max_cbs=64, decoder_row=ROW)
    out = torch.zeros(out_bytes + 8, dtype=torch.uint8, device=cuda)
    res = serve(eng, tbs, np.zeros(len(tbs)), arena, out, max_batch_tbs=1, pipeline_depth=1, timeout_s=30.0,
                max_wait_s=1e-4)
    expired = res.status == -6
    assert expired.sum() == res.stats["expired"] > 0
    assert np.all(res.status[~expired] == 0) and (~expired).sum() >= 1
    assert np.all(np.isnan(res.latency_s[expired])) and np.all(np.isfinite(res.latency_s[~expired]))
    assert res.stats["completed"] + res.stats["expired"] == len(tbs)
