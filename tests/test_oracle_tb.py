"""CPU checks of the transport-block path's checker and host logic.

* oracle/tb_ref.py reproduces py5gphy's segmentation, rate-matching lengths
  and CRCs (tests/golden/tb_vectors.npz, tests/golden/make_tb_golden.py);
* the library's segmentation (nrldpc_tb_segment, the same __host__ __device__
  code the device segmentation kernel runs) agrees with the oracle on random
  transport blocks, and every code-block configuration it produces derives
  through gen_ldpc_parameters to the same B and lifting size.
"""

import ctypes
import os

import numpy as np
import pytest

from tests.conftest import REPO

TB_GOLDEN = os.path.join(REPO, "tests", "golden", "tb_vectors.npz")


@pytest.fixture(scope="module")
def tbg():
    return np.load(TB_GOLDEN)


def test_tb_ref_matches_py5gphy(tbg):
    from oracle import tb_ref

    for B, bgn, C, cbz, L, F, K, Zc in tbg["cbs"]:
        assert tb_ref.cbs_info(int(B), int(bgn)) == (C, cbz, L, F, K, Zc), (B, bgn)
    er = tbg["er"]
    last = None
    for G, C, Qm, r, e in er:
        if (G, C, Qm) != last:
            lst = tb_ref.er_list(int(G), int(C), int(Qm))
            last = (G, C, Qm)
        assert lst[r] == e
    for i, (poly, n) in enumerate(zip(tbg["crc_poly"], tbg["crc_len"])):
        bits = np.unpackbits(tbg[f"crc_in_{i}"])[: int(n)]
        assert np.array_equal(tb_ref.crc_remainder_bits(bits, str(poly)), tbg[f"crc_out_{i}"]), (poly, n)


def _random_tbs(rng, count):
    from deeplearning_5g_ldpc_decoder_b200 import tb

    out = []
    while len(out) < count:
        A0 = float(np.exp(rng.uniform(np.log(200), np.log(1.2e6))))
        R = float(rng.uniform(0.2, 0.9))
        Qm = int(rng.choice([2, 4, 6, 8]))
        bgn = tb.select_bg(int(A0), R)
        A = tb.round_tbs(A0, bgn)
        C, _ = tb.code_block_count(A, bgn)
        G = tb.coded_bits(A, bgn, Qm, R)
        if -(-G // Qm // C) * Qm > 65535:
            continue
        out.append((A, G, Qm, int(rng.integers(4)), bgn))
    return out


def test_library_segmentation_matches_oracle(lib):
    from deeplearning_5g_ldpc_decoder_b200 import capi, tb
    from oracle import tb_ref

    rng = np.random.default_rng(7)
    for A, G, Qm, rv, bgn in _random_tbs(rng, 600):
        sg = tb.segment(A, G, Qm, bgn, rv)
        cbs, info = tb_ref.segment(A, G, Qm, bgn, rv)
        assert sg.C == info["C"] and sg.Kp == info["Kp"] and sg.Zc == info["Zc"] and sg.L_tb == info["L_tb"]
        for r, (cfg, start) in enumerate(cbs):
            assert sg.E(r) == cfg[3] and sg.llr_start(r) == start
            assert (sg.cb_cfg[0], sg.cb_cfg[1], sg.cb_cfg[2], sg.cb_cfg[4], sg.cb_cfg[5]) == \
                (cfg[0], cfg[1], cfg[2], cfg[4], cfg[5])
        # the per-code-block configuration is a valid reference configuration with the same derivation
        out = capi.LdpcConfig()
        c = capi.make_in_config(*sg.cb_cfg)
        assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(c)) == 0
        assert out.B == sg.Kp and out.Zc == sg.Zc and out.K - out.B == info["F"]


def test_select_bg_and_round_tbs():
    from deeplearning_5g_ldpc_decoder_b200 import tb
    from oracle import tb_ref

    for A in (24, 200, 292, 293, 1000, 3824, 3825, 10000, 500000):
        for R in (0.1, 0.25, 0.26, 0.5, 0.67, 0.68, 0.9):
            assert tb.select_bg(A, R) == tb_ref.select_bg(A, R), (A, R)
    rng = np.random.default_rng(3)
    for _ in range(2000):
        A0 = float(np.exp(rng.uniform(np.log(24), np.log(1.3e6))))
        for bgn in (1, 2):
            A = tb.round_tbs(A0, bgn)
            assert 24 <= A <= max(A0, 24) and A % 8 == 0
            tb_ref.cbs_info(A + (24 if A > 3824 else 16), bgn)   # raises if it does not split evenly


def test_segmentation_rejects_bad_blocks():
    from deeplearning_5g_ldpc_decoder_b200 import tb

    with pytest.raises(ValueError):
        tb.segment(1001, 3000, 2, 1)          # A not a multiple of 8
    with pytest.raises(ValueError):
        tb.segment(1000, 3001, 2, 1)          # G not a multiple of Qm
    with pytest.raises(ValueError):
        tb.segment(8000, 140000, 2, 1)        # one code block of E > 65535
    with pytest.raises(ValueError):
        tb.segment(99992, 300000, 2, 1)       # does not split into equal byte-aligned code blocks
    with pytest.raises(ValueError):
        tb.segment(1000, 3000, 3, 1)          # bad Qm


LBRM_GOLDEN = os.path.join(REPO, "tests", "golden", "lbrm_vectors.npz")


def test_limited_buffer_oracle_matches_py5gphy(oracle):
    """The oracle's limited-buffer rate matching and recovery reproduce py5gphy's
    (k0, selected bits, recovered soft values outside the filler positions)."""
    from oracle.oracle import in_config

    g = np.load(LBRM_GOLDEN)
    for i, (bgn, A, crc, E, rv, Qm, ncb) in enumerate(g["cases"]):
        cfg = in_config(*[int(x) for x in (bgn, A, crc, E, rv, Qm)])
        p = oracle.params(cfg, int(ncb))
        assert p.k0 == int(g[f"k0_{i}"][0]) and p.Ncb == int(ncb)
        rm = np.unpackbits(oracle.encode_ncb(g[f"pay_{i}"], cfg, int(ncb)))[: int(E)]
        assert np.array_equal(rm, g[f"rm_{i}"]), i
        h = oracle.rate_recover_ncb(cfg, int(ncb), 1280, g[f"llr_{i}"])[: p.N + 2 * p.Zc]
        keep = np.ones(p.N, dtype=bool)
        keep[p.B - 2 * p.Zc: p.K - 2 * p.Zc] = False
        assert np.array_equal(h[2 * p.Zc:][keep].astype(np.float64), g[f"rec_{i}"][keep]), i


def test_library_limited_buffer_segmentation(oracle):
    """Ncb = min(N, floor(3 TBS_LBRM / 2C)) per code block and k0 from it agree
    with the oracle's TS 38.212 restatement; a buffer that would cut into the
    systematic bits is rejected."""
    from oracle.oracle import in_config

    from deeplearning_5g_ldpc_decoder_b200 import tb

    rng = np.random.default_rng(17)
    checked = 0
    for A, G, Qm, rv, bgn in _random_tbs(rng, 300):
        C, _ = tb.code_block_count(A, bgn)
        lbrm = int(rng.integers(A // 2, 3 * A))
        try:
            sg = tb.segment(A, G, Qm, bgn, rv, tbs_lbrm=lbrm)
        except ValueError:
            full = tb.segment(A, G, Qm, bgn, rv)
            K = (22 if bgn == 1 else 10) * full.Zc
            assert (3 * lbrm) // (2 * C) < K - 2 * full.Zc
            continue
        p = oracle.params(in_config(*sg.cb_cfg[:6]), min((3 * lbrm) // (2 * C), 10 ** 9))
        assert sg.Ncb == p.Ncb and sg.k0 == p.k0, (A, G, Qm, rv, bgn, lbrm)
        assert sg.harq_elems == C * (p.N + 2 * p.Zc)
        checked += 1
    assert checked > 150
