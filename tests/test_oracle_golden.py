"""Pin the CPU oracle to the reference: every golden vector in
tests/golden/reference_vectors.npz was produced by the reference C library
built from its own sources (tests/golden/make_golden.py)."""

import numpy as np
import pytest

from golden_cases import algo_rows, decode_cases, expected, harq_sequences, lq_close
from oracle.oracle import dec_cfg, in_config


def test_params_match_reference(oracle, golden):
    for bgn, A, crc, B, Zc, iLS, K, F, N, k0 in golden["params"]:
        rc, p = oracle.derive(in_config(int(bgn), int(A), int(crc), 1200, 1, 2, 0))
        assert rc == 0
        assert (p.B, p.Zc, p.iLS, p.K, p.F, p.N, p.k0) == (B, Zc, iLS, K, F, N, k0)


def test_crc_matches_reference(oracle, golden):
    data = golden["crc_in"]
    for t in range(4):
        for j, L in enumerate(golden["crc_lens"]):
            assert oracle.crc(data[:L], t) == golden["crc_out"][t, j]


def test_encoder_matches_reference(oracle, golden):
    for key, cfg, _ in decode_cases(golden):
        rm = oracle.encode(golden[f"{key}_payload"], in_config(*cfg))
        assert np.array_equal(rm, golden[f"{key}_rm"]), key


@pytest.mark.parametrize("ai", range(6))
def test_decoders_match_reference(oracle, golden, ai):
    row = algo_rows(golden)[ai]
    for key, cfg, llr in decode_cases(golden):
        st, bits, its, lq = oracle.decode(llr, in_config(*cfg), dec_cfg(row))
        est, ebits, eits, elq = expected(golden, key, ai)
        assert st == est, key
        assert np.array_equal(bits, ebits), key
        assert its == eits, key
        assert lq_close(lq, elq, row[0], est == 0), key


def test_harq_sequences_match_reference(oracle, golden):
    row = [1, 8, 22936, 0, 1280, 32767, -32767]
    for hi, steps in harq_sequences(golden):
        buf = np.zeros(68 * 384, dtype=np.int16)
        for s in steps:
            st, bits, _, lq = oracle.decode(s["llr"], in_config(*s["cfg"]), dec_cfg(row), harq=buf)
            assert st == s["status"], (hi, s["cfg"])
            assert np.array_equal(bits, s["bits"])
            assert np.array_equal(lq, s["lq"])
            assert np.array_equal(buf[: len(s["buf"])], s["buf"])


def test_trained_tables_are_the_degree_rule(golden):
    """The reference's compiled-in algo-2 tables (c_lib/BG*_trained_ldpc_weights.c)
    are the degree rule repeated for 32 iterations with zero beta; the library's
    built-in table restates exactly that."""
    for bgn in (1, 2):
        off = golden[f"bg{bgn}_off"].astype(int)
        deg = np.diff(off)
        rule = np.where(deg <= 4, 26623, np.where(deg <= 8, 24575, 22527))
        assert np.array_equal(golden[f"bg{bgn}_trained_alpha"], np.tile(rule, (32, 1)))
        assert not golden[f"bg{bgn}_trained_beta"].any()
