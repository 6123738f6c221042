"""The scatter-form rate recovery's index arithmetic, checked on the CPU.

The fixed-point and mixed-size kernels place rate-matched LLR e at soft-buffer
position pos(e) when no LLR repeats (E <= N - F): symbol s = e / Qm through one
high multiply by ceil(2^32 / Qm) (s = e for Qm = 1), bit b = e - s Qm,
k = b (E / Qm) + s, compact position c = (c0 + k) mod (N - F), then the filler
gap and the 2 Zc punctured columns (csrc/nrldpc_decode_common.cuh
scatter_position and div_qm, csrc/nrldpc_mixed.cu recover_halves_mixed).  Here
that arithmetic is replayed with 32-bit unsigned semantics for every Qm, every
rv, both base graphs and a sweep of sizes, and compared with where the oracle's
rate recovery (a restatement of c_lib/ldpc_rate_recovery.c:24-65) puts each
LLR: every position must be in range, outside the filler, distinct, and the
oracle's.  No GPU needed."""

import numpy as np
import pytest

from oracle.oracle import in_config

M32 = (1 << 32) - 1


def qm_magic(qm):
    return 0 if qm <= 1 else ((1 << 32) + qm - 1) // qm & M32


def scatter_positions(p, E, Qm, ncb=0):
    """Device formula, vectorised: positions of LLRs 0..E-1 (circular buffer of
    ncb bits when 0 < ncb < N, as the transport-block engine derives it)."""
    e = np.arange(E, dtype=np.uint64)
    s = e if Qm == 1 else (e * np.uint64(qm_magic(Qm))) >> np.uint64(32)
    b = e - s * np.uint64(Qm)
    Nv = (ncb if 0 < ncb < p.N else p.N) - p.F
    fill_lo, fill_hi = p.B - 2 * p.Zc, p.K - 2 * p.Zc
    c0 = p.k0 if p.k0 < fill_lo else (fill_lo if p.k0 < fill_hi else p.k0 - p.F)
    c = (np.int64(c0) + (b * np.uint64(E // Qm) + s).astype(np.int64))
    c = np.where(c >= Nv, c - Nv, c)
    return np.where(c < p.B - 2 * p.Zc, c, c + p.F) + 2 * p.Zc


def cases():
    rng = np.random.default_rng(3)
    out = []
    for bgn in (1, 2):
        for Qm in (1, 2, 4, 6, 8):
            for rv in range(4):
                for _ in range(6):
                    A = 8 * int(rng.integers(2, (8400 if bgn == 1 else 3800) // 8))
                    R = float(rng.uniform(0.34 if bgn == 1 else 0.21, 0.95))
                    E = Qm * max(1, int(round((A + 24) / R / Qm)))
                    out.append((bgn, A, 1, E, rv, Qm))
    return out


@pytest.mark.parametrize("cfg", cases())
def test_scatter_positions_match_oracle_rate_recovery(oracle, cfg):
    rc, p = oracle.derive(in_config(*cfg))
    if rc != 0:
        pytest.skip("configuration rejected by gen_ldpc_parameters")
    E, Qm = cfg[3], cfg[5]
    Nv = p.N - p.F
    if E > Nv or E > 32000:
        pytest.skip("repetition: the kernels use the gather form")
    pos = scatter_positions(p, E, Qm)
    L = p.N + 2 * p.Zc
    assert pos.min() >= 2 * p.Zc and pos.max() < L
    assert not np.any((pos >= p.B) & (pos < p.K))
    assert len(np.unique(pos)) == E
    # the oracle's placement: LLR e carries the value e + 1
    llr = (np.arange(E) + 1).astype(np.int16)
    buf = oracle.rate_recover(in_config(*cfg), -32000, llr)
    where = np.full(E, -1)
    hit = (buf >= 1) & (np.arange(L) >= 2 * p.Zc)
    where[buf[hit].astype(np.int64) - 1] = np.nonzero(hit)[0]
    assert np.array_equal(where, pos)


def lbrm_cases():
    rng = np.random.default_rng(4)
    out = []
    for bgn in (1, 2):
        for Qm in (1, 2, 4, 8):
            for rv in range(4):
                A = 8 * int(rng.integers(40, (8400 if bgn == 1 else 3800) // 8))
                R = float(rng.uniform(0.5, 0.9))
                E = Qm * max(1, int(round((A + 24) / R / Qm)))
                out.append(((bgn, A, 1, E, rv, Qm), float(rng.uniform(0.3, 0.95))))
    return out


@pytest.mark.parametrize("cfg,frac", lbrm_cases())
def test_scatter_positions_with_limited_buffer(oracle, cfg, frac):
    """Limited-buffer rate matching (Ncb < N, TS 38.212 5.4.2.1) in the mixed
    kernel: compact length Ncb - F, k0 scaled by Ncb / N."""
    rc, p = oracle.derive(in_config(*cfg))
    if rc != 0:
        pytest.skip("configuration rejected by gen_ldpc_parameters")
    ncb = int(p.K - 2 * p.Zc + frac * (p.N - (p.K - 2 * p.Zc)))
    q = oracle.params(in_config(*cfg), ncb)
    E, Qm = cfg[3], cfg[5]
    if E > q.Ncb - q.F or E > 32000:
        pytest.skip("repetition: the kernels use the gather form")
    pos = scatter_positions(q, E, Qm, q.Ncb)
    assert pos.min() >= 2 * q.Zc and pos.max() < 2 * q.Zc + q.Ncb
    assert not np.any((pos >= q.B) & (pos < q.K)) and len(np.unique(pos)) == E
    llr = (np.arange(E) + 1).astype(np.int16)
    L = q.N + 2 * q.Zc
    buf = oracle.rate_recover_ncb(in_config(*cfg), q.Ncb, -32000, llr)[:L]
    where = np.full(E, -1)
    hit = (buf >= 1) & (np.arange(L) >= 2 * q.Zc)
    where[buf[hit].astype(np.int64) - 1] = np.nonzero(hit)[0]
    assert np.array_equal(where, pos)
