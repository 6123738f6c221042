"""Transport-block reference: segmentation, rate-matching lengths and CRCs.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the library's
transport-block path (nrldpc_tb_segment, the TB engine, the serving loop).
Nothing in the product imports it.

Restates, in plain Python/numpy:
* code-block segmentation, TS 38.212 5.2.2, as py5gphy/ldpc/ldpc_info.py:59-109
  (``get_cbs_info``: C, K', lifting size by the Kb rule, filler count);
* per-code-block rate-matching lengths, TS 38.212 5.4.2.1, as
  py5gphy/ldpc/nr_ldpc_ratematch.py:22-45 (``get_Er_ldpc``);
* CRC attach / check by shift-register division, as
  py5gphy/crc/crc.py:57-131 (``nr_crc_encode`` / ``nr_crc_decode``), with the
  TS 38.212 5.1 polynomials;
* base-graph choice, TS 38.212 7.2.2 (not in the reference; from the standard).
Pinned by tests/test_oracle_tb.py against vectors produced by py5gphy itself
(tests/golden/make_tb_golden.py).
"""

from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

LIFTING = sorted({a << j for a in (2, 3, 5, 7, 9, 11, 13, 15) for j in range(8) if (a << j) <= 384})
KCB = {1: 8448, 2: 3840}
KB_INFO = {1: 22, 2: 10}
# generator polynomial bits after the leading term, MSB first (TS 38.212 5.1)
POLY = {
    "16": 0x1021, "24A": 0x864CFB, "24B": 0x800063, "24C": 0xB2B117,
}
WIDTH = {"16": 16, "24A": 24, "24B": 24, "24C": 24}


def bg2_kb(B: int) -> int:
    return 10 if B > 640 else (9 if B > 560 else (8 if B > 192 else 6))


def cbs_info(B: int, bgn: int) -> Tuple[int, int, int, int, int, int]:
    """(C, cbz, L, F, K, Zc) for B = A + L_tb bits (get_cbs_info)."""
    Kcb = KCB[bgn]
    if B <= Kcb:
        L, C, Bd = 0, 1, B
    else:
        L = 24
        C = math.ceil(B / (Kcb - L))
        Bd = B + C * L
    if B % C or Bd % C:
        raise ValueError("transport block does not split evenly")
    cbz, Kd = B // C, Bd // C
    Kb = 22 if bgn == 1 else bg2_kb(B)
    Zc = next(z for z in LIFTING if z * Kb >= Kd)
    K = KB_INFO[bgn] * Zc
    return C, cbz, L, K - Kd, K, Zc


def er_list(G: int, C: int, Qm: int, NL: int = 1) -> List[int]:
    """Rate-matched length of each code block (get_Er_ldpc)."""
    g = NL * Qm
    lo = g * (G // (g * C))
    hi = g * (-(-G // (g * C)))
    n_lo = C - (G // g) % C
    return [lo if r < n_lo else hi for r in range(C)]


def crc_remainder_bits(bits: np.ndarray, poly: str) -> np.ndarray:
    """CRC bits of a 0/1 array by shift-register division (zero initial value)."""
    w = WIDTH[poly]
    p = POLY[poly]
    reg = 0
    top, mask = 1 << w, (1 << w) - 1
    for b in np.asarray(bits, dtype=np.int64).tolist():
        reg = (reg << 1) | int(b)
        if reg & top:
            reg ^= top | p
    for _ in range(w):
        reg <<= 1
        if reg & top:
            reg ^= top | p
    reg &= mask
    return np.array([(reg >> (w - 1 - i)) & 1 for i in range(w)], dtype=np.uint8)


def crc_attach(bits: np.ndarray, poly: str) -> np.ndarray:
    return np.concatenate([np.asarray(bits, dtype=np.uint8), crc_remainder_bits(bits, poly)])


def crc_check(bits_with_crc: np.ndarray, poly: str) -> bool:
    w = WIDTH[poly]
    data = np.asarray(bits_with_crc[:-w], dtype=np.uint8)
    return bool(np.array_equal(crc_remainder_bits(data, poly), np.asarray(bits_with_crc[-w:], dtype=np.uint8)))


def select_bg(A: int, R: float) -> int:
    if A <= 292 or (A <= 3824 and R <= 0.67) or R <= 0.25:
        return 2
    return 1


def segment(A: int, G: int, Qm: int, bgn: int, rv: int = 0):
    """Per-code-block decoder configurations of a transport block:
    list of ((bgn, A_cb, crctype, E_r, rv, Qm, 0), llr_start)."""
    L_tb = 24 if A > 3824 else 16
    B = A + L_tb
    C, cbz, L, F, K, Zc = cbs_info(B, bgn)
    crctype = (0 if L_tb == 16 else 1) if C == 1 else 2
    A_cb = A if C == 1 else cbz   # one code block: the decoder attaches / checks the TB CRC itself
    ers = er_list(G, C, Qm)
    out, start = [], 0
    for r in range(C):
        out.append(((bgn, A_cb, crctype, ers[r], rv, Qm, 0), start))
        start += ers[r]
    return out, dict(C=C, L_tb=L_tb, B=B, Kp=(B + C * L) // C, Zc=Zc, F=F, K=K)


def code_block_payloads(payload_bits: np.ndarray, A: int, bgn: int) -> List[np.ndarray]:
    """Transport-block bits + TB CRC split into the code blocks' information bits
    (before each code block's own CRC)."""
    poly = "24A" if A > 3824 else "16"
    tb = crc_attach(payload_bits[:A], poly)
    C, cbz, L, F, K, Zc = cbs_info(len(tb), bgn)
    if C == 1:
        return [np.asarray(payload_bits[:A], dtype=np.uint8)]
    return [tb[r * cbz:(r + 1) * cbz] for r in range(C)]
