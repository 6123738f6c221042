"""Host restatement (numpy float32) of the reference's max-log demapper and
LLR quantiser (c_lib/tx_rx_process.c:24-44, :101-268).

TEST INFRASTRUCTURE ONLY.  Given noisy symbols, it computes the int16 LLRs the
reference's demodulate_symbol + quantize_llr_to_int16 would produce, with the
same float32 operations in the same order, so the device front-end can be
checked bit for bit on the symbols it reports."""

from __future__ import annotations

import numpy as np

F = np.float32
INF = np.float32(3.0e38)

# (threshold in units of A, c1, s, c2): llr = (c1*A) * (s*r + c2*A) / nv for r < thr*A.
QAM16 = [[(-2, 8, 1, 1), (2, 4, 1, 0), (None, 8, 1, -1)],
         [(0, 4, 1, 2), (None, 4, -1, 2)]]
QAM64 = [[(-6, 16, 1, 3), (-4, 12, 1, 2), (-2, 8, 1, 1), (2, 4, 1, 0), (4, 8, 1, -1), (6, 12, 1, -2), (None, 16, 1, -3)],
         [(-6, 8, 1, 5), (-2, 4, 1, 4), (0, 8, 1, 3), (2, 8, -1, 3), (6, 4, -1, 4), (None, 8, -1, 5)],
         [(-4, 4, 1, 6), (0, 4, -1, -2), (4, 4, 1, -2), (None, 4, -1, 6)]]
QAM256 = [[(-14, 32, 1, 7), (-12, 28, 1, 6), (-10, 24, 1, 5), (-8, 20, 1, 4), (-6, 16, 1, 3), (-4, 12, 1, 2),
           (-2, 8, 1, 1), (2, 4, 1, 0), (4, 8, 1, -1), (6, 12, 1, -2), (8, 16, 1, -3), (10, 20, 1, -4),
           (12, 24, 1, -5), (14, 28, 1, -6), (None, 32, 1, -7)],
          [(-14, 16, 1, 11), (-12, 12, 1, 10), (-10, 8, 1, 9), (-6, 4, 1, 8), (-4, 8, 1, 7), (-2, 12, 1, 6),
           (0, 16, 1, 5), (2, 16, -1, 5), (4, 12, -1, 6), (6, 8, -1, 7), (10, 4, -1, 8), (12, 8, -1, 9),
           (14, 12, -1, 10), (None, 16, -1, 11)],
          [(-14, 8, 1, 13), (-10, 4, 1, 12), (-8, 8, 1, 11), (-6, 8, -1, -5), (-2, 4, -1, -4), (0, 8, -1, -3),
           (2, 8, 1, -3), (6, 4, 1, -4), (8, 8, 1, -5), (10, 8, -1, 11), (14, 4, -1, 12), (None, 8, -1, 13)],
          [(-12, 4, 1, 14), (-8, 4, -1, -10), (-4, 4, 1, 6), (0, 4, -1, -2), (4, 4, 1, -2), (8, 4, -1, 6),
           (12, 4, 1, -10), (None, 4, -1, 14)]]
NORM = {1: 2.0, 2: 2.0, 4: 10.0, 6: 42.0, 8: 170.0}


def constants(Qm: int, noise_power_db: float):
    A = F(1.0) / np.sqrt(F(NORM[Qm]), dtype=F)
    nv = np.power(F(10.0), F(noise_power_db) / F(10.0), dtype=F)
    return A, nv


def seg_llr(segs, r: np.ndarray, A, nv) -> np.ndarray:
    out = np.zeros_like(r)
    done = np.zeros(r.shape, dtype=bool)
    for thr, c1, s, c2 in segs:
        sel = ~done if thr is None else (~done & (r < F(thr) * A))
        lin = F(s) * r[sel] + F(c2) * A
        out[sel] = (F(c1) * A) * lin / nv
        done |= sel
    return out


def quantize(llr: np.ndarray) -> np.ndarray:
    scaled = (llr * F(128.0)).astype(F)
    q = np.where(scaled >= 0, scaled + F(0.5), scaled - F(0.5)).astype(F)
    q = np.trunc(q).astype(np.int64)
    return np.clip(q, -10000, 10000).astype(np.int16)


def demap(sym: np.ndarray, Qm: int, noise_power_db: float) -> np.ndarray:
    """sym float32 [..., 2] noisy symbols -> int16 LLRs [..., Qm]."""
    A, nv = constants(Qm, noise_power_db)
    re = sym[..., 0].astype(F)
    im = sym[..., 1].astype(F)
    if Qm == 1:
        return quantize((F(4.0) * (re + im)) * A / nv)[..., None]
    if Qm == 2:
        return np.stack([quantize((F(4.0) * re) * A / nv), quantize((F(4.0) * im) * A / nv)], axis=-1)
    tab = {4: QAM16, 6: QAM64, 8: QAM256}[Qm]
    out = []
    for segs in tab:
        out.append(quantize(seg_llr(segs, re, A, nv)))
        out.append(quantize(seg_llr(segs, im, A, nv)))
    return np.stack(out, axis=-1)


def bit_sign(b: np.ndarray) -> np.ndarray:
    return np.where(b != 0, F(-1.0), F(1.0)).astype(F)


def modulate(bits: np.ndarray, Qm: int) -> np.ndarray:
    """bits uint8 [..., Qm] -> float32 [..., 2] NR constellation points, the
    reference's float32 expressions in their order (c_lib/tx_rx_process.c:68-99)."""
    A = F(1.0) / np.sqrt(F(NORM[Qm]), dtype=F)
    s = [bit_sign(bits[..., j]) for j in range(Qm)]
    if Qm == 1:
        re = im = s[0] * A
    elif Qm == 2:
        re, im = s[0] * A, s[1] * A
    elif Qm == 4:
        re = (s[0] * (F(2.0) - s[2])) * A
        im = (s[1] * (F(2.0) - s[3])) * A
    elif Qm == 6:
        re = (s[0] * (F(4.0) - s[2] * (F(2.0) - s[4]))) * A
        im = (s[1] * (F(4.0) - s[3] * (F(2.0) - s[5]))) * A
    else:
        re = (s[0] * (F(8.0) - s[2] * (F(4.0) - s[4] * (F(2.0) - s[6])))) * A
        im = (s[1] * (F(8.0) - s[3] * (F(4.0) - s[5] * (F(2.0) - s[7])))) * A
    return np.stack([np.asarray(re, dtype=F), np.asarray(im, dtype=F)], axis=-1)
