"""Generate tests/golden/lbrm_vectors.npz: limited-buffer rate matching and
recovery from the reference's Python PHY.

py5gphy's ``get_k0`` / ``ratematch_ldpc`` / ``raterecover_ldpc``
(py5gphy/ldpc/nr_ldpc_ratematch.py:48-104, nr_ldpc_raterecover.py:15-68) take
the circular-buffer length Ncb as a parameter (the C library fixes Ncb = N).
For each case the codeword comes from the oracle's encoder (pinned to the
reference C encoder), with filler bits marked -1 as py5gphy expects; the
recovery input is integer-valued LLRs so the float sums are exact.

usage:  python tests/golden/make_lbrm_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle.refroot import REFERENCE_ROOT  # noqa: E402

sys.path.insert(0, REFERENCE_ROOT)

from py5gphy.ldpc import nr_ldpc_ratematch, nr_ldpc_raterecover  # noqa: E402

from oracle.oracle import Oracle, in_config  # noqa: E402

# (bgn, A, crctype, E, rv, Qm, Ncb)
CASES = [
    (1, 8424, 1, 9600, 0, 8, 18000), (1, 8424, 1, 12000, 1, 8, 18000), (1, 8424, 1, 30000, 2, 6, 16896),
    (1, 8424, 1, 25344, 3, 8, 20000), (1, 3816, 2, 7000, 1, 4, 8000), (1, 2000, 1, 6000, 3, 2, 4000),
    (2, 3816, 2, 8000, 1, 4, 9000), (2, 1000, 1, 2400, 2, 2, 2600), (2, 3816, 2, 20004, 3, 6, 12000),
    (2, 488, 1, 1920, 1, 2, 1600),
]


def main():
    orc = Oracle()
    rng = np.random.default_rng(99)
    out = {"cases": np.array(CASES, dtype=np.int64)}
    for i, (bgn, A, crc, E, rv, Qm, ncb) in enumerate(CASES):
        cfg = in_config(bgn, A, crc, E, rv, Qm)
        p = orc.params(cfg)
        pay = rng.integers(0, 256, A // 8, dtype=np.uint8)
        cw = orc.encode_codeword(pay, cfg)[: p.N + 2 * p.Zc].astype(np.int8)
        dn = cw[2 * p.Zc:].copy()
        dn[p.B - 2 * p.Zc: p.K - 2 * p.Zc] = -1
        k0 = nr_ldpc_ratematch.get_k0(Ncb=ncb, bgn=bgn, rv=rv, Zc=p.Zc)
        rm = nr_ldpc_ratematch.ratematch_ldpc(dn, ncb, E, k0, Qm)
        llr = rng.integers(-300, 300, E).astype(np.float64)
        rec = nr_ldpc_raterecover.raterecover_ldpc(llr, Ncb=ncb, N=p.N, k0=k0, Qm=Qm, Zc=p.Zc, K_apo=p.B, K=p.K)
        out[f"pay_{i}"] = pay
        out[f"k0_{i}"] = np.array([k0])
        out[f"rm_{i}"] = np.asarray(rm, dtype=np.uint8)
        out[f"llr_{i}"] = llr.astype(np.int16)
        out[f"rec_{i}"] = np.asarray(rec, dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "lbrm_vectors.npz"), **out)
    print(len(CASES), "cases")


if __name__ == "__main__":
    main()
