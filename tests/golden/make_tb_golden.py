"""Generate tests/golden/tb_vectors.npz from the reference's Python PHY.

Imports py5gphy from the reference tree and records, for the transport-block
formulas the library restates:
* ``get_cbs_info(B, bgn)`` (py5gphy/ldpc/ldpc_info.py:59-109) over transport
  blocks of one and many code blocks, both base graphs;
* ``get_Er_ldpc(G, C, Qm, 1)`` (py5gphy/ldpc/nr_ldpc_ratematch.py:22-45);
* ``nr_crc_encode`` (py5gphy/crc/crc.py:77-102) for CRC16 / 24A / 24B on seeded
  random payloads.

usage:  python tests/golden/make_tb_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.refroot import REFERENCE_ROOT  # noqa: E402

sys.path.insert(0, REFERENCE_ROOT)

from py5gphy.crc import crc  # noqa: E402
from py5gphy.ldpc import ldpc_info, nr_ldpc_ratematch  # noqa: E402


def valid_B(B, bgn):
    Kcb = {1: 8448, 2: 3840}[bgn]
    if B <= Kcb:
        return True
    C = -(-B // (Kcb - 24))
    return B % C == 0


def main():
    rng = np.random.default_rng(2024)
    cbs = []
    for bgn in (1, 2):
        cand = list(range(24, 4000, 8)) + list(range(4000, 200000, 1208)) + [1200016, 65560, 8448, 8449, 3840, 3841]
        for B in cand:
            if not valid_B(B, bgn):
                continue
            C, cbz, L, F, K, Zc = ldpc_info.get_cbs_info(B, bgn)
            cbs.append((B, bgn, C, cbz, L, F, K, Zc))
    er = []
    for _ in range(400):
        C = int(rng.integers(1, 150))
        Qm = int(rng.choice([1, 2, 4, 6, 8]))
        G = Qm * int(rng.integers(C, C * 20000))
        for r, e in enumerate(nr_ldpc_ratematch.get_Er_ldpc(G, C, Qm, 1)):
            er.append((G, C, Qm, r, int(e)))
    crcs_in, crcs_out, crcs_poly = [], [], []
    for poly in ("16", "24A", "24B"):
        for n in (1, 8, 24, 100, 1000, 8424):
            bits = rng.integers(0, 2, n).astype(np.int8)
            out = crc.nr_crc_encode(bits, poly)
            crcs_in.append(np.packbits(bits.astype(np.uint8)))
            crcs_out.append(np.asarray(out[n:], dtype=np.uint8))
            crcs_poly.append((poly, n))
    np.savez_compressed(
        os.path.join(HERE, "tb_vectors.npz"),
        cbs=np.array(cbs, dtype=np.int64), er=np.array(er, dtype=np.int64),
        crc_poly=np.array([p for p, _ in crcs_poly]), crc_len=np.array([n for _, n in crcs_poly]),
        **{f"crc_in_{i}": a for i, a in enumerate(crcs_in)}, **{f"crc_out_{i}": a for i, a in enumerate(crcs_out)})
    print(len(cbs), "segmentations,", len(er), "E values,", len(crcs_in), "CRCs")


if __name__ == "__main__":
    main()
