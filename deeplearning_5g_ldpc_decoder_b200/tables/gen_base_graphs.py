"""Generate ``csrc/nr_base_graphs.inc`` from the 3GPP TS 38.212 base-graph matrices.

The 5G NR LDPC base graphs (TS 38.212 Tables 5.3.2-2 and 5.3.2-3) are public
standard data: for each base graph BG1 (46 x 68) and BG2 (42 x 52) and each
lifting-size set iLS = 0..7 there is a matrix of circulant shifts V_ij, with
-1 marking a null (all-zero) circulant.

The reference project ships those matrices as MATLAB files
(``py5gphy/ldpc/tables/BG{1,2}S{0..7}.mat1``).  This script reads them and writes
one generated C include file in this project's own layout: one record per
non-null circulant, in row-major / column-ascending order, holding the base
row, base column and the eight raw shifts (one per iLS).  Everything else the
decoder needs (row offsets, degrees, shifts reduced mod Zc, the CSR views the
reference ABI hands out through ``gen_ldpc_parameters``) is derived from these
records at library load time.

The column-ascending edge order inside a row is the order in which the
reference's layered decoders visit a check node's edges
(``c_lib/ldpc_tables.c:30-68`` are CSR tables built row by row with
``np.nonzero`` in ``py5gphy/ldpc_c_parameters.py:49-78``); the floating-point
BP product order depends on it.

Usage (run in a checkout that has the reference tree)::

    python deeplearning_5g_ldpc_decoder_b200/tables/gen_base_graphs.py <reference-root>

The generated file is committed, so builds never need the reference tree.
"""

from __future__ import annotations

import os
import sys

import numpy as np


def load_matrices(ref_root: str, bgn: int) -> np.ndarray:
    from scipy import io

    mats = []
    for ils in range(8):
        path = os.path.join(ref_root, "py5gphy", "ldpc", "tables", f"BG{bgn}S{ils}.mat1")
        mats.append(np.asarray(io.loadmat(path)["BG"], dtype=np.int32))
    stack = np.stack(mats)  # [8, rows, cols]
    # The null pattern must be identical across the eight lifting sets.
    null = stack < 0
    assert (null == null[0]).all(), "null pattern differs between iLS sets"
    return stack


def edges(stack: np.ndarray):
    _, rows, cols = stack.shape
    out = []
    for r in range(rows):
        for c in range(cols):
            if stack[0, r, c] >= 0:
                out.append((r, c, [int(stack[s, r, c]) for s in range(8)]))
    return out


def render(bgn: int, stack: np.ndarray) -> str:
    _, rows, cols = stack.shape
    e = edges(stack)
    lines = [f"/* BG{bgn}: {rows} rows x {cols} columns, {len(e)} non-null circulants. */",
             f"static const nr_bg_edge_t kBG{bgn}Edges[{len(e)}] = {{"]
    for r, c, v in e:
        vs = ", ".join(f"{x:3d}" for x in v)
        lines.append(f"    {{{r:2d}, {c:2d}, {{{vs}}}}},")
    lines.append("};")
    return "\n".join(lines)


def main() -> None:
    ref_root = sys.argv[1] if len(sys.argv) > 1 else None
    if not ref_root:
        raise SystemExit("usage: gen_base_graphs.py <reference-root>")
    here = os.path.dirname(os.path.abspath(__file__))
    out = os.path.join(os.path.dirname(here), "csrc", "nr_base_graphs.inc")
    bg1 = load_matrices(ref_root, 1)
    bg2 = load_matrices(ref_root, 2)
    text = [
        "/* Generated by tables/gen_base_graphs.py from the 3GPP TS 38.212 base-graph",
        " * matrices (Tables 5.3.2-2 / 5.3.2-3).  Do not edit.",
        " * Record: {base row, base column, {V_ij for iLS 0..7}}, row-major, columns",
        " * ascending within a row.  Shifts are raw (not yet reduced mod Zc). */",
        render(1, bg1),
        "",
        render(2, bg2),
        "",
    ]
    with open(out, "w") as f:
        f.write("\n".join(text))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
