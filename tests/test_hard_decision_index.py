"""The hard-decision loops' group index, checked on the CPU.

The fixed-point, float and mixed-size kernels walk k = 0 .. G*Bp-1 over the
hard bits of the G code-block slots of a CTA (Bp = B rounded up to 32) and
split k into the slot gg = k / Bp and the bit i = k - gg*Bp with one high
multiply by ceil(2^32 / Bp) (csrc/nrldpc_decode_common.cuh bp_magic and
div_bp).  Here that arithmetic is replayed with 32-bit unsigned semantics for
every Bp a lifting size can produce and every k the loops reach, and compared
with the integer division.  No GPU needed."""

import numpy as np

from oracle.tb_ref import LIFTING as LIFTING_SIZES

M32 = (1 << 32) - 1


def bp_magic(bp):
    return (M32 // bp + 1) & M32


def test_group_index_is_exact_for_every_size():
    checked = 0
    for zc in LIFTING_SIZES:
        for cap in (384, 240):           # CTA lifted-row capacities: 384 (all kernels), 240 (mixed class 1)
            G = cap // zc
            if G == 0:
                continue
            kmax = 22 * zc                # B <= K = 22 Zc (BG1) or 10 Zc (BG2)
            for bp in range(32, ((kmax + 31) // 32) * 32 + 1, 32):
                k = np.arange(G * bp, dtype=np.uint64)
                gg = (k * np.uint64(bp_magic(bp))) >> np.uint64(32)
                assert np.array_equal(gg, k // np.uint64(bp)), (zc, cap, bp)
                checked += 1
    assert checked > 1000
