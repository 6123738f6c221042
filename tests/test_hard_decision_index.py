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


def test_four_position_step_index_is_exact_and_aligned():
    """The fixed-point kernel's CRC pass with B a multiple of 4: steps of four
    positions, Bq4 = roundup(B, 128) / 4 steps per slot.  The slot index is the
    same high multiply by ceil(2^32 / Bq4); each step's 16-byte loads start at
    LQ word gg*lq_len + i0 and table entry B-4-i0, both multiples of 4, and stay
    inside the block (i0 + 3 < B) and the table (B-4-i0 >= 0)."""
    checked = 0
    for zc in LIFTING_SIZES:
        G = 384 // zc
        for cols, kb in ((68, 22), (52, 10)):      # BG1, BG2: lq_len = cols*Zc, B <= K = kb*Zc
            lq_len = cols * zc
            assert lq_len % 4 == 0
            for B in range(4, kb * zc + 1, 4):
                bq4 = ((B + 127) & ~127) // 4
                assert bq4 % 32 == 0                  # a warp's 32 steps share one slot
                k = np.arange(G * bq4, dtype=np.uint64)
                gg = (k * np.uint64(bp_magic(bq4))) >> np.uint64(32)
                assert np.array_equal(gg, k // np.uint64(bq4)), (zc, B)
                i0 = 4 * (k - gg * np.uint64(bq4))
                live = i0 < B
                assert np.all(i0[live] + 3 < B)
                assert np.all((gg[live] * lq_len + i0[live]) % 4 == 0)
                assert np.all((B - 4 - i0[live].astype(np.int64)) >= 0)
                assert np.all((B - 4 - i0[live].astype(np.int64)) % 4 == 0)
                checked += 1
    assert checked > 1000


def test_mixed_four_position_step_index_is_exact():
    """The mixed-size kernel's CRC pass: slots of Bq4 = roundup(K, 128) / 4
    four-position steps (every block's B <= K of its graph), G = floor(capacity
    / Zc) slots for both CTA classes; the 16-byte LQ load of a step with work
    (i0 < B <= K) ends inside the slot's LQ (i0 + 3 < lq_len)."""
    checked = 0
    for zc in LIFTING_SIZES:
        for cap in (384, 240):
            G = cap // zc
            if G == 0:
                continue
            for cols, kb in ((68, 22), (52, 10)):
                K, lq_len = kb * zc, cols * zc
                bq4 = ((K + 127) & ~127) // 4
                assert bq4 % 32 == 0
                k = np.arange(G * bq4, dtype=np.uint64)
                gg = (k * np.uint64(bp_magic(bq4))) >> np.uint64(32)
                assert np.array_equal(gg, k // np.uint64(bq4)), (zc, cap, cols)
                i0 = 4 * (k - gg * np.uint64(bq4))
                assert np.all(i0[i0 < K] + 3 < lq_len)
                checked += 1
    assert checked > 150
