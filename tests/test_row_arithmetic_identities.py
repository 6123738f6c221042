"""The int16 identities the fixed-point row update relies on, checked on the CPU.

The kernels (csrc/nrldpc_fixed_row.cuh) rewrite the reference's per-edge
arithmetic (c_lib/fixedpoint_ldpc_decoder.c:103-144) into forms that are
cheaper on the GPU; each form must give the same int16 values.  Here every
identity is replayed per int16 half with numpy, over all 65536 values of the
message magnitude or belief where that is cheap and over seeded samples
elsewhere.  No GPU needed."""

import numpy as np
import pytest

M16 = 0xFFFF


def wrap16(x):
    """int16 wrap-around of an integer array."""
    return ((np.asarray(x, dtype=np.int64) + 32768) % 65536) - 32768


def u16(x):
    return np.asarray(x, dtype=np.int64) & M16


@pytest.mark.parametrize("flip", [False, True])
def test_negation_as_complement_plus_carry(flip):
    """-r with r = (flip ? -v : v) equals (v ^ ~mf) + (~mf & 1) per half
    (mf = 0xFFFF when flipped), modulo 2^16, for every int16 v."""
    v = np.arange(-32768, 32768, dtype=np.int64)
    mf = M16 if flip else 0
    nmf = M16 ^ mf
    r = wrap16(-v) if flip else v
    lhs = wrap16(-r)
    rhs = wrap16((u16(v) ^ nmf) + (nmf & 1))
    assert np.array_equal(lhs, rhs)
    # and the pass-2 form: lr = (v ^ mf) + (mf & 1)
    assert np.array_equal(wrap16(r), wrap16((u16(v) ^ mf) + (mf & 1)))


def _true_overflow(rel, lr):
    s = rel + lr
    return (s > 32767) | (s < -32768)


def _flag(rel, sum16, other):
    """The kernel's test: sign bit of (sum ^ rel) & ~(rel ^ other), per half."""
    return (((u16(sum16) ^ u16(rel)) & (M16 ^ (u16(rel) ^ u16(other)))) & 0x8000) != 0


def test_overflow_flag_from_flip_mask_is_exact_for_nonnegative_minima():
    """Open-max path (alpha >= 0): scaled minima v in [0, 32766], so testing the
    flip mask in place of the message's sign flags exactly the int16 overflows."""
    rng = np.random.default_rng(3)
    v = np.concatenate([np.arange(0, 32767, dtype=np.int64), rng.integers(0, 32767, 4096)])
    for rel in list(range(-32768, -32760)) + list(range(-5, 6)) + list(range(32760, 32768)) + \
            rng.integers(-32768, 32768, 48).tolist():
        for flip in (False, True):
            mf = M16 if flip else 0
            lr = -v if flip else v
            sum16 = wrap16(rel + lr)
            assert np.array_equal(_flag(rel, sum16, np.full_like(v, mf)), _true_overflow(rel, lr)), (rel, flip)


def test_shortcut_tests_miss_overflows_for_negative_minima():
    """Why the open-max path requires alpha >= 0 and the clamp path tests the
    message itself: with a negative alpha the scaled minima can be negative.
    An unflipped negative v makes the flip-mask test miss an overflow, and a
    flipped v = -32768 (whose negation stays -32768) makes the test on
    t = v ^ mf miss one; the message's own sign catches both."""
    # unflipped negative minimum: lr = v < 0, mf = 0
    rel, v = -32700, -100
    lr = v
    sum16 = int(wrap16(rel + lr))
    assert _true_overflow(rel, lr)
    assert not _flag(rel, sum16, 0)                  # flip mask
    assert _flag(rel, sum16, lr)                     # the message
    # flipped v = -32768: lr = -32768, t = v ^ mf = 0x7FFF
    rel, v = -100, -32768
    lr = int(wrap16(-v))
    sum16 = int(wrap16(rel + lr))
    t = (v & M16) ^ M16
    assert _true_overflow(rel, lr)
    assert not _flag(rel, sum16, t)                  # t = v ^ mf
    assert _flag(rel, sum16, lr)                     # the message


def test_open_max_scaling_equals_reference_offset_and_normalise():
    """(alpha * m + 2^14) >> 15 per half equals the reference's offset-then-
    normalise (c_lib/fixedpoint_ldpc_decoder.c:38-46) with beta = 0, max_llr =
    32767 and alpha >= 0, for every minimum m in [0, 32767], and stays in
    [0, 32766]."""
    m = np.arange(0, 32768, dtype=np.int64)
    for alpha in (0, 1, 16384, 22936, 26623, 32767):
        clipped = np.minimum(m, 32767)
        off = np.maximum(clipped - 0, 0)
        ref = wrap16((alpha * off + (1 << 14)) >> 15)
        fast = (alpha * m + (1 << 14)) >> 15
        assert np.array_equal(ref, fast), alpha
        assert fast.min() >= 0 and fast.max() <= 32766


def test_upper_clamp_at_32767_is_identity_on_int16():
    """With max_llr = 32767 the belief clamp min(max(s, min_llr), 32767) is
    max(s, min_llr) on every int16 s."""
    s = np.arange(-32768, 32768, dtype=np.int64)
    for min_llr in (-32768, -32767, -10000, 0):
        assert np.array_equal(np.minimum(np.maximum(s, min_llr), 32767), np.maximum(s, min_llr))
