"""The numpy restatement of the reference channel front-end (oracle/channel_ref.py)
pinned to the reference's own static functions: modulate_symbol,
demodulate_symbol and quantize_llr_to_int16 (c_lib/tx_rx_process.c:27-44,
:68-99, :234-268), exported by the shim translation unit that
oracle/build_ref.sh compiles around the reference source.  CPU only."""

import numpy as np
import pytest

from oracle import channel_ref

QMS = [1, 2, 4, 6, 8]


@pytest.mark.parametrize("Qm", QMS)
def test_modulation_matches_reference_on_every_bit_pattern(reflib, Qm):
    pats = ((np.arange(1 << Qm)[:, None] >> np.arange(Qm - 1, -1, -1)[None, :]) & 1).astype(np.uint8)
    want = reflib.modulate_symbols(pats, Qm)
    got = channel_ref.modulate(pats, Qm)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _symbols(Qm, rng, n=20000):
    """Random noisy symbols over and beyond the constellation, plus every
    segment boundary k*A exactly and one float either side of it."""
    A, _ = channel_ref.constants(Qm, 0.0)
    span = {1: 2, 2: 2, 4: 4, 6: 8, 8: 16}[Qm]
    x = rng.uniform(-1.3 * span, 1.3 * span, size=(n, 2)).astype(np.float32) * A
    ks = np.arange(-span, span + 1, dtype=np.float32)
    edges = (ks * A).astype(np.float32)
    e3 = np.concatenate([edges, np.nextafter(edges, np.float32(np.inf)), np.nextafter(edges, np.float32(-np.inf)),
                         np.float32([0.0, -0.0])])
    grid = np.stack(np.meshgrid(e3, e3[::-1]), axis=-1).reshape(-1, 2).astype(np.float32)
    return np.concatenate([x, grid])


@pytest.mark.parametrize("Qm", QMS)
def test_demapper_and_quantiser_match_reference(reflib, Qm):
    rng = np.random.default_rng(100 + Qm)
    sym = _symbols(Qm, rng)
    for noise_db in (-30.0, -12.0, -3.0, 0.0, 4.5, 10.0):
        want = reflib.demap_symbols(sym, Qm, noise_db)
        got = channel_ref.demap(sym, Qm, noise_db).reshape(-1)
        assert np.array_equal(got, want), (Qm, noise_db, int(np.sum(got != want)))
