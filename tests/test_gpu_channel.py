"""Device LLR front-end vs the host restatement of the reference demapper, on
the noisy symbols the device reports, plus noise statistics and the drop-in
tx_rx_process symbol."""

import ctypes

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import capi, channel_llrs, ldpc_decode, ldpc_encode
from oracle import channel_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def _pam(bits, m):
    a = np.ones(bits.shape[:-1], dtype=np.float64)
    for i in range(m - 1, 0, -1):
        a = (1 << (m - i)) - (1 - 2 * bits[..., i]) * a
    return (1 - 2 * bits[..., 0]) * a


@pytest.mark.parametrize("Qm", [1, 2, 4, 6, 8])
def test_demapper_bit_exact_and_noise_statistics(cuda, Qm):
    rng = np.random.default_rng(Qm)
    n, E = 64, 2400 // Qm * Qm
    rm = rng.integers(0, 256, size=(n, (E + 7) // 8), dtype=np.uint8)
    for noise_db in (-12.0, -3.0, 4.0):
        llr, sym = channel_llrs(torch.from_numpy(rm).to(cuda), E, Qm, noise_db, seed=7, return_symbols=True)
        llr, sym = llr.cpu().numpy(), sym.cpu().numpy()
        want = channel_ref.demap(sym, Qm, noise_db).reshape(n, E)
        assert np.array_equal(llr, want), noise_db
        # noise = received - transmitted constellation point
        bits = np.unpackbits(rm, axis=1)[:, :E].reshape(n, E // Qm, Qm).astype(np.float64)
        if Qm == 1:
            ideal = np.stack([1 - 2 * bits[..., 0]] * 2, axis=-1) / np.sqrt(2)
        else:
            m = Qm // 2
            ideal = np.stack([_pam(bits[..., 0::2], m), _pam(bits[..., 1::2], m)], axis=-1) / np.sqrt(
                channel_ref.NORM[Qm])
        noise = sym - ideal
        sigma = np.sqrt(10 ** (noise_db / 10) / 2)
        assert abs(noise.mean()) < 0.02 * sigma
        assert abs(noise.std() / sigma - 1) < 0.02


def test_tx_rx_process_dropin_and_seed(cuda, lib):
    rng = np.random.default_rng(3)
    rm = rng.integers(0, 256, size=300, dtype=np.uint8)
    outs = []
    for _ in range(2):
        lib.nrldpc_channel_seed(11)
        o = np.zeros(2400, np.int16)
        assert lib.tx_rx_process(rm.ctypes.data_as(ctypes.c_void_p), 2400, 8, ctypes.c_float(-40.0),
                                 o.ctypes.data_as(ctypes.c_void_p)) == 0
        outs.append(o)
    assert np.array_equal(outs[0], outs[1])
    bits = np.unpackbits(rm)[:2400]
    assert np.array_equal(outs[0] < 0, bits.astype(bool))       # 40 dB SNR: every hard decision right
    bad = np.zeros(8, np.int16)
    assert lib.tx_rx_process(rm.ctypes.data_as(ctypes.c_void_p), 2401, 8, ctypes.c_float(0.0),
                             bad.ctypes.data_as(ctypes.c_void_p)) == -1


def test_encode_channel_decode_chain_256qam(oracle, cuda):
    """Device encoder -> 256QAM channel -> decoder, checked against the oracle on
    the same LLRs.  At 20 dB most LLRs clip at +-10000 and the int16 decoder
    (like the reference's, c_lib/tx_rx_process.c:24-26) becomes overconfident
    and often fails; both behaviours must match the oracle exactly."""
    from oracle.oracle import dec_cfg, in_config

    cfg = (1, 8424, 1, 25344, 0, 8, 0)
    row = [1, 8, 22936, 0, 1280, 32767, -32767]
    pay = torch.randint(0, 256, (64, 1053), dtype=torch.uint8, device=cuda,
                        generator=torch.Generator(device=cuda).manual_seed(5))
    rm = ldpc_encode(pay, cfg)
    for esn0, min_pass in ((12.0, 0.95), (20.0, 0.0)):
        llr = channel_llrs(rm, 25344, 8, noise_power_db=-esn0, seed=1)
        res = ldpc_decode(llr, cfg, row)
        st = res.status.cpu().numpy()
        ok = (res.status == 0) & (res.hardbits[:, :1053] == pay).all(dim=1)
        assert ok.float().mean().item() >= min_pass, esn0
        host = llr.cpu().numpy()
        bits = res.hardbits.cpu().numpy()
        for i in range(0, 64, 8):
            es, eb, ei, _ = oracle.decode(host[i], in_config(*cfg), dec_cfg(row))
            assert st[i] == es and int(res.iterations[i]) == ei and np.array_equal(bits[i], eb), (esn0, i)


@pytest.mark.parametrize("Qm", [1, 2, 4, 6, 8])
def test_device_front_end_matches_reference_functions(cuda, reflib, Qm):
    """The device mapper and demapper against the reference's own static
    modulate_symbol / demodulate_symbol / quantize_llr_to_int16
    (c_lib/tx_rx_process.c:27, :68, :234), called through the reference build's
    channel shim.  At -300 dB of noise the noise term is far below half an ulp
    of every constellation coordinate, so the device reports the clean points."""
    rng = np.random.default_rng(40 + Qm)
    n, E = 16, 1200 // Qm * Qm
    rm = rng.integers(0, 256, size=(n, (E + 7) // 8), dtype=np.uint8)
    bits = np.unpackbits(rm, axis=1)[:, :E].reshape(-1, Qm)
    _, clean = channel_llrs(torch.from_numpy(rm).to(cuda), E, Qm, -300.0, seed=1, return_symbols=True)
    want = reflib.modulate_symbols(bits, Qm)
    assert np.array_equal(clean.cpu().numpy().reshape(-1, 2).view(np.uint32), want.view(np.uint32))
    for noise_db in (-15.0, -2.0, 5.0):
        llr, sym = channel_llrs(torch.from_numpy(rm).to(cuda), E, Qm, noise_db, seed=3, return_symbols=True)
        want = reflib.demap_symbols(sym.cpu().numpy(), Qm, noise_db)
        assert np.array_equal(llr.cpu().numpy().reshape(-1), want), noise_db
