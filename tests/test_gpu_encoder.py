"""Device encoder (CRC attach, QC-LDPC encoding, rate matching) vs the
reference's encoder outputs and the oracle, and an encode -> decode round trip."""

import ctypes

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import capi, ldpc_decode, ldpc_encode
from golden_cases import decode_cases
from oracle.oracle import in_config

pytestmark = pytest.mark.gpu


def test_dropin_encode_matches_reference_vectors(cuda, lib, golden):
    for key, cfg, _ in decode_cases(golden):
        pay = np.ascontiguousarray(golden[f"{key}_payload"])
        want = golden[f"{key}_rm"]
        for name in ("cuda_ldpc_5g_encode", "c_ldpc_5g_encode"):
            out = np.zeros_like(want)
            rc = getattr(lib, name)(pay.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(capi.make_in_config(*cfg)))
            assert rc == 0, (name, key)
            assert np.array_equal(out, want), (name, key)


def test_batched_encode_matches_oracle_everywhere(oracle, cuda):
    rng = np.random.default_rng(8)
    checked = 0
    for bgn in (1, 2):
        seen = set()
        for A in list(range(8, 640, 8)) + list(range(640, 8449, 56)):
            for crc in (1, 0, 2, 3):
                rc, p = oracle.derive(in_config(bgn, A, crc, 960, 0, 2, 0))
                if rc != 0 or p.Zc in seen:
                    continue
                seen.add(p.Zc)
                Qm = [1, 2, 4, 6, 8][len(seen) % 5]
                E = max(Qm, ((p.B * (3 + len(seen) % 4)) // 3 // Qm) * Qm)
                if len(seen) % 7 == 0:
                    E = min(65535 // Qm * Qm, (p.N * 2 // Qm) * Qm)      # repetition: E > N - F
                cfg = in_config(bgn, A, crc, E, len(seen) % 4, Qm, 0)
                n = 3
                pay = rng.integers(0, 256, size=(n, max(A // 8, 1)), dtype=np.uint8)[:, : A // 8]
                out = ldpc_encode(torch.from_numpy(np.ascontiguousarray(pay)).to(cuda),
                                  (bgn, A, crc, E, cfg.rv, Qm, 0)).cpu().numpy()
                for i in range(n):
                    assert np.array_equal(out[i], oracle.encode(pay[i], cfg)), (bgn, A, crc, E, Qm)
                checked += 1
    assert checked >= 90


def test_encode_decode_round_trip(cuda):
    cfg = (1, 8424, 1, 12672, 0, 4, 0)
    rng = np.random.default_rng(1)
    pay = torch.from_numpy(rng.integers(0, 256, size=(64, 1053), dtype=np.uint8)).to(cuda)
    rm = ldpc_encode(pay, cfg)
    bits = torch.from_numpy(np.unpackbits(rm.cpu().numpy(), axis=1)[:, :12672].astype(np.float32))
    noisy = (1.0 - 2.0 * bits) + 0.6 * torch.randn(bits.shape, generator=torch.Generator().manual_seed(2))
    llr = torch.clamp(torch.round(noisy * 128.0 * 2.0 / 0.36), -10000, 10000).to(torch.int16).to(cuda)
    res = ldpc_decode(llr, cfg, [1, 10, 22936, 0, 1280, 32767, -32767])
    torch.cuda.synchronize()
    assert (res.status == 0).all()
    assert torch.equal(res.hardbits[:, :1053], pay)
