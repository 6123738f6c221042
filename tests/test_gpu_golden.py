"""CUDA path vs the reference's own outputs (golden vectors made by the
reference C library, tests/golden/make_golden.py): batched API and the
drop-in single-code-block ABI."""

import ctypes

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import capi, ldpc_decode
from golden_cases import algo_rows, decode_cases, expected, harq_sequences, lq_close

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ai", range(6))
def test_batched_decode_matches_reference_vectors(cuda, golden, ai):
    row = algo_rows(golden)[ai]
    for key, cfg, llr in decode_cases(golden):
        # decode each vector next to a different partner to exercise the pair packing
        batch = np.stack([llr, llr[::-1].copy(), llr])
        res = ldpc_decode(torch.from_numpy(batch).to(cuda), cfg, row, return_app=True)
        torch.cuda.synchronize()
        est, ebits, eits, elq = expected(golden, key, ai)
        for r in (0, 2):
            assert int(res.status[r]) == est, key
            assert int(res.iterations[r]) == eits, key
            if eits > 0:
                assert np.array_equal(res.hardbits[r].cpu().numpy(), ebits), key
            assert lq_close(res.app[r].cpu().numpy(), elq, row[0], est == 0), key


@pytest.mark.parametrize("ai", [0, 1, 2, 3, 4])
def test_dropin_abi_matches_reference_vectors(cuda, lib, golden, ai):
    row = algo_rows(golden)[ai]
    dcfg = capi.make_decoder_config(row)
    for key, cfg, llr in decode_cases(golden):
        est, ebits, _, _ = expected(golden, key, ai)
        icfg = capi.make_in_config(*cfg)
        for name in ("cuda_ldpc_5g_decode", "c_ldpc_5g_decode"):
            bits = np.zeros_like(ebits)
            l16 = np.ascontiguousarray(llr, dtype=np.int16)
            rc = getattr(lib, name)(l16.ctypes.data_as(ctypes.c_void_p), bits.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(icfg), ctypes.byref(dcfg))
            assert rc == est, (name, key)
            assert np.array_equal(bits, ebits), (name, key)


def test_dropin_harq_sequences_match_reference(cuda, lib, golden):
    dcfg = capi.make_decoder_config([1, 8, 22936, 0, 1280, 32767, -32767])
    for hi, steps in harq_sequences(golden):
        for s in steps:
            icfg = capi.make_in_config(*s["cfg"])
            bits = np.zeros_like(s["bits"])
            l16 = np.ascontiguousarray(s["llr"], dtype=np.int16)
            rc = lib.cuda_ldpc_5g_decode(l16.ctypes.data_as(ctypes.c_void_p), bits.ctypes.data_as(ctypes.c_void_p),
                                         ctypes.byref(icfg), ctypes.byref(dcfg))
            assert rc == s["status"], (hi, s["cfg"])
            assert np.array_equal(bits, s["bits"]), (hi, s["cfg"])


def test_batched_harq_buffers_match_reference(cuda, golden):
    row = [1, 8, 22936, 0, 1280, 32767, -32767]
    for hi, steps in harq_sequences(golden):
        harq = torch.zeros((1, 68 * 384), dtype=torch.int16, device=cuda)
        for s in steps:
            res = ldpc_decode(torch.from_numpy(s["llr"][None, :].copy()).to(cuda), s["cfg"], row, return_app=True,
                              harq=harq)
            torch.cuda.synchronize()
            n = len(s["buf"])
            assert np.array_equal(harq[0, :n].cpu().numpy(), s["buf"]), (hi, s["cfg"])
            assert int(res.status[0]) == s["status"]
            assert np.array_equal(res.hardbits[0].cpu().numpy(), s["bits"])
            assert np.array_equal(res.app[0].cpu().numpy(), s["lq"])
