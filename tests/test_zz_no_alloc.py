"""nrldpc_decode_batch_noalloc: the decode entry point for callers that may not
allocate device memory (real-time receive pipelines that cannot take
cudaMalloc's synchronisation and latency mid-slot, host frameworks that own all
device memory).  Its scratch is a static device array of the library, so it
must give exactly the results of nrldpc_decode_batch, call after call, while
the device's free memory stays put.

Kept in its own file, collected last."""

import ctypes

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import capi
from oracle.oracle import in_config, make_llrs

pytestmark = pytest.mark.gpu

CASES = [
    # (in_config, decoder row, code blocks): the first needs more CTAs than the
    # static scratch holds, so each CTA loops over several work items.
    ((1, 8424, 1, 25344, 0, 8, 0), [1, 8, 22936, 0, 1280, 32767, -32767], 601),
    ((2, 488, 1, 1920, 0, 2, 0), [3, 10, 22936, 0, 1280, 32767, -32767], 257),
    ((1, 72, 2, 400, 2, 4, 0), [2, 12, 22936, 0, 1280, 32767, -32767], 101),
    ((2, 1000, 1, 3000, 1, 6, 0), [1, 6, 30000, 40, -900, 20000, -25000], 64),
]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _decode(fn, llr, cfg, row, outs, stream, harq=None):
    icfg = capi.make_in_config(*cfg)
    dcfg = capi.make_decoder_config(row)
    bits, status, iters, app = outs
    return fn(_ptr(llr), llr.shape[1], llr.shape[0], ctypes.byref(icfg), ctypes.byref(dcfg), _ptr(bits),
              bits.shape[1], _ptr(status), _ptr(iters), _ptr(app), app.shape[1],
              _ptr(harq) if harq is not None else ctypes.c_void_p(0), harq.shape[1] if harq is not None else 0,
              ctypes.c_void_p(stream))


def _outputs(n, cfg, dev):
    p = capi.gen_ldpc_parameters(capi.make_in_config(*cfg))
    return (torch.zeros((n, (p.B + 7) // 8), dtype=torch.uint8, device=dev),
            torch.full((n,), -7, dtype=torch.int32, device=dev),
            torch.full((n,), -7, dtype=torch.int32, device=dev),
            torch.zeros((n, p.N + 2 * p.Zc), dtype=torch.int16, device=dev))


def _inputs(oracle, cfg, n, seed):
    if cfg[3] > 20000:   # full-size code blocks: noisy LLRs, every iteration runs
        rng = np.random.default_rng(seed)
        return np.clip(rng.normal(size=(n, cfg[3])) * 900, -10000, 10000).astype(np.int16)
    llr, _ = make_llrs(oracle, in_config(*cfg), min(n, 48), noise_db=-1.5, seed=seed)
    reps = -(-n // llr.shape[0])
    return np.ascontiguousarray(np.tile(llr, (reps, 1))[:n])


def test_noalloc_matches_batched_entry_point_on_consecutive_calls(oracle, cuda, lib):
    stream = torch.cuda.current_stream(cuda).cuda_stream
    for ci, (cfg, row, n) in enumerate(CASES):
        llr = torch.from_numpy(_inputs(oracle, cfg, n, seed=ci)).to(cuda)
        want = _outputs(n, cfg, cuda)
        assert _decode(lib.nrldpc_decode_batch, llr, cfg, row, want, stream) == 0
        got = [_outputs(n, cfg, cuda) for _ in range(2)]
        torch.cuda.synchronize(cuda)
        free = []
        for call in range(2):
            free.append(torch.cuda.mem_get_info(cuda)[0])
            assert _decode(lib.nrldpc_decode_batch_noalloc, llr, cfg, row, got[call], stream) == 0
            torch.cuda.synchronize(cuda)
            for w, g in zip(want, got[call]):
                assert torch.equal(w, g), (cfg, row, call)
        free.append(torch.cuda.mem_get_info(cuda)[0])
        # After the per-device set-up of the very first call, calls allocate
        # nothing, including the first call of a new configuration.
        assert abs(free[2] - free[1]) <= (2 << 20), free
        if ci > 0:
            assert abs(free[1] - free[0]) <= (2 << 20), (ci, free)


def test_noalloc_combines_into_soft_buffers_like_batched_entry_point(oracle, cuda, lib):
    """HARQ: an rv 2 retransmission combined into the soft buffers an rv 0
    transmission left; every call starts from copies of the same buffers."""
    stream = torch.cuda.current_stream(cuda).cuda_stream
    row = [1, 10, 22936, 0, 1280, 32767, -32767]
    first, retx = (2, 488, 1, 1920, 0, 2, 0), (2, 488, 1, 1920, 2, 2, 1)
    n = 96
    p = capi.gen_ldpc_parameters(capi.make_in_config(*first))
    llr0 = torch.from_numpy(_inputs(oracle, first, n, seed=11)).to(cuda)
    llr2, _ = make_llrs(oracle, in_config(*retx[:6], 0), 48, noise_db=0.5, seed=12)
    llr2 = torch.from_numpy(np.ascontiguousarray(np.tile(llr2, (2, 1)))).to(cuda)
    stored = torch.zeros((n, p.N + 2 * p.Zc), dtype=torch.int16, device=cuda)
    assert _decode(lib.nrldpc_decode_batch, llr0, first, row, _outputs(n, first, cuda), stream, stored) == 0
    want, want_h = _outputs(n, retx, cuda), stored.clone()
    assert _decode(lib.nrldpc_decode_batch, llr2, retx, row, want, stream, want_h) == 0
    torch.cuda.synchronize(cuda)
    assert not torch.equal(want_h, stored)
    for call in range(2):
        got, got_h = _outputs(n, retx, cuda), stored.clone()
        assert _decode(lib.nrldpc_decode_batch_noalloc, llr2, retx, row, got, stream, got_h) == 0
        torch.cuda.synchronize(cuda)
        for w, g in zip(want, got):
            assert torch.equal(w, g), call
        assert torch.equal(want_h, got_h), call


def test_noalloc_rejects_float_algorithms(cuda, lib):
    cfg = (2, 488, 1, 1920, 0, 2, 0)
    llr = torch.zeros((2, 1920), dtype=torch.int16, device=cuda)
    outs = _outputs(2, cfg, cuda)
    for algo in (0, 4):
        row = [algo, 4, 22936, 0, 1280, 32767, -32767]
        assert _decode(lib.nrldpc_decode_batch_noalloc, llr, cfg, row, outs, 0) == capi.NRLDPC_ERR_ALGO
