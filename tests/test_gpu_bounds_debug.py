"""The small-case parity suite under the bounds-checked debug library.

libnrldpc_b200_debug.so is the same source compiled with -DNRLDPC_BOUNDS_CHECK:
every gather and scatter index of the decode kernels (belief words, edge
entries, message scratch, rate-matched LLR reads, CRC table entries) is
checked, and a violation is recorded instead of trapping (there is no
compute-sanitizer on this GPU pool; this build stands in for its memcheck).
Every lifting size of both base graphs, the queued (multi-wave) launches, the
mixed-size kernel, HARQ soft buffers and the no-allocation entry point run
through it.  Results must equal the release library's bit for bit, and no
violation may be recorded."""

import ctypes
import os

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import capi
from deeplearning_5g_ldpc_decoder_b200.build import DEBUG_LIB_PATH, build_library
from deeplearning_5g_ldpc_decoder_b200.mixed import MixedPlan, random_mixed_configs
from oracle.oracle import in_config, make_llrs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dbg(cuda):
    if not os.path.exists(DEBUG_LIB_PATH):
        build_library(debug=True)
    lib = capi.load_library(DEBUG_LIB_PATH)
    rec = (ctypes.c_uint32 * 4)()
    assert lib.nrldpc_bounds_check_status(rec, 1) == 1, "not the bounds-checked build"
    return lib


def _clean(lib):
    rec = (ctypes.c_uint32 * 4)()
    assert lib.nrldpc_bounds_check_status(rec, 1) == 1
    return list(rec)


def _decode(lib, llr, cfg, row, harq=None):
    p = capi.gen_ldpc_parameters(capi.make_in_config(*cfg), lib)
    n = llr.shape[0]
    dev = llr.device
    bits = torch.zeros((n, (p.B + 7) // 8), dtype=torch.uint8, device=dev)
    status = torch.full((n,), -9, dtype=torch.int32, device=dev)
    iters = torch.full((n,), -9, dtype=torch.int32, device=dev)
    app = torch.zeros((n, p.N + 2 * p.Zc), dtype=torch.float32 if row[0] in (0, 4) else torch.int16, device=dev)
    icfg, dcfg = capi.make_in_config(*cfg), capi.make_decoder_config(row)
    rc = lib.nrldpc_decode_batch(ctypes.c_void_p(llr.data_ptr()), llr.shape[1], n, ctypes.byref(icfg),
                                 ctypes.byref(dcfg), ctypes.c_void_p(bits.data_ptr()), bits.shape[1],
                                 ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(iters.data_ptr()),
                                 ctypes.c_void_p(app.data_ptr()), app.shape[1],
                                 ctypes.c_void_p(harq.data_ptr() if harq is not None else 0),
                                 harq.shape[1] if harq is not None else 0,
                                 ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert rc == 0
    torch.cuda.synchronize(dev)
    return bits, status, iters, app


def _size_configs(lib):
    """One (bgn, A, crctype) per lifting size and base graph that a payload reaches."""
    seen = {}
    for bgn in (1, 2):
        for A in range(8, (8448 if bgn == 1 else 3840) - 24 + 1, 8):
            for crc in (1, 0):
                p = capi.LdpcConfig()
                if lib.gen_ldpc_parameters(ctypes.byref(p), ctypes.byref(capi.make_in_config(bgn, A, crc, 960, 0, 2,
                                                                                               0))) == 0:
                    seen.setdefault((bgn, int(p.Zc)), (bgn, A, crc))
    return sorted(seen.values())


def test_every_lifting_size_in_bounds_and_identical(dbg, oracle, cuda):
    rel = capi.load_library()
    configs = _size_configs(rel)
    assert len(configs) >= 90
    rows = [[1, 6, 22936, 0, 1280, 32767, -32767], [4, 4, 22936, 0, 1280, 32767, -32767],
            [0, 3, 22936, 0, 1280, 32767, -32767]]
    for k, (bgn, A, crc) in enumerate(configs):
        B = A + (16 if crc == 0 else 24)
        E = 2 * ((B * 2 + 1) // 2)
        cfg = (bgn, A, crc, E, k % 4, 2, 0)
        llr, _ = make_llrs(oracle, in_config(*cfg), 3, noise_db=-1.0, seed=k)
        x = torch.from_numpy(llr).to(cuda)
        for row in rows if k % 3 == 0 else rows[:1]:
            want = _decode(rel, x, cfg, row)
            got = _decode(dbg, x, cfg, row)
            for w, g in zip(want, got):
                assert torch.equal(w, g), (cfg, row)
            assert _clean(dbg) == [0, 0, 0, 0], (cfg, row)


def test_queued_launches_harq_and_noalloc_in_bounds(dbg, cuda):
    rel = capi.load_library()
    rng = np.random.default_rng(5)
    cfg = (1, 8424, 1, 25344, 0, 8, 0)
    x = torch.from_numpy(np.clip(rng.normal(size=(700, 25344)) * 700 + 300, -10000, 10000).astype(np.int16)).to(cuda)
    for row in ([1, 4, 22936, 0, 1280, 32767, -32767], [4, 3, 22936, 0, 1280, 32767, -32767],
                [0, 2, 22936, 0, 1280, 32767, -32767]):
        h_rel = torch.zeros((700, 26112), dtype=torch.int16, device=cuda)
        h_dbg = h_rel.clone()
        want = _decode(rel, x, cfg, row, h_rel)
        got = _decode(dbg, x, cfg, row, h_dbg)
        for w, g in zip(want, got):
            assert torch.equal(w, g), row
        assert torch.equal(h_rel, h_dbg)
        assert _clean(dbg) == [0, 0, 0, 0], row
    # the no-allocation entry point runs the same kernel from its static scratch
    icfg, dcfg = capi.make_in_config(*cfg), capi.make_decoder_config([1, 4, 22936, 0, 1280, 32767, -32767])
    bits = torch.zeros((700, 1056), dtype=torch.uint8, device=cuda)
    st = torch.empty(700, dtype=torch.int32, device=cuda)
    it = torch.empty(700, dtype=torch.int32, device=cuda)
    assert dbg.nrldpc_decode_batch_noalloc(ctypes.c_void_p(x.data_ptr()), 25344, 700, ctypes.byref(icfg),
                                           ctypes.byref(dcfg), ctypes.c_void_p(bits.data_ptr()), 1056,
                                           ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(it.data_ptr()),
                                           ctypes.c_void_p(0), 0, ctypes.c_void_p(0), 0, ctypes.c_void_p(0)) == 0
    torch.cuda.synchronize()
    want = _decode(rel, x, cfg, [1, 4, 22936, 0, 1280, 32767, -32767])
    assert torch.equal(bits, want[0]) and torch.equal(st, want[1]) and torch.equal(it, want[2])
    assert _clean(dbg) == [0, 0, 0, 0]


def test_mixed_kernel_in_bounds(dbg, cuda):
    from deeplearning_5g_ldpc_decoder_b200 import channel_llrs, ldpc_encode

    cfgs = random_mixed_configs(240, seed=31)
    gen = torch.Generator(device=cuda).manual_seed(3)
    llrs = []
    for i, (bgn, A, crc, E, rv, Qm) in enumerate(cfgs):
        pay = torch.randint(0, 256, (1, A // 8), dtype=torch.uint8, device=cuda, generator=gen)
        llrs.append(channel_llrs(ldpc_encode(pay, (bgn, A, crc, E, rv, Qm, 0)), E, Qm, -(2.0 + 6.0 * (i % 4)),
                                 seed=i)[0])
    arena = torch.cat(llrs)
    row = [2, 8, 22936, 0, 1280, 32767, -32767]
    want = MixedPlan(cfgs, row, device=cuda).decode(arena, use_graph=False)
    got = MixedPlan(cfgs, row, device=cuda, lib=dbg).decode(arena, use_graph=False)
    torch.cuda.synchronize()
    for w, g in zip(want, got):
        assert torch.equal(w, g)
    assert _clean(dbg) == [0, 0, 0, 0]
