"""Host side of the C ABI (no GPU needed): the library loads, exports every
symbol declared in include/nrldpc_b200.h, derives parameters and CRCs exactly
like the reference, and validates arguments before touching a device."""

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from deeplearning_5g_ldpc_decoder_b200 import capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "nrldpc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for n in capi.EXPORTED_SYMBOLS:
        assert n in names, n


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", capi.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    for n in declared_functions():
        assert n in exported, n
        assert getattr(lib, n) is not None


def test_debug_library_exports_the_same_symbols_and_release_has_no_checks(lib):
    from deeplearning_5g_ldpc_decoder_b200.build import DEBUG_LIB_PATH, build_library

    path = DEBUG_LIB_PATH if os.path.exists(DEBUG_LIB_PATH) else build_library(debug=True)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    for n in declared_functions():
        assert n in exported, n
    assert b"bounds-checked" in capi.load_library(path).nrldpc_version()
    rec = (ctypes.c_uint32 * 4)(7, 7, 7, 7)
    assert lib.nrldpc_bounds_check_status(rec, 1) == 0 and list(rec) == [0, 0, 0, 0]
    assert b"bounds-checked" not in lib.nrldpc_version()


def test_record_layouts_match_reference():
    assert ctypes.sizeof(capi.LdpcInConfig) == 14
    assert ctypes.sizeof(capi.DecoderConfig) == 14
    assert ctypes.sizeof(capi.LdpcConfig) == 28 + 4 + 3 * 8  # 14 x u16, padding, 3 pointers


def test_gen_ldpc_parameters_matches_reference(lib, golden):
    for bgn, A, crc, B, Zc, iLS, K, F, N, k0 in golden["params"]:
        cfg = capi.make_in_config(int(bgn), int(A), int(crc), 1200, 1, 2, 0)
        out = capi.LdpcConfig()
        assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(cfg)) == 0
        assert (out.B, out.Zc, out.iLS, out.K, out.F, out.N, out.k0) == (B, Zc, iLS, K, F, N, k0)


def test_gen_ldpc_parameters_tables_match_reference_csr(lib, golden):
    for bgn, rows, nnz in ((1, 46, 316), (2, 42, 197)):
        # one configuration per lifting set
        seen = set()
        for row in golden["params"]:
            if row[0] != bgn or row[5] in seen:
                continue
            seen.add(int(row[5]))
            cfg = capi.make_in_config(bgn, int(row[1]), int(row[2]), 1200, 1, 2, 0)
            out = capi.LdpcConfig()
            assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(cfg)) == 0
            off = np.ctypeslib.as_array(out.HBG_offset_array, shape=(rows + 1,))
            col = np.ctypeslib.as_array(out.HBG_array, shape=(nnz,))
            vij = np.ctypeslib.as_array(out.Vij_array, shape=(nnz,))
            assert np.array_equal(off, golden[f"bg{bgn}_off"])
            assert np.array_equal(col, golden[f"bg{bgn}_col"])
            assert np.array_equal(vij, golden[f"bg{bgn}_vij"][out.iLS])
        assert seen == set(range(8))


def test_invalid_configs_rejected(lib):
    bad = [
        (3, 488, 1, 1920, 0, 2, 0),      # bgn
        (1, 488, 4, 1920, 0, 2, 0),      # crctype
        (1, 488, 1, 1920, 0, 3, 0),      # Qm
        (1, 488, 1, 1920, 0, 2, 2),      # HARQ_on
        (1, 488, 1, 1920, 4, 2, 0),      # rv
        (1, 488, 1, 1921, 0, 2, 0),      # E % Qm
        (1, 487, 1, 1920, 0, 2, 0),      # A % 8
        (1, 8432, 1, 30000, 0, 2, 0),    # BG1 B > 8448
        (2, 3824, 1, 9000, 0, 2, 0),     # BG2 B > 3840
    ]
    llr = np.zeros(40000, np.int16)
    bits = np.zeros(2048, np.uint8)
    dcfg = capi.make_decoder_config([1, 8, 22936, 0, 1280, 32767, -32767])
    for b in bad:
        cfg = capi.make_in_config(*b)
        out = capi.LdpcConfig()
        assert lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(cfg)) == -1, b
        for name in ("cuda_ldpc_5g_decode", "c_ldpc_5g_decode"):
            rc = getattr(lib, name)(llr.ctypes.data_as(ctypes.c_void_p), bits.ctypes.data_as(ctypes.c_void_p),
                                    ctypes.byref(cfg), ctypes.byref(dcfg))
            assert rc == capi.NRLDPC_ERR_CONFIG, (name, b)


def test_batched_argument_validation(lib):
    cfg = capi.make_in_config(2, 488, 1, 1920, 0, 2, 0)
    good = capi.make_decoder_config([1, 8, 22936, 0, 1280, 32767, -32767])
    badalgo = capi.make_decoder_config([5, 8, 22936, 0, 1280, 32767, -32767])
    vp = ctypes.c_void_p
    args = lambda d, n, ptr, stride: (ptr, stride, n, ctypes.byref(cfg), ctypes.byref(d), vp(0), 64, vp(0), vp(0),
                                      vp(0), 0, vp(0), 0, vp(0))
    assert lib.nrldpc_decode_batch(*args(good, 0, vp(0), 0)) == capi.NRLDPC_OK        # empty batch
    assert lib.nrldpc_decode_batch(*args(badalgo, 4, vp(0), 1920)) == capi.NRLDPC_ERR_ALGO
    assert lib.nrldpc_decode_batch(*args(good, 4, vp(0), 1920)) == capi.NRLDPC_ERR_ARG  # null LLRs
    assert lib.nrldpc_decode_batch(*args(good, 4, vp(16), 100)) == capi.NRLDPC_ERR_ARG  # stride < E
    assert lib.nrldpc_decode_batch(*args(good, -1, vp(16), 1920)) == capi.NRLDPC_ERR_ARG
    bad_cfg = capi.make_in_config(2, 488, 1, 1921, 0, 2, 0)
    assert lib.nrldpc_decode_batch(vp(16), 1921, 1, ctypes.byref(bad_cfg), ctypes.byref(good), vp(0), 64, vp(0),
                                   vp(0), vp(0), 0, vp(0), 0, vp(0)) == capi.NRLDPC_ERR_CONFIG


def test_calculate_crc_matches_reference(lib, golden):
    data = np.ascontiguousarray(golden["crc_in"])
    for t in range(4):
        for j, L in enumerate(golden["crc_lens"]):
            assert lib.calculate_crc(data.ctypes.data_as(ctypes.c_void_p), int(L), t) == golden["crc_out"][t, j]
    assert lib.calculate_crc(data.ctypes.data_as(ctypes.c_void_p), 10, 7) == 0   # unknown type reads as 0


def test_no_cpu_fallback_without_gpu(lib):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = capi.make_in_config(2, 488, 1, 1920, 0, 2, 0)
    dcfg = capi.make_decoder_config([1, 8, 22936, 0, 1280, 32767, -32767])
    llr = np.zeros(1920, np.int16)
    bits = np.zeros(64, np.uint8)
    rc = lib.cuda_ldpc_5g_decode(llr.ctypes.data_as(ctypes.c_void_p), bits.ctypes.data_as(ctypes.c_void_p),
                                 ctypes.byref(cfg), ctypes.byref(dcfg))
    assert rc == capi.NRLDPC_ERR_CUDA


def test_trained_weight_setters_validate(lib):
    assert lib.nrldpc_set_trained_weights(3, None, None, 1) == capi.NRLDPC_ERR_ARG
    a = np.zeros((2, 46), np.int16)
    assert lib.nrldpc_set_trained_weights(1, a.ctypes.data_as(ctypes.c_void_p), None, 0) == capi.NRLDPC_ERR_ARG
    assert lib.nrldpc_set_trained_weights(1, None, None, 0) == capi.NRLDPC_OK
    assert lib.nrldpc_set_degree_alpha(None) == capi.NRLDPC_OK
