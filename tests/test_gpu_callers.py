"""The drop-in boundary under the reference's own Python harness.

tests/golden/caller_vectors.npz was recorded by running the reference's
run_ldpc_trial (scripts/ldpc_c_sim_common.py:227-272) unchanged against the
reference C library, with the ctypes declarations its load_c_library installs
(:60-109), for every decoder row of the reference's C and CUDA sweep scripts.
Here the same calls are replayed through libnrldpc_b200.so with the same
declarations (ndpointer arguments, record pointers), in the harness's order:
encode, then every decoder row on one shared channel realisation with the
hard-bit buffer cleared before each decode.  Every encoded byte, status, hard
bit and the trial's returned (block error, bit error) arrays must be equal.
Both entry-point families are replayed: cuda_ldpc_5g_* (the CUDA sweep's
symbols) and c_ldpc_5g_* (the C sweep's)."""

import ctypes
import os

import numpy as np
import pytest
from numpy.ctypeslib import ndpointer

from deeplearning_5g_ldpc_decoder_b200 import capi

VEC = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "caller_vectors.npz")


def _ctype(desc: str):
    if desc.startswith("ndpointer:"):
        _, dt, flags = desc.split(":")
        return ndpointer(dtype=np.dtype(dt), flags=flags or None)
    if desc.startswith("pointer:"):
        name = desc.split(":")[1]
        return ctypes.POINTER({"LdpcInConfig": capi.LdpcInConfig, "DecoderConfig": capi.DecoderConfig}[name])
    return {"c_int": ctypes.c_int, "c_ulong": ctypes.c_size_t, "c_ushort": ctypes.c_uint16,
            "c_float": ctypes.c_float}[desc]


def _declarations(g):
    out = {}
    for d in g["declarations"]:
        name, sig = str(d).split("(", 1)
        parts = sig.rstrip(")").split(";")
        out[name] = ([_ctype(p) for p in parts if not p.startswith("->")], _ctype(parts[-1][2:]))
    return out


def _bind(lib, symbol, decl):
    fn = getattr(lib, symbol)
    fn.argtypes, fn.restype = decl
    return fn


@pytest.mark.gpu
@pytest.mark.parametrize("family", ["cuda", "c"])
def test_reference_harness_calls_replayed_through_dropin(cuda, family):
    g = np.load(VEC)
    decl = _declarations(g)
    lib = ctypes.CDLL(capi.LIB_PATH)     # own handle: the declarations below stay local to this test
    encode = _bind(lib, f"{family}_ldpc_5g_encode", decl["ldpc_5g_encode"])
    decode = _bind(lib, f"{family}_ldpc_5g_decode", decl["ldpc_5g_decode"])
    rows = [list(map(int, r)) for r in g["rows"]]
    for k in range(int(g["num_trials"])):
        cfg = capi.LdpcInConfig(*map(int, g[f"t{k}_cfg"]))
        info = g[f"t{k}_info"]
        rm = np.zeros((cfg.E + 7) // 8, dtype=np.uint8)
        assert encode(info, rm, ctypes.byref(cfg)) == 0
        assert np.array_equal(rm, g[f"t{k}_rm"]), k
        llr = g[f"t{k}_llr"]
        B = cfg.A + (16 if cfg.crctype == 0 else 24)
        hardbits = np.zeros((B + 7) // 8, dtype=np.uint8)
        info_bits = np.unpackbits(info, bitorder="big")[: cfg.A]
        block_err = np.zeros(len(rows))
        bit_err = np.zeros(len(rows))
        for r, vals in enumerate(rows):
            hardbits.fill(0)
            dcfg = capi.make_decoder_config(vals)
            st = decode(llr, hardbits, ctypes.byref(cfg), ctypes.byref(dcfg))
            assert st == g[f"t{k}_status"][r], (k, vals)
            assert np.array_equal(hardbits, g[f"t{k}_bits"][r]), (k, vals)
            block_err[r] = 0 if st == 0 else 1
            bit_err[r] = np.count_nonzero(np.unpackbits(hardbits, bitorder="big")[: cfg.A] != info_bits)
        assert np.array_equal(block_err, g[f"t{k}_block_err"]) and np.array_equal(bit_err, g[f"t{k}_bit_err"]), k


def test_table_config_loader_fields_from_dropin():
    """load_ldpc_table_config's view (deep_learning/ldpc_table_config.py:110-154)
    of gen_ldpc_parameters through this library equals the reference's (host
    code: no GPU needed)."""
    g = np.load(VEC)
    lib = ctypes.CDLL(capi.LIB_PATH)
    lib.gen_ldpc_parameters.argtypes = [ctypes.POINTER(capi.LdpcConfig), ctypes.POINTER(capi.LdpcInConfig)]
    lib.gen_ldpc_parameters.restype = ctypes.c_int
    seen = set()
    for k in range(int(g["num_trials"])):
        gi = int(g[f"t{k}_grid"][0])
        if gi in seen:
            continue
        seen.add(gi)
        icfg = capi.LdpcInConfig(*map(int, g[f"t{k}_cfg"]))
        c = capi.LdpcConfig()
        assert lib.gen_ldpc_parameters(ctypes.byref(c), ctypes.byref(icfg)) == 0
        want = g[f"table_{gi}"]
        rows, cols, nnz = {1: (46, 68, 316), 2: (42, 52, 197)}[c.bgn]
        assert [c.B, c.Zc, c.iLS, c.K, c.F, c.N, c.k0, rows, cols, nnz] == list(want)
        assert [c.HBG_array[i] for i in range(nnz)] == list(g[f"table_{gi}_cols"])
        assert [c.Vij_array[i] for i in range(nnz)] == list(g[f"table_{gi}_vij"])
        assert [c.HBG_offset_array[i] for i in range(rows + 1)] == list(g[f"table_{gi}_off"])
