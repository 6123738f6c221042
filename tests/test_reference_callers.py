"""The reference's own Python callers of the boundary, imported read-only from
the reference checkout and pointed at libnrldpc_b200.so (CPU; skipped where
the checkout is absent, e.g. on the GPU host, where
tests/test_gpu_callers.py replays their recorded calls instead).

* scripts/ldpc_c_sim_common.py:60-109 ``load_c_library`` binds this library's
  cuda_ldpc_5g_* and c_ldpc_5g_* symbols with its own ctypes declarations
  (tx_rx_process from the reference C library, as the CUDA sweep does:
  scripts/sim_cuda_ldpc_encoder_decoder.py:58-68);
* deep_learning/ldpc_table_config.py:110-154 ``load_ldpc_table_config`` returns
  identical LdpcTableConfig records from this library and from the reference C
  library for every (bgn, A, crctype, rv) of a sweep of sizes."""

import os
import sys

import numpy as np
import pytest

from deeplearning_5g_ldpc_decoder_b200 import capi
from oracle.oracle import REF_SO
from oracle.refroot import REFERENCE_ROOT, reference_available

pytestmark = pytest.mark.skipif(not reference_available() or not os.path.exists(REF_SO),
                                reason="reference checkout or its C library build not present")


@pytest.fixture(scope="module")
def ref_modules():
    for p in (os.path.join(REFERENCE_ROOT, "scripts"), REFERENCE_ROOT):
        if p not in sys.path:
            sys.path.insert(0, p)
    import ldpc_c_sim_common as sim
    from deep_learning import ldpc_table_config as tc

    return sim, tc


@pytest.mark.parametrize("family", ["cuda", "c"])
def test_load_c_library_binds_dropin_symbols(ref_modules, family):
    sim, _ = ref_modules
    lib = sim.load_c_library(capi.LIB_PATH, encode_symbol=f"{family}_ldpc_5g_encode",
                             decode_symbol=f"{family}_ldpc_5g_decode", channel_lib_path=REF_SO)
    assert lib.ldpc_5g_decode.argtypes is not None and lib.ldpc_5g_encode.restype is not None
    assert lib.tx_rx_process_fn is not None


def test_load_ldpc_table_config_identical(ref_modules):
    _, tc = ref_modules
    rng = np.random.default_rng(9)
    checked = 0
    for bgn in (1, 2):
        for A in sorted(set(rng.integers(2, 1056, 40).tolist()) | {8, 488, 3816, 8424}):
            A *= 8
            for crctype in (0, 1):
                B = A + (16 if crctype == 0 else 24)
                if B > (8448 if bgn == 1 else 3840) or A >= 65536:
                    continue
                E = int(np.ceil(3 * B / 8)) * 8
                rv = int(rng.integers(0, 4))
                args = (bgn, A, crctype, E, rv, 8)
                want = tc.load_ldpc_table_config(*args, lib_path=REF_SO)
                got = tc.load_ldpc_table_config(*args, lib_path=capi.LIB_PATH)
                assert got == want, args
                checked += 1
    assert checked > 100
    with pytest.raises(ValueError):
        tc.load_ldpc_table_config(2, 8000, 1, 9000, 0, 2, lib_path=capi.LIB_PATH)
