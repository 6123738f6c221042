"""Generate tests/golden/caller_vectors.npz by running the reference's own BLER
harness against the reference C library.

The reference's Python callers of the drop-in boundary cannot travel to the
GPU host, so this script records what they do here:

* ``load_c_library`` (scripts/ldpc_c_sim_common.py:60-109) binds the library's
  symbols; the ctypes declarations it installs (argtypes / restype of the
  encode, channel and decode functions) are recorded;
* ``run_ldpc_trial`` (scripts/ldpc_c_sim_common.py:227-272) is run unchanged
  on a recording proxy of that library for every decoder row of
  scripts/sim_c_ldpc_encoder_decoder.py:45-55 and
  scripts/sim_cuda_ldpc_encoder_decoder.py:41-48, over configurations built by
  the harness's own ``make_ldpc_config`` (:135-150) at SNRs converted by
  ``run_bler_sweep``'s rule (:286); every call's inputs, outputs and return
  value, and the trial's returned (block error, bit error) arrays, are stored;
* ``load_ldpc_table_config`` (deep_learning/ldpc_table_config.py:110-154) is
  run against the reference library on the same configurations.

tests/test_gpu_callers.py replays the recorded calls through
libnrldpc_b200.so with the recorded declarations.

usage:  oracle/build_ref.sh && python tests/golden/make_caller_golden.py
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle.oracle import REF_SO  # noqa: E402
from oracle.refroot import REFERENCE_ROOT  # noqa: E402

sys.path.insert(0, os.path.join(REFERENCE_ROOT, "scripts"))
sys.path.insert(0, REFERENCE_ROOT)

import ldpc_c_sim_common as sim  # noqa: E402
import sim_c_ldpc_encoder_decoder as sim_c  # noqa: E402
import sim_cuda_ldpc_encoder_decoder as sim_cuda  # noqa: E402
from deep_learning.ldpc_table_config import load_ldpc_table_config  # noqa: E402

# (Qm, rv, B, coderate, bgn, crctype) grid tuples, snr_power_db
GRID = [
    ((1, 0, 128, 1 / 3, 1, 0), [-3.0, -2.0]),       # the C sweep's configuration
    ((8, 0, 3840, 1 / 3, 1, 0), [0.8, 1.6]),        # the CUDA sweep's Qm 8 point
    ((2, 0, 3840, 1 / 3, 1, 0), [-4.2, -3.6]),      # the CUDA sweep's Qm 2 point
    ((4, 1, 512, 1 / 2, 2, 1), [2.0, 4.0]),
    ((6, 0, 1024, 2 / 3, 2, 3), [8.0, 10.0]),
]
TRIALS = 3


def describe(t) -> str:
    """Text form of one ctypes argtype / restype."""
    if hasattr(t, "_dtype_"):
        flags = [f for f in ("C_CONTIGUOUS", "F_CONTIGUOUS", "ALIGNED", "WRITEABLE")
                 if t._flags_ is not None and t._flags_ & np.ctypeslib.ndpointer(flags=f)._flags_]
        return f"ndpointer:{np.dtype(t._dtype_).str}:{','.join(flags)}"
    if hasattr(t, "_type_") and issubclass(t, ctypes._Pointer):
        return f"pointer:{t._type_.__name__}"
    return t.__name__


class Recorder:
    """Proxy of the loaded library that records every call the harness makes."""

    def __init__(self, lib):
        self.lib = lib
        self.calls = []

    def _wrap(self, name):
        fn = getattr(self.lib, name)

        def call(*args):
            rec = {"fn": name, "in": [np.array(a, copy=True) if isinstance(a, np.ndarray) else a for a in args]}
            ret = fn(*args)
            rec["out"] = [np.array(a, copy=True) if isinstance(a, np.ndarray) else None for a in args]
            rec["ret"] = int(ret)
            self.calls.append(rec)
            return ret
        return call

    def __getattr__(self, name):
        if name in ("ldpc_5g_encode", "tx_rx_process_fn", "ldpc_5g_decode"):
            return self._wrap(name)
        return getattr(self.lib, name)


def main() -> None:
    lib = sim.load_c_library(REF_SO)
    decl = {name: [describe(t) for t in getattr(lib, name).argtypes] + ["->" + getattr(lib, name).restype.__name__]
            for name in ("ldpc_5g_encode", "tx_rx_process_fn", "ldpc_5g_decode")}
    rows = [list(r) for r in sim_c.get_decoder_config_list()] + [list(r) for r in sim_cuda.get_decoder_config_list()]
    libc = ctypes.CDLL(None)
    out = {"rows": np.array(rows, dtype=np.int32)}
    trials = []
    for gi, (grid, snrs) in enumerate(GRID):
        assert sim.get_config_grid_rejection_reason(*grid) is None, grid
        cfg = sim.make_ldpc_config(*grid)
        tab = load_ldpc_table_config(cfg.bgn, cfg.A, cfg.crctype, cfg.E, cfg.rv, cfg.Qm, lib_path=REF_SO)
        out[f"table_{gi}"] = np.array([tab.B, tab.Zc, tab.iLS, tab.K, tab.F, tab.N, tab.k0, tab.num_rows,
                                       tab.num_cols, tab.num_edges], dtype=np.int32)
        out[f"table_{gi}_cols"] = np.array(tab.hbg_columns, dtype=np.int32)
        out[f"table_{gi}_vij"] = np.array(tab.vij, dtype=np.int32)
        out[f"table_{gi}_off"] = np.array(tab.row_offsets, dtype=np.int32)
        for snr in snrs:
            noise_db = -snr - 10 * np.log10(cfg.Qm)
            for t in range(TRIALS):
                seed = 100 * gi + 10 * int(snr * 10 % 10) + t
                np.random.seed(seed)
                libc.srand(ctypes.c_uint(seed))
                rec = Recorder(lib)
                block_err, bit_err = sim.run_ldpc_trial(rec, cfg, rows, noise_db)
                k = len(trials)
                enc = [c for c in rec.calls if c["fn"] == "ldpc_5g_encode"][0]
                chan = [c for c in rec.calls if c["fn"] == "tx_rx_process_fn"][0]
                decs = [c for c in rec.calls if c["fn"] == "ldpc_5g_decode"]
                assert len(decs) == len(rows)
                out[f"t{k}_cfg"] = np.array([cfg.bgn, cfg.A, cfg.crctype, cfg.E, cfg.rv, cfg.Qm, cfg.HARQ_on],
                                            dtype=np.int32)
                out[f"t{k}_grid"] = np.array([gi, snr, noise_db], dtype=np.float64)
                out[f"t{k}_info"] = enc["in"][0]
                out[f"t{k}_rm"] = enc["out"][1]
                out[f"t{k}_llr"] = chan["out"][4]
                out[f"t{k}_bits"] = np.stack([d["out"][1] for d in decs])
                out[f"t{k}_status"] = np.array([d["ret"] for d in decs], dtype=np.int32)
                out[f"t{k}_block_err"] = np.asarray(block_err, dtype=np.float64)
                out[f"t{k}_bit_err"] = np.asarray(bit_err, dtype=np.float64)
                trials.append(k)
    out["num_trials"] = np.array(len(trials))
    out["declarations"] = np.array([f"{k}({';'.join(v)})" for k, v in decl.items()])
    path = os.path.join(HERE, "caller_vectors.npz")
    np.savez_compressed(path, **out)
    st = np.array([out[f"t{k}_status"] for k in trials])
    print(f"wrote {path}: {len(trials)} trials x {len(rows)} decoder rows, status histogram "
          f"{dict(zip(*np.unique(st, return_counts=True)))}; declarations {list(out['declarations'])}")


if __name__ == "__main__":
    main()
