"""Generate the golden vectors in tests/golden/ from the REFERENCE C library.

The reference library is compiled from the reference's own sources by
``oracle/build_ref.sh`` into ``oracle/_ref/libnrLDPC_ref.so``.  For every case
below this script draws a seeded payload, encodes it with the reference's
``c_ldpc_5g_encode``, passes it through the reference's ``tx_rx_process``
(libc ``srand`` seeded per case), and decodes with the reference's
``c_ldpc_5g_decode``, recording:

* the int16 channel LLRs (decoder input),
* hard bits, return status and the final beliefs LQ (read through the shim
  accessors that expose the decoders' file-static arrays),
* the executed iteration count: the smallest max_iterations whose status is 0
  (decoding restarts from the same input, so a run with max_iterations = k is
  the state after k iterations), or max_iterations if it never converges,
* HARQ sequences (rv0 then rv2 combined), encoder outputs, CRC remainders,
  the base-graph CSR tables and the compiled-in algo-2 tables.

usage:  oracle/build_ref.sh && python tests/golden/make_golden.py
"""

from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle.oracle import RefLib, dec_cfg, in_config  # noqa: E402

DEFAULT_ROW = [1, 32, 22936, 0, 1280, 32767, -32767]

# (bgn, A, crctype, E, rv, Qm, snr_power_db, decoder rows, tag)
CASES = [
    (2, 488, 1, 1920, 0, 2, 0.0, "c1_bg2_zc64"),
    (2, 488, 1, 1920, 0, 2, -3.0, "c1_bg2_zc64_low"),
    (1, 8424, 1, 25344, 0, 8, 10.2, "c2_bg1_zc384_r13"),
    (1, 8424, 1, 9600, 0, 8, 16.0, "c2_bg1_zc384_r88"),
    (1, 2440, 1, 7392, 0, 2, -1.0, "c5_bg1_zc112"),
    (1, 488, 1, 1536, 0, 1, -3.0, "bg1_bpsk_small"),
    (1, 3816, 0, 11520, 1, 4, 2.0, "bg1_rv1_crc16_16qam"),
    (2, 1000, 2, 3000, 2, 6, 4.0, "bg2_rv2_crc24b_64qam"),
    (2, 3816, 3, 4800, 3, 8, 12.0, "bg2_rv3_crc24c_256qam"),
    (1, 24, 1, 120, 1, 2, 0.0, "bg1_tiny_zc3_rv1"),
    (2, 40, 3, 200, 3, 2, 0.0, "bg2_tiny"),
    (2, 1000, 1, 9000, 0, 2, -6.0, "bg2_repetition"),
    (1, 7000, 1, 8000, 0, 4, 30.0, "bg1_high_rate_noise"),
]
ALGOS = [
    [0, 8, 22936, 0, 1280, 20, -32768],     # BP row of scripts/sim_c_ldpc_encoder_decoder.py:49 (8 it)
    [1, 8, 22936, 0, 1280, 32767, -32767],
    [2, 8, 22936, 0, 1280, 32767, -32767],
    [3, 8, 22936, 0, 1280, 32767, -32767],
    [4, 8, 22936, 0, 1280, 32767, -32767],
    [1, 6, 26000, 64, 1000, 20000, -20000],  # offset min-sum + narrower clip
]
PER_CASE = 2


def iterations_of(ref: RefLib, llr, cfg, row, status):
    if status != 0:
        return row[1]
    for k in range(1, row[1] + 1):
        r = list(row)
        r[1] = k
        st, _, _ = ref.decode(llr, cfg, dec_cfg(r))
        if st == 0:
            return k
    raise AssertionError("converged run not reproduced")


def main() -> None:
    ref = RefLib()
    out = {}
    meta = []
    for ci, (bgn, A, crc, E, rv, Qm, snr, tag) in enumerate(CASES):
        cfg = in_config(bgn, A, crc, E, rv, Qm, 0)
        rc, p = ref.gen(cfg)
        assert rc == 0, tag
        rng = np.random.default_rng(1000 + ci)
        noise_db = -snr - 10 * np.log10(Qm)
        for k in range(1 if p.Zc >= 256 else PER_CASE):
            pay = rng.integers(0, 256, A // 8, dtype=np.uint8)
            rm = ref.encode(pay, cfg)
            ref.srand(1000 + 17 * ci + k)
            llr = ref.channel(rm, E, Qm, noise_db)
            key = f"{tag}_{k}"
            out[f"{key}_llr"] = llr
            out[f"{key}_payload"] = pay
            out[f"{key}_rm"] = rm
            for ai, row in enumerate(ALGOS):
                st, bits, lq = ref.decode(llr, cfg, dec_cfg(row))
                its = iterations_of(ref, llr, cfg, row, st)
                out[f"{key}_a{ai}_bits"] = bits
                out[f"{key}_a{ai}_lq"] = lq
                out[f"{key}_a{ai}_meta"] = np.array([st, its], dtype=np.int32)
            meta.append([bgn, A, crc, E, rv, Qm, k, ci])
    out["cases"] = np.array(meta, dtype=np.int32)
    out["algos"] = np.array(ALGOS, dtype=np.int32)
    out["tags"] = np.array([c[-1] for c in CASES])

    # HARQ: rv0 then rv2 of the same codeword combined into the soft buffer.
    harq_cases = [(2, 488, 1, 960, 2, -4.0), (1, 1976, 1, 3000, 4, -1.0)]
    for hi, (bgn, A, crc, E, Qm, snr) in enumerate(harq_cases):
        rng = np.random.default_rng(77 + hi)
        pay = rng.integers(0, 256, A // 8, dtype=np.uint8)
        row = [1, 8, 22936, 0, 1280, 32767, -32767]
        seq = []
        for step, (rv, harq_on) in enumerate([(0, 0), (2, 1), (3, 1)]):
            cfg = in_config(bgn, A, crc, E, rv, Qm, harq_on)
            rm = ref.encode(pay, cfg)
            ref.srand(500 + 10 * hi + step)
            llr = ref.channel(rm, E, Qm, -snr - 10 * np.log10(Qm))
            st, bits, lq = ref.decode(llr, cfg, dec_cfg(row))
            _, p = ref.gen(cfg)
            out[f"harq{hi}_s{step}_llr"] = llr
            out[f"harq{hi}_s{step}_bits"] = bits
            out[f"harq{hi}_s{step}_lq"] = lq
            out[f"harq{hi}_s{step}_buf"] = ref.harq_memory(p.N + 2 * p.Zc)
            seq.append([bgn, A, crc, E, rv, Qm, harq_on, st])
        out[f"harq{hi}_seq"] = np.array(seq, dtype=np.int32)

    # CRC remainders.
    rng = np.random.default_rng(5)
    crc_in = rng.integers(0, 256, 1056, dtype=np.uint8)
    lens = [1, 2, 3, 16, 61, 64, 480, 1056]
    crc_out = np.zeros((4, len(lens)), dtype=np.uint32)
    for t in range(4):
        for j, L in enumerate(lens):
            crc_out[t, j] = ref.lib.calculate_crc(crc_in.ctypes.data_as(ctypes.c_void_p), L, t)
    out["crc_in"] = crc_in
    out["crc_lens"] = np.array(lens, dtype=np.int32)
    out["crc_out"] = crc_out

    # Base-graph CSR tables and compiled-in algo-2 tables as the reference exports them.
    for bgn, rows, nnz in ((1, 46, 316), (2, 42, 197)):
        off = np.ctypeslib.as_array((ctypes.c_uint16 * (rows + 1)).in_dll(ref.lib, f"BG{bgn}_HBG_offset_array"))
        col = np.ctypeslib.as_array((ctypes.c_uint16 * nnz).in_dll(ref.lib, f"BG{bgn}_HBG_array"))
        vij = np.ctypeslib.as_array((ctypes.c_uint16 * (8 * nnz)).in_dll(ref.lib, f"BG{bgn}_HBG_Vij_array"))
        out[f"bg{bgn}_off"] = off.copy()
        out[f"bg{bgn}_col"] = col.copy()
        out[f"bg{bgn}_vij"] = vij.reshape(8, nnz).copy()
        ta = np.ctypeslib.as_array((ctypes.c_int16 * (32 * rows)).in_dll(ref.lib, f"BG{bgn}_trained_alpha_list"))
        tb = np.ctypeslib.as_array((ctypes.c_int16 * (32 * rows)).in_dll(ref.lib, f"BG{bgn}_trained_beta_list"))
        out[f"bg{bgn}_trained_alpha"] = ta.reshape(32, rows).copy()
        out[f"bg{bgn}_trained_beta"] = tb.reshape(32, rows).copy()

    # Derived parameters for every A of both base graphs and all CRC types (rv 1).
    prm = []
    for bgn in (1, 2):
        for crc in range(4):
            for A in range(8, 8449, 8):
                cfg = in_config(bgn, A, crc, 1200, 1, 2, 0)
                rc, p = ref.gen(cfg)
                if rc == 0:
                    prm.append([bgn, A, crc, p.B, p.Zc, p.iLS, p.K, p.F, p.N, p.k0])
    out["params"] = np.array(prm, dtype=np.int32)

    path = os.path.join(HERE, "reference_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
