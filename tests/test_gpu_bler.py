"""Block error rate against Es/N0: the device chain (ldpc_encode -> channel_llrs
-> ldpc_decode) against the reference's own chain (c_ldpc_5g_encode ->
tx_rx_process -> c_ldpc_5g_decode, the BLER loop of
scripts/ldpc_c_sim_common.py:227-343) on the same seeded payloads.

The device channel has its own noise generator, so the two chains see
different noise and agree only statistically: at every point the Wilson 95 %
intervals of the two block error rates must overlap.  Both sides are seeded,
so the test is deterministic.  SNR convention of the reference harness:
noise_power_db = -Es/N0 for unit-energy symbols (:286).

Points: BASELINE config 1 (BG2 Zc=64, A=488, E=1920, QPSK, algo 1, 10
iterations) across its waterfall, Es/N0 -3..0 dB (the BLER is already 0 at
the config's 0..3 dB); config 2 (BG1 Zc=384, A=8424, E=25344, 256QAM,
8 iterations) around its 1e-2 point with algo 1 and algo 0 (BP)."""

import json
import os

import numpy as np
import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import channel_llrs, ldpc_decode, ldpc_encode
from tests.bler_chain import overlap, payloads, reference_block_errors, wilson

pytestmark = pytest.mark.gpu

C1 = (2, 488, 1, 1920, 0, 2, 0)
C2 = (1, 8424, 1, 25344, 0, 8, 0)
ROW1 = [1, 10, 22936, 0, 1280, 32767, -32767]
ROW2 = [1, 8, 22936, 0, 1280, 32767, -32767]
ROW_BP = [0, 8, 22936, 0, 1280, 32767, -32767]

POINTS = [
    # (name, cfg, row, Es/N0 dB, blocks)
    *[("C1 algo1", C1, ROW1, es, 2000) for es in (-3.0, -2.5, -2.0, -1.5, -1.0, 0.0)],
    *[("C2 algo1", C2, ROW2, es, 800) for es in (10.4, 10.6, 10.8, 11.0)],
    *[("C2 algo0 BP", C2, ROW_BP, es, 800) for es in (10.4, 10.6, 10.8)],
]


def _device_errors(cfg, row, esn0, n, seed, dev):
    pay = torch.from_numpy(payloads(n, cfg[1], seed)).to(dev)
    llr = channel_llrs(ldpc_encode(pay, cfg), cfg[3], cfg[5], -esn0, seed=seed)
    res = ldpc_decode(llr, cfg, row)
    ok = (res.status == 0) & (res.hardbits[:, : cfg[1] // 8] == pay).all(dim=1)
    return int((~ok).sum().item())


def test_bler_curves_agree_within_wilson_intervals(cuda, reflib):
    table = []
    for k, (name, cfg, row, esn0, n) in enumerate(POINTS):
        seed = 1000 + k
        dev_err = _device_errors(cfg, row, esn0, n, seed, cuda)
        ref_err = reference_block_errors(cfg, row, -esn0, n, seed)
        ci_d, ci_r = wilson(dev_err, n), wilson(ref_err, n)
        table.append({"curve": name, "esn0_db": esn0, "blocks": n, "device_bler": dev_err / n,
                      "device_ci95": [round(x, 4) for x in ci_d], "reference_bler": ref_err / n,
                      "reference_ci95": [round(x, 4) for x in ci_r], "overlap": overlap(ci_d, ci_r)})
    print("\nBLER_TABLE " + json.dumps(table))
    out = os.environ.get("NRLDPC_BLER_TABLE")
    if out:
        with open(out, "w") as f:
            json.dump(table, f, indent=1)
    bad = [t for t in table if not t["overlap"]]
    assert not bad, bad
    # the sweep crosses the waterfall: each curve has points with errors and points nearly without
    for name in {t["curve"] for t in table}:
        rates = [t["reference_bler"] for t in table if t["curve"] == name]
        assert max(rates) > 0.05 and min(rates) < 0.05, (name, rates)
