"""Iterate over the golden vectors produced by tests/golden/make_golden.py."""

from __future__ import annotations

import numpy as np


def decode_cases(g):
    """Yield (key, in_config tuple, llr) for every golden decode case."""
    tags = [str(t) for t in g["tags"]]
    for bgn, A, crc, E, rv, Qm, k, ci in g["cases"]:
        key = f"{tags[ci]}_{k}"
        yield key, (int(bgn), int(A), int(crc), int(E), int(rv), int(Qm), 0), g[f"{key}_llr"]


def algo_rows(g):
    return [list(map(int, r)) for r in g["algos"]]


def expected(g, key, ai):
    st, its = g[f"{key}_a{ai}_meta"]
    return int(st), g[f"{key}_a{ai}_bits"], int(its), g[f"{key}_a{ai}_lq"]


def harq_sequences(g):
    hi = 0
    while f"harq{hi}_seq" in g.files:
        steps = []
        for s, row in enumerate(g[f"harq{hi}_seq"]):
            bgn, A, crc, E, rv, Qm, harq_on, st = map(int, row)
            steps.append(dict(cfg=(bgn, A, crc, E, rv, Qm, harq_on), status=st, llr=g[f"harq{hi}_s{s}_llr"],
                              bits=g[f"harq{hi}_s{s}_bits"], lq=g[f"harq{hi}_s{s}_lq"],
                              buf=g[f"harq{hi}_s{s}_buf"]))
        yield hi, steps
        hi += 1


BP_RTOL = 1e-3        # elementwise bound on BP final LLRs
BP_ATOL = 2e-2        # LLR units (1/128 of an int16 quantum is 0.0078)
BP_TIGHT_RTOL = 1e-4  # ... and fewer than BP_TIGHT_FRAC of the LLRs beyond this
BP_TIGHT_FRAC = 1e-2


def lq_close(a: np.ndarray, b: np.ndarray, algo: int, converged: bool = True) -> bool:
    """Final-belief comparison: exact for every algorithm except BP (algo 0).

    BP calls tanhf/atanhf: CUDA's float functions on the device, the host
    libm's in the reference; they differ by an ulp or two now and then and
    layered BP amplifies that a little.  Hard decisions, status and iteration
    counts are compared exactly elsewhere."""
    if algo != 0:
        return bool(np.array_equal(a, b))
    if not converged:
        # A BP run that never converges is chaotic: hard decisions are compared
        # exactly elsewhere; here the LLRs must agree in sign and roughly in size.
        return bool(np.mean(np.sign(a) == np.sign(b)) > 0.999 and np.allclose(a, b, rtol=1e-2, atol=0.5))
    if not np.allclose(a, b, rtol=BP_RTOL, atol=BP_ATOL):
        return False
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-6)
    return bool(np.mean(rel > BP_TIGHT_RTOL) < BP_TIGHT_FRAC)
