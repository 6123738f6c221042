"""Autograd restatement of the reference's unrolled layered min-sum model.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the training
kernels (nrldpc_train_forward / nrldpc_train_backward).  Nothing in the product
imports it.

Restates ``CTableNeuralLayeredMinSumDecoder.forward``
(deep_learning/deeplearning_ldpc_model.py:315-410) as plain torch float32 ops
so autograd produces the reference's gradients: per iteration t and base-graph
row r, lifted LLRs of the row are gathered (:356-359), the old messages
subtracted (:359), the first minimum found with ``torch.min`` (first index),
the second minimum as the minimum over the other entries (:364-371),
``alpha * clamp(u - beta, min=0)`` formed (:373-376), signed by the product of
the signs (sign +1 at 0, :361-365), added back and optionally clipped (:378-381),
then scattered into a copy of LQ (:383-386).  Base-graph tables come from the
C oracle (``Oracle.graph``).  Pinned by tests/test_oracle_train.py against
vectors produced by the reference model itself (tests/golden/make_train_golden.py).
"""

from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np
import torch

from .oracle import Oracle, in_config


class MinSumGraph:
    """Per-row lifted column indices [Zc, degree] of one configuration."""

    def __init__(self, bgn, A, crctype, E, rv=0, Qm=2, oracle: Optional[Oracle] = None):
        o = oracle or Oracle()
        p, col, shift, off = o.graph(in_config(bgn, A, crctype, E, rv, Qm))
        self.params = p
        self.Zc, self.B, self.rows = p.Zc, p.B, p.rows
        self.n = p.N + 2 * p.Zc
        self.degrees = [int(off[r + 1] - off[r]) for r in range(p.rows)]
        z = np.arange(p.Zc)[:, None]
        self.row_cols: List[torch.Tensor] = []
        for r in range(p.rows):
            c = col[off[r]:off[r + 1]][None, :]
            s = shift[off[r]:off[r + 1]][None, :]
            self.row_cols.append(torch.from_numpy((c * p.Zc + (s + z) % p.Zc).astype(np.int64)))


def minsum_unrolled(graph: MinSumGraph, llr: torch.Tensor, alpha: torch.Tensor, beta: torch.Tensor,
                    clip: Optional[float] = None, detach: bool = False) -> Tuple[torch.Tensor, List[torch.Tensor]]:
    """llr [batch, n]; alpha, beta [T, rows] -> (final LQ, per-iteration LQ list)."""
    batch = llr.shape[0]
    T = alpha.shape[0]
    lq = llr.clone()
    if clip is not None:
        lq = lq.clamp(-clip, clip)
    cols = [c.to(llr.device) for c in graph.row_cols]
    msgs = [llr.new_zeros((batch, graph.Zc, d)) for d in graph.degrees]
    per_iter = []
    for t in range(T):
        for r, d in enumerate(graph.degrees):
            flat = cols[r].reshape(-1)
            rel = lq[:, flat].reshape(batch, graph.Zc, d) - msgs[r]
            x = rel.detach() if detach else rel
            sgn = torch.where(x < 0, -torch.ones_like(x), torch.ones_like(x))
            mag = x.abs()
            m1, i1 = torch.min(mag, dim=2)
            first = torch.nn.functional.one_hot(i1, num_classes=d).to(torch.bool)
            m2, _ = torch.min(mag.masked_fill(first, float("inf")), dim=2)
            u = torch.where(first, m2.unsqueeze(2), m1.unsqueeze(2))
            out = alpha[t, r] * torch.clamp(u - beta[t, r], min=0.0)
            new = torch.prod(sgn, dim=2, keepdim=True) * sgn * out
            v = x + new
            if clip is not None:
                v = v.clamp(-clip, clip)
            nxt = lq.clone()
            nxt[:, flat] = v.reshape(batch, -1)
            lq = nxt
            msgs[r] = new
        per_iter.append(lq.clone())
    return lq, per_iter


def bce_loss(llr: torch.Tensor, target: torch.Tensor, B: int) -> torch.Tensor:
    """BCEWithLogits(-LLR[:, :B], target), mean (deep_learning/ldpc_model_trainer.py:141-147)."""
    return torch.nn.functional.binary_cross_entropy_with_logits(-llr[:, :B], target)
