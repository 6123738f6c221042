"""Generate tests/golden/train_vectors.npz from the REFERENCE PyTorch model.

Runs the reference's ``CTableNeuralLayeredMinSumDecoder``
(deep_learning/deeplearning_ldpc_model.py) imported from the reference tree,
with its table config loaded through the reference C library built by
``oracle/build_ref.sh``.  For each case it records the model's inputs (decoder
layout LLRs, raw alpha / beta), forward outputs (final and per-iteration LLRs)
and the gradients of a BCE loss with intermediate-iteration terms (the
trainer's loss, deep_learning/ldpc_model_trainer.py:141-150 and :216-233) with
respect to raw_alpha, raw_beta and the input LLRs.

Input LLRs: seeded payload -> reference c_ldpc_5g_encode -> reference
tx_rx_process (int16) -> rate recovery (fill 1280) -> /128, the conversion of
deep_learning/ldpc_c_baseline_evaluation.py:157-176.

usage:  oracle/build_ref.sh && python tests/golden/make_train_golden.py
"""

from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
from oracle.refroot import REFERENCE_ROOT as REFERENCE  # noqa: E402

sys.path.insert(0, REFERENCE)

from deep_learning.deeplearning_ldpc_model import CTableNeuralLayeredMinSumDecoder  # noqa: E402
from deep_learning.ldpc_table_config import load_ldpc_table_config  # noqa: E402

from oracle.oracle import REF_SO, Oracle, RefLib, in_config  # noqa: E402

# name: (bgn, A, crctype, E, Qm, noise_db, T, batch, mode, clip, detach, inter_weight, seed)
CASES = {
    "bg2_checkpoint": (2, 488, 1, 1920, 2, 1.0, 3, 3, "checkpoint", None, False, 0.25, 11),
    "bg2_degree_clip_detach": (2, 488, 1, 1920, 2, 1.5, 2, 2, "degree", 12.0, True, 0.0, 12),
    "bg1_single_clip": (1, 2440, 1, 7392, 2, 0.5, 2, 2, "single", 20.0, False, 0.5, 13),
}


def model_inputs(ref: RefLib, orc: Oracle, bgn, A, crctype, E, Qm, noise_db, batch, rng):
    cfg = in_config(bgn, A, crctype, E, 0, Qm)
    _, p = orc.derive(cfg)
    llrs, targets = [], []
    for _ in range(batch):
        payload = rng.integers(0, 256, A // 8, dtype=np.uint8)   # A is a multiple of 8 in every case
        rm = ref.encode(payload, cfg)
        ch = ref.channel(rm, E, Qm, noise_db)
        harq = orc.rate_recover(cfg, 1280, ch)
        llrs.append(harq[: p.N + 2 * p.Zc].astype(np.float32) / 128.0)
        cw = orc.encode_codeword(payload, cfg)
        targets.append(cw[: p.B].astype(np.float32))   # information + CRC bits (systematic part)
    return np.stack(llrs), np.stack(targets)


def main():
    torch.manual_seed(0)
    ref = RefLib()
    orc = Oracle()
    out = {}
    for name, (bgn, A, crctype, E, Qm, noise_db, T, batch, mode, clip, detach, w, seed) in CASES.items():
        rng = np.random.default_rng(seed)
        ref.srand(seed)
        llr, target = model_inputs(ref, orc, bgn, A, crctype, E, Qm, noise_db, batch, rng)
        tc = load_ldpc_table_config(bgn, A, crctype, E, 0, Qm, 0, lib_path=REF_SO)
        kwargs = dict(num_iterations=T, learnable_scaling=True, learnable_beta=True, alpha_mode=mode,
                      clip_llr=clip, detach_check_update_inputs=detach, init_beta=0.02)
        model = CTableNeuralLayeredMinSumDecoder(tc, **kwargs)
        with torch.no_grad():
            model.raw_alpha.add_(torch.from_numpy(rng.normal(0.0, 0.6, tuple(model.raw_alpha.shape))).float())
            model.raw_beta.add_(torch.from_numpy(rng.normal(0.0, 0.8, tuple(model.raw_beta.shape))).float())
        x = torch.from_numpy(llr).requires_grad_(True)
        tgt = torch.from_numpy(target)
        bits, final, iters = model(x, return_llr=True, return_iteration_llrs=True)
        crit = torch.nn.BCEWithLogitsLoss()
        loss = crit(-final[:, : tc.B], tgt)
        if w > 0 and T > 1:
            loss = loss + w * torch.stack([crit(-it[:, : tc.B], tgt) for it in iters[:-1]]).mean()
        loss.backward()
        prefix = name + "/"
        out[prefix + "config"] = np.array([bgn, A, crctype, E, Qm, T, batch, int(detach)], dtype=np.int64)
        out[prefix + "clip"] = np.array([clip if clip is not None else 0.0], dtype=np.float32)
        out[prefix + "mode"] = np.array(mode)
        out[prefix + "inter_weight"] = np.array([w], dtype=np.float32)
        out[prefix + "llr"] = llr
        out[prefix + "target"] = target
        out[prefix + "raw_alpha"] = model.raw_alpha.detach().numpy().copy()
        out[prefix + "raw_beta"] = model.raw_beta.detach().numpy().copy()
        out[prefix + "alpha"] = model.alpha().detach().numpy().copy()
        out[prefix + "beta"] = model.beta().detach().numpy().copy()
        out[prefix + "final"] = final.detach().numpy()
        out[prefix + "iters"] = torch.stack(iters).detach().numpy()
        out[prefix + "bits"] = bits.numpy().astype(np.uint8)
        out[prefix + "loss"] = np.array([loss.item()], dtype=np.float64)
        out[prefix + "g_raw_alpha"] = model.raw_alpha.grad.numpy().copy()
        out[prefix + "g_raw_beta"] = model.raw_beta.grad.numpy().copy()
        out[prefix + "g_llr"] = x.grad.numpy().copy()
        print(name, "loss", loss.item(), "n", llr.shape, "|g_alpha|", float(model.raw_alpha.grad.norm()))
    np.savez_compressed(os.path.join(HERE, "train_vectors.npz"), **out)


if __name__ == "__main__":
    main()
