"""CPU checks of the training path's checker and host logic.

* The torch restatement of the reference's unrolled min-sum model
  (oracle/minsum_torch.py) reproduces the vectors the reference model produced
  (tests/golden/train_vectors.npz, tests/golden/make_train_golden.py): forward
  bit-exact, gradients to float32 summation-order tolerance.
* The host side of NeuralLayeredMinSumDecoder (parameter mapping, alpha tables
  per mode, int16 export, CRC targets) without launching a kernel.
"""

import os

import numpy as np
import pytest
import torch

from tests.conftest import REPO

TRAIN_GOLDEN = os.path.join(REPO, "tests", "golden", "train_vectors.npz")
CASES = ["bg2_checkpoint", "bg2_degree_clip_detach", "bg1_single_clip"]


@pytest.fixture(scope="module")
def tg():
    return np.load(TRAIN_GOLDEN)


def case(tg, name):
    bgn, A, crc, E, Qm, T, batch, det = (int(v) for v in tg[name + "/config"])
    clip = float(tg[name + "/clip"][0]) or None
    return dict(bgn=bgn, A=A, crc=crc, E=E, Qm=Qm, T=T, batch=batch, detach=bool(det), clip=clip,
                mode=str(tg[name + "/mode"]), w=float(tg[name + "/inter_weight"][0]))


def alpha_table(mode, alpha, degrees, T):
    R = len(degrees)
    if mode == "single":
        return alpha.reshape(1, 1).expand(T, R)
    if mode == "checkpoint":
        return alpha
    uniq = sorted(set(degrees))
    return torch.stack([alpha[uniq.index(d)] for d in degrees]).reshape(1, R).expand(T, R)


def grad_close(got, want, rtol=2e-4):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    scale = max(np.abs(want).max(), 1e-30)
    err = np.abs(got - want).max() / scale
    assert err < rtol, f"max abs diff {err:.3e} of max |grad|"


@pytest.mark.parametrize("name", CASES)
def test_restatement_matches_reference_model(tg, oracle, name):
    from oracle.minsum_torch import MinSumGraph, bce_loss, minsum_unrolled

    c = case(tg, name)
    g = MinSumGraph(c["bgn"], c["A"], c["crc"], c["E"], 0, c["Qm"], oracle=oracle)
    raw_a = torch.tensor(tg[name + "/raw_alpha"], requires_grad=True)
    raw_b = torch.tensor(tg[name + "/raw_beta"], requires_grad=True)
    lo, hi = 0.5, 1.0 - 1e-6
    alpha = (lo + (hi - lo) * torch.sigmoid(raw_a)).clamp(lo, hi)
    beta = torch.sigmoid(raw_b).clamp(0.0, 1.0 - 1e-6)
    assert torch.equal(alpha.detach(), torch.tensor(tg[name + "/alpha"]))
    x = torch.tensor(tg[name + "/llr"], requires_grad=True)
    final, its = minsum_unrolled(g, x, alpha_table(c["mode"], alpha, g.degrees, c["T"]), beta, c["clip"],
                                 c["detach"])
    assert torch.equal(final.detach(), torch.tensor(tg[name + "/final"]))
    for t, it in enumerate(its):
        assert torch.equal(it.detach(), torch.tensor(tg[name + "/iters"][t]))
    tgt = torch.tensor(tg[name + "/target"])
    loss = bce_loss(final, tgt, g.B)
    if c["w"] > 0 and c["T"] > 1:
        loss = loss + c["w"] * torch.stack([bce_loss(i, tgt, g.B) for i in its[:-1]]).mean()
    assert abs(loss.item() - float(tg[name + "/loss"][0])) < 1e-6
    loss.backward()
    grad_close(raw_a.grad, tg[name + "/g_raw_alpha"])
    grad_close(raw_b.grad, tg[name + "/g_raw_beta"])
    grad_close(x.grad, tg[name + "/g_llr"])


@pytest.mark.parametrize("name", CASES)
def test_module_parameter_mapping(tg, name):
    from deeplearning_5g_ldpc_decoder_b200.train import NeuralLayeredMinSumDecoder

    c = case(tg, name)
    m = NeuralLayeredMinSumDecoder((c["bgn"], c["A"], c["crc"], c["E"], 0, c["Qm"], 0), num_iterations=c["T"],
                                   alpha_mode=c["mode"], clip_llr=c["clip"], detach_check_update_inputs=c["detach"],
                                   init_beta=0.02)
    assert tuple(m.raw_alpha.shape) == tg[name + "/raw_alpha"].shape
    assert tuple(m.raw_beta.shape) == tg[name + "/raw_beta"].shape
    assert m.n == tg[name + "/llr"].shape[1]
    with torch.no_grad():
        m.raw_alpha.copy_(torch.tensor(tg[name + "/raw_alpha"]))
        m.raw_beta.copy_(torch.tensor(tg[name + "/raw_beta"]))
    assert torch.equal(m.alpha().detach(), torch.tensor(tg[name + "/alpha"]))
    assert torch.equal(m.beta().detach(), torch.tensor(tg[name + "/beta"]))
    tab = m.alpha_table().detach()
    assert tab.shape == (c["T"], m.num_rows)
    want = alpha_table(c["mode"], torch.tensor(tg[name + "/alpha"]), m.row_degrees, c["T"])
    assert torch.equal(tab, want)


def test_module_validation_and_init():
    from deeplearning_5g_ldpc_decoder_b200.train import NeuralLayeredMinSumDecoder

    cfg = (2, 488, 1, 1920, 0, 2, 0)
    with pytest.raises(ValueError):
        NeuralLayeredMinSumDecoder(cfg, alpha_mode="row")
    with pytest.raises(ValueError):
        NeuralLayeredMinSumDecoder(cfg, alpha_min=0.9, alpha_max=0.5)
    with pytest.raises(ValueError):
        NeuralLayeredMinSumDecoder(cfg, init_alpha=0.4)           # below alpha_min
    with pytest.raises(ValueError):
        NeuralLayeredMinSumDecoder(cfg, alpha_mode="checkpoint", init_alpha=np.full((3, 3), 0.7))
    m = NeuralLayeredMinSumDecoder(cfg, num_iterations=4, alpha_mode="degree",
                                   init_alpha_degree_values=[0.8] * 4 + [0.75] * 4 + [0.7] * 11)
    assert m.unique_row_degrees == tuple(sorted(set(m.row_degrees)))
    a = m.alpha().detach().numpy()
    for i, d in enumerate(m.unique_row_degrees):
        assert abs(a[i] - (0.8 if d <= 4 else (0.75 if d <= 8 else 0.7))) < 1e-5
    m2 = NeuralLayeredMinSumDecoder(cfg, learnable_scaling=False, learnable_beta=False)
    assert m2.trainable_parameters() == []
    assert "checkpoint_MB" in m2.memory_summary(16)


def test_int16_export():
    from deeplearning_5g_ldpc_decoder_b200.train import (DEFAULT_DEGREE_ALPHA, NeuralLayeredMinSumDecoder,
                                                         export_degree_alpha_table, export_int16_tables)

    cfg = (2, 488, 1, 1920, 0, 2, 0)
    m = NeuralLayeredMinSumDecoder(cfg, num_iterations=5, alpha_mode="checkpoint", init_beta=0.1)
    with torch.no_grad():
        m.raw_alpha.add_(torch.linspace(-1, 1, m.raw_alpha.numel()).reshape(m.raw_alpha.shape))
    a, b = export_int16_tables(m)
    assert a.dtype == np.int16 and a.shape == (5, m.num_rows) and b.shape == a.shape
    want = np.rint(m.alpha_table().detach().double().numpy() * 32767.0)
    assert np.array_equal(a, want.astype(np.int16))
    assert np.all(b == np.int16(round(0.1 * 128)))
    _, bq = export_int16_tables(m, beta_scale=32767.0)
    assert np.all(np.abs(bq.astype(np.int64) - round(0.1 * 32767)) <= 1)
    with pytest.raises(ValueError):
        export_degree_alpha_table(m)
    md = NeuralLayeredMinSumDecoder(cfg, num_iterations=5, alpha_mode="degree", init_alpha=0.66)
    tab = export_degree_alpha_table(md)
    assert tab.shape == (19,)
    for d in range(1, 20):
        assert tab[d - 1] == (round(0.66 * 32767) if d in md.unique_row_degrees else DEFAULT_DEGREE_ALPHA[d - 1])


@pytest.mark.parametrize("bgn,A,crc,E", [(2, 488, 1, 1920), (1, 2440, 1, 7392), (2, 200, 0, 600),
                                         (1, 4000, 2, 12000), (2, 1000, 3, 3000)])
def test_crc_targets_match_encoder(oracle, bgn, A, crc, E):
    from oracle.oracle import in_config

    from deeplearning_5g_ldpc_decoder_b200.train import crc_bits

    cfg = in_config(bgn, A, crc, E, 0, 2)
    _, p = oracle.derive(cfg)
    rng = np.random.default_rng(A)
    pays = rng.integers(0, 256, (4, A // 8), dtype=np.uint8)
    bits = torch.from_numpy(np.unpackbits(pays, axis=1)[:, :A].astype(np.int64))
    t = torch.cat([bits, crc_bits(bits, crc)], 1).numpy()
    for i in range(4):
        assert np.array_equal(t[i], oracle.encode_codeword(pays[i], cfg)[: p.B])


def test_training_checkpoint_sizes_and_float64_fit():
    """One code block of every configuration fits in shared memory, float64
    included (BG1 Zc384: 26112 doubles, 209 KB, since the backward keeps LQ and
    dLQ in one array); a configuration the parameter derivation rejects raises
    instead of launching."""
    from deeplearning_5g_ldpc_decoder_b200 import capi
    from deeplearning_5g_ldpc_decoder_b200.train import checkpoint_sizes

    lq, msg = checkpoint_sizes(capi.make_in_config(1, 8424, 1, 25344, 0, 2, 0), 2, 1, True)
    assert lq == 2 * 1 * 68 * 384 and msg == 2 * 1 * 46 * 6 * 384
    with pytest.raises(ValueError):
        checkpoint_sizes(capi.make_in_config(3, 8424, 1, 25344, 0, 2, 0), 2, 1, False)
    lq, msg = checkpoint_sizes(capi.make_in_config(1, 8424, 1, 25344, 0, 2, 0), 2, 3, False)
    assert lq == 2 * 3 * 68 * 384 and msg == 2 * 3 * 46 * 4 * 384
