"""GPU parity of the training kernels (nrldpc_train_forward / nrldpc_train_backward).

* forward bit-exact against the reference model's vectors and, at the
  configurations of the learned min-sum workload (BG2 Zc64 and BG1 Zc112,
  10 unrolled iterations), against the torch restatement of the model;
* gradients against the reference model's vectors, against autograd through the
  restatement, and against central finite differences of the kernel's own
  forward (norm-wise relative error < 1e-3);
* learned parameters exported to the int16 algo-2 / algo-3 tables and decoded
  bit-exactly against the C oracle with the same tables.
"""

import numpy as np
import pytest
import torch

from tests.test_oracle_train import CASES, alpha_table, case, grad_close, tg  # noqa: F401

pytestmark = pytest.mark.gpu

WORKLOADS = {"bg2_zc64": (2, 488, 1, 1920, 0, 2, 0), "bg1_zc112": (1, 2440, 1, 7392, 0, 2, 0)}


def _model(cfg, T, mode, clip=None, detach=False, seed=0, beta=0.03):
    from deeplearning_5g_ldpc_decoder_b200.train import NeuralLayeredMinSumDecoder

    m = NeuralLayeredMinSumDecoder(cfg, num_iterations=T, alpha_mode=mode, clip_llr=clip,
                                   detach_check_update_inputs=detach, init_beta=beta).cuda()
    g = torch.Generator().manual_seed(seed)
    with torch.no_grad():
        m.raw_alpha.add_(torch.randn(m.raw_alpha.shape, generator=g).cuda() * 0.5)
        m.raw_beta.add_(torch.randn(m.raw_beta.shape, generator=g).cuda() * 0.5)
    return m


def _loss(model, llr, target, w=0.25):
    from deeplearning_5g_ldpc_decoder_b200.train import decoder_loss

    _, final, its = model(llr, return_llr=True, return_iteration_llrs=True)
    loss = decoder_loss(final, target, model.B)
    if w > 0 and len(its) > 1:
        loss = loss + w * torch.stack([decoder_loss(x, target, model.B) for x in its[:-1]]).mean()
    return loss


@pytest.mark.parametrize("name", CASES)
def test_kernels_match_reference_model_vectors(cuda, tg, name):  # noqa: F811
    from deeplearning_5g_ldpc_decoder_b200.train import NeuralLayeredMinSumDecoder

    c = case(tg, name)
    m = NeuralLayeredMinSumDecoder((c["bgn"], c["A"], c["crc"], c["E"], 0, c["Qm"], 0), num_iterations=c["T"],
                                   alpha_mode=c["mode"], clip_llr=c["clip"], detach_check_update_inputs=c["detach"],
                                   init_beta=0.02).cuda()
    with torch.no_grad():
        m.raw_alpha.copy_(torch.tensor(tg[name + "/raw_alpha"]))
        m.raw_beta.copy_(torch.tensor(tg[name + "/raw_beta"]))
    x = torch.tensor(tg[name + "/llr"], device=cuda, requires_grad=True)
    tgt = torch.tensor(tg[name + "/target"], device=cuda)
    bits, final, its = m(x, return_llr=True, return_iteration_llrs=True)
    assert torch.equal(final.detach().cpu(), torch.tensor(tg[name + "/final"]))
    assert torch.equal(bits.cpu().to(torch.uint8), torch.tensor(tg[name + "/bits"]))
    for t, it in enumerate(its):
        assert torch.equal(it.detach().cpu(), torch.tensor(tg[name + "/iters"][t]))
    from deeplearning_5g_ldpc_decoder_b200.train import decoder_loss

    loss = decoder_loss(final, tgt, m.B)
    if c["w"] > 0 and c["T"] > 1:
        loss = loss + c["w"] * torch.stack([decoder_loss(i, tgt, m.B) for i in its[:-1]]).mean()
    assert abs(loss.item() - float(tg[name + "/loss"][0])) < 1e-6
    loss.backward()
    grad_close(m.raw_alpha.grad.cpu(), tg[name + "/g_raw_alpha"])
    grad_close(m.raw_beta.grad.cpu(), tg[name + "/g_raw_beta"])
    grad_close(x.grad.cpu(), tg[name + "/g_llr"])


@pytest.mark.parametrize("wl", sorted(WORKLOADS))
@pytest.mark.parametrize("mode,clip,detach", [("checkpoint", None, False), ("degree", 25.0, False),
                                              ("single", None, True)])
def test_kernels_match_restatement_at_workload_sizes(cuda, oracle, wl, mode, clip, detach):
    from oracle.minsum_torch import MinSumGraph, minsum_unrolled

    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS[wl]
    T = 10
    m = _model(cfg, T, mode, clip, detach, seed=3)
    batch = 48 if wl == "bg2_zc64" else 12
    llr, target = make_training_batch(m, batch, ebn0_to_noise_power_db(1.0, 2, m.B, cfg[3]), seed=5)
    x = llr.clone().requires_grad_(True)
    loss = _loss(m, x, target)
    loss.backward()
    g = MinSumGraph(*cfg[:6], oracle=oracle)
    ra = m.raw_alpha.detach().clone().requires_grad_(True)
    rb = m.raw_beta.detach().clone().requires_grad_(True)
    lo, hi = m.alpha_min, m.alpha_max
    a = (lo + (hi - lo) * torch.sigmoid(ra)).clamp(lo, hi)
    b = torch.sigmoid(rb).clamp(0.0, 1.0 - 1e-6)
    x2 = llr.clone().requires_grad_(True)
    fin, its = minsum_unrolled(g, x2, alpha_table(mode, a, g.degrees, T), b, clip, detach)
    _, kfin = m(llr, return_llr=True)
    assert torch.equal(kfin, fin.detach()), "forward differs from the restatement"
    from deeplearning_5g_ldpc_decoder_b200.train import decoder_loss

    ref = decoder_loss(fin, target, m.B) + 0.25 * torch.stack([decoder_loss(i, target, m.B) for i in its[:-1]]).mean()
    assert abs(ref.item() - loss.item()) < 1e-6
    ref.backward()
    grad_close(m.raw_alpha.grad.cpu(), ra.grad.cpu(), rtol=1e-4)
    grad_close(m.raw_beta.grad.cpu(), rb.grad.cpu(), rtol=1e-4)
    grad_close(x.grad.cpu(), x2.grad.cpu(), rtol=1e-4)


def _flat_params(m):
    return torch.cat([m.raw_alpha.detach().reshape(-1), m.raw_beta.detach().reshape(-1)])


def _set_flat(m, v):
    na = m.raw_alpha.numel()
    with torch.no_grad():
        m.raw_alpha.copy_(v[:na].reshape(m.raw_alpha.shape))
        m.raw_beta.copy_(v[na:].reshape(m.raw_beta.shape))


def _loss64(m, llr, target):
    """Loss of the kernel forward, accumulated in float64."""
    with torch.no_grad():
        _, final, its = m(llr, return_llr=True, return_iteration_llrs=True)
        t = target.double()

        def bce(z):
            logits = -z[:, : m.B].double()
            return torch.nn.functional.binary_cross_entropy_with_logits(logits, t)

        return float(bce(final) + 0.25 * torch.stack([bce(i) for i in its[:-1]]).mean())


@pytest.mark.parametrize("wl,mode", [("bg2_zc64", "checkpoint"), ("bg2_zc64", "degree"), ("bg1_zc112", "single")])
def test_gradient_vs_central_finite_differences(cuda, wl, mode):
    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS[wl]
    T = 10
    m = _model(cfg, T, mode, seed=7)
    batch = 16 if wl == "bg2_zc64" else 4
    llr, target = make_training_batch(m, batch, ebn0_to_noise_power_db(1.5, 2, m.B, cfg[3]), seed=9)
    m.zero_grad()
    loss = _loss(m, llr, target)
    loss.backward()
    g = torch.cat([m.raw_alpha.grad.reshape(-1), m.raw_beta.grad.reshape(-1)]).double().cpu()
    p0 = _flat_params(m)
    h = 1e-3
    fd = torch.zeros_like(g)
    for i in range(p0.numel()):
        e = torch.zeros_like(p0)
        e[i] = h
        _set_flat(m, p0 + e)
        fp = _loss64(m, llr, target)
        _set_flat(m, p0 - e)
        fm = _loss64(m, llr, target)
        fd[i] = (fp - fm) / (2 * h)
    _set_flat(m, p0)
    rel = float((fd - g).norm() / g.norm())
    assert rel < 1e-3, f"norm-wise relative error {rel:.3e}"
    # a random direction through all parameters at once
    v = torch.randn(p0.shape, generator=torch.Generator().manual_seed(1)).to(p0.device)
    v = v / v.norm()
    _set_flat(m, p0 + h * v)
    fp = _loss64(m, llr, target)
    _set_flat(m, p0 - h * v)
    fm = _loss64(m, llr, target)
    _set_flat(m, p0)
    dd = (fp - fm) / (2 * h)
    an = float(g @ v.double().cpu())
    assert abs(dd - an) < 1e-3 * abs(an) + 1e-9, (dd, an)


def test_gradient_wrt_llr_finite_differences(cuda):
    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS["bg2_zc64"]
    m = _model(cfg, 6, "checkpoint", seed=11)
    llr, target = make_training_batch(m, 8, ebn0_to_noise_power_db(1.0, 2, m.B, cfg[3]), seed=13)
    x = llr.clone().requires_grad_(True)
    _loss(m, x, target).backward()
    gx = x.grad.double().cpu()
    h = 1e-3
    gen = torch.Generator().manual_seed(2)
    for _ in range(4):
        v = torch.randn(llr.shape, generator=gen).to(llr.device)
        v = v / v.norm()
        fp = _loss64(m, llr + h * v, target)
        fm = _loss64(m, llr - h * v, target)
        dd = (fp - fm) / (2 * h)
        an = float((gx * v.double().cpu()).sum())
        assert abs(dd - an) < 1e-3 * abs(an) + 1e-9, (dd, an)


def test_learned_tables_decode_bit_exact_vs_c(cuda, oracle):
    from oracle.oracle import dec_cfg, in_config

    from deeplearning_5g_ldpc_decoder_b200 import ldpc_decode
    from deeplearning_5g_ldpc_decoder_b200.decoder import channel_llrs, ldpc_encode, set_degree_alpha, \
        set_trained_weights
    from deeplearning_5g_ldpc_decoder_b200.train import (ebn0_to_noise_power_db, export_degree_alpha_table,
                                                         export_int16_tables, install_learned_tables,
                                                         train_learned_minsum)

    cfg = WORKLOADS["bg2_zc64"]
    icfg = in_config(*cfg)
    n = 64
    pay = torch.randint(0, 256, (n, cfg[1] // 8), dtype=torch.uint8, device=cuda,
                        generator=torch.Generator(device=cuda).manual_seed(4))
    llr = channel_llrs(ldpc_encode(pay, cfg), cfg[3], 2, ebn0_to_noise_power_db(1.0, 2, 512, cfg[3]), seed=17)
    llr_h = llr.cpu().numpy()
    try:
        for mode, algo in (("checkpoint", 2), ("degree", 3)):
            model, _, best = train_learned_minsum(cfg, num_iterations=10, epochs=3, batch_size=256, lr=5e-2,
                                                  alpha_mode=mode, learnable_beta=True, init_beta=0.05, seed=1)
            assert np.isfinite(best)
            install_learned_tables(model)
            a, b = export_int16_tables(model)
            oracle.set_trained(2, a, b)
            if mode == "degree":
                oracle.set_degree_alpha(export_degree_alpha_table(model))
            row = [algo, 10, 22936, 3, 1280, 32767, -32767]
            res = ldpc_decode(llr, cfg, row, return_app=True)
            torch.cuda.synchronize()
            hb, st_d, it_d, app = (res.hardbits.cpu().numpy(), res.status.cpu().numpy(),
                                   res.iterations.cpu().numpy(), res.app.cpu().numpy())
            for i in range(n):
                st, bits, it, lq = oracle.decode(llr_h[i], icfg, dec_cfg(row))
                assert st_d[i] == st and it_d[i] == it, (mode, i)
                assert np.array_equal(hb[i], bits), (mode, i)
                assert np.array_equal(app[i], lq), (mode, i)
    finally:
        set_trained_weights(2, None)
        set_degree_alpha(None)
        oracle.set_trained(2, None)
        oracle.set_degree_alpha(None)
