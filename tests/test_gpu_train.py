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
    """Forward bit-exact given the reference's alpha / beta values; gradients of the
    loss with respect to raw_alpha, raw_beta and the LLRs within float32
    summation-order tolerance.  (torch's CUDA sigmoid may differ from its CPU
    sigmoid in the last bit, so the forward check feeds the recorded alpha / beta.)"""
    from deeplearning_5g_ldpc_decoder_b200.train import MinSumUnrolled, NeuralLayeredMinSumDecoder, decoder_loss

    c = case(tg, name)
    cfg = (c["bgn"], c["A"], c["crc"], c["E"], 0, c["Qm"], 0)
    m = NeuralLayeredMinSumDecoder(cfg, num_iterations=c["T"], alpha_mode=c["mode"], clip_llr=c["clip"],
                                   detach_check_update_inputs=c["detach"], init_beta=0.02).cuda()
    x = torch.tensor(tg[name + "/llr"], device=cuda)
    a_tab = alpha_table(c["mode"], torch.tensor(tg[name + "/alpha"]), m.row_degrees, c["T"]).contiguous().cuda()
    b_tab = torch.tensor(tg[name + "/beta"]).cuda()
    final, its = MinSumUnrolled.apply(x, a_tab, b_tab, cfg, c["clip"], c["detach"], True)
    assert torch.equal(final.cpu(), torch.tensor(tg[name + "/final"]))
    assert torch.equal(its.cpu(), torch.tensor(tg[name + "/iters"]))
    assert torch.equal((final < 0).cpu().to(torch.uint8), torch.tensor(tg[name + "/bits"]))

    with torch.no_grad():
        m.raw_alpha.copy_(torch.tensor(tg[name + "/raw_alpha"]))
        m.raw_beta.copy_(torch.tensor(tg[name + "/raw_beta"]))
    xg = x.clone().requires_grad_(True)
    tgt = torch.tensor(tg[name + "/target"], device=cuda)
    _, fin, it_list = m(xg, return_llr=True, return_iteration_llrs=True)
    loss = decoder_loss(fin, tgt, m.B)
    if c["w"] > 0 and c["T"] > 1:
        loss = loss + c["w"] * torch.stack([decoder_loss(i, tgt, m.B) for i in it_list[:-1]]).mean()
    assert abs(loss.item() - float(tg[name + "/loss"][0])) < 1e-5
    loss.backward()
    grad_close(m.raw_alpha.grad.cpu(), tg[name + "/g_raw_alpha"])
    grad_close(m.raw_beta.grad.cpu(), tg[name + "/g_raw_beta"])
    grad_close(xg.grad.cpu(), tg[name + "/g_llr"])


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


def _loss_value(m, llr, target, w=0.25):
    with torch.no_grad():
        return float(_loss(m, llr, target, w))


# Finite differences run on the float64 kernels: the min-sum loss is continuous
# and piecewise smooth, with a kink wherever two check-row minima swap, and in
# float32 the rounding noise at a step small enough to avoid kinks swamps the
# difference quotient.  (The float32 kernels are tied to autograd by the tests
# above.)  Near convergence the pieces are wide and a step of 1e-7 sees one; in
# the low-SNR regime the gradient is large (~1e3) and the pieces narrow, so the
# step is 1e-10 -- the difference quotient converges to the kernel's gradient as
# the step shrinks in both regimes.  The channel LLRs are multiples of 1/128, so
# two magnitudes of a check row are often exactly equal: the loss then has a
# kink AT the evaluation point, where autograd (and the kernels) route the
# gradient to the first minimum and a central difference averages the two
# one-sided slopes.  The checks therefore run at generic points: the LLRs get a
# small continuous jitter.
def _generic(llr, seed):
    g = torch.Generator().manual_seed(seed)
    return llr.double() + 1e-3 * torch.randn(llr.shape, generator=g, dtype=torch.float64).to(llr.device)

@pytest.mark.parametrize("wl,mode,ebn0,h", [("bg2_zc64", "checkpoint", 1.5, 1e-7), ("bg2_zc64", "degree", 2.0, 1e-7),
                                            ("bg1_zc112", "single", 1.5, 1e-7),
                                            ("bg2_zc64", "checkpoint", 0.0, 1e-10),
                                            ("bg2_zc64", "degree", 1.0, 1e-10)])
def test_gradient_vs_central_finite_differences(cuda, wl, mode, ebn0, h):
    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS[wl]
    T = 10
    m = _model(cfg, T, mode, seed=7).double()
    batch = 16 if wl == "bg2_zc64" else 4
    llr, target = make_training_batch(m, batch, ebn0_to_noise_power_db(ebn0, 2, m.B, cfg[3]), seed=9)
    llr, target = _generic(llr, 21), target.double()
    m.zero_grad()
    _loss(m, llr, target).backward()
    g = torch.cat([m.raw_alpha.grad.reshape(-1), m.raw_beta.grad.reshape(-1)]).cpu()
    assert g.dtype == torch.float64 and float(g.norm()) > 0
    p0 = _flat_params(m)
    fd = torch.zeros_like(g)
    for i in range(p0.numel()):
        e = torch.zeros_like(p0)
        e[i] = h
        _set_flat(m, p0 + e)
        fp = _loss_value(m, llr, target)
        _set_flat(m, p0 - e)
        fm = _loss_value(m, llr, target)
        fd[i] = (fp - fm) / (2 * h)
    _set_flat(m, p0)
    rel = float((fd - g).norm() / g.norm())
    assert rel < 1e-3, f"norm-wise relative error {rel:.3e}"
    # a random direction through all parameters at once
    v = torch.randn(p0.shape, generator=torch.Generator().manual_seed(1), dtype=torch.float64).to(p0.device)
    v = v / v.norm()
    _set_flat(m, p0 + h * v)
    fp = _loss_value(m, llr, target)
    _set_flat(m, p0 - h * v)
    fm = _loss_value(m, llr, target)
    _set_flat(m, p0)
    dd = (fp - fm) / (2 * h)
    an = float(g @ v.cpu())
    assert abs(dd - an) < 1e-3 * abs(an), (dd, an)


def test_gradient_wrt_llr_finite_differences(cuda):
    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS["bg2_zc64"]
    m = _model(cfg, 6, "checkpoint", seed=11).double()
    llr, target = make_training_batch(m, 8, ebn0_to_noise_power_db(1.0, 2, m.B, cfg[3]), seed=13)
    llr, target = _generic(llr, 22), target.double()
    x = llr.clone().requires_grad_(True)
    _loss(m, x, target).backward()
    gx = x.grad.cpu()
    h = 1e-7
    gen = torch.Generator().manual_seed(2)
    for _ in range(4):
        v = torch.randn(llr.shape, generator=gen, dtype=torch.float64).to(llr.device)
        v = v / v.norm()
        dd = (_loss_value(m, llr + h * v, target) - _loss_value(m, llr - h * v, target)) / (2 * h)
        an = float((gx * v.cpu()).sum())
        assert abs(dd - an) < 1e-3 * abs(an), (dd, an)


def test_float64_kernels_agree_with_float32_path(cuda):
    """The float64 instantiation computes the same function: forwards agree to
    float32 rounding on a well-conditioned batch."""
    from deeplearning_5g_ldpc_decoder_b200.train import ebn0_to_noise_power_db, make_training_batch

    cfg = WORKLOADS["bg2_zc64"]
    m = _model(cfg, 4, "checkpoint", seed=5)
    llr, _ = make_training_batch(m, 8, ebn0_to_noise_power_db(3.0, 2, m.B, cfg[3]), seed=3)
    _, f32 = m(llr, return_llr=True)
    m64 = _model(cfg, 4, "checkpoint", seed=5).double()
    _, f64 = m64(llr.double(), return_llr=True)
    assert f64.dtype == torch.float64
    err = ((f64 - f32.double()).abs().max() / f64.abs().max()).detach()
    assert float(err) < 1e-4


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
