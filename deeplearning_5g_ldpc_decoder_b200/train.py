"""Differentiable unrolled layered float min-sum for learning alpha / beta.

``NeuralLayeredMinSumDecoder`` mirrors the reference's
``CTableNeuralLayeredMinSumDecoder`` (deep_learning/deeplearning_ldpc_model.py:72-410):
same constructor arguments, parameter names (``raw_alpha``, ``raw_beta``),
alpha sharing modes (single / checkpoint / degree, sigmoid-bounded to
[alpha_min, alpha_max]), sigmoid-bounded beta per [iteration, row], optional
LLR clipping and detached check-update inputs, and the same forward outputs.
The decoder itself runs in two hand-written CUDA kernels wrapped in
``MinSumUnrolled`` (a ``torch.autograd.Function``): the forward keeps one
checkpoint of the decoder state per iteration and the backward recomputes each
iteration from its checkpoint while back-propagating, instead of storing every
intermediate tensor.

``export_int16_tables`` turns learned alpha / beta into the int16 tables of the
fixed-point decoders (algo 2: per [iteration, row]; algo 3: per degree).
"""

from __future__ import annotations

import ctypes
from typing import Optional, Sequence, Tuple, Union

import numpy as np
import torch
import torch.nn as nn

from . import capi

INF_CLIP = 0.0   # "no clipping" at the C ABI


def _cfg(config) -> capi.LdpcInConfig:
    if isinstance(config, capi.LdpcInConfig):
        return config
    return capi.make_in_config(*config)


def _vp(t: Optional[torch.Tensor]) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def checkpoint_sizes(cfg: capi.LdpcInConfig, T: int, batch: int, f64: bool) -> Tuple[int, int]:
    """(reals of the LQ checkpoints, uint32 words of the message checkpoints)."""
    lib = capi.load_library()
    lq, msg = ctypes.c_int64(0), ctypes.c_int64(0)
    rc = lib.nrldpc_train_checkpoint_words(ctypes.byref(cfg), T, batch, int(f64), ctypes.byref(lq), ctypes.byref(msg))
    if rc != 0:
        raise ValueError(f"configuration not supported by the training kernels ({'float64' if f64 else 'float32'}): {rc}")
    return int(lq.value), int(msg.value)


class MinSumUnrolled(torch.autograd.Function):
    """(llr [batch, n], alpha [T, R], beta [T, R]) -> (final [batch, n], per-iteration [T, batch, n]).

    Runs in the dtype of ``llr``: float32 (training) or float64 (gradient checks)."""

    @staticmethod
    def forward(ctx, llr, alpha_tab, beta_tab, config, clip, detach, want_iters):
        lib = capi.load_library()
        cfg = _cfg(config)
        f64 = llr.dtype == torch.float64
        dt = torch.float64 if f64 else torch.float32
        llr = llr.contiguous().to(dt)
        alpha_tab = alpha_tab.contiguous().to(dt)
        beta_tab = beta_tab.contiguous().to(dt)
        T, R = alpha_tab.shape
        batch, n = llr.shape
        if beta_tab.shape != (T, R):
            raise ValueError("alpha and beta tables must both be [iterations, rows]")
        dev = llr.device
        lq_elems, msg_words = checkpoint_sizes(cfg, T, batch, f64)
        final = torch.empty_like(llr)
        iters = torch.empty((T, batch, n), dtype=dt, device=dev) if want_iters else None
        ck_lq = torch.empty(lq_elems, dtype=dt, device=dev)
        ck_lr = torch.empty(max(msg_words, 2), dtype=torch.int32, device=dev)
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        fn = lib.nrldpc_train_forward_f64 if f64 else lib.nrldpc_train_forward
        clip_arg = (ctypes.c_double if f64 else ctypes.c_float)(clip or INF_CLIP)
        with torch.cuda.device(dev):
            rc = fn(_vp(llr), batch, ctypes.byref(cfg), T, _vp(alpha_tab), _vp(beta_tab), clip_arg, _vp(final),
                    _vp(iters), _vp(ck_lq), _vp(ck_lr), stream)
        if rc != 0:
            raise RuntimeError(f"nrldpc_train_forward failed: {rc}")
        ctx.save_for_backward(llr, alpha_tab, beta_tab, ck_lq, ck_lr)
        ctx.cfg = (cfg.bgn, cfg.A, cfg.crctype, cfg.E, cfg.rv, cfg.Qm, cfg.HARQ_on)
        ctx.clip = clip
        ctx.detach = detach
        if iters is None:
            iters = torch.empty((0,), dtype=dt, device=dev)
            ctx.mark_non_differentiable(iters)
        return final, iters

    @staticmethod
    def backward(ctx, g_final, g_iters):
        lib = capi.load_library()
        llr, alpha_tab, beta_tab, ck_lq, ck_lr = ctx.saved_tensors
        cfg = _cfg(ctx.cfg)
        f64 = llr.dtype == torch.float64
        T, R = alpha_tab.shape
        batch, n = llr.shape
        dev = llr.device
        g_llr = torch.empty_like(llr)
        g_alpha = torch.zeros_like(alpha_tab)
        g_beta = torch.zeros_like(beta_tab)
        gf = g_final.contiguous().to(llr.dtype) if g_final is not None else None
        gi = (g_iters.contiguous().to(llr.dtype)
              if (g_iters is not None and g_iters.numel() == T * batch * n) else None)
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        fn = lib.nrldpc_train_backward_f64 if f64 else lib.nrldpc_train_backward
        clip_arg = (ctypes.c_double if f64 else ctypes.c_float)(ctx.clip or INF_CLIP)
        with torch.cuda.device(dev):
            rc = fn(_vp(llr), batch, ctypes.byref(cfg), T, _vp(alpha_tab), _vp(beta_tab), clip_arg, int(ctx.detach),
                    _vp(ck_lq), _vp(ck_lr), _vp(gf), _vp(gi), _vp(g_llr), _vp(g_alpha), _vp(g_beta), stream)
        if rc != 0:
            raise RuntimeError(f"nrldpc_train_backward failed: {rc}")
        return g_llr, g_alpha, g_beta, None, None, None, None


def _inverse_bounded_sigmoid(values, lo: float, hi: float) -> torch.Tensor:
    v = torch.as_tensor(values, dtype=torch.float32)
    if bool(torch.any(v <= lo)) or bool(torch.any(v >= hi)):
        raise ValueError(f"bounded sigmoid values must satisfy {lo} < value < {hi}")
    x = ((v - lo) / (hi - lo)).clamp(1e-6, 1.0 - 1e-6)
    return torch.log(x / (1.0 - x))


def _inverse_sigmoid(value: float) -> torch.Tensor:
    v = torch.tensor(float(value)).clamp(1e-6, 1.0 - 1e-6)
    return torch.log(v / (1.0 - v))


class NeuralLayeredMinSumDecoder(nn.Module):
    """Trainable unrolled layered min-sum on the B200 kernels (see module docstring)."""

    def __init__(self, config, num_iterations: int = 8, learnable_scaling: bool = True,
                 learnable_beta: bool = True, init_alpha: Union[float, Sequence, torch.Tensor] = 0.75,
                 init_beta: float = 0.0, alpha_mode: str = "single", alpha_min: float = 0.5,
                 alpha_max: float = 1.0 - 1e-6, init_alpha_degree_values: Optional[Sequence[float]] = None,
                 clip_llr: Optional[float] = None, detach_check_update_inputs: bool = False):
        super().__init__()
        if alpha_mode not in {"single", "checkpoint", "degree"}:
            raise ValueError("alpha_mode must be 'single', 'checkpoint', or 'degree'")
        if not 0.0 < alpha_min < alpha_max < 1.0:
            raise ValueError("alpha_min and alpha_max must satisfy 0 < alpha_min < alpha_max < 1")
        self.in_config = tuple(int(v) for v in (config if not isinstance(config, capi.LdpcInConfig) else (
            config.bgn, config.A, config.crctype, config.E, config.rv, config.Qm, config.HARQ_on)))
        if len(self.in_config) == 6:
            self.in_config = self.in_config + (0,)
        p = capi.gen_ldpc_parameters(capi.make_in_config(*self.in_config))
        self.bgn, self.Zc, self.B, self.K, self.N = p.bgn, p.Zc, p.B, p.K, p.N
        self.n = p.N + 2 * p.Zc
        self.num_rows = capi.BG_ROWS[p.bgn]
        offs = [p.HBG_offset_array[i] for i in range(self.num_rows + 1)]
        self.row_degrees = [offs[r + 1] - offs[r] for r in range(self.num_rows)]
        self.num_iterations = int(num_iterations)
        self.clip_llr = clip_llr
        self.detach_check_update_inputs = bool(detach_check_update_inputs)
        self.alpha_mode = alpha_mode
        self.alpha_min, self.alpha_max = float(alpha_min), float(alpha_max)
        self.unique_row_degrees = tuple(sorted(set(self.row_degrees)))
        idx = {d: i for i, d in enumerate(self.unique_row_degrees)}
        self.register_buffer("row_alpha_degree_indices",
                             torch.tensor([idx[d] for d in self.row_degrees], dtype=torch.long))
        raw_alpha = self._make_raw_alpha(init_alpha, init_alpha_degree_values)
        raw_beta = _inverse_sigmoid(init_beta).repeat(self.num_iterations, self.num_rows)
        if learnable_scaling:
            self.raw_alpha = nn.Parameter(raw_alpha)
        else:
            self.register_buffer("raw_alpha", raw_alpha)
        if learnable_beta:
            self.raw_beta = nn.Parameter(raw_beta)
        else:
            self.register_buffer("raw_beta", raw_beta)

    def _make_raw_alpha(self, init_alpha, init_alpha_degree_values):
        lo, hi = self.alpha_min, self.alpha_max
        if self.alpha_mode == "single":
            if not isinstance(init_alpha, (int, float)):
                t = torch.as_tensor(init_alpha, dtype=torch.float32)
                if tuple(t.shape) != (1,):
                    raise ValueError("single-mode init_alpha table must have shape (1,)")
                return _inverse_bounded_sigmoid(t, lo, hi)
            return _inverse_bounded_sigmoid(float(init_alpha), lo, hi).reshape(1)
        if self.alpha_mode == "checkpoint":
            shape = (self.num_iterations, self.num_rows)
            if isinstance(init_alpha, (int, float)):
                return _inverse_bounded_sigmoid(float(init_alpha), lo, hi).expand(shape).clone()
            t = torch.as_tensor(init_alpha, dtype=torch.float32)
            if tuple(t.shape) != shape:
                raise ValueError(f"checkpoint-mode init_alpha must have shape {shape}")
            return _inverse_bounded_sigmoid(t, lo, hi)
        nd = len(self.unique_row_degrees)
        if init_alpha_degree_values is not None:
            t = torch.as_tensor(init_alpha_degree_values, dtype=torch.float32)
            if t.numel() == nd:
                sel = t
            elif t.numel() >= max(self.unique_row_degrees):
                sel = torch.stack([t[d - 1] for d in self.unique_row_degrees])
            else:
                raise ValueError("init_alpha_degree_values: one value per unique degree or a 1-based degree table")
            return _inverse_bounded_sigmoid(sel, lo, hi)
        if isinstance(init_alpha, (int, float)):
            return _inverse_bounded_sigmoid(float(init_alpha), lo, hi).repeat(nd)
        t = torch.as_tensor(init_alpha, dtype=torch.float32)
        if tuple(t.shape) != (nd,):
            raise ValueError(f"degree-mode init_alpha must have shape ({nd},)")
        return _inverse_bounded_sigmoid(t, lo, hi)

    def alpha(self) -> torch.Tensor:
        a = self.alpha_min + (self.alpha_max - self.alpha_min) * torch.sigmoid(self.raw_alpha)
        return a.clamp(min=self.alpha_min, max=self.alpha_max)

    def beta(self) -> torch.Tensor:
        return torch.sigmoid(self.raw_beta).clamp(min=0.0, max=1.0 - 1e-6)

    def alpha_table(self) -> torch.Tensor:
        """Alpha per [iteration, row]."""
        a = self.alpha()
        T, R = self.num_iterations, self.num_rows
        if self.alpha_mode == "single":
            return a.reshape(1, 1).expand(T, R)
        if self.alpha_mode == "checkpoint":
            return a
        return a[self.row_alpha_degree_indices].reshape(1, R).expand(T, R)

    def forward(self, llr: torch.Tensor, return_llr: bool = False, return_iteration_llrs: bool = False):
        single = llr.dim() == 1
        if single:
            llr = llr.unsqueeze(0)
        if llr.dim() != 2 or llr.shape[1] != self.n:
            raise ValueError(f"llr must have shape [batch, {self.n}]")
        final, iters = MinSumUnrolled.apply(llr, self.alpha_table(), self.beta(), self.in_config, self.clip_llr,
                                            self.detach_check_update_inputs, bool(return_iteration_llrs))
        bits = (final < 0).to(torch.int64)
        iteration_llrs = list(iters.unbind(0)) if return_iteration_llrs else None
        if single:
            bits, final = bits.squeeze(0), final.squeeze(0)
            if iteration_llrs is not None:
                iteration_llrs = [x.squeeze(0) for x in iteration_llrs]
        if return_llr and return_iteration_llrs:
            return bits, final, iteration_llrs
        if return_llr:
            return bits, final
        if return_iteration_llrs:
            return bits, iteration_llrs
        return bits

    def trainable_parameters(self):
        """Names and shapes of the trainable parameters."""
        return [(name, tuple(p.shape)) for name, p in self.named_parameters() if p.requires_grad]

    def alpha_parameter_shape(self) -> Tuple[int, ...]:
        return tuple(self.raw_alpha.shape)

    def memory_summary(self, batch_size: int, dtype_bytes: int = 4) -> dict:
        """Decoder state per batch in MB (reference convention: LQ + one message per
        edge), plus what the training kernels keep: one checkpoint of LQ and of the
        compressed messages (4 words per lifted row) per iteration."""
        lq = batch_size * self.n
        lr = batch_size * sum(self.row_degrees) * self.Zc
        ck = self.num_iterations * batch_size * (self.n + 4 * self.num_rows * self.Zc)
        mb = 1024.0 * 1024.0
        return {"LQ_MB": lq * dtype_bytes / mb, "Lr_MB": lr * dtype_bytes / mb,
                "total_message_MB": (lq + lr) * dtype_bytes / mb, "checkpoint_MB": ck * 4 / mb}


# Default algo-3 table, Q15 per exact degree 1..19
# (c_lib/degree_fixedpoint_ldpc_decoder.c:23-43: <=4 -> 26623, 5..8 -> 24575, >8 -> 22527).
DEFAULT_DEGREE_ALPHA = np.array([26623] * 4 + [24575] * 4 + [22527] * 11, dtype=np.int16)


def _q(x: np.ndarray, scale: float) -> np.ndarray:
    return np.clip(np.rint(x * scale), -32768, 32767).astype(np.int16)


def export_int16_tables(model: NeuralLayeredMinSumDecoder, beta_scale: float = 128.0) -> Tuple[np.ndarray, np.ndarray]:
    """Learned alpha / beta -> algo-2 tables [iterations, rows] int16.

    alpha: Q15, round(alpha * 32767) (c_lib/BG1_trained_ldpc_weights.c:11-14).
    beta: subtracted from int16 LLR magnitudes by the fixed-point decoder, so the
    default scale is the LLR quantisation step, round(beta * 128) (the scale the
    float decoder maps int16 beta with, c_lib/floatpoint_ldpc_decoder.c:319);
    pass beta_scale=32767 for the Q15 form the weights file's header describes."""
    with torch.no_grad():
        a = model.alpha_table().detach().cpu().double().numpy()
        b = model.beta().detach().cpu().double().numpy()
    return _q(a, 32767.0), _q(b, beta_scale)


def export_degree_alpha_table(model: NeuralLayeredMinSumDecoder) -> np.ndarray:
    """Degree-mode alpha -> the 19-entry algo-3 table (Q15, entry d-1 for degree d);
    degrees the base graph does not have keep the default values."""
    if model.alpha_mode != "degree":
        raise ValueError("export_degree_alpha_table needs alpha_mode='degree'")
    with torch.no_grad():
        a = model.alpha().detach().cpu().double().numpy()
    tab = DEFAULT_DEGREE_ALPHA.copy()
    for i, d in enumerate(model.unique_row_degrees):
        tab[d - 1] = _q(a[i : i + 1], 32767.0)[0]
    return tab


def install_learned_tables(model: NeuralLayeredMinSumDecoder, beta_scale: float = 128.0) -> None:
    """Install the exported tables into the fixed-point decoders: algo 2 for the
    model's base graph and, in degree mode, the algo-3 degree table."""
    from .decoder import set_degree_alpha, set_trained_weights

    alpha, beta = export_int16_tables(model, beta_scale)
    set_trained_weights(model.bgn, alpha, beta)
    if model.alpha_mode == "degree":
        set_degree_alpha(export_degree_alpha_table(model))


def recovered_llrs(llr_int16: torch.Tensor, config, fill: Optional[int] = None) -> torch.Tensor:
    """Rate-matched int16 LLRs [batch, E] -> decoder-layout float LLRs
    [batch, N+2Zc] (int16 / 128), through the device rate recovery.

    fill=None sets filler positions [B, K) to 10 x max |channel LLR| per block,
    as the training data path does (py5gphy/ldpc/nr_ldpc_raterecover.py:55-57);
    an int uses that int16 value (the C path's filling_bit_value)."""
    from .decoder import code_params, ldpc_decode

    res = ldpc_decode(llr_int16, config, [4, 0, 0, 0, 0 if fill is None else int(fill), 32767, -32767],
                      return_app=True)
    app = res.app
    if fill is None:
        p = code_params(config)
        if p.K > p.B:
            big = llr_int16.abs().amax(dim=1, keepdim=True).float() * (10.0 / 128.0)
            app[:, p.B : p.K] = big.expand(-1, p.K - p.B)
    return app


def ebn0_to_noise_power_db(ebn0_db: float, Qm: int, B: int, E: int) -> float:
    """Noise power (dB, unit-energy symbols) for an Eb/N0 with Eb the energy per
    information+CRC bit: Es/N0 = Eb/N0 + 10 log10(Qm B / E)."""
    return -(float(ebn0_db) + 10.0 * float(np.log10(Qm * B / E)))


# TS 38.212 5.1 generator polynomials (without the leading term), by the C ABI's
# crctype: 0 CRC16, 1 CRC24A, 2 CRC24B, 3 CRC24C.
_CRC_POLY = {0: (16, 0x1021), 1: (24, 0x864CFB), 2: (24, 0x800063), 3: (24, 0xB2B117)}
_crc_tables = {}


def _crc_bit_table(A: int, crctype: int) -> np.ndarray:
    """[A, L] 0/1: CRC bits contributed by a single 1 at message position i,
    x^(A-1-i) * x^L mod g(x) (the CRC is linear with a zero initial value)."""
    key = (A, crctype)
    if key not in _crc_tables:
        L, poly = _CRC_POLY[crctype]
        top, mask = 1 << L, (1 << L) - 1
        rem = np.zeros(A, dtype=np.int64)
        r = poly
        for i in range(A - 1, -1, -1):
            rem[i] = r
            r <<= 1
            if r & top:
                r = (r ^ poly) & mask
        _crc_tables[key] = ((rem[:, None] >> (L - 1 - np.arange(L))[None, :]) & 1).astype(np.float32)
    return _crc_tables[key]


def crc_bits(bits: torch.Tensor, crctype: int) -> torch.Tensor:
    """CRC (MSB first) of each row of a [batch, A] 0/1 tensor, computed on its device
    as parities of a matrix product (counts < 2^24, exact in fp32)."""
    tab = torch.from_numpy(_crc_bit_table(bits.shape[1], crctype)).to(bits.device)
    counts = bits.to(torch.float32) @ tab
    return (counts.to(torch.int64) & 1).to(bits.dtype)


def make_training_batch(model: NeuralLayeredMinSumDecoder, batch_size: int, noise_power_db: float,
                        seed: int, device=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """One training batch generated on the device: seeded payloads -> device LDPC
    encoder and rate matching -> QAM + AWGN + max-log LLRs -> int16 -> device rate
    recovery -> decoder-layout float LLRs.  Returns (llr [batch, n] float32,
    target [batch, B] float32 information+CRC bits), the contract of
    make_c_table_training_batch (deep_learning/ldpc_training_data.py:24-79)."""
    from .decoder import channel_llrs, code_params, ldpc_encode

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    bgn, A, crctype, E, rv, Qm, _ = model.in_config
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    nbytes = (A + 7) // 8
    pay = torch.randint(0, 256, (batch_size, nbytes), dtype=torch.uint8, device=dev, generator=gen)
    if A % 8:
        pay[:, -1] &= (0xFF << (8 - A % 8)) & 0xFF
    rm = ldpc_encode(pay, model.in_config)
    llr16 = channel_llrs(rm, E, Qm, noise_power_db, seed=int(seed))
    llr = recovered_llrs(llr16, model.in_config)
    bits = torch.stack([(pay >> (7 - k)) & 1 for k in range(8)], dim=2).reshape(batch_size, -1)[:, :A]
    target = torch.cat([bits, crc_bits(bits, crctype)], dim=1).to(torch.float32)
    return llr, target


def decoder_loss(llr: torch.Tensor, target: torch.Tensor, B: int, loss_type: str = "bce",
                 llr_margin: float = 5.0) -> torch.Tensor:
    """Supervised loss on the information+CRC bits
    (deep_learning/ldpc_model_trainer.py:141-150): BCEWithLogits(-LLR[:, :B]) or
    softplus(margin - signed LLR)."""
    if loss_type == "bce":
        return torch.nn.functional.binary_cross_entropy_with_logits(-llr[:, :B], target)
    signed = (1.0 - 2.0 * target) * llr[:, :B]
    return torch.nn.functional.softplus(llr_margin - signed).mean()


def train_learned_minsum(config, num_iterations: int = 8, epochs: int = 50, batch_size: int = 4096,
                         lr: float = 1e-2, noise_power_db: Optional[float] = None,
                         ebn0_db_range: Optional[Tuple[float, float]] = (0.0, 3.0),
                         loss_type: str = "bce", llr_margin: float = 5.0, intermediate_loss_weight: float = 0.0,
                         intermediate_loss_stride: int = 4, seed: int = 0, verbose: bool = False, **model_kwargs):
    """Adam + cosine-annealed training of alpha / beta on device-generated batches,
    with gradient-norm clipping at 1.0, intermediate-iteration supervision and
    best-state tracking (deep_learning/ldpc_model_trainer.py:49-321).  One noise
    level per batch: uniform Eb/N0 in ebn0_db_range, or a fixed noise_power_db.
    Returns (model restored to its best state, best state dict, best loss)."""
    if intermediate_loss_weight < 0 or intermediate_loss_stride <= 0:
        raise ValueError("intermediate_loss_weight must be >= 0 and intermediate_loss_stride > 0")
    if loss_type not in ("bce", "margin"):
        raise ValueError("loss_type must be 'bce' or 'margin'")
    model = NeuralLayeredMinSumDecoder(config, num_iterations=num_iterations, **model_kwargs).cuda()
    opt = torch.optim.Adam(model.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs, eta_min=lr * 0.05)
    rng = np.random.default_rng(seed)
    best_loss, best_state = float("inf"), None
    bgn, A, crctype, E, rv, Qm, _ = model.in_config
    for epoch in range(epochs):
        if noise_power_db is not None:
            npdb = float(noise_power_db)
        else:
            npdb = ebn0_to_noise_power_db(rng.uniform(*ebn0_db_range), Qm, model.B, E)
        llr, target = make_training_batch(model, batch_size, npdb, seed=seed * 1000003 + epoch)
        opt.zero_grad(set_to_none=True)
        want_iters = intermediate_loss_weight > 0
        out = model(llr, return_llr=True, return_iteration_llrs=want_iters)
        final = out[1]
        loss = decoder_loss(final, target, model.B, loss_type, llr_margin)
        if want_iters:
            sup = out[2][intermediate_loss_stride - 1 :: intermediate_loss_stride]
            if sup and len(out[2]) % intermediate_loss_stride == 0:
                sup = sup[:-1]   # the final iteration is already the main term
            if sup:
                loss = loss + intermediate_loss_weight * torch.stack(
                    [decoder_loss(x, target, model.B, loss_type, llr_margin) for x in sup]).mean()
        if not torch.isfinite(loss):
            raise FloatingPointError("non-finite training loss")
        loss.backward()
        torch.nn.utils.clip_grad_norm_(model.parameters(), max_norm=1.0)
        opt.step()
        sched.step()
        lv = float(loss.detach())
        if lv < best_loss:
            best_loss = lv
            best_state = {k: v.detach().cpu().clone() for k, v in model.state_dict().items()}
        if verbose:
            print(f"epoch {epoch + 1}/{epochs} noise_power_db={npdb:.2f} loss={lv:.6f}")
    if best_state is not None:
        model.load_state_dict(best_state)
    return model, best_state, best_loss
