"""PyTorch-facing API of the B200 LDPC receive path.

PyTorch provides device memory and streams; the work is done by the CUDA
kernels in ``libnrldpc_b200.so``, called through its C ABI with raw device
pointers on the caller's current stream.  There is no CPU fallback: without a
CUDA device or without the library every call raises.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence, Union

import torch

from . import capi
from .capi import DecoderConfig, LdpcInConfig, make_decoder_config, make_in_config


@dataclass
class DecodeResult:
    hardbits: torch.Tensor            # uint8 [n, ceil(B/8)], MSB first
    status: torch.Tensor              # int32 [n]: 0 CRC pass, 1 not converged
    iterations: torch.Tensor          # int32 [n]: iterations executed
    app: Optional[torch.Tensor]       # [n, N+2Zc] final beliefs (int16, or float32 for algos 0/4)


def _as_in_config(cfg: Union[LdpcInConfig, Sequence[int], dict]) -> LdpcInConfig:
    if isinstance(cfg, LdpcInConfig):
        return cfg
    if isinstance(cfg, dict):
        return make_in_config(**cfg)
    return make_in_config(*cfg)


def _as_decoder_config(cfg: Union[DecoderConfig, Sequence[int]]) -> DecoderConfig:
    if isinstance(cfg, DecoderConfig):
        return cfg
    return make_decoder_config(cfg)


def code_params(inconfig) -> capi.LdpcConfig:
    """Derived parameters (B, Zc, K, N, ...) exactly as gen_ldpc_parameters."""
    return capi.gen_ldpc_parameters(_as_in_config(inconfig))


def _row_stride(t: torch.Tensor) -> int:
    """Elements between rows; torch leaves the stride of a size-1 dim arbitrary."""
    return t.stride(0) if t.shape[0] > 1 else t.shape[1]


def _check(rc: int, what: str) -> None:
    if rc == capi.NRLDPC_OK:
        return
    msg = {capi.NRLDPC_ERR_CUDA: "CUDA error", capi.NRLDPC_ERR_CONFIG: "invalid LDPC configuration",
           capi.NRLDPC_ERR_ALGO: "invalid decoder algorithm", capi.NRLDPC_ERR_ARG: "invalid argument"}
    raise RuntimeError(f"{what} failed: {msg.get(rc, rc)}")


def ldpc_decode(llr: torch.Tensor, inconfig, decoder_config, *, return_app: bool = False,
                harq: Optional[torch.Tensor] = None, out: Optional[DecodeResult] = None) -> DecodeResult:
    """Decode a batch of code blocks that share one configuration.

    llr: int16 CUDA tensor [n, L] (L >= E), rate-matched order, row-contiguous.
    inconfig: LdpcInConfig or (bgn, A, crctype, E, rv, Qm, HARQ_on).
    decoder_config: DecoderConfig or [algo, max_iterations, alpha, beta,
        filling_bit_value, max_llr, min_llr].
    harq: optional int16 CUDA tensor [n, >= N+2Zc] of soft buffers; combined
        into when inconfig.HARQ_on == 1 and always updated.
    """
    cfg = _as_in_config(inconfig)
    dcfg = _as_decoder_config(decoder_config)
    if not llr.is_cuda or llr.dtype != torch.int16 or llr.dim() != 2:
        raise ValueError("llr must be an int16 CUDA tensor of shape [n, L]")
    if llr.shape[0] > 1 and (llr.stride(1) != 1 or llr.stride(0) < llr.shape[1]):
        llr = llr.contiguous()
    elif llr.shape[0] <= 1 and llr.stride(1) != 1:
        llr = llr.contiguous()
    p = code_params(cfg)
    n = llr.shape[0]
    nb = (p.B + 7) // 8
    dev = llr.device
    if out is None:
        bits = torch.zeros((n, nb), dtype=torch.uint8, device=dev)
        status = torch.empty(n, dtype=torch.int32, device=dev)
        iters = torch.empty(n, dtype=torch.int32, device=dev)
        app = None
        if return_app:
            dt = torch.float32 if dcfg.algo in (0, 4) else torch.int16
            app = torch.empty((n, p.N + 2 * p.Zc), dtype=dt, device=dev)
        out = DecodeResult(bits, status, iters, app)
    if harq is not None:
        if not harq.is_cuda or harq.dtype != torch.int16 or harq.stride(1) != 1 or harq.shape[0] != n:
            raise ValueError("harq must be an int16 CUDA tensor [n, >= N+2Zc]")
    lib = capi.load_library()
    stream = torch.cuda.current_stream(dev).cuda_stream
    with torch.cuda.device(dev):
        rc = lib.nrldpc_decode_batch(
            ctypes.c_void_p(llr.data_ptr()), _row_stride(llr), n, ctypes.byref(cfg), ctypes.byref(dcfg),
            ctypes.c_void_p(out.hardbits.data_ptr()), _row_stride(out.hardbits),
            ctypes.c_void_p(out.status.data_ptr()), ctypes.c_void_p(out.iterations.data_ptr()),
            ctypes.c_void_p(out.app.data_ptr() if out.app is not None else 0),
            _row_stride(out.app) if out.app is not None else 0,
            ctypes.c_void_p(harq.data_ptr() if harq is not None else 0),
            _row_stride(harq) if harq is not None else 0,
            ctypes.c_void_p(stream))
    _check(rc, "nrldpc_decode_batch")
    return out


def ldpc_encode(info: torch.Tensor, inconfig, ncb: int = 0) -> torch.Tensor:
    """Encode a batch of payloads (uint8 CUDA tensor [n, >= A/8], MSB first) into
    rate-matched bits packed MSB first: uint8 [n, ceil(E/8)].  0 < ncb < N selects
    limited-buffer rate matching over a circular buffer of ncb bits."""
    cfg = _as_in_config(inconfig)
    if not info.is_cuda or info.dtype != torch.uint8 or info.dim() != 2:
        raise ValueError("info must be a uint8 CUDA tensor of shape [n, A/8]")
    if info.shape[1] < (cfg.A + 7) // 8:
        raise ValueError(f"info rows must hold ceil(A/8) = {(cfg.A + 7) // 8} bytes")
    if info.stride(1) != 1:
        info = info.contiguous()
    n = info.shape[0]
    out = torch.zeros((n, (cfg.E + 7) // 8), dtype=torch.uint8, device=info.device)
    lib = capi.load_library()
    stream = torch.cuda.current_stream(info.device).cuda_stream
    with torch.cuda.device(info.device):
        if ncb and 0 < ncb < code_params(cfg).N:
            rc = lib.nrldpc_encode_batch_ncb(ctypes.c_void_p(info.data_ptr()), _row_stride(info), n,
                                             ctypes.byref(cfg), int(ncb), ctypes.c_void_p(out.data_ptr()),
                                             _row_stride(out), ctypes.c_void_p(stream))
        else:
            rc = lib.nrldpc_encode_batch(ctypes.c_void_p(info.data_ptr()), _row_stride(info), n, ctypes.byref(cfg),
                                         ctypes.c_void_p(out.data_ptr()), _row_stride(out), ctypes.c_void_p(stream))
    _check(rc, "nrldpc_encode_batch")
    return out


def channel_llrs(rm: torch.Tensor, E: int, Qm: int, noise_power_db: float, seed: int = 0,
                 return_symbols: bool = False):
    """Device LLR front-end: packed rate-matched bits (uint8 CUDA [n, ceil(E/8)])
    -> NR QAM -> AWGN (power 10^(noise_power_db/10)) -> max-log LLRs quantised
    to int16 like the reference channel.  Returns int16 [n, E] (and the noisy
    symbols float [n, E/Qm, 2] when asked)."""
    if not rm.is_cuda or rm.dtype != torch.uint8 or rm.dim() != 2:
        raise ValueError("rm must be a uint8 CUDA tensor [n, ceil(E/8)]")
    if rm.stride(1) != 1:
        rm = rm.contiguous()
    n = rm.shape[0]
    llr = torch.empty((n, E), dtype=torch.int16, device=rm.device)
    sym = torch.empty((n, E // Qm, 2), dtype=torch.float32, device=rm.device) if return_symbols else None
    lib = capi.load_library()
    stream = torch.cuda.current_stream(rm.device).cuda_stream
    with torch.cuda.device(rm.device):
        rc = lib.nrldpc_channel_batch(ctypes.c_void_p(rm.data_ptr()), _row_stride(rm), n, E, Qm,
                                      ctypes.c_float(noise_power_db), ctypes.c_uint64(seed),
                                      ctypes.c_void_p(llr.data_ptr()), E,
                                      ctypes.c_void_p(sym.data_ptr() if sym is not None else 0),
                                      ctypes.c_void_p(stream))
    _check(rc, "nrldpc_channel_batch")
    return (llr, sym) if return_symbols else llr


def ldpc_decode_host(llr, inconfig, decoder_config):
    """Decode from host (numpy / CPU tensor) LLRs through the host-buffer C ABI;
    returns numpy (hardbits, status, iterations)."""
    import numpy as np

    cfg = _as_in_config(inconfig)
    dcfg = _as_decoder_config(decoder_config)
    a = np.ascontiguousarray(llr.numpy() if isinstance(llr, torch.Tensor) else llr, dtype=np.int16)
    p = code_params(cfg)
    n = a.shape[0]
    nb = (p.B + 7) // 8
    bits = np.zeros((n, nb), dtype=np.uint8)
    status = np.zeros(n, dtype=np.int32)
    iters = np.zeros(n, dtype=np.int32)
    lib = capi.load_library()
    rc = lib.nrldpc_decode_batch_host(a.ctypes.data_as(ctypes.c_void_p), a.shape[1], n, ctypes.byref(cfg),
                                      ctypes.byref(dcfg), bits.ctypes.data_as(ctypes.c_void_p), nb,
                                      status.ctypes.data_as(ctypes.c_void_p), iters.ctypes.data_as(ctypes.c_void_p),
                                      None)
    _check(rc, "nrldpc_decode_batch_host")
    return bits, status, iters


def set_trained_weights(bgn: int, alpha=None, beta=None) -> None:
    """Install algo-2 tables [T][rows] (int16 Q15 alpha, int16 beta); None restores the built-in table."""
    import numpy as np

    lib = capi.load_library()
    if alpha is None:
        _check(lib.nrldpc_set_trained_weights(bgn, None, None, 0), "nrldpc_set_trained_weights")
        return
    a = np.ascontiguousarray(alpha, dtype=np.int16)
    b = np.ascontiguousarray(beta if beta is not None else np.zeros_like(a), dtype=np.int16)
    if a.ndim != 2 or a.shape[1] != capi.BG_ROWS[bgn] or b.shape != a.shape:
        raise ValueError("alpha/beta must be [T, rows] int16")
    _check(lib.nrldpc_set_trained_weights(bgn, a.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                                          a.shape[0]), "nrldpc_set_trained_weights")


def set_degree_alpha(table=None) -> None:
    """Install the 19-entry degree->alpha table of algo 3 (None restores the default)."""
    import numpy as np

    lib = capi.load_library()
    if table is None:
        lib.nrldpc_set_degree_alpha(None)
        return
    t = np.ascontiguousarray(table, dtype=np.int16)
    if t.shape != (19,):
        raise ValueError("degree alpha table must have 19 entries")
    lib.nrldpc_set_degree_alpha(t.ctypes.data_as(ctypes.c_void_p))
