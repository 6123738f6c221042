"""The decoder as a PyTorch dispatcher operator: ``torch.ops.nrldpc.ldpc_decode``.

The operator wraps the same C-ABI call as ``decoder.ldpc_decode``
(``nrldpc_decode_batch`` on the caller's current stream).  Registering it with
``torch.library`` makes it visible to the dispatcher: it has a fake (meta)
implementation, so shape propagation, FakeTensor tracing and torch.compile
see its outputs without running it, and it has only a CUDA kernel, so a CPU
tensor is rejected by the dispatcher instead of falling back to anything.

    bits, status, iterations, app = torch.ops.nrldpc.ldpc_decode(
        llr, [bgn, A, crctype, E, rv, Qm, HARQ_on],
        [algo, max_iterations, alpha, beta, filling_bit_value, max_llr, min_llr],
        return_app)

Outputs: uint8 [n, ceil(B/8)] hard bits (MSB first), int32 [n] status, int32
[n] executed iterations, and the final beliefs [n, N+2Zc] (int16; float32 for
algos 0 and 4) when ``return_app``, else an empty [n, 0] tensor of that type.
"""

from __future__ import annotations

from typing import List, Tuple

import torch

from . import decoder

Tensor = torch.Tensor


def _shapes(llr: Tensor, inconfig: List[int], decoder_config: List[int], return_app: bool):
    if len(inconfig) != 7 or len(decoder_config) != 7:
        raise ValueError("inconfig and decoder_config must each have 7 entries")
    p = decoder.code_params(list(inconfig))
    if p.Zc == 0:
        raise ValueError("invalid LDPC configuration")
    n = llr.shape[0]
    app_dt = torch.float32 if decoder_config[0] in (0, 4) else torch.int16
    app_cols = p.N + 2 * p.Zc if return_app else 0
    return n, (p.B + 7) // 8, app_dt, app_cols


@torch.library.custom_op("nrldpc::ldpc_decode", mutates_args=(), device_types="cuda")
def ldpc_decode_op(llr: Tensor, inconfig: List[int], decoder_config: List[int],
                   return_app: bool = False) -> Tuple[Tensor, Tensor, Tensor, Tensor]:
    n, nb, app_dt, app_cols = _shapes(llr, inconfig, decoder_config, return_app)
    res = decoder.ldpc_decode(llr, list(inconfig), list(decoder_config), return_app=return_app)
    app = res.app if res.app is not None else torch.empty((n, 0), dtype=app_dt, device=llr.device)
    return res.hardbits, res.status, res.iterations, app


@ldpc_decode_op.register_fake
def _ldpc_decode_fake(llr, inconfig, decoder_config, return_app=False):
    if llr.dtype != torch.int16 or llr.dim() != 2:
        raise ValueError("llr must be an int16 tensor of shape [n, L]")
    n, nb, app_dt, app_cols = _shapes(llr, inconfig, decoder_config, return_app)
    return (llr.new_empty((n, nb), dtype=torch.uint8), llr.new_empty((n,), dtype=torch.int32),
            llr.new_empty((n,), dtype=torch.int32), llr.new_empty((n, app_cols), dtype=app_dt))
