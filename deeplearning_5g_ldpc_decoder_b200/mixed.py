"""Mixed-size batches: one persistent kernel decodes code blocks that mix base
graphs, lifting sizes, rates, modulations, redundancy versions and CRC types,
replayed from a CUDA graph (C ABI: nrldpc_mixed_plan_*)."""

from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import torch

from . import capi
from .capi import LdpcInConfig


# nrldpc_mixed_plan_autotune's candidates, in its order (NRLDPC_MIXED_AUTOTUNE_CANDIDATES).
AUTOTUNE_CANDIDATES = 8
AUTOTUNE_NAMES = [f"{cls}, {ctas} CTA/SM, {order}"
                  for cls in ("right-sized CTAs", "384-thread CTAs")
                  for order in ("largest-first", "interleaved")
                  for ctas in (2, 1)]


class Block(ctypes.Structure):
    """nrldpc_block_t."""

    _fields_ = [("cfg", LdpcInConfig), ("llr_offset", ctypes.c_int64), ("bits_offset", ctypes.c_int64)]


def _declare(lib):
    if getattr(lib, "_mixed_declared", False):
        return
    vp, i32 = ctypes.c_void_p, ctypes.c_int32
    lib.nrldpc_mixed_plan_create.argtypes = [ctypes.POINTER(Block), i32, ctypes.POINTER(capi.DecoderConfig),
                                             ctypes.POINTER(vp)]
    lib.nrldpc_mixed_plan_create.restype = i32
    lib.nrldpc_mixed_plan_execute.argtypes = [vp, vp, vp, vp, vp, i32, vp]
    lib.nrldpc_mixed_plan_execute.restype = i32
    lib.nrldpc_mixed_plan_autotune.argtypes = [vp, vp, vp, vp, vp, vp, vp]
    lib.nrldpc_mixed_plan_autotune.restype = i32
    lib.nrldpc_mixed_plan_select.argtypes = [vp, i32]
    lib.nrldpc_mixed_plan_select.restype = i32
    lib.nrldpc_mixed_plan_destroy.argtypes = [vp]
    lib.nrldpc_mixed_plan_destroy.restype = i32
    lib._mixed_declared = True


class MixedPlan:
    """Plan for one batch composition.

    configs: per block (bgn, A, crctype, E, rv, Qm).  By default the LLRs of
    block i occupy llr_arena[llr_offsets[i] : llr_offsets[i] + E_i] and its
    hard bits bits_arena[bits_offsets[i] : + ceil(B_i/8)], packed back to back.
    `lib` selects another build of the library (the bounds-checked debug one).
    """

    def __init__(self, configs: Sequence[Sequence[int]], decoder_config, device=None, lib=None):
        self.lib = lib or capi.load_library()
        _declare(self.lib)
        self.configs = [tuple(int(v) for v in c[:6]) for c in configs]
        n = len(self.configs)
        blocks = (Block * n)()
        self.llr_offsets, self.bits_offsets, self.nbytes = [], [], []
        lo = bo = 0
        for i, (bgn, A, crc, E, rv, Qm) in enumerate(self.configs):
            p = capi.gen_ldpc_parameters(capi.make_in_config(bgn, A, crc, E, rv, Qm, 0), self.lib)
            nb = (p.B + 7) // 8
            blocks[i].cfg = capi.make_in_config(bgn, A, crc, E, rv, Qm, 0)
            blocks[i].llr_offset = lo
            blocks[i].bits_offset = bo
            self.llr_offsets.append(lo)
            self.bits_offsets.append(bo)
            self.nbytes.append(nb)
            lo += E
            bo += nb
        self.llr_len, self.bits_len = lo, bo
        self.decoder_config = capi.make_decoder_config(decoder_config) if not isinstance(
            decoder_config, capi.DecoderConfig) else decoder_config
        self.device = torch.device(device or "cuda")
        self._plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = self.lib.nrldpc_mixed_plan_create(blocks, n, ctypes.byref(self.decoder_config),
                                                   ctypes.byref(self._plan))
        if rc != 0:
            raise RuntimeError(f"nrldpc_mixed_plan_create failed: {rc}")
        self.num_blocks = n

    def pack_llrs(self, llrs: List[torch.Tensor]) -> torch.Tensor:
        return torch.cat([t.reshape(-1).to(torch.int16) for t in llrs]).to(self.device)

    def outputs(self):
        return (torch.zeros(self.bits_len, dtype=torch.uint8, device=self.device),
                torch.empty(self.num_blocks, dtype=torch.int32, device=self.device),
                torch.empty(self.num_blocks, dtype=torch.int32, device=self.device))

    def decode(self, llr_arena: torch.Tensor, use_graph: bool = True, out=None):
        bits, status, iters = out if out is not None else self.outputs()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        with torch.cuda.device(self.device):
            rc = self.lib.nrldpc_mixed_plan_execute(self._plan, ctypes.c_void_p(llr_arena.data_ptr()),
                                                    ctypes.c_void_p(bits.data_ptr()),
                                                    ctypes.c_void_p(status.data_ptr()),
                                                    ctypes.c_void_p(iters.data_ptr()), int(use_graph),
                                                    ctypes.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"nrldpc_mixed_plan_execute failed: {rc}")
        return bits, status, iters

    def autotune(self, llr_arena: torch.Tensor, out=None):
        bits, status, iters = out if out is not None else self.outputs()
        ms = (ctypes.c_float * AUTOTUNE_CANDIDATES)()
        stream = torch.cuda.current_stream(self.device).cuda_stream
        with torch.cuda.device(self.device):
            best = self.lib.nrldpc_mixed_plan_autotune(self._plan, ctypes.c_void_p(llr_arena.data_ptr()),
                                                       ctypes.c_void_p(bits.data_ptr()),
                                                       ctypes.c_void_p(status.data_ptr()),
                                                       ctypes.c_void_p(iters.data_ptr()), ms, ctypes.c_void_p(stream))
        if best < 0:
            raise RuntimeError(f"nrldpc_mixed_plan_autotune failed: {best}")
        return best, list(ms)

    def select(self, candidate: int) -> None:
        """Use autotuner candidate `candidate` (AUTOTUNE_NAMES order) without timing."""
        with torch.cuda.device(self.device):
            rc = self.lib.nrldpc_mixed_plan_select(self._plan, int(candidate))
        if rc != 0:
            raise RuntimeError(f"nrldpc_mixed_plan_select failed: {rc}")

    def block_bits(self, bits: torch.Tensor, i: int) -> torch.Tensor:
        return bits[self.bits_offsets[i]: self.bits_offsets[i] + self.nbytes[i]]

    def close(self):
        if self._plan:
            self.lib.nrldpc_mixed_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def random_mixed_configs(n: int, seed: int = 0, bg1_share: float = 0.6, rate=(0.2, 0.92), qms=(2, 4, 6, 8),
                         lib=None, rvs=(0, 1, 2, 3)):
    """Configurations of the mixed-size workload: lifting size uniform over the
    51 sizes (redrawn where a base graph cannot reach it), BG1 with probability
    bg1_share, code rate uniform in `rate`, Qm from `qms`, rv from `rvs` and CRC24
    type random.  Returns a list of (bgn, A, crctype, E, rv, Qm)."""
    import numpy as np

    lib = lib or capi.load_library()
    rng = np.random.default_rng(seed)
    by_zc = {1: {}, 2: {}}
    for bgn in (1, 2):
        for crc in (1, 2, 3):
            for A in range(8, (8448 if bgn == 1 else 3840) - 24 + 1, 8):
                cfg = capi.make_in_config(bgn, A, crc, 960, 0, 2, 0)
                out = capi.LdpcConfig()
                if lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(cfg)) == 0:
                    by_zc[bgn].setdefault(int(out.Zc), []).append((A, crc, int(out.B)))
    sizes = sorted(by_zc[1])
    out = []
    while len(out) < n:
        bgn = 1 if rng.random() < bg1_share else 2
        zc = sizes[rng.integers(len(sizes))]
        if zc not in by_zc[bgn]:
            continue
        A, crc, B = by_zc[bgn][zc][rng.integers(len(by_zc[bgn][zc]))]
        Qm = int(qms[rng.integers(len(qms))])
        R = rng.uniform(*rate)
        E = int(round(B / R / Qm)) * Qm
        if E < Qm or E > 65535:
            continue
        out.append((bgn, A, crc, E, int(rvs[rng.integers(len(rvs))]), Qm))
    return out
