"""Transport blocks: segmentation, device encode for test traffic, the batched
decode engine and the serving loop (C ABI in include/nrldpc_b200.h).

* ``segment`` / ``select_bg`` / ``round_tbs`` — TS 38.212 5.2.2 segmentation,
  7.2.2 base-graph choice, and transport-block sizes that segment into equal
  byte-aligned code blocks (the property TS 38.214's size rule guarantees).
* ``TbEngine`` — decode batches of transport blocks on the device: on-device
  segmentation, one mixed-size persistent launch for all code blocks,
  on-device transport-block CRC and payload gather.
* ``serve`` — the native continuous-batching loop over an arrival trace with
  HBM-budget admission; per-block verdict latency.
* ``encode_transport_blocks`` — test traffic: payload -> transport-block CRC ->
  code blocks (CRC24B when several) -> device LDPC encoder -> device channel,
  into one LLR arena.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import capi

TB_DTYPE = np.dtype([("A", "<i4"), ("G", "<i4"), ("Qm", "<u2"), ("rv", "<u2"), ("bgn", "<u2"), ("flags", "<u2"),
                     ("llr_offset", "<i8"), ("out_offset", "<i8"), ("tbs_lbrm", "<i4"), ("pad", "<i4"),
                     ("harq_offset", "<i8")])
HARQ_COMBINE = capi.NRLDPC_TB_HARQ_COMBINE   # add this transmission to the stored soft buffers
HARQ_STORE = capi.NRLDPC_TB_HARQ_STORE       # keep the combined soft buffers for a retransmission
assert TB_DTYPE.itemsize == ctypes.sizeof(capi.TbDesc)


@dataclass
class Segmentation:
    C: int
    L_tb: int
    Kp: int
    Zc: int
    E_lo: int
    E_hi: int
    n_lo: int
    cb_cfg: Tuple[int, int, int, int, int, int, int]   # (bgn, A_cb, crctype, E_lo, rv, Qm, 0)
    Ncb: int = 0          # circular-buffer length of every code block
    k0: int = 0
    harq_elems: int = 0   # int16 soft-buffer elements of the whole block: C (N + 2Zc)

    def E(self, r: int) -> int:
        return self.E_lo if r < self.n_lo else self.E_hi

    def llr_start(self, r: int) -> int:
        return r * self.E_lo if r < self.n_lo else self.n_lo * self.E_lo + (r - self.n_lo) * self.E_hi


def segment(A: int, G: int, Qm: int, bgn: int, rv: int = 0, tbs_lbrm: int = 0) -> Segmentation:
    """TS 38.212 5.2.2 segmentation; tbs_lbrm > 0 adds limited-buffer rate matching."""
    lib = capi.load_library()
    d = capi.TbDesc(A, G, Qm, rv, bgn, 0, 0, 0, int(tbs_lbrm), 0, 0)
    info = capi.TbInfo()
    if lib.nrldpc_tb_segment(ctypes.byref(d), ctypes.byref(info)) != 0:
        raise ValueError(f"invalid transport block A={A} G={G} Qm={Qm} bgn={bgn} rv={rv} tbs_lbrm={tbs_lbrm}")
    c = info.cb_cfg
    return Segmentation(info.C, info.L_tb, info.Kp, info.Zc, info.E_lo, info.E_hi, info.n_lo,
                        (c.bgn, c.A, c.crctype, c.E, c.rv, c.Qm, 0), info.Ncb, info.k0, info.harq_elems)


def code_block_count(A: int, bgn: int) -> Tuple[int, int]:
    """(C, L_tb): code blocks and transport-block CRC length (TS 38.212 5.2.2)."""
    L = 24 if A > 3824 else 16
    B = A + L
    Kcb = 8448 if bgn == 1 else 3840
    return (1 if B <= Kcb else -(-B // (Kcb - 24))), L


def coded_bits(A: int, bgn: int, Qm: int, R: float) -> int:
    """G for a target code rate R: (A + CRCs) / R rounded to whole symbols."""
    C, L = code_block_count(A, bgn)
    B = A + L + (24 * C if C > 1 else 0)
    return Qm * max(1, int(round(B / R / Qm)))


def select_bg(A: int, R: float) -> int:
    """TS 38.212 7.2.2: base graph 2 if A <= 292, or A <= 3824 and R <= 0.67, or R <= 0.25."""
    return int(capi.load_library().nrldpc_tb_select_bg(int(A), int(math.floor(R * 1024))))


def round_tbs(A: float, bgn: int) -> int:
    """Nearest transport-block size at or below A (at least 24) that segments into
    equal byte-aligned code blocks: a multiple of 8 for one code block, else
    (A + 24) a multiple of 8 C (TS 38.214 5.1.3.2's form)."""
    A = max(24, int(A))
    Kcb = 8448 if bgn == 1 else 3840
    while True:
        L = 24 if A > 3824 else 16
        if A + L <= Kcb:
            return (A // 8) * 8
        C = -(-(A + 24) // (Kcb - 24))
        A2 = 8 * C * ((A + 24) // (8 * C)) - 24
        B = A2 + 24
        if A2 > 3824 and -(-B // (Kcb - 24)) == C:
            return A2
        A = A2 if A2 < A else A - 8


def tb_array(rows: Sequence[Tuple[int, ...]]) -> np.ndarray:
    """(A, G, Qm, rv, bgn, llr_offset, out_offset[, tbs_lbrm[, flags, harq_offset]]) rows
    -> nrldpc_tb_t records."""
    a = np.zeros(len(rows), dtype=TB_DTYPE)
    for i, r in enumerate(rows):
        A, G, Qm, rv, bgn, lo, oo = r[:7]
        lbrm = r[7] if len(r) > 7 else 0
        flags = r[8] if len(r) > 8 else 0
        ho = r[9] if len(r) > 9 else 0
        a[i] = (A, G, Qm, rv, bgn, flags, lo, oo, lbrm, 0, ho)
    return a


class TbEngine:
    """Batched transport-block decoder (algos 1-3) on the current CUDA device."""

    def __init__(self, max_tbs: int, max_cbs: int, decoder_row=(1, 10, 22936, 0, 1280, 32767, -32767)):
        self.lib = capi.load_library()
        self.max_tbs, self.max_cbs = int(max_tbs), int(max_cbs)
        self.handle = ctypes.c_void_p()
        dc = capi.make_decoder_config(decoder_row)
        rc = self.lib.nrldpc_tb_engine_create(self.max_tbs, self.max_cbs, ctypes.byref(dc), ctypes.byref(self.handle))
        if rc != 0:
            raise RuntimeError(f"nrldpc_tb_engine_create failed: {rc}")

    def close(self):
        if self.handle:
            self.lib.nrldpc_tb_engine_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def decode(self, tbs: np.ndarray, llr, out, stream=None, harq=None):
        """tbs: nrldpc_tb_t records (numpy); llr: int16 CUDA arena; out: uint8 CUDA
        arena; harq: int16 CUDA soft-buffer arena for blocks with HARQ flags.
        Returns (status, iterations) int32 CUDA tensors."""
        import torch

        dev = llr.device
        d_tbs = torch.from_numpy(tbs.view(np.uint8).copy()).to(dev)
        n = len(tbs)
        status = torch.empty(n, dtype=torch.int32, device=dev)
        iters = torch.empty(n, dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        rc = self.lib.nrldpc_tb_engine_decode(self.handle, ctypes.c_void_p(d_tbs.data_ptr()), n,
                                              ctypes.c_void_p(llr.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                              ctypes.c_void_p(status.data_ptr()), ctypes.c_void_p(iters.data_ptr()),
                                              ctypes.c_void_p(harq.data_ptr() if harq is not None else 0),
                                              ctypes.c_void_p(s.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"nrldpc_tb_engine_decode failed: {rc}")
        self._keep = d_tbs   # alive until the stream has consumed it
        return status, iters

    def views(self):
        """Device pointers (ints) of the last batch's code-block bits, status,
        iterations and each transport block's first code block."""
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        self.lib.nrldpc_tb_engine_views(self.handle, *[ctypes.byref(p) for p in ptrs])
        return [p.value for p in ptrs]


@dataclass
class ServeResult:
    status: np.ndarray        # int32 per block: 0 pass, 1 fail, -5 dropped, -6 expired, -2 bad configuration
    latency_s: np.ndarray     # verdict - arrival (NaN when dropped or expired)
    stats: dict
    cb_first: Optional[np.ndarray] = None   # with record=True: block i's code blocks start here in
    cb_status: Optional[np.ndarray] = None  # the per-code-block status, iterations and hard bits
    cb_iterations: Optional[np.ndarray] = None
    cb_bits: Optional[np.ndarray] = None    # [code blocks][1056] bytes


def serve(engine: TbEngine, tbs: np.ndarray, arrival_s: np.ndarray, llr, out, *, max_batch_tbs: int = 4096,
          max_batch_cbs: Optional[int] = None, llr_budget_bytes: int = 8 << 30, pipeline_depth: int = 2,
          timeout_s: float = 120.0, max_wait_s: float = 0.0, record: bool = False, stream=None) -> ServeResult:
    """Serve an arrival trace through the native loop (nrldpc_serve_run).
    max_wait_s > 0 drops admitted blocks that wait longer for a batch
    (NRLDPC_TB_EXPIRED); record=True also returns every decoded code block's
    status, iterations and hard bits (a device copy per block: for checks)."""
    import torch

    n = len(tbs)
    arrival = np.ascontiguousarray(arrival_s, dtype=np.float64)
    tbs = np.ascontiguousarray(tbs)
    status = np.zeros(n, dtype=np.int32)
    lat = np.zeros(n, dtype=np.float64)
    cfg = capi.ServeConfig(int(max_batch_tbs), int(max_batch_cbs or engine.max_cbs), int(llr_budget_bytes),
                           int(pipeline_depth), 0, float(timeout_s), float(max_wait_s))
    rec = None
    if record:
        counts = np.array([segment(int(t["A"]), int(t["G"]), int(t["Qm"]), int(t["bgn"]), int(t["rv"]),
                                   int(t["tbs_lbrm"])).C for t in tbs], dtype=np.int64)
        first = np.ascontiguousarray(np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.int64))
        total = max(int(counts.sum()), 1)
        rec = (first, torch.full((total,), -9, dtype=torch.int32, device=llr.device),
               torch.full((total,), -9, dtype=torch.int32, device=llr.device),
               torch.zeros((total, 1056), dtype=torch.uint8, device=llr.device))
        cfg.h_cb_first = first.ctypes.data
        cfg.d_cb_status = rec[1].data_ptr()
        cfg.d_cb_iterations = rec[2].data_ptr()
        cfg.d_cb_bits = rec[3].data_ptr()
    st = capi.ServeStats()
    s = stream if stream is not None else torch.cuda.current_stream(llr.device)
    rc = engine.lib.nrldpc_serve_run(engine.handle, ctypes.byref(cfg), tbs.ctypes.data_as(ctypes.c_void_p),
                                     arrival.ctypes.data_as(ctypes.c_void_p), n, ctypes.c_void_p(llr.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), status.ctypes.data_as(ctypes.c_void_p),
                                     lat.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st),
                                     ctypes.c_void_p(s.cuda_stream))
    if rc != 0:
        raise RuntimeError(f"nrldpc_serve_run failed: {rc}")
    stats = {k: getattr(st, k) for k, _ in capi.ServeStats._fields_}
    if rec is None:
        return ServeResult(status, lat, stats)
    s.synchronize()
    return ServeResult(status, lat, stats, rec[0], rec[1].cpu().numpy(), rec[2].cpu().numpy(), rec[3].cpu().numpy())


def tb_crc(payload: np.ndarray, A: int) -> np.ndarray:
    """Transport-block CRC bits (CRC16 for A <= 3824, else CRC24A) of A payload
    bits given as bytes, through the library's calculate_crc."""
    lib = capi.load_library()
    data = np.ascontiguousarray(payload[: A // 8], dtype=np.uint8)
    L = 24 if A > 3824 else 16
    r = int(lib.calculate_crc(data.ctypes.data_as(ctypes.c_void_p), A // 8, 1 if L == 24 else 0))
    return np.array([(r >> (L - 1 - i)) & 1 for i in range(L)], dtype=np.uint8)


def encode_transport_blocks(payloads: List[np.ndarray], tbs: np.ndarray, noise_power_db: Sequence[float],
                            seed: int = 0, device=None):
    """Test traffic.  payloads[i]: A_i/8 bytes; tbs: records (A, G, Qm, rv, bgn,
    llr_offset set here contiguously, out_offset set here).  Returns
    (tbs with offsets, int16 CUDA LLR arena, total output bytes)."""
    import torch

    from .decoder import channel_llrs, ldpc_encode

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    tbs = tbs.copy()
    llr_off, out_off = 0, 0
    segs = []
    for i in range(len(tbs)):
        sg = segment(int(tbs[i]["A"]), int(tbs[i]["G"]), int(tbs[i]["Qm"]), int(tbs[i]["bgn"]), int(tbs[i]["rv"]),
                     int(tbs[i]["tbs_lbrm"]))
        segs.append(sg)
        tbs[i]["llr_offset"] = llr_off
        tbs[i]["out_offset"] = out_off
        llr_off += int(tbs[i]["G"])
        out_off += int(tbs[i]["A"]) // 8
    arena = torch.zeros(max(llr_off, 1), dtype=torch.int16, device=dev)
    for i, sg in enumerate(segs):
        A = int(tbs[i]["A"])
        pay = np.ascontiguousarray(payloads[i][: A // 8], dtype=np.uint8)
        if sg.C == 1:
            chunks = [pay]
        else:
            tb_bits = np.concatenate([np.unpackbits(pay), tb_crc(pay, A)])
            chunk_bits = sg.cb_cfg[1]
            chunks = [np.packbits(tb_bits[r * chunk_bits:(r + 1) * chunk_bits]) for r in range(sg.C)]
        # code blocks of one E share a configuration: one encoder and one channel call each
        for lo, hi in ((0, sg.n_lo), (sg.n_lo, sg.C)):
            if hi <= lo:
                continue
            E = sg.E(lo)
            cfg = (sg.cb_cfg[0], sg.cb_cfg[1], sg.cb_cfg[2], E, sg.cb_cfg[4], sg.cb_cfg[5], 0)
            info = torch.from_numpy(np.stack(chunks[lo:hi])).to(dev)
            rm = ldpc_encode(info, cfg, ncb=sg.Ncb)
            llr = channel_llrs(rm, E, cfg[5], float(noise_power_db[i]), seed=seed * 1000003 + i * 7 + lo)
            start = int(tbs[i]["llr_offset"]) + sg.llr_start(lo)
            arena[start:start + (hi - lo) * E] = llr.reshape(-1)
    return tbs, arena, out_off
