"""ctypes wrappers of the CPU oracle and of the reference library build.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() (as the
checker) and bench.py's CPU-baseline leg.  Nothing in the product imports it.

* ``Oracle``  — ``oracle/liboracle.so``, this project's C restatement of the
  reference receive path (``oracle/nr_ldpc_oracle.c``).
* ``RefLib``  — ``oracle/_ref/libnrLDPC_ref.so``, the reference C library built
  from its own sources by ``oracle/build_ref.sh`` (only where the reference
  tree was available at build time).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnrLDPC_ref.so")


class InConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint16) for n in ("bgn", "A", "crctype", "E", "rv", "Qm", "HARQ_on")]


class DecCfg(ctypes.Structure):
    _fields_ = [
        ("algo", ctypes.c_uint16),
        ("max_iterations", ctypes.c_uint16),
        ("alpha", ctypes.c_uint16),
        ("beta", ctypes.c_uint16),
        ("filling_bit_value", ctypes.c_int16),
        ("max_llr", ctypes.c_int16),
        ("min_llr", ctypes.c_int16),
    ]


class OrcParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "bgn", "A", "crctype", "E", "rv", "Qm", "HARQ_on", "B", "Zc", "iLS", "K", "F", "N", "k0",
        "rows", "cols", "nnz", "Ncb")]


class RefConfig(ctypes.Structure):
    """Layout of the reference's ldpc_config_t (c_lib/nr_ldpc.h:54-79)."""

    _fields_ = [(n, ctypes.c_uint16) for n in (
        "bgn", "A", "crctype", "E", "rv", "Qm", "HARQ_on", "B", "Zc", "iLS", "K", "F", "N", "k0")] + [
        ("Vij_array", ctypes.POINTER(ctypes.c_uint16)),
        ("HBG_array", ctypes.POINTER(ctypes.c_uint16)),
        ("HBG_offset_array", ctypes.POINTER(ctypes.c_uint16)),
    ]


def in_config(bgn, A, crctype, E, rv=0, Qm=2, HARQ_on=0) -> InConfig:
    return InConfig(bgn, A, crctype, E, rv, Qm, HARQ_on)


def dec_cfg(row) -> DecCfg:
    """[algo, max_iterations, alpha, beta, filling_bit_value, max_llr, min_llr]."""
    return DecCfg(*[int(v) for v in row])


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def build_oracle() -> str:
    src = os.path.join(HERE, "nr_ldpc_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


class Oracle:
    def __init__(self, path: str | None = None):
        self.lib = ctypes.CDLL(path or build_oracle())
        L = self.lib
        L.orc_derive.argtypes = [ctypes.POINTER(InConfig), ctypes.POINTER(OrcParams)]
        L.orc_crc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_crc.restype = ctypes.c_uint32
        L.orc_rate_recover.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int16, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(InConfig),
                                 ctypes.POINTER(DecCfg), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_decode.restype = ctypes.c_int32
        L.orc_decode_many.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.POINTER(InConfig),
                                      ctypes.POINTER(DecCfg), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                      ctypes.c_void_p]
        L.orc_decode_many.restype = ctypes.c_int32
        L.orc_encode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(InConfig)]
        L.orc_encode.restype = ctypes.c_int32
        L.orc_encode_codeword.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(InConfig)]
        L.orc_encode_codeword.restype = ctypes.c_int32
        L.orc_channel.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint16, ctypes.c_float,
                                  ctypes.c_uint64, ctypes.c_void_p]
        L.orc_channel.restype = ctypes.c_int
        L.orc_set_trained.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.orc_set_degree_alpha.argtypes = [ctypes.c_void_p]
        L.orc_set_ncb.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_int]
        L.orc_set_ncb.restype = ctypes.c_int
        L.orc_encode_params.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(OrcParams)]
        L.orc_encode_params.restype = ctypes.c_int32
        L.orc_decode_recovered.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(OrcParams),
                                           ctypes.POINTER(DecCfg), ctypes.c_void_p, ctypes.c_void_p]
        L.orc_decode_recovered.restype = ctypes.c_int32
        L.orc_graph.argtypes = [ctypes.POINTER(OrcParams), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_graph.restype = ctypes.c_int
        self.harq = np.zeros(68 * 384, dtype=np.int16)

    def derive(self, cfg: InConfig):
        p = OrcParams()
        rc = self.lib.orc_derive(ctypes.byref(cfg), ctypes.byref(p))
        return rc, p

    def params(self, cfg: InConfig, ncb: int = 0) -> OrcParams:
        """Derived parameters, with limited-buffer rate matching when 0 < ncb < N."""
        rc, p = self.derive(cfg)
        if rc != 0 or self.lib.orc_set_ncb(ctypes.byref(p), int(ncb)) != 0:
            raise ValueError("invalid configuration")
        return p

    def encode_ncb(self, payload: np.ndarray, cfg: InConfig, ncb: int) -> np.ndarray:
        p = self.params(cfg, ncb)
        payload = np.ascontiguousarray(payload, dtype=np.uint8)
        out = np.zeros((cfg.E + 7) // 8 + 8, dtype=np.uint8)
        assert self.lib.orc_encode_params(_p(payload), _p(out), ctypes.byref(p)) == 0
        return out[: (cfg.E + 7) // 8].copy()

    def rate_recover_ncb(self, cfg: InConfig, ncb: int, fill: int, llr: np.ndarray, harq: np.ndarray | None = None):
        """Soft buffer after rate recovery with circular-buffer length ncb; with
        cfg.HARQ_on the LLRs are added to `harq` (int16 wrap-around, in place)."""
        p = self.params(cfg, ncb)
        h = np.zeros(68 * 384, dtype=np.int16) if harq is None else harq
        llr = np.ascontiguousarray(llr, dtype=np.int16)
        self.lib.orc_rate_recover(ctypes.byref(p), fill, _p(llr), _p(h))
        return h

    def decode_soft(self, harq: np.ndarray, cfg: InConfig, dcfg: DecCfg):
        """Decode a recovered soft buffer: (status, bits, iterations, final LQ)."""
        rc, p = self.derive(cfg)
        bits = np.zeros((p.B + 7) // 8, dtype=np.uint8)
        lq = np.zeros(p.N + 2 * p.Zc, dtype=np.float32 if dcfg.algo in (0, 4) else np.int16)
        it = ctypes.c_int32(0)
        h = np.ascontiguousarray(harq, dtype=np.int16)
        st = self.lib.orc_decode_recovered(_p(h), _p(bits), ctypes.byref(p), ctypes.byref(dcfg), _p(lq),
                                           ctypes.byref(it))
        return int(st), bits, int(it.value), lq

    def graph(self, cfg: InConfig):
        """(params, col[nnz], shift[nnz] = Vij mod Zc, off[rows+1]) of one configuration."""
        rc, p = self.derive(cfg)
        if rc != 0:
            raise ValueError("invalid LDPC configuration")
        col = np.zeros(316, dtype=np.int32)
        shift = np.zeros(316, dtype=np.int32)
        off = np.zeros(47, dtype=np.int32)
        nnz = self.lib.orc_graph(ctypes.byref(p), _p(col), _p(shift), _p(off))
        return p, col[:nnz].copy(), shift[:nnz].copy(), off[: p.rows + 1].copy()

    def crc(self, data: np.ndarray, crctype: int) -> int:
        data = np.ascontiguousarray(data, dtype=np.uint8)
        return int(self.lib.orc_crc(_p(data), len(data), crctype))

    def rate_recover(self, cfg: InConfig, fill: int, llr: np.ndarray, harq: np.ndarray | None = None):
        rc, p = self.derive(cfg)
        assert rc == 0
        llr = np.ascontiguousarray(llr, dtype=np.int16)
        h = self.harq if harq is None else harq
        self.lib.orc_rate_recover(ctypes.byref(p), fill, _p(llr), _p(h))
        return h[: p.N + 2 * p.Zc].copy()

    def decode(self, llr: np.ndarray, cfg: InConfig, dcfg: DecCfg, harq: np.ndarray | None = None):
        """Returns (status, hardbits, iterations, final LQ)."""
        rc, p = self.derive(cfg)
        if rc != 0:
            return -2, None, 0, None
        llr = np.ascontiguousarray(llr, dtype=np.int16)
        bits = np.zeros((p.B + 7) // 8, dtype=np.uint8)
        lq = np.zeros(p.N + 2 * p.Zc, dtype=np.float32 if dcfg.algo in (0, 4) else np.int16)
        it = ctypes.c_int32(0)
        h = self.harq if harq is None else harq
        st = self.lib.orc_decode(_p(llr), _p(bits), ctypes.byref(cfg), ctypes.byref(dcfg), _p(h), _p(lq),
                                 ctypes.byref(it))
        return int(st), bits, int(it.value), lq

    def decode_many(self, llr: np.ndarray, cfg: InConfig, dcfg: DecCfg):
        rc, p = self.derive(cfg)
        assert rc == 0
        llr = np.ascontiguousarray(llr, dtype=np.int16)
        n = llr.shape[0]
        nb = (p.B + 7) // 8
        bits = np.zeros((n, nb), dtype=np.uint8)
        status = np.zeros(n, dtype=np.int32)
        iters = np.zeros(n, dtype=np.int32)
        rc = self.lib.orc_decode_many(_p(llr), llr.shape[1], n, ctypes.byref(cfg), ctypes.byref(dcfg), _p(bits), nb,
                                      _p(status), _p(iters))
        assert rc == 0, rc
        return status, bits, iters

    def encode(self, payload: np.ndarray, cfg: InConfig) -> np.ndarray:
        payload = np.ascontiguousarray(payload, dtype=np.uint8)
        out = np.zeros((cfg.E + 7) // 8, dtype=np.uint8)
        rc = self.lib.orc_encode(_p(payload), _p(out), ctypes.byref(cfg))
        assert rc == 0, rc
        return out

    def encode_codeword(self, payload: np.ndarray, cfg: InConfig) -> np.ndarray:
        rc, p = self.derive(cfg)
        assert rc == 0
        payload = np.ascontiguousarray(payload, dtype=np.uint8)
        out = np.zeros(p.N + 2 * p.Zc, dtype=np.uint8)
        self.lib.orc_encode_codeword(_p(payload), _p(out), ctypes.byref(cfg))
        return out

    def channel(self, rm_bytes: np.ndarray, E: int, Qm: int, noise_db: float, seed: int) -> np.ndarray:
        rm_bytes = np.ascontiguousarray(rm_bytes, dtype=np.uint8)
        out = np.zeros(E, dtype=np.int16)
        rc = self.lib.orc_channel(_p(rm_bytes), E, Qm, noise_db, seed, _p(out))
        assert rc == 0
        return out

    def set_trained(self, bgn: int, alpha=None, beta=None):
        if alpha is None:
            self.lib.orc_set_trained(bgn, None, None, 0)
            return
        a = np.ascontiguousarray(alpha, dtype=np.int16)
        b = np.ascontiguousarray(beta if beta is not None else np.zeros_like(a), dtype=np.int16)
        self.lib.orc_set_trained(bgn, _p(a), _p(b), a.shape[0])

    def set_degree_alpha(self, tab=None):
        if tab is None:
            self.lib.orc_set_degree_alpha(None)
        else:
            t = np.ascontiguousarray(tab, dtype=np.int16)
            self.lib.orc_set_degree_alpha(_p(t))


def make_llrs(orc: Oracle, cfg: InConfig, n: int, noise_db: float, seed: int = 0):
    """Seeded payloads -> oracle encoder -> oracle channel.  Returns
    (llr [n, E] int16, payload [n, A/8] uint8)."""
    rng = np.random.default_rng(seed)
    A = cfg.A
    llr = np.zeros((n, cfg.E), dtype=np.int16)
    pay = rng.integers(0, 256, size=(n, max(A // 8, 1)), dtype=np.uint8)[:, : A // 8]
    for i in range(n):
        rm = orc.encode(pay[i], cfg)
        llr[i] = orc.channel(rm, cfg.E, cfg.Qm, noise_db, seed * 1000003 + i)
    return llr, pay


class RefLib:
    """The reference C library built from its sources (oracle/_ref)."""

    def __init__(self, path: str | None = None):
        path = path or REF_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        for name in ("c_ldpc_5g_decode",):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(InConfig), ctypes.POINTER(DecCfg)]
            f.restype = ctypes.c_int32
        L.c_ldpc_5g_encode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(InConfig)]
        L.c_ldpc_5g_encode.restype = ctypes.c_int32
        L.tx_rx_process.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint16, ctypes.c_float,
                                    ctypes.c_void_p]
        L.tx_rx_process.restype = ctypes.c_int
        L.gen_ldpc_parameters.argtypes = [ctypes.POINTER(RefConfig), ctypes.POINTER(InConfig)]
        L.gen_ldpc_parameters.restype = ctypes.c_int
        L.calculate_crc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.calculate_crc.restype = ctypes.c_uint32
        for acc in ("ref_fixed_lq", "ref_degree_lq", "ref_neural_lq"):
            getattr(L, acc).restype = ctypes.POINTER(ctypes.c_int16)
        L.ref_float_lq.restype = ctypes.POINTER(ctypes.c_float)
        L.ref_modulate_symbols.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint16, ctypes.c_void_p]
        L.ref_demap_symbols.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint16, ctypes.c_float,
                                        ctypes.c_void_p, ctypes.c_void_p]
        self.libc = ctypes.CDLL(None)

    def modulate_symbols(self, bits: np.ndarray, Qm: int) -> np.ndarray:
        """The reference's modulate_symbol (c_lib/tx_rx_process.c:68) on each group
        of Qm bits: uint8 [n, Qm] -> float32 [n, 2]."""
        b = np.ascontiguousarray(bits, dtype=np.uint8).reshape(-1, Qm)
        out = np.zeros((b.shape[0], 2), dtype=np.float32)
        self.lib.ref_modulate_symbols(_p(b), b.shape[0], Qm, _p(out))
        return out

    def demap_symbols(self, sym: np.ndarray, Qm: int, noise_power_db: float, want_float: bool = False):
        """The reference's demodulate_symbol + quantize_llr_to_int16
        (c_lib/tx_rx_process.c:234, :27) on given noisy symbols float32 [n, 2],
        with the noise variance computed as tx_rx_process does (:298)."""
        s = np.ascontiguousarray(sym, dtype=np.float32).reshape(-1, 2)
        q = np.zeros(s.shape[0] * Qm, dtype=np.int16)
        f = np.zeros(s.shape[0] * Qm, dtype=np.float32) if want_float else None
        self.lib.ref_demap_symbols(_p(s), s.shape[0], Qm, ctypes.c_float(noise_power_db), _p(q),
                                   _p(f) if f is not None else None)
        return (q, f) if want_float else q

    def srand(self, seed: int):
        self.libc.srand(ctypes.c_uint(seed))

    def gen(self, cfg: InConfig):
        rc_cfg = RefConfig()
        rc = self.lib.gen_ldpc_parameters(ctypes.byref(rc_cfg), ctypes.byref(cfg))
        return rc, rc_cfg

    def encode(self, payload: np.ndarray, cfg: InConfig) -> np.ndarray:
        payload = np.ascontiguousarray(payload, dtype=np.uint8)
        out = np.zeros((cfg.E + 7) // 8 + 8, dtype=np.uint8)
        rc = self.lib.c_ldpc_5g_encode(_p(payload), _p(out), ctypes.byref(cfg))
        assert rc == 0, rc
        return out[: (cfg.E + 7) // 8].copy()

    def channel(self, rm_bytes: np.ndarray, E: int, Qm: int, noise_db: float) -> np.ndarray:
        rm_bytes = np.ascontiguousarray(rm_bytes, dtype=np.uint8)
        out = np.zeros(E, dtype=np.int16)
        rc = self.lib.tx_rx_process(_p(rm_bytes), E, Qm, ctypes.c_float(noise_db), _p(out))
        assert rc == 0
        return out

    def decode(self, llr: np.ndarray, cfg: InConfig, dcfg: DecCfg):
        """Returns (status, hardbits, final LQ copy)."""
        rc, p = self.gen(cfg)
        llr = np.ascontiguousarray(llr, dtype=np.int16)
        B = p.B if rc == 0 else 8448
        bits = np.zeros((B + 7) // 8, dtype=np.uint8)
        st = self.lib.c_ldpc_5g_decode(_p(llr), _p(bits), ctypes.byref(cfg), ctypes.byref(dcfg))
        lq = None
        if rc == 0 and st >= 0:
            n = p.N + 2 * p.Zc
            acc = {1: self.lib.ref_fixed_lq, 2: self.lib.ref_neural_lq, 3: self.lib.ref_degree_lq,
                   0: self.lib.ref_float_lq, 4: self.lib.ref_float_lq}[dcfg.algo]
            lq = np.ctypeslib.as_array(acc(), shape=(n,)).copy()
        return int(st), bits, lq

    def harq_memory(self, n: int) -> np.ndarray:
        arr = (ctypes.c_int16 * (68 * 384)).in_dll(self.lib, "HARQ_memory")
        return np.ctypeslib.as_array(arr)[:n].copy()
