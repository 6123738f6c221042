"""ctypes binding of ``libnrldpc_b200.so`` (the C ABI in include/nrldpc_b200.h).

The record classes mirror the reference's ctypes structs
(scripts/ldpc_c_sim_common.py:32-57, deep_learning/ldpc_table_config.py:19-54)
field for field, so either set of classes can be passed to either library.
"""

from __future__ import annotations

import ctypes
import os
import threading

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libnrldpc_b200.so")

NRLDPC_OK = 0
NRLDPC_NOT_CONVERGED = 1
NRLDPC_ERR_CUDA = -1
NRLDPC_ERR_CONFIG = -2
NRLDPC_ERR_ALGO = -3
NRLDPC_ERR_ARG = -4

BG_ROWS = {1: 46, 2: 42}
BG_COLS = {1: 68, 2: 52}
BG_NNZ = {1: 316, 2: 197}


class LdpcInConfig(ctypes.Structure):
    """ldpc_in_config_t: seven uint16_t (c_lib/nr_ldpc.h:42-50)."""

    _fields_ = [(n, ctypes.c_uint16) for n in ("bgn", "A", "crctype", "E", "rv", "Qm", "HARQ_on")]


class DecoderConfig(ctypes.Structure):
    """ldpc_decoder_cfg_t (c_lib/nr_ldpc.h:82-90)."""

    _fields_ = [
        ("algo", ctypes.c_uint16),
        ("max_iterations", ctypes.c_uint16),
        ("alpha", ctypes.c_uint16),
        ("beta", ctypes.c_uint16),
        ("filling_bit_value", ctypes.c_int16),
        ("max_llr", ctypes.c_int16),
        ("min_llr", ctypes.c_int16),
    ]


class LdpcConfig(ctypes.Structure):
    """ldpc_config_t (c_lib/nr_ldpc.h:54-79)."""

    _fields_ = [(n, ctypes.c_uint16) for n in (
        "bgn", "A", "crctype", "E", "rv", "Qm", "HARQ_on", "B", "Zc", "iLS", "K", "F", "N", "k0")] + [
        ("Vij_array", ctypes.POINTER(ctypes.c_uint16)),
        ("HBG_array", ctypes.POINTER(ctypes.c_uint16)),
        ("HBG_offset_array", ctypes.POINTER(ctypes.c_uint16)),
    ]


class TbDesc(ctypes.Structure):
    """nrldpc_tb_t: one transport block of a batch (32 bytes)."""

    _fields_ = [("A", ctypes.c_int32), ("G", ctypes.c_int32), ("Qm", ctypes.c_uint16), ("rv", ctypes.c_uint16),
                ("bgn", ctypes.c_uint16), ("flags", ctypes.c_uint16), ("llr_offset", ctypes.c_int64),
                ("out_offset", ctypes.c_int64), ("tbs_lbrm", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("harq_offset", ctypes.c_int64)]


class TbInfo(ctypes.Structure):
    """nrldpc_tb_info_t: segmentation of one transport block."""

    _fields_ = [("C", ctypes.c_int32), ("L_tb", ctypes.c_int32), ("Kp", ctypes.c_int32), ("Zc", ctypes.c_int32),
                ("E_lo", ctypes.c_int32), ("E_hi", ctypes.c_int32), ("n_lo", ctypes.c_int32),
                ("cb_cfg", LdpcInConfig), ("Ncb", ctypes.c_int32), ("k0", ctypes.c_int32),
                ("harq_elems", ctypes.c_int64)]


class ServeConfig(ctypes.Structure):
    """nrldpc_serve_cfg_t."""

    _fields_ = [("max_batch_tbs", ctypes.c_int32), ("max_batch_cbs", ctypes.c_int32),
                ("llr_budget_bytes", ctypes.c_int64), ("pipeline_depth", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("timeout_s", ctypes.c_double), ("max_wait_s", ctypes.c_double),
                ("h_cb_first", ctypes.c_void_p), ("d_cb_bits", ctypes.c_void_p), ("d_cb_status", ctypes.c_void_p),
                ("d_cb_iterations", ctypes.c_void_p)]


class ServeStats(ctypes.Structure):
    """nrldpc_serve_stats_t."""

    _fields_ = [("admitted", ctypes.c_int64), ("dropped", ctypes.c_int64), ("completed", ctypes.c_int64),
                ("failed", ctypes.c_int64), ("batches", ctypes.c_int64), ("wall_s", ctypes.c_double),
                ("mean_batch_tbs", ctypes.c_double), ("expired", ctypes.c_int64)]


NRLDPC_TB_DROPPED = -5
NRLDPC_TB_EXPIRED = -6
NRLDPC_TB_HARQ_COMBINE = 1
NRLDPC_TB_HARQ_STORE = 2


def make_decoder_config(values) -> DecoderConfig:
    """Row [algo, max_iterations, alpha, beta, filling_bit_value, max_llr, min_llr]
    (scripts/ldpc_c_sim_common.py:112-122)."""
    return DecoderConfig(*[int(v) for v in values])


def make_in_config(bgn, A, crctype, E, rv=0, Qm=2, HARQ_on=0) -> LdpcInConfig:
    return LdpcInConfig(bgn, A, crctype, E, rv, Qm, HARQ_on)


_lock = threading.Lock()
_lib = None

EXPORTED_SYMBOLS = (
    "gen_ldpc_parameters",
    "cuda_ldpc_5g_decode",
    "c_ldpc_5g_decode",
    "cuda_ldpc_5g_encode",
    "c_ldpc_5g_encode",
    "calculate_crc",
    "tx_rx_process",
    "nrldpc_encode_batch",
    "nrldpc_encode_batch_ncb",
    "nrldpc_channel_batch",
    "nrldpc_channel_seed",
    "nrldpc_decode_batch",
    "nrldpc_decode_batch_host",
    "nrldpc_decode_batch_noalloc",
    "nrldpc_train_forward",
    "nrldpc_train_backward",
    "nrldpc_train_forward_f64",
    "nrldpc_train_backward_f64",
    "nrldpc_train_checkpoint_words",
    "nrldpc_set_trained_weights",
    "nrldpc_set_degree_alpha",
    "nrldpc_mixed_plan_create",
    "nrldpc_mixed_plan_execute",
    "nrldpc_mixed_plan_autotune",
    "nrldpc_mixed_plan_select",
    "nrldpc_mixed_plan_destroy",
    "nrldpc_tb_segment",
    "nrldpc_tb_select_bg",
    "nrldpc_tb_engine_create",
    "nrldpc_tb_engine_destroy",
    "nrldpc_tb_engine_decode",
    "nrldpc_tb_engine_views",
    "nrldpc_serve_run",
    "nrldpc_kernel_launch_count",
    "nrldpc_version",
    "nrldpc_bounds_check_status",
)


def load_library(path: str | None = None) -> ctypes.CDLL:
    """Load the CUDA library (building it first if it is missing and nvcc exists).

    Raises if the library cannot be found or built: there is no CPU fallback.
    """
    global _lib
    with _lock:
        if _lib is not None and path is None:
            return _lib
        p = path or LIB_PATH
        if not os.path.exists(p):
            from .build import build_library

            p = build_library()
        lib = ctypes.CDLL(p)
        _declare(lib)
        if path is None:
            _lib = lib
        return lib


def _declare(lib: ctypes.CDLL) -> None:
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    lib.gen_ldpc_parameters.argtypes = [ctypes.POINTER(LdpcConfig), ctypes.POINTER(LdpcInConfig)]
    lib.gen_ldpc_parameters.restype = ctypes.c_int
    for name in ("cuda_ldpc_5g_decode", "c_ldpc_5g_decode"):
        f = getattr(lib, name)
        f.argtypes = [vp, vp, ctypes.POINTER(LdpcInConfig), ctypes.POINTER(DecoderConfig)]
        f.restype = i32
    for name in ("cuda_ldpc_5g_encode", "c_ldpc_5g_encode"):
        f = getattr(lib, name)
        f.argtypes = [vp, vp, ctypes.POINTER(LdpcInConfig)]
        f.restype = i32
    lib.nrldpc_encode_batch.argtypes = [vp, i64, i32, ctypes.POINTER(LdpcInConfig), vp, i64, vp]
    lib.nrldpc_channel_batch.argtypes = [vp, i64, i32, i32, i32, ctypes.c_float, ctypes.c_uint64, vp, i64, vp, vp]
    lib.nrldpc_channel_batch.restype = i32
    lib.nrldpc_channel_seed.argtypes = [ctypes.c_uint64]
    lib.nrldpc_channel_seed.restype = None
    lib.tx_rx_process.argtypes = [vp, ctypes.c_size_t, ctypes.c_uint16, ctypes.c_float, vp]
    lib.tx_rx_process.restype = ctypes.c_int
    lib.nrldpc_encode_batch.restype = i32
    lib.calculate_crc.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.calculate_crc.restype = ctypes.c_uint32
    lib.nrldpc_decode_batch.argtypes = [vp, i64, i32, ctypes.POINTER(LdpcInConfig), ctypes.POINTER(DecoderConfig),
                                        vp, i64, vp, vp, vp, i64, vp, i64, vp]
    lib.nrldpc_decode_batch.restype = i32
    lib.nrldpc_decode_batch_noalloc.argtypes = [vp, i64, i32, ctypes.POINTER(LdpcInConfig),
                                                ctypes.POINTER(DecoderConfig), vp, i64, vp, vp, vp, i64, vp, i64, vp]
    lib.nrldpc_decode_batch_noalloc.restype = i32
    lib.nrldpc_decode_batch_host.argtypes = [vp, i64, i32, ctypes.POINTER(LdpcInConfig),
                                             ctypes.POINTER(DecoderConfig), vp, i64, vp, vp, vp]
    lib.nrldpc_decode_batch_host.restype = i32
    f32 = ctypes.c_float
    lib.nrldpc_train_forward.argtypes = [vp, i32, ctypes.POINTER(LdpcInConfig), i32, vp, vp, f32, vp, vp, vp, vp, vp]
    lib.nrldpc_train_forward.restype = i32
    lib.nrldpc_train_backward.argtypes = [vp, i32, ctypes.POINTER(LdpcInConfig), i32, vp, vp, f32, i32, vp, vp, vp,
                                          vp, vp, vp, vp, vp]
    lib.nrldpc_train_backward.restype = i32
    f64 = ctypes.c_double
    lib.nrldpc_train_forward_f64.argtypes = [vp, i32, ctypes.POINTER(LdpcInConfig), i32, vp, vp, f64, vp, vp, vp, vp,
                                             vp]
    lib.nrldpc_train_forward_f64.restype = i32
    lib.nrldpc_train_backward_f64.argtypes = [vp, i32, ctypes.POINTER(LdpcInConfig), i32, vp, vp, f64, i32, vp, vp,
                                              vp, vp, vp, vp, vp, vp]
    lib.nrldpc_train_backward_f64.restype = i32
    lib.nrldpc_train_checkpoint_words.argtypes = [ctypes.POINTER(LdpcInConfig), i32, i32, i32,
                                                  ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    lib.nrldpc_train_checkpoint_words.restype = i32
    lib.nrldpc_encode_batch_ncb.argtypes = [vp, i64, i32, ctypes.POINTER(LdpcInConfig), i32, vp, i64, vp]
    lib.nrldpc_encode_batch_ncb.restype = i32
    lib.nrldpc_tb_segment.argtypes = [ctypes.POINTER(TbDesc), ctypes.POINTER(TbInfo)]
    lib.nrldpc_tb_segment.restype = i32
    lib.nrldpc_tb_select_bg.argtypes = [i32, i32]
    lib.nrldpc_tb_select_bg.restype = i32
    lib.nrldpc_tb_engine_create.argtypes = [i32, i32, ctypes.POINTER(DecoderConfig), ctypes.POINTER(vp)]
    lib.nrldpc_tb_engine_create.restype = i32
    lib.nrldpc_tb_engine_destroy.argtypes = [vp]
    lib.nrldpc_tb_engine_destroy.restype = i32
    lib.nrldpc_tb_engine_decode.argtypes = [vp, vp, i32, vp, vp, vp, vp, vp, vp]
    lib.nrldpc_tb_engine_decode.restype = i32
    lib.nrldpc_tb_engine_views.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                           ctypes.POINTER(vp)]
    lib.nrldpc_tb_engine_views.restype = i32
    lib.nrldpc_serve_run.argtypes = [vp, ctypes.POINTER(ServeConfig), vp, vp, i32, vp, vp, vp, vp,
                                     ctypes.POINTER(ServeStats), vp]
    lib.nrldpc_serve_run.restype = i32
    lib.nrldpc_set_trained_weights.argtypes = [ctypes.c_uint16, vp, vp, i32]
    lib.nrldpc_set_trained_weights.restype = i32
    lib.nrldpc_set_degree_alpha.argtypes = [vp]
    lib.nrldpc_set_degree_alpha.restype = i32
    lib.nrldpc_kernel_launch_count.argtypes = []
    lib.nrldpc_kernel_launch_count.restype = i64
    lib.nrldpc_version.argtypes = []
    lib.nrldpc_version.restype = ctypes.c_char_p
    lib.nrldpc_bounds_check_status.argtypes = [vp, i32]
    lib.nrldpc_bounds_check_status.restype = i32


def gen_ldpc_parameters(cfg: LdpcInConfig, lib=None) -> LdpcConfig:
    lib = lib or load_library()
    out = LdpcConfig()
    if lib.gen_ldpc_parameters(ctypes.byref(out), ctypes.byref(cfg)) != 0:
        raise ValueError("invalid LDPC configuration")
    return out


def kernel_launch_count(lib=None) -> int:
    return int((lib or load_library()).nrldpc_kernel_launch_count())
