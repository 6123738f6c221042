"""B200-native 5G NR LDPC receive path: rate recovery, layered decoding
(BP, fixed/trained/degree min-sum, float min-sum) and CRC early termination,
as hand-written sm_100a CUDA behind the reference's C ABI."""

from .capi import (  # noqa: F401
    DecoderConfig,
    LdpcConfig,
    LdpcInConfig,
    load_library,
    make_decoder_config,
    make_in_config,
)

__all__ = [
    "DecoderConfig",
    "LdpcConfig",
    "LdpcInConfig",
    "load_library",
    "make_decoder_config",
    "make_in_config",
    "ldpc_decode",
    "ldpc_decode_host",
    "ldpc_encode",
    "channel_llrs",
]


def __getattr__(name):
    # torch is imported lazily so the ctypes layer works without it.
    if name in ("ldpc_decode", "ldpc_decode_host", "ldpc_encode", "channel_llrs", "code_params", "set_trained_weights", "set_degree_alpha",
                "DecodeResult"):
        from . import decoder

        return getattr(decoder, name)
    if name == "ops":
        # importing it registers torch.ops.nrldpc.ldpc_decode
        import importlib

        return importlib.import_module(".ops", __name__)
    raise AttributeError(name)
