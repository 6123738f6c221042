"""torch.ops.nrldpc.ldpc_decode without a GPU: the fake (meta) implementation's
output shapes and types under FakeTensorMode, and the dispatcher's refusal of
CPU tensors (the operator has a CUDA kernel only)."""

import pytest
import torch
from torch._subclasses.fake_tensor import FakeTensorMode

from deeplearning_5g_ldpc_decoder_b200 import code_params, ops  # noqa: F401  (registers the operator)

CASES = [((2, 488, 1, 1920, 0, 2, 0), 1), ((1, 8424, 1, 25344, 0, 8, 0), 0), ((1, 72, 2, 400, 2, 4, 0), 4),
         ((2, 1000, 1, 3000, 1, 6, 0), 3)]


@pytest.mark.parametrize("cfg,algo", CASES)
@pytest.mark.parametrize("return_app", [False, True])
def test_fake_shapes(cfg, algo, return_app):
    p = code_params(cfg)
    row = [algo, 8, 22936, 0, 1280, 32767, -32767]
    with FakeTensorMode():
        llr = torch.empty((7, cfg[3]), dtype=torch.int16, device="cuda")
        bits, status, iters, app = torch.ops.nrldpc.ldpc_decode(llr, list(cfg), row, return_app)
    assert bits.shape == (7, (p.B + 7) // 8) and bits.dtype == torch.uint8
    assert status.shape == (7,) and status.dtype == torch.int32 and iters.dtype == torch.int32
    assert app.shape == (7, p.N + 2 * p.Zc if return_app else 0)
    assert app.dtype == (torch.float32 if algo in (0, 4) else torch.int16)
    assert bits.device.type == "cuda"


def test_cpu_tensors_have_no_kernel():
    with pytest.raises(NotImplementedError):
        torch.ops.nrldpc.ldpc_decode(torch.zeros((2, 1920), dtype=torch.int16), [2, 488, 1, 1920, 0, 2, 0],
                                     [1, 10, 22936, 0, 1280, 32767, -32767], False)


def test_fake_rejects_bad_inputs():
    with FakeTensorMode():
        llr = torch.empty((3, 100), dtype=torch.int16, device="cuda")
        with pytest.raises(ValueError):
            torch.ops.nrldpc.ldpc_decode(llr, [2, 8000, 1, 9000, 0, 2, 0], [1, 8, 1, 0, 0, 1, -1], False)
        with pytest.raises(ValueError):
            torch.ops.nrldpc.ldpc_decode(llr.float(), [2, 488, 1, 1920, 0, 2, 0], [1, 8, 1, 0, 0, 1, -1], False)
