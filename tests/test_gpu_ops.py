"""torch.ops.nrldpc.ldpc_decode on the GPU: same results as the ctypes API,
torch.library.opcheck (schema, fake implementation, dispatch), and use inside
a torch.compile'd function."""

import pytest
import torch

from deeplearning_5g_ldpc_decoder_b200 import ldpc_decode, ops  # noqa: F401
from oracle.oracle import in_config, make_llrs

pytestmark = pytest.mark.gpu

CFG = [2, 488, 1, 1920, 0, 2, 0]


def test_op_equals_ctypes_api_and_passes_opcheck(oracle, cuda):
    llr_h, _ = make_llrs(oracle, in_config(*CFG), 40, noise_db=-1.0, seed=3)
    llr = torch.from_numpy(llr_h).to(cuda)
    for row in ([1, 10, 22936, 0, 1280, 32767, -32767], [0, 10, 22936, 0, 1280, 32767, -32767],
                [4, 10, 22936, 0, 1280, 32767, -32767]):
        want = ldpc_decode(llr, CFG, row, return_app=True)
        bits, status, iters, app = torch.ops.nrldpc.ldpc_decode(llr, CFG, row, True)
        assert torch.equal(bits, want.hardbits) and torch.equal(status, want.status)
        assert torch.equal(iters, want.iterations) and torch.equal(app, want.app)
        torch.library.opcheck(ops.ldpc_decode_op, (llr, CFG, row, True),
                              test_utils=("test_schema", "test_faketensor"))
        torch.library.opcheck(ops.ldpc_decode_op, (llr, CFG, row, False),
                              test_utils=("test_schema", "test_faketensor"))


def test_op_inside_torch_compile(oracle, cuda):
    llr_h, pay = make_llrs(oracle, in_config(*CFG), 64, noise_db=-1.0, seed=4)
    llr = torch.from_numpy(llr_h).to(cuda)
    row = [1, 10, 22936, 0, 1280, 32767, -32767]
    payload = torch.from_numpy(pay).to(cuda)

    def block_errors(x):
        bits, status, _, _ = torch.ops.nrldpc.ldpc_decode(x, CFG, row, False)
        ok = (status == 0) & (bits[:, : CFG[1] // 8] == payload).all(dim=1)
        return (~ok).sum()

    eager = block_errors(llr)
    compiled = torch.compile(block_errors, fullgraph=True)(llr)
    assert int(compiled) == int(eager)
