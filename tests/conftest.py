import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_vectors.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


@pytest.fixture(scope="session")
def reflib():
    from oracle.oracle import REF_SO, RefLib

    if not os.path.exists(REF_SO):
        pytest.skip("reference library not built here (oracle/build_ref.sh needs the reference tree)")
    return RefLib()


@pytest.fixture(scope="session")
def lib():
    from deeplearning_5g_ldpc_decoder_b200 import capi

    return capi.load_library()


@pytest.fixture(scope="session")
def cuda():
    """The GPU tests must run on the CUDA path; they fail (not skip) without a GPU."""
    import torch

    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    torch.cuda.init()
    return torch.device("cuda:0")
