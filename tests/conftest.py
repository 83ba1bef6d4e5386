import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def small_states():
    from gexs_b200 import synth
    return synth.make_states(3000, 40, 1001)


@pytest.fixture(scope="session")
def small_lines(small_states):
    from gexs_b200 import synth
    return synth.make_lines(small_states, 4000, 100.0, 4000.0, 2001, broadening_seed=3001)


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from gexs_b200 import Context
    return Context(0)
