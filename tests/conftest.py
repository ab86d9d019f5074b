import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "donof.jl_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libdonofb200.so")


@pytest.fixture(scope="session")
def cuda_ctx():
    import torch
    import donof_b200 as d

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = d.Context(0)
    yield ctx
    ctx.close()
