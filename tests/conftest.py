import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a) and libhpblas1.so")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_golden(name):
    """Yield (meta, arrays-dict) per case of a golden .npz file."""
    import re
    z = np.load(GOLDEN / name)
    meta = json.loads(bytes(z["meta"]).decode())
    groups = [dict() for _ in meta]
    for k in z.files:
        if k == "meta":
            continue
        m = re.fullmatch(r"(\w+?)__(\d+)", k)
        groups[int(m.group(2))][m.group(1)] = z[k]
    return list(zip(meta, groups))


@pytest.fixture(scope="session")
def gpu():
    """(Context, torch) on cuda:0; the context runs on torch's current stream."""
    import torch
    from high_precision_blas1_b200 import Context
    ctx = Context(0, torch.cuda.current_stream().cuda_stream)
    yield ctx, torch
    torch.cuda.synchronize()
    ctx.close()
