import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libpbgpu.so")


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


GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")


def load_golden():
    from parbutterfly_b200.graph import BipartiteGraph
    z = np.load(GOLDEN)
    names = sorted({k.split("/")[0] for k in z.files})
    out = {}
    for n in names:
        nv, nu, m = (int(x) for x in z[f"{n}/dims"])
        g = BipartiteGraph(nv, nu, z[f"{n}/offsetsV"].astype(np.uint32), z[f"{n}/edgesV"].astype(np.uint32),
                           z[f"{n}/offsetsU"].astype(np.uint32), z[f"{n}/edgesU"].astype(np.uint32))
        rec = {k[len(n) + 1:]: z[k] for k in z.files if k.startswith(n + "/")}
        out[n] = (g, rec)
    return out


@pytest.fixture(scope="session")
def golden():
    return load_golden()


@pytest.fixture(scope="session")
def ctx():
    from parbutterfly_b200.butterflies import Context
    c = Context(0)
    yield c
    c.close()
