import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    with np.load(os.path.join(GOLDEN, "aggregation_golden.npz")) as z:
        return {k: z[k] for k in z.files}


def golden_csr(g, key):
    from oracle.oracle import Csr
    off = g[key + "/offsets"]
    return Csr(len(off) - 1, off, g[key + "/indices"], g[key + "/values"])


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("CUDA device required")
    import thermofem_b200 as tf
    return tf.Context(0)


def to_device(a, dtype=None, index_dtype=None):
    """oracle.Csr or (offsets, indices, values) -> thermofem_b200.DeviceCsr."""
    import torch
    import thermofem_b200 as tf
    if isinstance(a, tuple):
        off, idx, val = a
    else:
        off, idx, val = a.offsets, a.indices, a.values
    return tf.DeviceCsr.from_host(off, idx, val, dtype=dtype or torch.float64, index_dtype=index_dtype or torch.int32)
