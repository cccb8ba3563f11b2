import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def rel_max(a, b):
    """max_i |a_i - b_i| / RMS(|b_i|) over rows (vectors) or entries."""
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if b.ndim == 2:
        scale = np.sqrt((b ** 2).sum(1).mean())
        return float(np.sqrt(((a - b) ** 2).sum(1)).max() / scale)
    scale = np.sqrt((b ** 2).mean())
    return float(np.abs(a - b).max() / scale)


def rel_rms(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
