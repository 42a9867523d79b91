import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def load_golden(path):
    z = np.load(path)
    g = {k: z[k] for k in z.files}
    L = int(g["num_levels"])
    g["levels"] = [(g[f"in{l}_src"], g[f"in{l}_dst"], g[f"in{l}_dsrc"], g[f"in{l}_ddst"],
                    g[f"in{l}_w"]) for l in range(L)]
    g["name"] = os.path.basename(path)[:-4]
    return g


@pytest.fixture(params=GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def golden(request):
    return load_golden(request.param)

