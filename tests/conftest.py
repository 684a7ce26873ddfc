import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_names():
    """The mesh cases of tests/golden (flow_cases.npz holds the incompressible-step runs)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("flow_"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    g = {k: z[k] for k in z.files}
    s = g["sizes"]
    g["n_cells"], g["n_internal_faces"], g["n_faces"] = int(s[0]), int(s[1]), int(s[2])
    return g


def golden_hierarchy(g):
    return [{f: g[f"lev{k}_{f}"] for f in ("l", "u", "weight", "agg", "faceMap", "faceFlip")}
            for k in range(int(g["nlevels"]))]


def perf_dict(a):
    return dict(initialResidual=a[0], finalResidual=a[1], residualSum=a[2], normFactor=a[3], iterations=int(a[4]),
                converged=bool(a[5]))


@pytest.fixture(params=golden_names())
def golden(request):
    return load_golden(request.param)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
