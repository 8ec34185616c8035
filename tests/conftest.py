import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: large inputs")


def golden_cases():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    n_grp = int(d["n_grp"])
    N = len(d["dims"])
    d["groups"] = [{"memo_mode": int(d[f"g{g}_memo_mode"]), "begin_imten": int(d[f"g{g}_begin_imten"]),
                    "n_imten": int(d[f"g{g}_n_imten"]), "o_opt": [int(x) for x in d[f"g{g}_o_opt"]]}
                   for g in range(n_grp)]
    d["N"] = N
    d["dims_list"] = [int(x) for x in d["dims"]]
    return d


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    import adatm_b200 as A
    A.lib()
    return A
