import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    """A golden fixture written by the reference (tests/golden/make_golden.py)."""
    import numpy as np
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    if "meta_keys" not in z.files:          # the coefficient-program fixtures carry no metadata
        return z, {}
    meta = dict(zip([str(k) for k in z["meta_keys"]], [str(v) for v in z["meta_vals"]]))
    return z, meta


# the assembled-problem fixtures; those with "_pc_" also hold the ILU(0)/SSOR-preconditioned CG
# and pin the oracle only (the GPU tests run over GOLDEN_CASES)
_ALL = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and not f.startswith("integrand_"))
GOLDEN_CASES = [n for n in _ALL if "_pc_" not in n and "_ds_" not in n]
PC_CASES = [n for n in _ALL if "_pc_" in n]
DS_CASES = [n for n in _ALL if "_ds_" in n]     # free space with ds (Robin) terms: oracle only
INTEGRAND_CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f.startswith("integrand_"))
