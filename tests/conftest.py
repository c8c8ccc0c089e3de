import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases(kind=None):
    out = []
    for name in sorted(os.listdir(GOLDEN)):
        p = os.path.join(GOLDEN, name, "golden.npz")
        if not os.path.exists(p):
            continue
        z = np.load(p)
        large = "sha_list_1" in z.files
        if kind == "large" and not large:
            continue
        if kind == "small" and large:
            continue
        if kind == "lanczos" and (large or "steps" not in z.files):
            continue
        if kind == "tpq" and (large or "tpq" not in z.files):
            continue
        if kind == "lobpcg" and (large or "lobpcg_steps" not in z.files):
            continue
        if kind == "lanczos_or_tpq" and (large or ("steps" not in z.files and "tpq" not in z.files)):
            continue
        if kind == "eigenvector" and (large or "energy_state" not in z.files):
            continue
        out.append(name)
    return out


def case_dir(name):
    return os.path.join(GOLDEN, name)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name, "golden.npz")))
