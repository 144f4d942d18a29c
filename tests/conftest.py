"""Shared pytest configuration: the ``gpu`` marker and golden-fixture loading."""

import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")


def load_golden(name: str) -> dict:
    """Inputs and upstream FP64 outputs of one synthetic configuration (see tests/golden/make_golden.py)."""
    d = dict(np.load(os.path.join(GOLDEN, f"{name}.npz"), allow_pickle=False))
    inp = {k: v for k, v in d.items() if not k.startswith("ref_")}
    ref = {k[4:]: v for k, v in d.items() if k.startswith("ref_")}
    inp["nk"] = tuple(int(x) for x in inp["nk"])
    for k in ("beta", "mu"):
        inp[k] = float(inp[k])
    for k in ("niw", "niv_core", "niv_shell"):
        inp[k] = int(inp[k])
    for k in ("chi_loc_sum_dens", "chi_loc_sum_magn"):
        inp[k] = complex(inp[k])
    return inp, ref


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b))) / scale


GOLDEN_CONFIGS = ("t1", "t1b", "t2", "t3", "t4e", "t5e", "t3a")
