"""Shared helpers for the parity tests."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)

import make_golden  # noqa: E402
from ns2d import abi  # noqa: E402


def load_case(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    p = abi.params_from_arrays(z["param_names"], z["params"])
    outs = [z[f"out{i}"] for i in range(int(z["n_out"]))]
    return p, z["w0"], outs


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / scale)
