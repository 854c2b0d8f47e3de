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
    names = [str(s) for s in z["param_names"]]
    kw = {}
    for n, v in zip(names, z["params"]):
        t = dict(abi.Params._fields_)[n]
        kw[n] = float(v) if t.__name__ == "c_double" else int(v)
    p = abi.default_params(**kw)
    outs = [z[f"out{i}"] for i in range(int(z["n_out"]))]
    return p, z["w0"], outs


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.max(np.abs(b))
    if scale == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / scale)
