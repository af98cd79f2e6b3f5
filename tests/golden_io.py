"""Helpers that load the committed golden fixtures."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cplx(a):
    a = np.asarray(a, dtype=np.float64)
    return a[..., 0] + 1j * a[..., 1]


def sdet_kats():
    with open(os.path.join(HERE, "sdet_kats.json")) as f:
        k = json.load(f)
    out = {}
    for key, v in k.items():
        if isinstance(v, list):
            out[key] = cplx(v)
        else:
            out[key] = v
    return out
