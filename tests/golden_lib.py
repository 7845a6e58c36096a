"""Loads the golden fixtures of tests/golden/ (made by tests/golden/make_golden.py)."""
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load(path):
    z = np.load(path)
    ins = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    outs = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return ins, outs


def model(ins):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import model_from_arrays
    return model_from_arrays(ins)


def orbit_keys(outs):
    return sorted({k.split("_")[0] for k in outs if k.startswith("orbit") and k.endswith("_tall")})
