"""Loader for the committed golden fixtures (produced from the reference by make_golden.py)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NAMES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
               if not os.path.basename(p).startswith("softening"))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    bodies = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    return bodies, z
