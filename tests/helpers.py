"""Shared test helpers: golden fixtures, relative errors, GPU runners."""
from __future__ import annotations

import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SMALL_CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                     if not os.path.basename(p).startswith(("cfg_", "poisson_")))
GRAD_KEYS = ("g_pos", "g_scl", "g_rot", "g_dr", "g_di")
FWD_TOL = 1e-5   # relative L2, forward vs the FP64 oracle
GRAD_TOL = 1e-4  # relative L2, every gradient vs the FP64 oracle


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def params_of(z):
    return (z["positions"], z["scales"], z["rotations"], z["density_r"], z["density_i"])


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    b = np.asarray(b, dtype=a.dtype)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))
