"""Generate tests/golden/poisson_masks.npz by running the REFERENCE's own
variable-density Poisson-disc mask generator
(3DGS/3dgsVC/data/mask_generator.py: gen_pdf, PoissonDiscGenerator,
gen_poisson_mask), which needs numpy only.

For each case the global numpy state is seeded (np.random.seed(seed)), as a
caller of the reference would, and the reference's mask is stored packed
together with its pdf's SHA-256 and a seeded sample of pdf values.  The
pixel visiting order the reference draws is np.random.permutation(ny*nz)
from that state, i.e. np.random.RandomState(seed).permutation(ny*nz).

    python tests/golden/make_poisson_golden.py --reference /path/to/GS_TMI
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# (ny, nz, accel, calib, seed)
CASES = [
    (32, 28, 4.0, 8, 1),
    (48, 40, 6.0, 12, 2),
    (64, 64, 8.0, 16, 3),
    (128, 96, 6.0, 24, 4),
    (256, 160, 8.0, 24, 5),
    (16, 16, 4.0, 24, 6),     # calibration square wider than the plane (negative slice start)
    (32, 32, 12.0, 24, 7),    # calibration alone reaches the target
    (37, 53, 5.0, 10, 8),     # odd sizes
]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout (contains 3DGS/)")
    a = ap.parse_args()
    sys.path.insert(0, os.path.join(a.reference, "3DGS", "3dgsVC", "data"))
    import mask_generator as mg

    out = {}
    for k, (ny, nz, accel, calib, seed) in enumerate(CASES):
        np.random.seed(seed)
        mask = np.asarray(mg.gen_poisson_mask((ny, nz), accel, calib), dtype=np.int8)
        pdf = mg.gen_pdf((ny, nz), accel, calib, 2.0)
        pick = np.random.RandomState(1000 + k).randint(0, ny * nz, 64)
        out[f"case{k}_params"] = np.array([ny, nz, accel, calib, seed], np.float64)
        out[f"case{k}_mask"] = np.packbits(mask.reshape(-1))
        out[f"case{k}_pdf_sha256"] = np.frombuffer(hashlib.sha256(np.ascontiguousarray(pdf).tobytes()).digest(),
                                                   np.uint8)
        out[f"case{k}_pdf_pick"] = pick.astype(np.int64)
        out[f"case{k}_pdf_values"] = pdf.reshape(-1)[pick]
        print(ny, nz, accel, calib, seed, int(mask.sum()))
    np.savez_compressed(os.path.join(HERE, "poisson_masks.npz"), ncases=np.array(len(CASES)), **out)


if __name__ == "__main__":
    main()
