"""Poisson-disc k-space masks on the CPU: the oracle's sequential dart
throwing and the package's numpy restatement of the pdf and exclusion radius
against golden masks made by the reference's own generator
(tests/golden/make_poisson_golden.py; mask_generator.py:22-63, :132-390)."""
import hashlib
import os

import numpy as np
import pytest

from gs_tmi_b200 import masks
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "poisson_masks.npz")


def cases():
    g = np.load(GOLDEN)
    for k in range(int(g["ncases"])):
        ny, nz, accel, calib, seed = g[f"case{k}_params"]
        ny, nz, calib, seed = int(ny), int(nz), int(calib), int(seed)
        mask = np.unpackbits(g[f"case{k}_mask"])[:ny * nz].reshape(ny, nz).astype(np.int8)
        yield (ny, nz, float(accel), calib, seed), mask, g, k


@pytest.mark.parametrize("k", range(8))
def test_pdf_restatement_matches_reference(k):
    (ny, nz, accel, calib, seed), _, g, k = list(cases())[k]
    pdf = masks.gen_pdf((ny, nz), accel, calib)
    sha = hashlib.sha256(np.ascontiguousarray(pdf).tobytes()).digest()
    assert sha == g[f"case{k}_pdf_sha256"].tobytes()
    assert np.array_equal(pdf.reshape(-1)[g[f"case{k}_pdf_pick"]], g[f"case{k}_pdf_values"])


@pytest.mark.parametrize("k", range(8))
def test_oracle_matches_reference_masks(k):
    (ny, nz, accel, calib, seed), ref, _, _ = list(cases())[k]
    order = np.random.RandomState(seed).permutation(ny * nz).astype(np.int32)
    radius = masks.exclusion_radius((ny, nz), accel, calib)
    out = oracle.poisson_mask(radius, order, (ny, nz), calib, masks.target_points((ny, nz), accel))
    assert np.array_equal(out, ref)
    assert int(out.sum()) == max(masks.target_points((ny, nz), accel), int(ref.sum()))
