"""CPU oracle for the complex-Gaussian tile voxelizer -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker.  The product package
(``gs_tmi_b200``) never imports it and has no CPU fallback.

The numerical core lives in ``gsv_oracle.c`` (built by ``oracle/Makefile``
into ``oracle/_build/liborc.so``).  It restates, in FP64 with an FP32
inclusion predicate shared bit-for-bit with the CUDA kernels:

* preprocess  -- 3DGS/3dgsVC/gaussian/tile_voxelizer.py:282-290, :77-84
* binning     -- 3DGS/3dgsVC/gaussian/tile_voxelizer.py:87-162
* forward     -- 3DGS/3dgsVC/gaussian/tile_voxelizer.py:210-244 and
                 3DGS/3dgsVC/gaussian/cuda_ext/tile_voxelize_cuda_kernel.cu:118-135
* backward    -- tile_voxelize_cuda_kernel.cu:233-252 plus the torch autograd
                 chain through tile_voxelizer.py:282-290

Parity of this oracle with the reference itself is pinned by
``tests/golden/`` (fixtures generated by running the reference's own
PyTorch path; see ``tests/golden/make_golden.py``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")
_lib = None
_lock = threading.Lock()

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


def build() -> str:
    """Compile ``liborc.so`` if it is missing or older than its source."""
    src = os.path.join(_HERE, "gsv_oracle.c")
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_preprocess_f32.argtypes = [_f32p, _f32p, _f32p, _i64, _i32, _i32, _i32, _vp, _vp, _vp]
            L.orc_preprocess_f32.restype = None
            L.orc_qcoef_from_covinv_f32.argtypes = [_f32p, _f32p, _i64, _f32p]
            L.orc_qcoef_from_covinv_f32.restype = None
            L.orc_count_pairs.argtypes = [_f32p, _f32p, _i64, _i32, _i32, _i32, _i32, _i32p, _i32p]
            L.orc_count_pairs.restype = _i64
            L.orc_fill_pairs.argtypes = [_i32p, _i32p, _i64, _i32, _i32, _i32, _i32, _i32p, _i32p]
            L.orc_fill_pairs.restype = None
            common = [_i32] + [_vp] * 11 + [_i64, _i32, _i32, _i32, _i32, _i32p, _i32p]
            L.orc_forward.argtypes = common + [_f64p, _vp]
            L.orc_forward.restype = ctypes.c_int
            L.orc_backward.argtypes = common + [_i64, _f64p, _vp, _vp, _vp, _vp, _vp]
            L.orc_backward.restype = ctypes.c_int
            L.orc_candidate_evals.argtypes = [_i32p, _i32, _i32, _i32, _i32]
            L.orc_candidate_evals.restype = _i64
            L.orc_boundary_voxels.argtypes = [_f32p, _f32p, _f32p, _i64, _i32, _i32, _i32, _i32,
                                              _i32p, _i32p, ctypes.c_double,
                                              np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")]
            L.orc_boundary_voxels.restype = _i64
            L.orc_extent_check.argtypes = [_f32p, _f32p, _f32p, _i64, _i32, _i32, _i32, _i32p, _i32p,
                                           np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")]
            L.orc_extent_check.restype = _i64
            L.orc_poisson_mask.argtypes = [_f64p, _i32p, _i32, _i32, _i32, _i64,
                                           np.ctypeslib.ndpointer(dtype=np.int8, flags="C_CONTIGUOUS")]
            L.orc_poisson_mask.restype = _i64
            L.orc_set_predicate.argtypes = [ctypes.c_int]
            L.orc_set_predicate.restype = ctypes.c_int
            L.orc_predicate_flips.argtypes = [ctypes.c_int, _vp, _vp, _vp, _vp, _i64, _i32, _i32, _i32, _i32,
                                              _i32p, _i32p, ctypes.c_int, ctypes.c_int,
                                              np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS"), _vp]
            L.orc_predicate_flips.restype = ctypes.c_int
            L.orc_num_threads.argtypes = []
            L.orc_num_threads.restype = ctypes.c_int
            _lib = L
    return _lib


# Inclusion tests the oracle can evaluate (gsv_oracle.c, ORC_PRED_*):
ROWFORM = 0        # the kernels' voxel-unit row form, shared bit for bit
REFERENCE = 1      # the reference CUDA kernel's op order, IEEE division by hs
REFERENCE_RCP = 2  # the same with the division as a product by the reciprocal
_pred_lock = threading.Lock()


def _with_predicate(mode, fn):
    with _pred_lock:
        old = lib().orc_set_predicate(int(mode))
        try:
            return fn()
        finally:
            lib().orc_set_predicate(old)


def _c(a, dtype):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


# --------------------------------------------------------------------------
# preprocess / binning
# --------------------------------------------------------------------------

def preprocess_f32(positions, scales, rotations, shape):
    """FP32 center_vox [n,3], radius_vox [n] and kernel Q coefficients [n,6]."""
    p, s, q = _c(positions, np.float32), _c(scales, np.float32), _c(rotations, np.float32)
    n = p.shape[0]
    center = np.empty((n, 3), np.float32)
    radius = np.empty((n,), np.float32)
    qc = np.empty((n, 6), np.float32)
    lib().orc_preprocess_f32(p, s, q, n, *shape, _ptr(center), _ptr(radius), _ptr(qc))
    return center, radius, qc


def build_tile_pairs(center_vox, radius_vox, shape, tile_size):
    """(tile_ranges int32 [T,2], pair_ids int32 [P]) with ascending gid per tile.

    Mirrors tile_voxelizer.py:87-162 (canonical stable order)."""
    c, r = _c(center_vox, np.float32), _c(radius_vox, np.float32)
    n = c.shape[0]
    counts = np.zeros(max(n, 1), np.int32)
    box = np.zeros((max(n, 1), 6), np.int32)
    total = lib().orc_count_pairs(c, r, n, *shape, tile_size, counts, box)
    if total < 0:
        raise ValueError("a Gaussian has an empty tile box (negative radius)")
    d, h, w = shape
    ts = tile_size
    ntiles = -(-d // ts) * -(-h // ts) * -(-w // ts)
    ranges = np.zeros((ntiles, 2), np.int32)
    pair_ids = np.zeros(max(total, 1), np.int32)
    lib().orc_fill_pairs(counts, box, n, *shape, ts, ranges, pair_ids)
    return ranges, pair_ids[:total]


def candidate_evals(tile_ranges, shape, tile_size):
    return int(lib().orc_candidate_evals(_c(tile_ranges, np.int32), *shape, tile_size))


# --------------------------------------------------------------------------
# forward / backward
# --------------------------------------------------------------------------

def _args(compat, a, b, c, dr, di, hs, o64):
    a, b, c = _c(a, np.float32), _c(b, np.float32), _c(c, np.float32)
    dr, di, hs = _c(dr, np.float32), _c(di, np.float32), _c(hs, np.float32)
    o64 = o64 or {}
    keys = ("a", "b", "c", "dr", "di")
    ov = [_c(o64.get(k), np.float64) for k in keys]
    keep = [a, b, c, dr, di, hs] + ov
    ptrs = [_ptr(x) for x in keep]
    return keep, ptrs


def forward(params, shape, tile_size, tile_ranges, pair_ids, overrides64=None, compat=False,
            half_shape=None, predicate=ROWFORM):
    """FP64 complex volume [d,h,w] and stats (candidates, included).

    ``params`` = (positions, scales, rotations, density_r, density_i) or, with
    ``compat=True``, (center_vox, cov_inv[n,9], None, density_r, density_i).
    ``overrides64`` maps a/b/c/dr/di to FP64 arrays used for the arithmetic
    while the FP32 ``params`` fix the inclusion predicate (finite differences).
    ``predicate`` selects the FP32 inclusion test (ROWFORM, REFERENCE,
    REFERENCE_RCP); everything else stays FP64.
    """
    a, b, c, dr, di = params
    n = np.asarray(dr).shape[0]
    keep, ptrs = _args(compat, a, b, c, dr, di, half_shape, overrides64)
    d, h, w = shape
    vol = np.zeros(d * h * w * 2, np.float64)
    stats = np.zeros(2, np.int64)
    tr, pid = _c(tile_ranges, np.int32), _c(pair_ids, np.int32)
    if pid.size == 0:
        pid = np.zeros(1, np.int32)
    _with_predicate(predicate, lambda: lib().orc_forward(int(compat), *ptrs, n, d, h, w, tile_size, tr, pid, vol,
                                                        _ptr(stats)))
    del keep
    return (vol[0::2] + 1j * vol[1::2]).reshape(d, h, w), stats


def backward(params, shape, tile_size, tile_ranges, pair_ids, grad_vol, overrides64=None,
             compat=False, half_shape=None, predicate=ROWFORM):
    """FP64 gradients.  params mode -> (d_pos[n,3], d_scale[n,3], d_rot[n,4],
    d_rho_r[n], d_rho_i[n]); compat mode -> (d_center[n,3], d_cov_inv[n,3,3],
    None, d_rho_r[n], d_rho_i[n])."""
    a, b, c, dr, di = params
    n = np.asarray(dr).shape[0]
    keep, ptrs = _args(compat, a, b, c, dr, di, half_shape, overrides64)
    d, h, w = shape
    gv = np.empty(d * h * w * 2, np.float64)
    g = np.asarray(grad_vol).reshape(-1)
    gv[0::2] = g.real
    gv[1::2] = g.imag
    nn = max(n, 1)
    o1 = np.zeros(nn * 3)
    o2 = np.zeros(nn * (9 if compat else 3))
    o3 = np.zeros(nn * 4)
    o4 = np.zeros(nn)
    o5 = np.zeros(nn)
    tr, pid = _c(tile_ranges, np.int32), _c(pair_ids, np.int32)
    npairs = pid.size
    if npairs == 0:
        pid = np.zeros(1, np.int32)
    _with_predicate(predicate, lambda: lib().orc_backward(int(compat), *ptrs, n, d, h, w, tile_size, tr, pid,
                                                         npairs, gv, _ptr(o1), _ptr(o2), _ptr(o3), _ptr(o4),
                                                         _ptr(o5)))
    del keep
    if compat:
        return o1[: n * 3].reshape(n, 3), o2[: n * 9].reshape(n, 3, 3), None, o4[:n], o5[:n]
    return (o1[: n * 3].reshape(n, 3), o2[: n * 3].reshape(n, 3), o3[: n * 4].reshape(n, 4), o4[:n],
            o5[:n])


def voxelize(positions, scales, rotations, density_r, density_i, shape, tile_size):
    """Whole path on the CPU: preprocess, bin, FP64 forward."""
    center, radius, _ = preprocess_f32(positions, scales, rotations, shape)
    ranges, pids = build_tile_pairs(center, radius, shape, tile_size)
    vol, stats = forward((positions, scales, rotations, density_r, density_i), shape, tile_size,
                         ranges, pids)
    return vol, ranges, pids, stats


# --------------------------------------------------------------------------
# finite differences (FP64, inclusion predicate frozen at the base point)
# --------------------------------------------------------------------------

def fd_gradient(params, shape, tile_size, tile_ranges, pair_ids, grad_vol, which, index, h=1e-6,
                compat=False, half_shape=None):
    """Central difference of L = sum(Re(conj(g) * vol)) w.r.t. one scalar.

    ``which`` in a/b/c/dr/di names the parameter array, ``index`` the flat
    element.  The FP32 params keep the inclusion set fixed, so L is smooth in
    the perturbed FP64 copy and the difference converges at O(h^2)."""
    names = ("a", "b", "c", "dr", "di")
    base = {k: None if v is None else np.asarray(v, np.float64).copy() for k, v in zip(names, params)}
    g = np.asarray(grad_vol)

    def loss(delta):
        ov = {k: (v.copy() if v is not None else None) for k, v in base.items()}
        ov[which].reshape(-1)[index] += delta
        vol, _ = forward(params, shape, tile_size, tile_ranges, pair_ids, overrides64=ov,
                         compat=compat, half_shape=half_shape)
        return float(np.sum(vol.real * g.real + vol.imag * g.imag))

    return (loss(h) - loss(-h)) / (2 * h)


def predicate_flips(params, shape, tile_size, tile_ranges, pair_ids, mode_a=ROWFORM, mode_b=REFERENCE,
                    compat=False, half_shape=None, voxel_flags=False):
    """Listed candidates on which two FP32 inclusion tests disagree.

    Returns {"both", "a_only", "b_only", "candidates"} and, with
    ``voxel_flags``, a boolean [d,h,w] mask of the voxels with a
    disagreement.  ``params`` as in :func:`forward` (densities unused)."""
    a, b, c = params[:3]
    a, b, c = _c(a, np.float32), _c(b, np.float32), _c(c, np.float32)
    hs = _c(half_shape, np.float32)
    n = a.shape[0]
    d, h, w = shape
    out = np.zeros(4, np.int64)
    flags = np.zeros(d * h * w, np.uint8) if voxel_flags else None
    tr, pid = _c(tile_ranges, np.int32), _c(pair_ids, np.int32)
    if pid.size == 0:
        pid = np.zeros(1, np.int32)
    lib().orc_predicate_flips(int(compat), _ptr(a), _ptr(b), _ptr(c), _ptr(hs), n, d, h, w, tile_size, tr, pid,
                              int(mode_a), int(mode_b), out, _ptr(flags))
    res = {"both": int(out[0]), "a_only": int(out[1]), "b_only": int(out[2]), "candidates": int(out[3])}
    if voxel_flags:
        return res, flags.reshape(d, h, w).astype(bool)
    return res


def boundary_voxels(positions, scales, rotations, shape, tile_size, tile_ranges, pair_ids, tol=1e-4):
    """Boolean [d,h,w] mask of voxels with a listed pair whose FP64
    Mahalanobis distance is within ``tol`` of the 9.0 cutoff."""
    d, h, w = shape
    flags = np.zeros(d * h * w, np.uint8)
    pid = _c(pair_ids, np.int32)
    if pid.size == 0:
        pid = np.zeros(1, np.int32)
    lib().orc_boundary_voxels(_c(positions, np.float32), _c(scales, np.float32), _c(rotations, np.float32),
                              np.asarray(positions).shape[0], d, h, w, tile_size, _c(tile_ranges, np.int32),
                              pid, float(tol), flags)
    return flags.reshape(d, h, w).astype(bool)


def extent_check(positions, scales, rotations, shape, tile_ranges, pair_ids):
    """Checks the tile-8 kernels' extent cull against the shared FP32
    predicate: returns (included pairs the cull would drop -- must be 0,
    {"listed", "kept", "slots_kept"} counts)."""
    d, h, w = shape
    stats = np.zeros(3, np.int64)
    pid = _c(pair_ids, np.int32)
    if pid.size == 0:
        pid = np.zeros(1, np.int32)
    bad = lib().orc_extent_check(_c(positions, np.float32), _c(scales, np.float32), _c(rotations, np.float32),
                                 np.asarray(positions).shape[0], d, h, w, _c(tile_ranges, np.int32), pid, stats)
    return int(bad), {"listed": int(stats[0]), "kept": int(stats[1]), "slots_kept": int(stats[2])}


def num_threads() -> int:
    return int(lib().orc_num_threads())


def poisson_mask(radius, order, shape, calib, target):
    """Sequential variable-density Poisson-disc dart throwing
    (3DGS/3dgsVC/data/mask_generator.py:241-390): int8 [ny, nz] mask for the
    exclusion radius map `radius` (FP64 [ny, nz]) and pixel visiting order
    `order` (a permutation of ny*nz)."""
    ny, nz = shape
    out = np.zeros(ny * nz, np.int8)
    lib().orc_poisson_mask(_c(radius, np.float64).reshape(-1), _c(order, np.int32), ny, nz, int(calib),
                           int(target), out)
    return out.reshape(ny, nz)
