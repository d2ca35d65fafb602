"""gs_tmi_b200 -- B200 (sm_100a) complex-Gaussian tile voxelizer for 3DGSMR.

Drop-in for the reference ``gaussian.TileVoxelizer`` plugin: same
constructor / forward signature and autograd behaviour, backed by the C ABI
in ``include/gsv.h`` (``lib/libgsv_b200.so``, built with
``python gs_tmi_b200/build.py``).  Importing this package fails loudly when
the library is missing: there is no CPU path.
"""
from .tile_voxelizer import (  # noqa: F401
    TileVoxelizer,
    _TileVoxelizeCUDA,
    build_tile_pairs,
    num_tiles,
    prepare_and_bin,
    voxelize,
)

__all__ = ["TileVoxelizer", "build_tile_pairs", "voxelize", "num_tiles", "prepare_and_bin"]
