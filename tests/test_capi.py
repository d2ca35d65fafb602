"""C ABI checks that need no GPU: the library loads, exports every entry
point include/*.h declares (and the ctypes table binds them all), and the
pure-host queries behave.  No kernel is launched here."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^GSV_API\s+[\w\s\*]+?\b(gsv_\w+)\s*\(", text, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("gsv_prepare", "gsv_bin", "gsv_forward", "gsv_backward", "gsv_tile_forward",
                 "gsv_tile_backward", "gsv_build_tile_pairs_count", "gsv_build_tile_pairs_fill"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from gs_tmi_b200 import _lib

    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\sT\s+(gsv_\w+)$", out, flags=re.M))
    missing = declared_symbols() - exported
    assert not missing, missing
    # the ctypes table covers the whole ABI, and nothing beyond it is exported
    assert set(_lib.SIGNATURES) == declared_symbols()
    assert exported == declared_symbols()
    for name in _lib.SIGNATURES:
        assert getattr(_lib.lib, name) is not None


def test_host_queries():
    from gs_tmi_b200._lib import GsvShape, lib

    assert lib.gsv_abi_version() == 4
    s = GsvShape(64, 64, 64, 8)
    assert lib.gsv_num_tiles(s) == 512
    assert lib.gsv_num_tiles(GsvShape(20, 12, 16, 8)) == 3 * 2 * 2
    assert lib.gsv_num_tiles(GsvShape(0, 4, 4, 8)) == -1
    assert lib.gsv_gauss_workspace_bytes(20000, s) > 20000 * 48
    assert lib.gsv_gauss_workspace_bytes(-1, s) == 0
    plain = lib.gsv_pair_workspace_bytes(292047, s, 0)
    det = lib.gsv_pair_workspace_bytes(292047, s, 1)
    assert plain >= 292047 * 16 and det >= plain + 292047 * 48
    for code in range(6):
        assert lib.gsv_status_string(code)


def test_entry_points_reject_bad_arguments_without_launching():
    """Argument validation happens on the host before any CUDA call."""
    import ctypes

    from gs_tmi_b200._lib import GSV_ERR_INVALID_ARGUMENT, GsvParams, GsvShape, lib

    bad = GsvShape(0, 8, 8, 8)
    p = GsvParams(None, None, None, None, None, 10)
    assert lib.gsv_prepare(ctypes.byref(p), bad, None, 0, None, None) == GSV_ERR_INVALID_ARGUMENT
    assert lib.gsv_prepare(ctypes.byref(p), GsvShape(8, 8, 8, 8), None, 0, None, None) == GSV_ERR_INVALID_ARGUMENT
    assert lib.gsv_tile_forward(*([None] * 7), 0, 1, 0, 8, 8, 8, None, None, None) == GSV_ERR_INVALID_ARGUMENT
    assert lib.gsv_forward(bad, 0, None, None, 0, None, None) == GSV_ERR_INVALID_ARGUMENT


def test_module_surface_matches_reference():
    """Constructor / forward signatures of the drop-in plugin
    (3DGS/3dgsVC/gaussian/tile_voxelizer.py:247-322)."""
    import inspect

    import gs_tmi_b200

    init = inspect.signature(gs_tmi_b200.TileVoxelizer.__init__)
    assert list(init.parameters)[:7] == ["self", "volume_shape", "tile_size", "max_radius", "use_cuda",
                                         "strict_cuda", "device"]
    assert init.parameters["tile_size"].default == 8 and init.parameters["max_radius"].default == 20
    fwd = inspect.signature(gs_tmi_b200.TileVoxelizer.forward)
    assert list(fwd.parameters) == ["self", "positions", "scales", "rotations", "density", "chunk_size"]
    btp = inspect.signature(gs_tmi_b200.build_tile_pairs)
    assert list(btp.parameters) == ["center_vox", "radius_vox", "volume_shape", "tile_size"]


def test_no_cpu_fallback():
    import torch

    import gs_tmi_b200

    with pytest.raises(RuntimeError):
        gs_tmi_b200.TileVoxelizer((8, 8, 8), use_cuda=False)
    if not torch.cuda.is_available():
        with pytest.raises(RuntimeError):
            gs_tmi_b200.TileVoxelizer((8, 8, 8))
        with pytest.raises(ValueError):
            gs_tmi_b200.build_tile_pairs(torch.zeros(2, 3), torch.ones(2), (8, 8, 8), 8)


def test_ctypes_structs_match_the_header(tmp_path):
    """Every struct of include/gsv.h has the size and field offsets its
    ctypes mirror assumes (gcc compiles a probe against the header)."""
    import ctypes
    import shutil

    from gs_tmi_b200 import _lib

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    mirrors = {"gsv_shape": _lib.GsvShape, "gsv_params": _lib.GsvParams, "gsv_grads": _lib.GsvGrads,
               "gsv_batch_item": _lib.GsvBatchItem, "gsv_tuning": _lib.GsvTuning,
               "gsv_density_rows": _lib.GsvDensityRows, "gsv_density_config": _lib.GsvDensityConfig}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gsv.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, cls in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_density_host_queries():
    from gs_tmi_b200 import density
    from gs_tmi_b200._lib import GSV_ERR_INVALID_ARGUMENT, lib

    assert lib.gsv_density_workspace_bytes(0) == 0
    assert lib.gsv_density_workspace_bytes(100_000) >= 100_000 * (36 * 4 + 16)
    assert lib.gsv_density_control(None, None, None, None, None, None, None, 0, None) == GSV_ERR_INVALID_ARGUMENT
    assert lib.gsv_normal_fill(None, 4, 0, None, None) == GSV_ERR_INVALID_ARGUMENT
    assert density.initial_rows(50_000, 500_000) == 100_352
    assert density.initial_rows(1000, 500_000) == 65_536
    assert density.initial_rows(400_000, 500_000) == 500_000
    assert density.initial_rows(600_000, 500_000) == 600_000


def test_flag_and_status_constants_mirror_the_header():
    """Every GSV_FLAG_*, GSV_BACKWARD_*, GSV_TUNE_*, GSV_DENSITY_* and GSV_BIN_*
    #define of include/gsv.h has the same value in the ctypes binding."""
    import re

    from gs_tmi_b200 import _lib

    text = open(os.path.join(ROOT, "include", "gsv.h")).read()
    defs = dict(re.findall(r"^#define\s+(GSV_(?:FLAG|BACKWARD|TUNE|DENSITY|BIN)_\w+)\s+(0x[0-9a-fA-F]+|\d+)", text,
                           flags=re.M))
    assert "GSV_FLAG_SCAN_STALLED" in defs and "GSV_BIN_COUNTING" in defs
    for name, value in defs.items():
        assert getattr(_lib, name) == int(value, 0), name
