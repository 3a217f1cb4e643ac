"""The C ABI library builds, loads and exports every entry point declared in
include/olcuda.h, and the ctypes structures match the C layouts.  CPU only:
no entry point that computes is called."""

from __future__ import annotations

import ctypes
from pathlib import Path
import re
import subprocess

import pytest

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "olcuda.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"OLC_API\s+[\w\s\*]+?\b(olc_\w+)\s*\(", text)))


def test_header_declares_the_bound_entry_points():
    from ordinarylight_b200 import _native

    assert declared_symbols() == sorted(_native.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol(native_library):
    for name in declared_symbols():
        assert hasattr(native_library, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(REPO / "ordinarylight_b200" / "_lib" / "libolcuda.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (olc_\w+)", out))
    assert set(declared_symbols()) <= exported


def test_abi_version_and_error_path_without_gpu(native_library):
    import re

    header = (REPO / "include" / "olcuda.h").read_text()
    assert native_library.olc_abi_version() == int(re.search(r"#define OLC_ABI_VERSION (\d+)", header).group(1))
    # a null context is rejected before any device work
    assert native_library.olc_destroy(None) == 0
    from ordinarylight_b200 import _native

    stats = _native.OlcRenderStats()
    cam = _native.OlcCamera()
    rc = native_library.olc_render(None, ctypes.byref(cam), 1, 1, 1, 0, None, 0, ctypes.byref(stats))
    assert rc == _native.OLC_ERR_VALUE
    assert b"context" in native_library.olc_last_error(None)


def test_struct_layouts_match_the_c_header(tmp_path):
    from ordinarylight_b200 import _native

    structs = {"olc_config": _native.OlcConfig, "olc_scene_desc": _native.OlcSceneDesc,
               "olc_camera": _native.OlcCamera, "olc_render_stats": _native.OlcRenderStats,
               "olc_bvh_info": _native.OlcBvhInfo, "olc_launch_record": _native.OlcLaunchRecord,
               "olc_scene_stats": _native.OlcSceneStats, "olc_pool_info": _native.OlcPoolInfo,
               "olc_job": _native.OlcJob}
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname in structs:
        lines.append(f'  printf("{cname} %zu\\n", sizeof({cname}));')
    lines.append('  printf("scene.volume_density %zu\\n", offsetof(olc_scene_desc, volume_density));')
    lines.append('  printf("stats.gpu_ms %zu\\n", offsetof(olc_render_stats, gpu_ms));')
    lines.append('  printf("job.out_rgba %zu\\n", offsetof(olc_job, out_rgba));')
    lines.append("  return 0; }")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], check=True)
    sizes = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for cname, ctype in structs.items():
        assert int(sizes[cname]) == ctypes.sizeof(ctype), cname
    assert int(sizes["scene.volume_density"]) == _native.OlcSceneDesc.volume_density.offset
    assert int(sizes["stats.gpu_ms"]) == _native.OlcRenderStats.gpu_ms.offset
    assert int(sizes["job.out_rgba"]) == _native.OlcJob.out_rgba.offset


def test_missing_library_fails_loudly(tmp_path):
    from ordinarylight_b200 import _native

    with pytest.raises(_native.NativeLibraryMissing):
        _native.load(tmp_path / "absent.so")
