"""The Python mirrors of the C ABI's structs (math_b200/ntrace.py, math_b200/denoise.py) have the
layout the headers declare: a small C program compiled here prints sizeof and every field's offset
of each struct, and the ctypes Structure must agree field by field (CPU only)."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

# C struct name -> (module, ctypes class name)
MIRRORS = {
    "nt_surface": ("ntrace", "Surface"),
    "nt_build_opts": ("ntrace", "BuildOpts"),
    "nt_render_opts": ("ntrace", "RenderOpts"),
    "nt_stats": ("ntrace", "Stats"),
    "nt_peaks": ("ntrace", "Peaks"),
    "nt_mesh_info": ("ntrace", "MeshInfo"),
    "nt_denoiser_layout": ("denoise", "Layout"),
}


def _mirror(module, name):
    if module == "ntrace":
        from math_b200 import ntrace as m
    else:
        from math_b200 import denoise as m
    return getattr(m, name)


@pytest.fixture(scope="module")
def c_layouts(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc:
        pytest.skip("no C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "ntrace.h"', '#include "ntrace_denoise.h"',
             "int main(void) {"]
    for cname, (module, pyname) in MIRRORS.items():
        cls = _mirror(module, pyname)
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0; }"]
    d = tmp_path_factory.mktemp("abi")
    src = d / "layout.c"
    exe = d / "layout"
    src.write_text("\n".join(lines))
    proc = subprocess.run([cc, "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                          capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    layouts = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        layouts.setdefault(cname, {})[field] = int(value)
    return layouts


@pytest.mark.parametrize("cname", sorted(MIRRORS))
def test_ctypes_mirror_matches_the_header(c_layouts, cname):
    module, pyname = MIRRORS[cname]
    cls = _mirror(module, pyname)
    c = c_layouts[cname]
    assert ctypes.sizeof(cls) == c["size"], (cname, ctypes.sizeof(cls), c["size"])
    for field, _ in cls._fields_:
        assert getattr(cls, field).offset == c[field], (cname, field)


def test_frame_module_reports_stats_fields_only():
    """math_b200.frame prints a subset of nt_stats (by the mirror's field names)."""
    from math_b200 import frame, ntrace

    names = {f for f, _ in ntrace.Stats._fields_}
    assert set(frame.STAT_KEYS) <= names, set(frame.STAT_KEYS) - names
