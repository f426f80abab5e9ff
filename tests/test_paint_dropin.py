"""The C++ drop-in (math_b200/paint.hpp): a program written against the reference's painter interface
(PaintObjects, Visible* objects, Paintbrush, PainterNotifier, paint<N,T>) compiles and links against the
library; on a GPU it paints the same image as the Python scene API does for the same scene."""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT

SRC = ROOT / "tests" / "cpp" / "paint_dropin.cpp"


def _build(tmp_path: Path) -> Path:
    exe = tmp_path / "paint_dropin"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
                    "-L", str(ROOT / "math_b200"), "-lntrace", "-Wl,-rpath," + str(ROOT / "math_b200"), "-pthread"],
                   check=True)
    return exe


def test_dropin_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert exe.exists()
    # argument checking runs without a GPU
    assert subprocess.run([str(exe)], capture_output=True).returncode == 2


@pytest.mark.gpu
def test_dropin_paints_like_the_scene_api(require_gpu, tmp_path):
    from math_b200 import scenes

    exe = _build(tmp_path)
    verts, facets = scenes.icosphere(2)
    mesh = tmp_path / "mesh.bin"
    with open(mesh, "wb") as f:
        np.array([len(verts), len(facets)], np.int32).tofile(f)
        verts.astype(np.float32).tofile(f)
        facets.astype(np.int32).tofile(f)
    out = tmp_path / "out.bin"
    screen, spp, depth, passes = 32, 16, 5, 2
    run = subprocess.run([str(exe), str(mesh), str(out), str(screen), str(spp), str(depth), str(passes)],
                         capture_output=True, text=True)
    assert run.returncode == 0, run.stderr
    assert f"passes {passes} pixels {passes * screen * screen}" in run.stdout
    img = np.fromfile(out, np.float32).reshape(-1, 3)

    spec = scenes.make_spec(3, verts, facets, screen=screen, spp=spp, max_depth=depth, seed=0)
    s = scenes.build_scene(spec)
    for _ in range(passes):
        s.render(spp, max_depth=depth, seed=0)
    expect, _ = s.image()
    err = np.sqrt(((img - expect) ** 2).sum() / (expect ** 2).sum())
    assert err < 1e-5
