"""A compiled C++ caller of the drop-in templates (tests/dropin/dropin_main.cpp,
built with g++ against include/ and libbgt.so): Thinning2D<unsigned char>,
Thinning3D<float> and both CenterlineExtraction<unsigned char> overloads,
their new[] outputs delete[]d by the caller, compared with the oracle; and
the failure path (invalid sizes return 0 segments with delete[]-able
outputs, a failed Thinning2D leaves a zero-filled output)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import pyoracle as po
from tests.helpers import blobs2d, blobs3d

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "begputhinning_b200")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "dropin_main")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "dropin", "dropin_main.cpp"), "-L", PKG, "-lbgt",
           f"-Wl,-rpath,{PKG}", "-I/usr/local/cuda/include", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


def test_dropin_program_links(exe):
    """Compiles and links against libbgt.so without a GPU (runs nothing)."""
    assert os.path.exists(exe)


def _run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


@pytest.mark.gpu
def test_dropin_thinning(exe, tmp_path):
    rng = np.random.default_rng(12)
    img = blobs2d(rng, 150, 233, 25)
    p = tmp_path / "a.raw"
    img.tofile(p)
    _run(exe, "thin2d_u8", p, 233, 150, tmp_path / "a.out")
    got = np.fromfile(tmp_path / "a.out", np.uint8).reshape(img.shape)
    assert np.array_equal(got, po.thin2d(img)[0])
    vol = blobs3d(rng, 30, 41, 52, 6)
    q = tmp_path / "v.raw"
    vol.tofile(q)
    _run(exe, "thin3d_f32", q, 52, 41, 30, tmp_path / "v.out")
    got3 = np.fromfile(tmp_path / "v.out", np.uint8).reshape(vol.shape)
    assert np.array_equal(got3, po.thin3d(vol)[0])


@pytest.mark.gpu
def test_dropin_centerline(exe, tmp_path):
    rng = np.random.default_rng(13)
    img = blobs2d(rng, 180, 200, 30)
    p = tmp_path / "c.raw"
    img.tofile(p)
    _run(exe, "cl2d_u8", p, 200, 180, 10, 3, tmp_path / "c")
    ref = po.centerline2d(img, 10, 3)
    for name, want in (("x", ref.x), ("y", ref.y)):
        got = np.fromfile(tmp_path / f"c.{name}", np.float32)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), name
    assert np.array_equal(np.fromfile(tmp_path / "c.idx", np.uint32), ref.idx)
    vol = blobs3d(rng, 34, 40, 44, 6)
    q = tmp_path / "d.raw"
    vol.tofile(q)
    _run(exe, "cl3d_u8", q, 44, 40, 34, 5, 2, tmp_path / "d")
    ref3 = po.centerline3d(vol, 5, 2)
    for name, want in (("x", ref3.x), ("y", ref3.y), ("z", ref3.z)):
        got = np.fromfile(tmp_path / f"d.{name}", np.float32)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), name
    assert np.array_equal(np.fromfile(tmp_path / "d.idx", np.uint32), ref3.idx)


@pytest.mark.gpu
def test_dropin_failure_path(exe):
    out = _run(exe, "bad_sizes").split("\n")
    assert out[0] == "cl2d 0 0"
    assert out[1] == "cl3d 0 0"
    assert out[2] == "thin2d 0"
