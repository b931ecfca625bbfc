"""The C++ adapters (include/shinobi/shinobi.hpp) with the reference's class
and method names: tests/cpp/adapter_example.cpp must compile against the
header and the library, fail cleanly without a device, and on a GPU produce
the oracle's primary hits and direct-illumination frame for a uniform and a
two-level grid."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "shinobi_b200")
CUDA = "/usr/local/cuda"


def _compile(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libshinobi_b200.so")):
        import __graft_entry__
        __graft_entry__.build()
    exe = str(tmp_path / "adapter_example")
    cmd = ["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "cpp", "adapter_example.cpp"),
           "-L", LIBDIR, "-lshinobi_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{LIBDIR}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}", "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def _write_scene(path, sc):
    with open(path, "wb") as f:
        f.write(struct.pack("II", sc.vertices.shape[0], sc.indices.shape[0]))
        f.write(np.ascontiguousarray(sc.vertices, np.float32).tobytes())
        f.write(np.ascontiguousarray(sc.indices, np.uint32).tobytes())


def test_adapter_compiles_and_fails_cleanly_without_device(tmp_path):
    import torch
    exe = _compile(tmp_path)
    if torch.cuda.is_available():
        pytest.skip("a device is present: covered by the GPU test")
    sc = scenes.uniform_soup(100, seed=1)
    _write_scene(tmp_path / "s.bin", sc)
    r = subprocess.run([exe, str(tmp_path / "s.bin"), str(tmp_path / "o.bin"), "0", "32", "24"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 3, (r.stdout, r.stderr)
    assert "no device" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_adapter_primary_hits_match_oracle(tmp_path, gpu, kind):
    exe = _compile(tmp_path)
    sc = scenes.uniform_soup(20000, seed=7, offset_scale=0.02)
    _write_scene(tmp_path / "s.bin", sc)
    rx, ry = 256, 192
    r = subprocess.run([exe, str(tmp_path / "s.bin"), str(tmp_path / "o.bin"), str(kind), str(rx), str(ry)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.stdout, r.stderr)
    raw = np.fromfile(tmp_path / "o.bin", np.uint32)
    n = rx * ry
    tri, t, rgb = raw[:n], raw[n:2 * n].view(np.float32), raw[2 * n:].view(np.float32).reshape(n, 3)
    b = oracle.bounds(sc.vertices, sc.indices)
    if kind == 0:
        g = oracle.build_uniform(sc.vertices, sc.indices, b, oracle.resolution(sc.num_triangles, b, 5.0))
    elif kind == 2:  # SAHGridBuilder: the resolution of least SAH cost
        g = oracle.build_uniform(sc.vertices, sc.indices, b, oracle.sah_resolution(sc.vertices, sc.indices, b)["res"])
    else:
        g = oracle.build_two_level(sc.vertices, sc.indices, b,
                                   oracle.resolution(sc.num_triangles, b, 1.0 / 16.0, 1, 2), 4.0, 16)
    cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, rx, ry)
    o, d = oracle.primary_rays(cam)
    rt, rtt = oracle.trace_closest(g, o, d)[:2]
    assert np.count_nonzero(rt != oracle.MISS) > 1000
    assert np.array_equal(tri, rt)
    assert np.array_equal(t.view(np.uint32), rtt.view(np.uint32))
    light = dict(position=(0.3, 1.2, 0.3), edge1=(0.4, 0.0, 0.0), edge2=(0.0, 0.0, 0.4),
                 normal=(0.0, -1.0, 0.0), intensity=(4.0, 4.0, 4.0))
    ro, rd, _ = oracle.direct_rays(o, d, rt, rtt, 4, 1, 0, light)
    occ, _ = oracle.trace_any(g, ro, rd, np.full(ro.shape[0], 0.9999, np.float32))
    frame, _ = oracle.shade_direct(sc.vertices, sc.indices, o, d, rt, rtt, 4, 1, 0, light, occ)
    assert np.array_equal(rgb.view(np.uint32), frame.view(np.uint32))
    assert (frame > 0).any()
    assert "Grid resolution" in r.stdout
