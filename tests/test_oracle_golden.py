"""Pin the oracle to the reference's own code through the committed fixtures
in tests/golden/ (made by tests/golden/make_golden.py from the reference
sources compiled in place).  CPU only."""
import os

import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _canon_ranges(r):
    """Empty ranges carry no information; the reference writes [k, k] with k
    the running offset, the oracle (like the GPU build) writes [0, 0]."""
    r = r.copy()
    r[r[:, 0] == r[:, 1]] = 0
    return r


@pytest.mark.parametrize("case", [0, 1, 2])
def test_uniform_build_matches_reference_hostbuild(case):
    """TwoLevelGridBuilderHost::hostBuild (src/Control/Algorithm/TwoLevelGridBuilder.cpp:28-213)
    on scenes where every top cell is a single leaf: cell ranges and the
    reference array equal the oracle's uniform build."""
    z = _load("hostbuild_uniform.npz")
    g = lambda n: z[f"c{case}_{n}"]  # noqa: E731
    u = oracle.build_uniform(g("vertices"), g("indices"), g("bounds"), g("res"))
    assert np.array_equal(_canon_ranges(u.cells), _canon_ranges(g("leaves")))
    assert np.array_equal(u.indices, g("refs"))


@pytest.mark.parametrize("case", [0, 1, 2])
def test_two_level_cell_words_match_reference_hostbuild(case):
    """Same scenes through the oracle's two-level build: every top cell word
    (leaf begin, leaf resolution, not-empty bit) equals hostBuild's, the leaf
    ranges and references too."""
    z = _load("hostbuild_uniform.npz")
    g = lambda n: z[f"c{case}_{n}"]  # noqa: E731
    t = oracle.build_two_level(g("vertices"), g("indices"), g("bounds"), g("res"), 4.0, 16)
    assert np.array_equal(t.cells, g("cellwords"))
    assert np.array_equal(_canon_ranges(t.leaves), _canon_ranges(g("leaves")))
    assert np.array_equal(t.indices, g("refs"))


def test_resolution_rule_on_fixture_scenes():
    """The fixture's top resolution was computed by the oracle's rule; it
    must still be a cube root of lambda*N/V within the clamp."""
    z = _load("hostbuild_uniform.npz")
    for case in range(int(z["num_cases"])):
        res = z[f"c{case}_res"]
        assert res.shape == (3,) and np.all(res >= 1) and np.all(res <= 2048)


def _cameras():
    return [scenes.CAMERA_SOUP, scenes.CAMERA_CLUSTER, scenes.CAMERA_HEIGHTFIELD,
            scenes.Camera((1.0, -2.0, 0.5), (0.3, 0.9, -0.1), (0.0, 0.0, 1.0), 60.0, 333, 77)]


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_camera_and_primary_directions_bit_exact(k):
    """Camera::init (src/Primitive/Camera.h:41-60) and RegularPixelSampler<1,1>
    + getDirection (src/Primitive/PixelSampler.h:40-52): bit-exact."""
    z = _load("camera.npz")
    cam = _cameras()[k]
    stored = z[f"cam{k}"]
    assert np.allclose(stored[:10], [*cam.eye, *cam.forward, *cam.up, cam.fov_deg])
    assert int(stored[10]) == cam.res_x and int(stored[11]) == cam.res_y
    c9 = oracle.camera(cam)
    assert np.array_equal(c9.view(np.uint32), z[f"c9_{k}"].view(np.uint32))
    _, d = oracle.primary_rays(cam)
    ids = z[f"ids_{k}"]
    assert np.array_equal(d[ids].view(np.uint32), z[f"dirs_{k}"].view(np.uint32))


def test_closest_hits_match_reference_intersector():
    """SimpleIntersector (Moller-Trumbore, src/Intersector/SimpleIntersector.hpp:38-89)
    brute force vs the oracle's watertight brute force: identical hit ids on
    every ray; distances agree to the precision of the reference's test, and
    the oracle's distance is within 1e-5 relative of the FP64 one (plus 1e-8
    absolute: a few rays start within 1e-4 of the surface, where FP32
    cancellation in the origin-relative vertices sets the floor)."""
    z = _load("mt_closest.npz")
    tri, t = oracle.trace_brute(z["vertices"], z["indices"], z["org"], z["dir"])[:2]
    assert np.array_equal(tri, z["tri"])
    hit = tri != oracle.MISS
    assert hit.sum() > 3000
    rel = np.abs(t[hit] - z["t"][hit]) / np.abs(z["t"][hit])
    assert rel.max() < 1e-4
    t64 = oracle.t_fp64(z["vertices"], z["indices"], tri, z["org"], z["dir"])
    assert np.all(np.abs(t[hit] - t64[hit]) <= 1e-5 * np.abs(t64[hit]) + 1e-8)


def test_cosine_sampler_matches_reference():
    """CosineHemisphereSampler (src/Utils/HemisphereSamplers.hpp:54-72) with the
    host sinf/cosf vs the oracle's deterministic sincos(2 pi u): within a few ulp."""
    z = _load("cosine.npz")
    out = oracle.cosine_local(z["u1"], z["u2"])
    assert np.max(np.abs(out - z["dirs"])) < 1e-6


def test_cell_word_packing_matches_reference():
    """TwoLevelGridCell (src/Control/Structure/TwoLevelGrid.hpp:72-151):
    x = leaf begin, y = resX | resY<<8 | resZ<<16 | notEmpty<<30 -- the
    layout the oracle and the CUDA build write."""
    rows = _load("cellword.npz")["rows"]
    for rx, ry, rz, ne, lb, w0, w1 in rows.tolist():
        assert w0 == lb
        assert w1 == (rx | (ry << 8) | (rz << 16) | (0x40000000 if ne else 0))


# ---- oracle self-consistency (no fixture needed) ---------------------------------


def test_oracle_grid_traversal_equals_brute_force():
    sc = scenes.uniform_soup(4000, seed=3, offset_scale=0.03)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    g = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    o, d = scenes.random_rays(5000, seed=4)
    tri_g, t_g = oracle.trace_closest(g, o, d)[:2]
    tri_b, t_b = oracle.trace_brute(sc.vertices, sc.indices, o, d)[:2]
    assert np.array_equal(tri_g, tri_b)
    assert np.array_equal(t_g.view(np.uint32), t_b.view(np.uint32))
    t2 = oracle.build_two_level(sc.vertices, sc.indices, b, oracle.resolution(sc.num_triangles, b, 1 / 16, 1, 2), 4.0)
    tri_2, t_2 = oracle.trace_closest(t2, o, d)[:2]
    assert np.array_equal(tri_2, tri_b)


def test_oracle_sincos_accuracy():
    u = np.linspace(0, 1, 100001, endpoint=False, dtype=np.float32)
    s, c = oracle.sincos_2pi(u)
    ang = 2 * np.pi * u.astype(np.float64)
    assert np.max(np.abs(s - np.sin(ang))) < 2e-6
    assert np.max(np.abs(c - np.cos(ang))) < 2e-6


def test_oracle_philox_known_answer():
    """Philox4x32-10 known-answer vectors (Salmon et al., SC'11, Random123 kat_vectors)."""
    ctr = np.array([[0, 0, 0, 0], [0xFFFFFFFF] * 4, [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]], np.uint32)
    keys = [(0, 0), (0xFFFFFFFF, 0xFFFFFFFF), (0xA4093822, 0x299F31D0)]
    expect = [[0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8],
              [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD],
              [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]]
    for i in range(3):
        out = oracle.philox(ctr[i:i + 1], *keys[i])
        assert out[0].tolist() == expect[i]
