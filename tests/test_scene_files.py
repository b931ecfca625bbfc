"""Scene files: the library's OBJ/MTL, camera and light readers against the
reference's own readers (FWObject::read, CameraManager::read,
LightSourceLoader::loadFromFile, compiled in place as the checker) -- on
the reference's ruins scene and on small files with the cases its parser
treats specially -- and the committed ruins fixture against both."""
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
RUINS = os.path.join(os.environ.get("SHINOBI_REFERENCE", "/root/reference"), "scenes", "ruins")


def _ref():
    if oracle.ref_lib() is None or not os.path.exists(os.path.join(RUINS, "ruins.obj")):
        pytest.skip("reference tree / checker library not available")


def _same_obj(mine, ref):
    assert np.array_equal(mine["vertices"].view(np.uint32), ref["vertices"].view(np.uint32))
    assert np.array_equal(mine["indices"], ref["indices"].astype(np.uint32))
    assert np.array_equal(mine["face_material"], ref["face_material"].astype(np.uint32))
    m = ref["materials"]
    assert np.array_equal(mine["diffuse"][:, :3].view(np.uint32), m[:, 0:3].view(np.uint32))
    assert np.array_equal(mine["specular"][:, :3].view(np.uint32), m[:, 3:6].view(np.uint32))
    assert np.array_equal(mine["specular"][:, 3].view(np.uint32), m[:, 6].view(np.uint32))


def test_ruins_obj_matches_reference_reader():
    import shinobi_b200 as shn
    _ref()
    mine = shn.read_obj(os.path.join(RUINS, "ruins.obj"))
    ref = oracle.ref_read_obj(os.path.join(RUINS, "ruins.obj"))
    _same_obj(mine, ref)
    assert mine["vertices"].shape == (24625, 3) and mine["indices"].shape == (38665, 3)
    assert mine["material_names"][0] == "Default" and len(mine["material_names"]) == 10


def test_ruins_camera_and_light_match_reference_readers():
    import shinobi_b200 as shn
    _ref()
    cam = shn.read_camera(os.path.join(RUINS, "camera.cfg"))
    rc = oracle.ref_read_camera(os.path.join(RUINS, "camera.cfg"))
    mine = np.array(list(cam.eye) + list(cam.forward) + list(cam.up) + [cam.fov_deg, cam.res_x, cam.res_y],
                    np.float32)
    assert np.array_equal(mine.view(np.uint32), rc.view(np.uint32))
    lt = shn.read_light(os.path.join(RUINS, "light.cfg"))
    rl = oracle.ref_read_light(os.path.join(RUINS, "light.cfg"))
    mine = np.array([x for k in ("position", "edge1", "edge2", "normal", "intensity") for x in lt[k]], np.float32)
    assert np.array_equal(mine.view(np.uint32), rl.view(np.uint32))


def test_ruins_fixture_is_what_both_readers_load():
    import shinobi_b200 as shn
    _ref()
    z = np.load(os.path.join(HERE, "golden", "ruins.npz"))
    mine = shn.read_obj(os.path.join(RUINS, "ruins.obj"))
    _same_obj(mine, {k: z[k] for k in ("vertices", "indices", "face_material", "materials")})


EDGE_OBJ = """# comment line
mtllib edge.mtl
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
V 0.5 0.5 1
v 2 2 2 # a trailing comment rejects the line
v 1 2 3 4
vp 1 2
vt 0 0
vt 1 0 0.5
vn 0 0 1
g group
o object
s 1
f 1 2 3
usemtl Brick
f 1/1 2/2 3/2 4/1
usemtl Default
f 1//1 2//1 5//1
usemtl Glass
F 1/1/1 2/2/1 3/1/1 4/2/1 5/1/1
fo 2 3 5
f 1 2
f 1 2 3 # comment
usemtl Brick\r
f  3  4  5  \r
l 1 2
"""

EDGE_MTL = """newmtl Brick
Kd 0.5 0.25 0.125
Ks 0.1 0.2 0.3
Ns 10
newmtl Unused
Kd 0.9 0.9 0.9
newmtl Glass
kd 0.1 0.1 0.1
KS 1 1 1
Ka 0.2 0.2 0.2
Ns 2.5
"""


def test_edge_cases_match_reference_reader(tmp_path):
    """Fans of quads and pentagons, v / v/t / v//n / v/t/n references, upper
    case keywords, lines the reference rejects (trailing comments, a fourth
    coordinate, two-vertex faces, unknown entities), materials in order of
    first use, an .mtl material the OBJ does not use (its coefficients land
    on the previous material, as in the reference) and a coefficient keyword
    whose second letter is upper case (ignored)."""
    import shinobi_b200 as shn
    _ref()
    (tmp_path / "edge.obj").write_bytes(EDGE_OBJ.encode())
    (tmp_path / "edge.mtl").write_bytes(EDGE_MTL.encode())
    mine = shn.read_obj(str(tmp_path / "edge.obj"))
    ref = oracle.ref_read_obj(str(tmp_path / "edge.obj"))
    _same_obj(mine, ref)
    assert mine["vertices"].shape[0] == 5
    assert mine["indices"].shape[0] == 1 + 2 + 1 + 3 + 1 + 1
    assert mine["material_names"] == ["Default", "Brick", "Glass"]
    assert mine["skipped_lines"] > 0


def test_camera_rotation_and_light_normal_match_reference(tmp_path):
    import shinobi_b200 as shn
    _ref()
    (tmp_path / "cam.cfg").write_text("#camera parameters\nposition 1 2 3\norientation 0 0.6 0.8\nup 0 1 0\n"
                                      "rotation 10 20 30\nresX 640\nresY 480\nFOV 45\n")
    (tmp_path / "light.cfg").write_text("position 1 2 3\n# a comment\nnormal 0 -1 0\nintensity 5 6 7\n"
                                        "edge1 1 0 0\nedge2 0 0 1\n")
    cam = shn.read_camera(str(tmp_path / "cam.cfg"))
    rc = oracle.ref_read_camera(str(tmp_path / "cam.cfg"))
    mine = np.array(list(cam.eye) + list(cam.forward) + list(cam.up) + [cam.fov_deg, cam.res_x, cam.res_y],
                    np.float32)
    assert np.array_equal(mine.view(np.uint32), rc.view(np.uint32))
    lt = shn.read_light(str(tmp_path / "light.cfg"))
    rl = oracle.ref_read_light(str(tmp_path / "light.cfg"))
    mine = np.array([x for k in ("position", "edge1", "edge2", "normal", "intensity") for x in lt[k]], np.float32)
    assert np.array_equal(mine.view(np.uint32), rl.view(np.uint32))


def test_bad_face_index_is_refused(tmp_path):
    import shinobi_b200 as shn
    (tmp_path / "bad.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(shn.ShinobiError) as e:
        shn.read_obj(str(tmp_path / "bad.obj"))
    assert e.value.status == shn._abi.SHN_ERR_INVALID
