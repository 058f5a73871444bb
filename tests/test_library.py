"""The C-ABI library loads, exports every symbol include/cupbr_c.h declares,
and its host-only entry points (scene description, XML / OBJ parsing, file
writers) behave -- no GPU needed, nothing here launches a kernel."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import _native as N
from cupbr_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cupbr_c.h")
from conftest import REFERENCE_ROOT

REF_SCENES = os.path.join(REFERENCE_ROOT, "res", "Scenes")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|uint32_t|const char\*)\s+(cupbr_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    syms = declared_symbols()
    assert len(syms) > 60
    lib = C.CDLL(N.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    unbound = [s for s in syms if s not in N.exported_symbols()]
    assert not unbound, unbound


def test_errors_are_reported_not_printed():
    with pytest.raises(cb.CupbrError) as e:
        N.call("cupbr_renderer_create", 99, C.byref(C.c_void_p()))
    assert "unknown rendering method" in str(e.value)
    with pytest.raises(cb.CupbrError):
        N.call("cupbr_camera_default", 0, 0, C.byref(N.Camera()))


def test_material_and_camera_defaults_match_reference():
    m = N.Material()
    N.call("cupbr_material_default", C.byref(m))
    d = scenes.MaterialDesc()
    assert m.type == d.type and m.albedo_d.tuple() == d.albedo_d and m.albedo_e.tuple() == d.albedo_e
    assert m.shininess == np.float32(d.shininess) and m.roughness == 1.0 and m.eta == 1.5
    assert m.sigma_s.tuple() == (1, 1, 1) and m.sigma_a.tuple() == (1, 1, 1) and m.g == 0
    cam = cb.Camera(1920, 1080)  # Camera.cpp:6-11
    assert cam.position() == (0, 0, 0) and cam.z_axis() == (0, 0, 1) and cam.y_axis() == (0, 1, 0)
    assert cam.x_axis()[0] == np.float32(1920) / np.float32(1080)


def _parse(path):
    h = C.c_void_p()
    N.call("cupbr_scene_parse_xml", path.encode(), C.byref(h))
    return cb.Scene(h.value)


def test_xml_round_trip(tmp_path):
    desc = scenes.material_test_scene(0)
    desc.volume = ((0.1, 0.2, 0.3), (0.01, 0.02, 0.03), 0.4)
    path = desc.to_xml(str(tmp_path / "mixed.xml"))
    sc = _parse(path)
    info = sc.info()
    assert info["objects"] == len(desc.objects) and info["lights"] == len(desc.lights)
    assert info["committed"] == 0 and info["env_width"] == desc.env.shape[1]
    for i, o in enumerate(desc.objects):
        got = sc.object(i)
        assert got.type == o.type
        assert got.material.type == o.material.type
        assert got.material.albedo_d.tuple() == tuple(np.float32(o.material.albedo_d).tolist())
        if o.type in (scenes.MESH, scenes.TRIANGLE):
            assert np.array_equal(sc.object_triangles(i), o.triangles())
        if o.type == scenes.MESH:
            assert np.array_equal(np.array([*got.box_lo.tuple(), *got.box_hi.tuple()], np.float32), o.box())
    for i, l in enumerate(desc.lights):
        got = sc.light(i)
        assert got.type == l.type and got.radiance.tuple() == tuple(np.float32(l.radiance).tolist())
    sc.destroy()


@pytest.mark.parametrize("bad, msg", [
    ("<header><scene_size>1</scene_size><light_count>0</light_count></header>", "geometry"),
    ("<header><scene_size>1</scene_size><light_count>0</light_count></header><geometry><geometry1>"
     "<type>CONE</type><material><type>LAMBERT</type></material></geometry1></geometry>", "not a valid geometry"),
    ("<header><scene_size>1</scene_size><light_count>0</light_count></header><geometry><geometry1>"
     "<type>SPHERE</type><position>0,0</position><radius>1</radius><material><type>LAMBERT</type></material>"
     "</geometry1></geometry>", "three components"),
    ("<header><scene_size>0</scene_size><light_count>0</light_count>", "closing tag"),
    ("<header><scene_size>0</scene_size><light_count>1</light_count></header><lights><light1><type>SPOT</type>"
     "</light1></lights>", "not a valid light"),
])
def test_malformed_xml_fails_loudly(tmp_path, bad, msg):
    p = tmp_path / "bad.xml"
    p.write_text(bad)
    with pytest.raises(cb.CupbrError) as e:
        _parse(str(p))
    assert msg in str(e.value)


def test_obj_loader_semantics(tmp_path):
    # "f a/b/c" references, polygons keep their first three vertices, unused
    # vertices still widen the box (ObjLoader.cpp:29-65)
    p = tmp_path / "m.obj"
    p.write_text("# c\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 5 5 5\nvn 0 0 1\nf 1/1/1 2/2/1 3/3/1 4/4/1\n")
    h = C.c_void_p()
    N.call("cupbr_scene_create", C.byref(h))
    sc = cb.Scene(h.value)
    m = N.Material()
    N.call("cupbr_material_default", C.byref(m))
    N.call("cupbr_scene_add_mesh_obj", sc._h, str(p).encode(), N.Vec3(1, 2, 3), N.Vec3(2, 2, 2), C.byref(m), None)
    o = sc.object(0)
    assert o.triangle_count == 1
    assert o.box_hi.tuple() == (11.0, 12.0, 13.0) and o.box_lo.tuple() == (1.0, 2.0, 3.0)
    assert np.array_equal(sc.object_triangles(0)[0], np.array([1, 2, 3, 3, 2, 3, 1, 4, 3], np.float32))
    p.write_text("v 0 0 0\nf 1 2 3\n")
    with pytest.raises(cb.CupbrError):
        N.call("cupbr_scene_add_mesh_obj", sc._h, str(p).encode(), N.Vec3(0, 0, 0), N.Vec3(1, 1, 1), C.byref(m), None)


def test_mesh_arguments_validated():
    h = C.c_void_p()
    N.call("cupbr_scene_create", C.byref(h))
    sc = cb.Scene(h.value)
    v = np.zeros((3, 3), np.float32)
    idx = np.array([[0, 1, 3]], np.uint32)
    with pytest.raises(cb.CupbrError, match="out of range"):
        N.call("cupbr_scene_add_mesh", sc._h, v.ctypes.data, 3, idx.ctypes.data, 1, N.Vec3(0, 0, 0),
               N.Vec3(1, 1, 1), None, None)
    v[0, 0] = np.nan
    idx[0, 2] = 2
    with pytest.raises(cb.CupbrError, match="non-finite"):
        N.call("cupbr_scene_add_mesh", sc._h, v.ctypes.data, 3, idx.ctypes.data, 1, N.Vec3(0, 0, 0),
               N.Vec3(1, 1, 1), None, None)


@pytest.mark.parametrize("field,value,msg", [("nx", 0, "empty density grid"), ("majorant", 0.0, "majorant"),
                                             ("albedo", 1.5, "albedo"), ("g", 1.0, r"\|g\|"), ("q", 1.0, "q must")])
def test_medium_description_validated(field, value, msg):
    d = N.MediumDesc(4, 4, 4, N.Vec3(-1, -1, 1), N.Vec3(1, 1, 3), 8.5, 0.9, 0.3, 0.5)
    setattr(d, field, value)
    h = C.c_void_p()
    with pytest.raises(cb.CupbrError, match=msg):
        N.call("cupbr_medium_create", C.byref(d), C.byref(h))


def test_medium_parameter_count():
    # 1 (medium albedo) + 3 per object + 3 per light; an empty scene needs no GPU
    h = C.c_void_p()
    N.call("cupbr_scene_create", C.byref(h))
    n = C.c_uint32()
    N.call("cupbr_medium_param_count", h, C.byref(n))
    N.call("cupbr_scene_destroy", h)
    assert n.value == 1


@pytest.mark.skipif(not os.path.isdir(REF_SCENES), reason="reference scene files not present")
def test_reference_scene_files_parse(tmp_path):
    """Every shipped scene parses.  Those naming res/hdrtest.hdr (absent from
    the reference tree) fail with an I/O error instead of crashing, and parse
    once their <environment> element is removed."""
    seen = 0
    for f in sorted(os.listdir(REF_SCENES)):
        path = os.path.join(REF_SCENES, f)
        text = open(path).read()
        size = int(re.search(r"<scene_size>\s*(\d+)", text).group(1))
        cwd = os.getcwd()
        os.chdir(REFERENCE_ROOT)  # asset paths in these files are relative to the project root
        try:
            if "hdrtest.hdr" in text:
                with pytest.raises(cb.CupbrError, match="environment"):
                    _parse(path)
                stripped = tmp_path / f
                stripped.write_text(re.sub(r"<environment>.*?</environment>", "", text, flags=re.S))
                path = str(stripped)
            sc = _parse(path)
        finally:
            os.chdir(cwd)
        assert sc.info()["objects"] == size
        seen += 1
    assert seen == 12


def test_bmp_and_pfm_writers(tmp_path):
    rgba = np.arange(4 * 3 * 4, dtype=np.uint8).reshape(3, 4, 4)
    p = str(tmp_path / "x.bmp")
    N.call("cupbr_save_bmp", p.encode(), rgba.ctypes.data, 4, 3)
    raw = open(p, "rb").read()
    assert raw[:2] == b"BM" and len(raw) == 54 + rgba.size
    assert raw[54:58] == bytes([rgba[0, 0, 2], rgba[0, 0, 1], rgba[0, 0, 0], rgba[0, 0, 3]])
    rgb = np.random.default_rng(0).random((3, 4, 3), dtype=np.float32)
    q = str(tmp_path / "x.pfm")
    N.call("cupbr_save_pfm", q.encode(), rgb.ctypes.data, 4, 3)
    assert np.array_equal(scenes.read_pfm(q), rgb)


def test_pick_and_update_material_validate_arguments():
    desc = scenes.cornell_box()
    h = C.c_void_p()
    N.call("cupbr_scene_create", C.byref(h))
    sc = cb.Scene(h.value)
    m = N.Material()
    N.call("cupbr_material_default", C.byref(m))
    N.call("cupbr_scene_add_sphere", sc._h, N.Vec3(0, 0, 3), 1.0, C.byref(m), None)
    idx = C.c_int32(-1)
    cam = cb.Camera(8, 8)
    with pytest.raises(cb.CupbrError, match="outside"):
        N.call("cupbr_scene_pick", sc._h, C.byref(cam._c), 8, 0, 8, 8, C.byref(m), C.byref(idx))
    with pytest.raises(cb.CupbrError, match="out of range"):
        sc.update_material(1, desc.objects[0].material)
    # an uncommitted scene updates its host copy only (no GPU needed)
    sc.update_material(0, scenes.MaterialDesc(scenes.GGX, albedo_s=(0.5, 0.5, 0.5), roughness=0.3))
    o = sc.object(0)
    assert o.material.type == scenes.GGX and abs(o.material.roughness - 0.3) < 1e-7


def test_batch_arguments_validated():
    h = C.c_void_p()
    N.call("cupbr_scene_create", C.byref(h))
    sc = cb.Scene(h.value)  # never committed
    v = (N.View * 1)()
    v[0].scene, v[0].camera, v[0].width, v[0].height, v[0].spp = h.value, cb.Camera(4, 4)._c, 4, 4, 1
    v[0].device_image = 16
    out = C.c_void_p()
    with pytest.raises(cb.CupbrError, match="not committed"):
        N.call("cupbr_batch_create", v, 1, 5, C.byref(out))
    with pytest.raises(cb.CupbrError, match="no views"):
        N.call("cupbr_batch_create", v, 0, 5, C.byref(out))
    with pytest.raises(cb.CupbrError, match="max_depth"):
        N.call("cupbr_batch_create", v, 1, 0, C.byref(out))
    del sc


def test_camera_extension_element(tmp_path):
    """<camera> (position + yaw/pitch or look_at) gives the reference Camera's
    axes for that state (Camera.cpp:82-88); no element gives Camera(w, h)."""
    desc = scenes.cornell_box()
    desc.camera = ((0.2, 0.1, -0.5), 1.3, 0.2)
    sc = _parse(desc.to_xml(str(tmp_path / "cam.xml")))
    cam = sc.camera(640, 480)
    a = np.float32(640) / np.float32(480)
    f = np.float32
    z = np.array([np.cos(f(1.3)) * np.cos(f(0.2)), np.sin(f(0.2)), np.sin(f(1.3)) * np.cos(f(0.2))], np.float32)
    h = np.array([z[2], 0, -z[0]], np.float32)
    x = a * h / np.float32(np.linalg.norm(h))
    y = np.cross(z, x) / a
    assert np.allclose(cam.position(), (0.2, 0.1, -0.5))
    assert np.allclose(cam.z_axis(), z, atol=1e-6) and np.allclose(cam.x_axis(), x, atol=1e-6)
    assert np.allclose(cam.y_axis(), y, atol=1e-6)
    plain = _parse(scenes.cornell_box().to_xml(str(tmp_path / "plain.xml"))).camera(640, 480)
    assert plain.z_axis() == (0, 0, 1) and plain.x_axis()[0] == a
    (tmp_path / "la.xml").write_text(open(tmp_path / "plain.xml").read() +
                                     "<camera><position>0,0,0</position><look_at>1,0,1</look_at></camera>")
    la = _parse(str(tmp_path / "la.xml")).camera(8, 8)
    assert np.allclose(la.z_axis(), (np.sqrt(0.5), 0, np.sqrt(0.5)), atol=1e-6)
