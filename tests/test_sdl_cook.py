"""Host-side scene cooking through the library's SDL parser (no GPU needed).

The parser follows the reference grammar (Engine/Source/SDL/SdlCommandParser.cpp:84-560,
SdlInlinePacketInterface.cpp:48-245); cooking follows the actors it supports (AModel,
AModelLight, ARectangleLight, AImageDome) and bakes actor transforms (TDecomposedTransform:
T * R * S) into world-space triangles.
"""

import math
import os
import tempfile

import numpy as np
import pytest

import photon_gpu
import scenes


def _cook(text, wd="."):
    return photon_gpu.CookedScene(text, wd)


def test_cornell_cooks_to_generator_triangles():
    s = scenes.cornell()
    c = _cook(scenes.to_sdl(s))
    ref = np.concatenate([g.tris for g in s.groups])
    assert np.array_equal(c.tris.view(np.uint32), ref.view(np.uint32))
    assert (c.width, c.height, c.spp, c.estimator) == (256, 256, 64, 0)
    assert c.emitters.shape == (1, 4) and np.allclose(c.emitters[0], [17, 12, 4, 0])
    # light triangles are the last group
    assert np.all(c.tri_emitter[-2:] == 1) and np.all(c.tri_emitter[:-2] == 0)
    # camera looking down +z with +y up: camera x = -x (world), y = +y, z = -z
    cam = c.camera
    assert np.allclose(cam[0:3], [278, 273, -800])
    assert np.allclose(cam[3:6], [-1, 0, 0]) and np.allclose(cam[6:9], [0, 1, 0]) and np.allclose(cam[9:12], [0, 0, -1])
    # 40 degree horizontal field of view on a 36 mm sensor
    assert abs(cam[14] - (0.018 / math.tan(math.radians(20.0)))) < 1e-6


def test_bvpt_and_materials():
    s = scenes.cornell_glossy(estimator="bvpt")
    c = _cook(scenes.to_sdl(s))
    assert c.estimator == 1
    assert c.num_materials == len(s.groups)
    assert _cook(scenes.to_sdl(scenes.cornell(estimator="bvptdl"))).estimator == 2


def test_sample_filters():
    import dataclasses

    for name, code in photon_gpu.FILTERS.items():
        s = dataclasses.replace(scenes.cornell(8, 8, 1), sample_filter=name)
        assert _cook(scenes.to_sdl(s)).sample_filter == code
    # without a sample-filter clause the path-tracing visualizer uses Blackman-Harris
    text = scenes.to_sdl(scenes.cornell(8, 8, 1)).replace("[enum sample-filter box] ", "")
    assert "sample-filter" not in text
    assert _cook(text).sample_filter == photon_gpu.FILTERS["bh"]


def test_streamed_fragments_equal_whole_text():
    text = scenes.to_sdl(scenes.cornell(32, 32, 4))
    whole = _cook(text)
    # split the text at arbitrary points, including inside comments and tokens
    pieces = [text[i:i + 97] for i in range(0, len(text), 97)]
    eng_text = "// leading comment\n" + "".join(pieces)
    again = _cook(eng_text)
    assert np.array_equal(whole.tris, again.tris)


def test_reference_style_scene_with_transforms_and_area_light():
    text = """#version 1.1.0;
option(single-frame-render-session) @session = [vector2 frame-size "40 30"] [string visualizer @visualizer]
    [string observer @observer] [string sample-source @sampler];
observer(single-lens) @observer = [real fov-degrees 50] [vector3 pos "0 0 16"] [vector3 dir "0 0 -1"] [vector3 up-axis "0 1 0"];
sample-source(stratified) @sampler = [integer samples 40];
visualizer(path-tracing) @visualizer = [enum sample-filter box] [enum estimator bneept];
geometry(rectangle) @boxWall = [real width 1] [real height 1];
image(constant) @white = [real-array values "0.7 0.7 0.7"][enum color-space LSRGB];
// top light
actor(rectangle-light) @topLight = [spectrum color "1 1 1"][real watts 500][real width 3][real height 3];
translate(@topLight) = [vector3 amount "0 4.75 0"];
rotate(@topLight)    = [vector3 axis "1 0 0"] [real degrees 90];
material(matte-opaque) @wallMat = [image albedo @white];
actor(model) @bottomWall = [geometry geometry @boxWall] [material material @wallMat];
actor(model).translate(@bottomWall) = [vector3 amount "0 -5 0"];
actor(model).rotate(@bottomWall)    = [vector3 axis "1 0 0"] [real degrees -90];
actor(model).scale(@bottomWall)     = [vector3 amount "10 10 10"];
"""
    c = _cook(text)
    assert (c.width, c.height, c.spp) == (40, 30, 40)
    assert c.tris.shape[0] == 4
    light = c.tris[c.tri_emitter == 1]
    floor = c.tris[c.tri_emitter == 0]
    # the light lies in the plane y = 4.75 (rectangle in XY rotated +90 deg about x), facing -y
    assert np.allclose(light[:, :, 1], 4.75, atol=1e-5)
    n = np.cross(light[:, 1] - light[:, 0], light[:, 2] - light[:, 0])
    assert np.all(n[:, 1] < 0)
    # the floor is the 10 x 10 square at y = -5 facing +y
    assert np.allclose(floor[:, :, 1], -5.0, atol=1e-5)
    assert np.isclose(np.abs(floor[:, :, 0]).max(), 5.0, atol=1e-5)
    n = np.cross(floor[:, 1] - floor[:, 0], floor[:, 2] - floor[:, 0])
    assert np.all(n[:, 1] > 0)
    # radiance = watts / (area * pi * energy(white)), the reference's putEnergy normalisation
    expected = 500.0 / (9.0 * math.pi * 0.999678004)
    assert np.allclose(c.emitters[0, :3], expected, rtol=1e-5)


def test_environment_dome(tmp_path):
    s = scenes.ggx_sphere(level=2, width=16, height=16, spp=1)
    scenes.write_pfm(str(tmp_path / "env.pfm"), np.full((1, 1, 3), 0.1, np.float32))
    c = _cook(scenes.to_sdl(s), str(tmp_path))
    env = c.emitters[c.emitters[:, 3] == 1]
    assert env.shape[0] == 1 and np.allclose(env[0, :3], 0.1)
    # dome radius: 1.01 x the farthest bound corner from the origin
    tris = c.tris.reshape(-1, 3)
    lo, hi = tris.min(0), tris.max(0)
    corners = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    r = max(1.0, np.linalg.norm(corners, axis=1).max() * 1.01)
    assert np.isclose(c.camera[15], 4 * math.pi * r * r, rtol=1e-5)


@pytest.mark.parametrize("content", [
    b"PF\n4 2\n-1.0\n" + bytes(4 * 2 * 3 * 4 - 4),          # one float short
    b"PF\n100000 100000\n-1.0\n" + bytes(48),             # a header that claims 120 GB
    b"PF\n-4 2\n-1.0\n" + bytes(96),                       # negative width
    b"PF\n4 2\n0\n" + bytes(96),                           # scale 0 (no byte order)
    b"P6\n4 2\n255\n" + bytes(24),                         # not a PFM
])
def test_malformed_dome_images_are_reported(content, tmp_path):
    s = scenes.ggx_sphere(level=2, width=16, height=16, spp=1)
    (tmp_path / "env.pfm").write_bytes(content)
    with pytest.raises(photon_gpu.PhotonGpuError) as err:
        _cook(scenes.to_sdl(s), str(tmp_path))
    assert "cannot read dome image" in str(err.value)


def test_little_and_big_endian_dome_images(tmp_path):
    s = scenes.ggx_sphere(level=2, width=16, height=16, spp=1)
    for scale, order in ((-1.0, "<f4"), (1.0, ">f4")):
        (tmp_path / "env.pfm").write_bytes(f"PF\n1 1\n{scale}\n".encode() + np.array([0.25, 0.5, 2.0], order).tobytes())
        c = _cook(scenes.to_sdl(s), str(tmp_path))
        env = c.emitters[c.emitters[:, 3] == 1]
        assert np.array_equal(env[0, :3], np.array([0.25, 0.5, 2.0], np.float32))


@pytest.mark.parametrize("snippet, message", [
    ("geometry(sphere) @g = [real radius 1];\nactor(model) @a = [geometry geometry @g] [material material @m];\n"
     "material(matte-opaque) @m = ;", "not supported"),
    ("actor(model) @a = [geometry geometry @g] [material material @m] [bad", "clause"),
])
def test_errors_are_reported(snippet, message):
    base = scenes.to_sdl(scenes.cornell(8, 8, 1))
    with pytest.raises(photon_gpu.PhotonGpuError) as err:
        _cook(base + snippet)
    assert message in str(err.value)


@pytest.mark.parametrize("old, new, message", [
    ('frame-size "8 8"', 'frame-size "0 8"', "resolution"),
    ('frame-size "8 8"', 'frame-size "8 -2"', "resolution"),
    ('frame-size "8 8"', 'frame-size "8.5 8"', "resolution"),
    ('frame-size "8 8"', 'frame-size "65536 65537"', "resolution"),
    ('frame-size "8 8"', 'frame-size "8"', "two numbers"),
    ("[integer samples 1]", "[integer samples 0]", "whole number"),
    ("[integer samples 1]", "[integer samples -3]", "whole number"),
])
def test_bad_session_numbers_are_reported(old, new, message):
    base = scenes.to_sdl(scenes.cornell(8, 8, 1))
    assert old in base
    with pytest.raises(photon_gpu.PhotonGpuError) as err:
        _cook(base.replace(old, new))
    assert message in str(err.value)


def test_degenerate_triangles_are_dropped():
    s = scenes.cornell(8, 8, 1)
    g = s.groups[0]
    bad = np.zeros((1, 3, 3), np.float32)
    g.tris = np.concatenate([g.tris, bad])
    c = _cook(scenes.to_sdl(s))
    assert c.tris.shape[0] == 36


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian", "ascii"])
def test_ply_meshes_cook_to_the_same_triangles(fmt, tmp_path):
    s = scenes.cornell(16, 16, 4)
    scenes.write_meshes(s, str(tmp_path), fmt)
    c = _cook(scenes.to_sdl(s, mesh_format="ply"), str(tmp_path))
    ref = np.concatenate([g.tris for g in s.groups])
    assert np.array_equal(c.tris.view(np.uint32), ref.view(np.uint32))


def _write_custom_ply(path, header_props, vertex_rows, face_rows, extra=""):
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\n")
        f.write(f"element vertex {len(vertex_rows)}\n{header_props}")
        f.write(f"element face {len(face_rows)}\nproperty list uchar int vertex_indices\n{extra}end_header\n")
        for r in vertex_rows:
            f.write(" ".join(str(x) for x in r) + "\n")
        for r in face_rows:
            f.write(" ".join(str(x) for x in r) + "\n")


def _ply_scene_text():
    """A one-mesh scene whose mesh is read from g0.ply."""
    tri = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32)
    s = scenes.Scene("ply", 8, 8, 1, 8, cam_pos=(0.5, 0.5, -3.0), cam_dir=(0.0, 0.0, 1.0), cam_up=(0.0, 1.0, 0.0),
                     fov_deg=40.0, groups=[scenes.MeshGroup(tri, scenes.WHITE)])
    return scenes.to_sdl(s, mesh_format="ply")


def test_ply_extra_properties_and_elements(tmp_path):
    # shared vertices, an extra per-vertex colour, a trailing edge element with a list
    props = "property double x\nproperty double y\nproperty double z\nproperty uchar red\n"
    verts = [(0, 0, 0, 1), (1, 0, 0, 2), (0, 1, 0, 3), (1, 1, 0, 4)]
    faces = [(3, 0, 1, 2), (3, 2, 1, 3)]
    path = tmp_path / "g0.ply"
    _write_custom_ply(path, props, verts, faces, extra="element edge 1\nproperty list uchar int vertex_pair\n")
    with open(path, "a") as f:
        f.write("2 0 3\n")
    c = _cook(_ply_scene_text(), str(tmp_path))
    want = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 0], [1, 0, 0], [1, 1, 0]]], np.float32)
    assert np.array_equal(c.tris, want)


@pytest.mark.parametrize("faces", [[(4, 0, 1, 2, 3)], [(3, 0, 1, 7)]])
def test_ply_rejects_polygons_and_bad_indices(faces, tmp_path):
    props = "property float x\nproperty float y\nproperty float z\n"
    _write_custom_ply(tmp_path / "g0.ply", props, [(0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)], faces)
    with pytest.raises(photon_gpu.PhotonGpuError, match="PLY"):
        _cook(_ply_scene_text(), str(tmp_path))


_PLY_XYZ = b"property float x\nproperty float y\nproperty float z\n"
_PLY_FACE = b"element face 1\nproperty list uchar int vertex_indices\n"


@pytest.mark.parametrize("content, message", [
    (b"plx\nformat ascii 1.0\n", "not a PLY file"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE, "no end_header"),
    (b"ply\nformat binary_middle_endian 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE + b"end_header\n",
     "unknown format"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\nproperty float x\nproperty float y\n" + _PLY_FACE
     + b"end_header\n0 0\n1 0\n0 1\n3 0 1 2\n", "needs x, y and z"),
    (b"ply\nformat ascii 1.0\n" + _PLY_FACE + b"element vertex 3\n" + _PLY_XYZ
     + b"end_header\n3 0 1 2\n0 0 0\n1 0 0\n0 1 0\n", "must follow the vertex element"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ
     + b"element face 1\nproperty list uchar float vertex_indices\nend_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n",
     "must be integers"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ + b"property short q\n" + _PLY_FACE
     .replace(b"int", b"int128") + b"end_header\n", "unknown property type"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE + b"end_header\n0 0 0\n1 0 0\n0 1\n",
     "PLY: truncated"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE + b"end_header\n0 0 0\n1 0 0\n0 1 x\n3 0 1 2\n",
     "truncated or malformed ASCII body"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE + b"end_header\n"
     + np.zeros(9, "<f4").tobytes() + b"\x03" + np.arange(2, dtype="<i4").tobytes(), "truncated binary body"),
    # element counts far beyond the body: rejected before anything is sized by them
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1000000000\n" + _PLY_XYZ + _PLY_FACE
     + b"end_header\n" + np.zeros(9, "<f4").tobytes(), "truncated body"),
    (b"ply\nformat ascii 1.0\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE.replace(b"face 1", b"face 400000000000")
     + b"end_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n", "truncated body"),
    # an element with a huge count and no properties: rows of zero bytes would loop without reading
    (b"ply\nformat ascii 1.0\nelement junk 18446744073709551615\nelement vertex 3\n" + _PLY_XYZ + _PLY_FACE
     + b"end_header\n0 0 0\n1 0 0\n0 1 0\n3 0 1 2\n", "has rows but no properties"),
])
def test_ply_malformed_files_are_reported(content, message, tmp_path):
    (tmp_path / "g0.ply").write_bytes(content)
    with pytest.raises(photon_gpu.PhotonGpuError) as err:
        _cook(_ply_scene_text(), str(tmp_path))
    assert message in str(err.value)


def test_ply_big_endian_doubles_and_short_indices(tmp_path):
    # scalar types other than float / int, in big-endian order
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], ">f8")
    body = verts.tobytes() + b"\x03" + np.array([0, 1, 2], ">u2").tobytes()
    head = (b"ply\nformat binary_big_endian 1.0\nelement vertex 3\nproperty double x\nproperty double y\n"
            b"property double z\nelement face 1\nproperty list uchar ushort vertex_indices\nend_header\n")
    (tmp_path / "g0.ply").write_bytes(head + body)
    c = _cook(_ply_scene_text(), str(tmp_path))
    assert np.array_equal(c.tris, verts.astype(np.float32)[None])
