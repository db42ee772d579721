"""Textured materials and the OBJ / MTL / PNG asset path.

CPU: the PNG reader on every row filter and colour type, an OBJ + MTL + PNG
round trip of the textured Cornell box to the same arrays and the same oracle
frames, the oracle's texture fetch against a numpy restatement of its
definition, and textures against constant materials.  GPU: the library
against the oracle on textured scenes (FP32 and FP16 storage, the three
renderer types) and on the scene read back from OBJ."""
import struct
import zlib

import numpy as np
import pytest

import oracle_py as op
from crisoptix_b200 import _abi, assets, scenes
from helpers import scene_size_of, small_config_params, static

W, H = 48, 40


def _png(rows: np.ndarray, color: int) -> bytes:
    """Filter-0 PNG of (H, W, C) uint8 rows with colour type `color`."""
    h, w = rows.shape[:2]
    raw = np.concatenate([np.zeros((h, 1), np.uint8), rows.reshape(h, -1)], axis=1)

    def chunk(k, b):
        return struct.pack(">I", len(b)) + k + b + struct.pack(">I", zlib.crc32(k + b) & 0xFFFFFFFF)

    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, color, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw.tobytes())) + chunk(b"IEND", b""))


@pytest.mark.parametrize("filter_type", [0, 1, 2, 3, 4])
def test_png_filters_round_trip(filter_type):
    rng = np.random.default_rng(filter_type)
    a = rng.integers(0, 256, (9, 13, 4), dtype=np.uint8)
    a[3:5] = a[2]  # repeated rows and smooth runs exercise the predictors
    a[:, 4:8] = np.arange(4, dtype=np.uint8)[None, :, None] * 40
    assert (assets.decode_png_rgba(assets.encode_png_rgba(a, filter_type)) == a).all()


def test_png_colour_types_expand_like_stbi_rgba():
    rng = np.random.default_rng(1)
    g = rng.integers(0, 256, (5, 7, 1), dtype=np.uint8)
    ga = rng.integers(0, 256, (5, 7, 2), dtype=np.uint8)
    rgb = rng.integers(0, 256, (5, 7, 3), dtype=np.uint8)
    out = assets.decode_png_rgba(_png(g, 0))
    assert (out[..., :3] == g).all() and (out[..., 3] == 255).all()
    out = assets.decode_png_rgba(_png(ga, 4))
    assert (out[..., :3] == ga[..., :1]).all() and (out[..., 3] == ga[..., 1]).all()
    out = assets.decode_png_rgba(_png(rgb, 2))
    assert (out[..., :3] == rgb).all() and (out[..., 3] == 255).all()
    with pytest.raises(ValueError):
        assets.decode_png_rgba(b"not a png")


def _tex_np(rgba, uv):
    """numpy float32 restatement of the texture fetch's definition."""
    t = rgba.astype(np.float32) / np.float32(255.0)
    h, w = rgba.shape[:2]
    f = np.float32
    u, v = uv[:, 0].astype(f), uv[:, 1].astype(f)
    u = np.where(np.isfinite(u), u, f(0))
    v = np.where(np.isfinite(v), v, f(0))
    x = (u - np.floor(u)) * f(w) - f(0.5)
    y = (v - np.floor(v)) * f(h) - f(0.5)
    xf, yf = np.floor(x), np.floor(y)
    a = np.floor((x - xf) * f(256) + f(0.5)) * f(1 / 256)
    b = np.floor((y - yf) * f(256) + f(0.5)) * f(1 / 256)
    i0, j0 = xf.astype(np.int64) % w, yf.astype(np.int64) % h
    i1, j1 = (i0 + 1) % w, (j0 + 1) % h
    w00, w10, w01, w11 = (f(1) - a) * (f(1) - b), a * (f(1) - b), (f(1) - a) * b, a * b
    return (((w00[:, None] * t[j0, i0] + w10[:, None] * t[j0, i1]) + w01[:, None] * t[j1, i0]) +
            w11[:, None] * t[j1, i1]).astype(f)


def test_oracle_texture_fetch_matches_its_definition():
    rng = np.random.default_rng(2)
    for h, w in ((1, 1), (3, 5), (8, 8), (17, 2)):
        tex = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
        uv = np.concatenate([rng.uniform(-3, 3, (4000, 2)), rng.normal(0, 1e-7, (200, 2)),
                             [[np.nan, 0.2], [np.inf, -np.inf], [0.5 / w, 0.5 / h], [1.0, 1.0], [-1.0, 2.0]]])
        uv = uv.astype(np.float32)
        got = op.tex_sample(tex, uv)
        assert (got == _tex_np(tex, uv)).all()
    # at texel centres the fetch is the texel itself
    tex = rng.integers(0, 256, (4, 6, 4), dtype=np.uint8)
    jj, ii = np.mgrid[0:4, 0:6]
    uv = np.stack([(ii.ravel() + 0.5) / 6, (jj.ravel() + 0.5) / 4], axis=1).astype(np.float32)
    assert np.allclose(op.tex_sample(tex, uv), tex.reshape(-1, 4) / 255.0, atol=1e-6)


def test_obj_round_trip(tmp_path):
    desc, cam = scenes.textured_cornell_box()
    path = str(tmp_path / "box.obj")
    assets.save_obj(path, desc)
    back = assets.load_obj(path)
    for name in ("positions", "normals", "uvs", "indices", "triangle_material", "emitter_faces"):
        assert (np.asarray(getattr(back, name)) == np.asarray(getattr(desc, name))).all(), name
    # SpecTexUsage is a per-model argument (src/Model.cpp:9), not in the MTL
    assert (back.materials["spec_usage"] == 0).all()
    back.materials["spec_usage"] = desc.materials["spec_usage"]
    assert back.materials.tobytes() == desc.materials.tobytes()
    # textures are numbered in order of first use; every slot reads the same texels
    assert ((back.material_textures >= 0) == (desc.material_textures >= 0)).all()
    assert len(back.textures) == len(desc.textures)
    for tb, td in zip(back.material_textures.ravel(), desc.material_textures.ravel()):
        if td >= 0:
            assert (back.textures[tb] == desc.textures[td]).all()
    assert [(tuple(np.float32(c)), f, n) for c, f, n in back.emitters] == \
           [(tuple(np.float32(c)), f, n) for c, f, n in desc.emitters]
    p = small_config_params(scene_size_of(desc))
    a, b = op.Oracle.from_scene(desc, W, H, p), op.Oracle.from_scene(back, W, H, p)
    oa, ob = np.zeros((H, W, 3), np.float32), np.zeros((H, W, 3), np.float32)
    for f in range(2):
        a.render_frame(cam, oa)
        b.render_frame(cam, ob)
        assert oa.tobytes() == ob.tobytes()


def test_obj_flip_uv_fan_and_defaults(tmp_path):
    (tmp_path / "q.mtl").write_text("newmtl lit\nKe 5 5 5\nnewmtl plain\n")
    (tmp_path / "q.obj").write_text(
        "mtllib q.mtl\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0.25\nvt 1 0.25\nvt 1 1\nvt 0 1\n"
        "usemtl plain\nf 1/1 2/2 3/3 4/4\nusemtl lit\nf -4/-4 -2/-2 -1/-1\n")
    d = assets.load_obj(str(tmp_path / "q.obj"), flip_uv=True)
    assert d.indices.shape == (3, 3)  # quad fanned into two, plus one
    assert len(d.positions) == 9  # corners without vn get the face normal: a vertex each
    assert np.allclose(d.uvs[:3, 1], [0.75, 0.75, 0.0])
    assert np.allclose(d.normals[:6], [0, 0, 1])  # generated face normals
    plain, lit = d.materials
    assert tuple(plain["diffuse"]) == (1, 1, 1) and plain["roughness"] == 1.0
    assert tuple(lit["emission"]) == (5, 5, 5) and d.emitters[0][1:] == (0, 1)
    assert d.material_textures is None


def test_textures_change_the_oracle_frame_and_match_constants():
    """A 1 x 1 texture of value c reads c / 255 (to rounding), so the frame
    matches the untextured scene with that constant; the textured box does
    not."""
    desc, cam = scenes.cornell_box()
    p = small_config_params(scene_size_of(desc))
    mats = desc.materials.copy()
    mats[0]["diffuse"] = (200 / 255, 100 / 255, 50 / 255)
    const = scenes.Scene(**{**desc.__dict__, "materials": mats})
    mt = np.full((len(mats), 3), -1, np.int32)
    mt[0, 0] = 0
    tex = scenes.Scene(**{**desc.__dict__, "uvs": np.zeros((len(desc.positions), 2), np.float32),
                          "textures": [np.array([[[200, 100, 50, 255]]], np.uint8)], "material_textures": mt})
    a, b = op.Oracle.from_scene(const, W, H, p), op.Oracle.from_scene(tex, W, H, p)
    oa, ob = np.zeros((H, W, 3), np.float32), np.zeros((H, W, 3), np.float32)
    a.render_frame(cam, oa)
    b.render_frame(cam, ob)
    assert np.abs(oa - ob).max() <= 1e-4 * max(1.0, float(np.abs(oa).max()))
    t, _ = scenes.textured_cornell_box()
    c = op.Oracle.from_scene(t, W, H, p)
    oc = np.zeros((H, W, 3), np.float32)
    c.render_frame(cam, oc)
    assert np.isfinite(oc).all() and np.abs(oc - oa).mean() > 0.05


# ---- GPU parity -----------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("storage", [_abi.STORAGE_FP32, _abi.STORAGE_FP16])
@pytest.mark.parametrize("rtype", [_abi.CONDITIONAL_RESTIR, _abi.RESTIR_PT, _abi.PATH_TRACER])
def test_textured_parity(cuda_device, rtype, storage):
    from helpers import orbit
    from test_parity_gpu import run_parity

    desc, cam = scenes.textured_cornell_box()
    p = small_config_params(scene_size_of(desc), renderer_type=rtype, storage=storage)
    run_parity(desc, cam, p, W, H, 3, lambda c, f: orbit(c, f, 30))


@pytest.mark.gpu
def test_obj_scene_parity(cuda_device, tmp_path):
    from test_parity_gpu import run_parity

    desc, cam = scenes.textured_cornell_box()
    path = str(tmp_path / "box.obj")
    assets.save_obj(path, desc)
    back = assets.load_obj(path, spec_usage=_abi.SPEC_OCC_ROUGH_METAL)  # every material: the ORM workflow
    run_parity(back, cam, small_config_params(scene_size_of(back)), W, H, 3, static)


@pytest.mark.gpu
def test_adjoint_rejects_textures(cuda_device):
    from crisoptix_b200 import CrisbError, Scene
    from crisoptix_b200.adjoint import PtAdjoint

    desc, cam = scenes.textured_cornell_box()
    with pytest.raises(CrisbError):
        PtAdjoint(Scene(desc), W, H, small_config_params(scene_size_of(desc), renderer_type=_abi.PATH_TRACER))


def test_flat_scene_keeps_textures():
    """The flattened soup of a textured scene reads the same texels at the
    same corners, so the oracle renders it identically."""
    desc, cam = scenes.textured_cornell_box()
    flat = scenes.flat_scene(desc)
    assert flat.textured and len(flat.textures) == len(desc.textures)
    assert (flat.flatten_uvs() == desc.flatten_uvs()).all()
    p = small_config_params(scene_size_of(desc))
    a, b = op.Oracle.from_scene(desc, W, H, p), op.Oracle.from_scene(flat, W, H, p)
    oa, ob = np.zeros((H, W, 3), np.float32), np.zeros((H, W, 3), np.float32)
    a.render_frame(cam, oa)
    b.render_frame(cam, ob)
    assert oa.tobytes() == ob.tobytes()


@pytest.mark.parametrize("version", [7400, 7500])
def test_fbx_round_trip(tmp_path, version):
    """save_fbx -> load_fbx keeps every triangle corner's position, normal and
    uv bit for bit, the materials, textures and emitters; the oracle renders
    the read scene as the original (32- and 64-bit node records)."""
    desc, cam = scenes.textured_cornell_box()
    path = str(tmp_path / "box.fbx")
    assets.save_fbx(path, desc, version=version)
    back = assets.load_fbx(path)
    ti, tb = np.asarray(desc.indices).reshape(-1, 3), np.asarray(back.indices).reshape(-1, 3)
    for name in ("positions", "normals", "uvs"):
        a, b = np.asarray(getattr(desc, name))[ti], np.asarray(getattr(back, name))[tb]
        assert a.tobytes() == b.tobytes(), name
    assert (np.asarray(back.triangle_material) == np.asarray(desc.triangle_material)).all()
    assert (back.materials["spec_usage"] == 0).all()
    back.materials["spec_usage"] = desc.materials["spec_usage"]
    assert back.materials.tobytes() == desc.materials.tobytes()
    assert ((back.material_textures >= 0) == (desc.material_textures >= 0)).all()
    for tbk, td in zip(back.material_textures.ravel(), desc.material_textures.ravel()):
        if td >= 0:
            assert (back.textures[tbk] == desc.textures[td]).all()
    assert [(tuple(np.float32(c)), f, n) for c, f, n in back.emitters] == \
           [(tuple(np.float32(c)), f, n) for c, f, n in desc.emitters]
    assert np.asarray(back.emitter_faces).tobytes() == np.asarray(desc.emitter_faces).tobytes()
    p = small_config_params(scene_size_of(desc))
    a, b = op.Oracle.from_scene(desc, W, H, p), op.Oracle.from_scene(back, W, H, p)
    oa, ob = np.zeros((H, W, 3), np.float32), np.zeros((H, W, 3), np.float32)
    for f in range(2):
        a.render_frame(cam, oa)
        b.render_frame(cam, ob)
        assert oa.tobytes() == ob.tobytes()


def _fbx_graph_file(path, ascii=False):
    """A quad and a triangle with per-corner indexed normals and uvs, one
    material slot, used by two models: `child` (rotated 90 degrees about z,
    scaled 2) under `parent` (translated by (1, 2, 3)), and `other` at the
    origin with no material."""
    N = assets.FbxNode
    verts = np.array([0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0, 2, 0, 0], np.float64)
    pvi = np.array([0, 1, 2, -4, 1, 4, -3], np.int32)  # quad (0 1 2 3), triangle (1 4 2)
    normals = np.array([0, 0, 1, 0, 0, -1], np.float64)
    nidx = np.array([0, 0, 0, 0, 1, 1, 1], np.int32)
    uvs = np.array([0, 0, 1, 0, 1, 1, 0, 1, 0.5, 0.25], np.float64)
    uvidx = np.array([0, 1, 2, 3, 1, 4, 2], np.int32)
    geom = N("Geometry", [10, "g\x00\x01Geometry", "Mesh"], [
        N("Vertices", [verts]), N("PolygonVertexIndex", [pvi]),
        N("LayerElementNormal", [0], [N("MappingInformationType", ["ByPolygonVertex"]),
                                      N("ReferenceInformationType", ["IndexToDirect"]),
                                      N("Normals", [normals]), N("NormalsIndex", [nidx])]),
        N("LayerElementUV", [0], [N("MappingInformationType", ["ByPolygonVertex"]),
                                  N("ReferenceInformationType", ["IndexToDirect"]),
                                  N("UV", [uvs]), N("UVIndex", [uvidx])]),
        N("LayerElementMaterial", [0], [N("MappingInformationType", ["AllSame"]),
                                        N("ReferenceInformationType", ["IndexToDirect"]),
                                        N("Materials", [np.array([0], np.int32)])])])
    parent = N("Model", [20, "parent\x00\x01Model", "Null"], [N("Properties70", [], [
        assets.fbx_p("Lcl Translation", "Lcl Translation", 1.0, 2.0, 3.0)])])
    child = N("Model", [21, "child\x00\x01Model", "Mesh"], [N("Properties70", [], [
        assets.fbx_p("Lcl Rotation", "Lcl Rotation", 0.0, 0.0, 90.0),
        assets.fbx_p("Lcl Scaling", "Lcl Scaling", 2.0, 2.0, 2.0)])])
    other = N("Model", [22, "other\x00\x01Model", "Mesh"], [N("Properties70")])
    mat = N("Material", [30, "red\x00\x01Material", ""], [N("Properties70", [], [
        assets.fbx_p("DiffuseColor", "Color", 0.8, 0.4, 0.2), assets.fbx_p("DiffuseFactor", "Number", 0.5),
        assets.fbx_p("EmissiveColor", "Color", 0.0, 0.0, 0.0)])])
    conns = [N("C", ["OO", 20, 0]), N("C", ["OO", 21, 20]), N("C", ["OO", 22, 0]), N("C", ["OO", 10, 21]),
             N("C", ["OO", 10, 22]), N("C", ["OO", 30, 21])]
    top = [N("Objects", [], [geom, parent, child, other, mat]), N("Connections", [], conns)]
    if ascii:
        assets.write_fbx_ascii_tree(str(path), top)
    else:
        assets.write_fbx_tree(str(path), top, version=7400)


def test_fbx_scene_graph_transforms_fans_and_layers(tmp_path):
    path = tmp_path / "graph.fbx"
    _fbx_graph_file(path)
    d = assets.load_fbx(str(path), flip_uv=True)
    P = np.asarray(d.positions, np.float64)[np.asarray(d.indices).reshape(-1, 3)]
    Nn = np.asarray(d.normals, np.float64)[np.asarray(d.indices).reshape(-1, 3)]
    U = np.asarray(d.uvs, np.float64)[np.asarray(d.indices).reshape(-1, 3)]
    assert P.shape == (6, 3, 3)  # (quad -> 2 triangles + 1 triangle) x 2 models
    # the child model: rotate 90 degrees about z, scale 2, then translate (1, 2, 3)
    to_world = lambda v: np.array([-2 * v[1] + 1, 2 * v[0] + 2, 2 * v[2] + 3])  # noqa: E731
    quad = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0)]
    expect = [to_world(quad[0]), to_world(quad[1]), to_world(quad[2])]
    np.testing.assert_allclose(P[0], expect, atol=1e-6)
    np.testing.assert_allclose(P[1], [to_world(quad[0]), to_world(quad[2]), to_world(quad[3])], atol=1e-6)
    np.testing.assert_allclose(P[2], [to_world((1, 0, 0)), to_world((2, 0, 0)), to_world((1, 1, 0))], atol=1e-6)
    np.testing.assert_allclose(P[3:], np.array([[quad[0], quad[1], quad[2]], [quad[0], quad[2], quad[3]],
                                                [(1, 0, 0), (2, 0, 0), (1, 1, 0)]], np.float64))
    np.testing.assert_allclose(Nn[:2], np.tile([0, 0, 1.0], (2, 3, 1)), atol=1e-6)  # z normals stay z
    np.testing.assert_allclose(Nn[2], np.tile([0, 0, -1.0], (3, 1)), atol=1e-6)
    np.testing.assert_allclose(U[0], [[0, 1], [1, 1], [1, 0]])  # flipped v
    np.testing.assert_allclose(U[2], [[1, 1], [0.5, 0.75], [1, 0]])
    # the child's slot 0 is the red material, diffuse times its factor; the
    # other model has no material: the reference's fallbacks
    assert list(d.triangle_material) == [0, 0, 0, 1, 1, 1]
    np.testing.assert_allclose(d.materials["diffuse"][0], [0.4, 0.2, 0.1], rtol=1e-6)
    np.testing.assert_allclose(d.materials["diffuse"][1], [1, 1, 1])
    assert float(d.materials["roughness"][1]) == 1.0 and d.emitters == []


def test_fbx_ascii_reads_like_binary(tmp_path):
    """The ASCII form of the same trees gives the same scenes: the textured
    box through save_fbx, the scene graph through the node writer."""
    desc, _ = scenes.textured_cornell_box()
    assets.save_fbx(str(tmp_path / "b.fbx"), desc)
    assets.save_fbx(str(tmp_path / "a.fbx"), desc, ascii=True)
    _fbx_graph_file(tmp_path / "gb.fbx")
    _fbx_graph_file(tmp_path / "ga.fbx", ascii=True)
    assert (tmp_path / "a.fbx").read_text().startswith("; FBX")
    for bn, an in (("b.fbx", "a.fbx"), ("gb.fbx", "ga.fbx")):
        b, a = assets.load_fbx(str(tmp_path / bn)), assets.load_fbx(str(tmp_path / an))
        for name in ("positions", "normals", "uvs", "indices", "triangle_material", "emitter_faces"):
            assert np.asarray(getattr(a, name)).tobytes() == np.asarray(getattr(b, name)).tobytes(), (an, name)
        assert a.materials.tobytes() == b.materials.tobytes()


def test_fbx_rejects_non_fbx(tmp_path):
    (tmp_path / "h.fbx").write_text("; FBX 7.4.0 project file\nFBXHeaderExtension:  {\n}\n")
    (tmp_path / "x.fbx").write_text("solid cube\nfacet normal 0 0 1\n")
    for name in ("h.fbx", "x.fbx"):  # no Objects; not FBX at all
        with pytest.raises(ValueError):
            assets.load_fbx(str(tmp_path / name))


def test_fbx_transform_chain_pivots_orders_and_geometric(tmp_path):
    """The FBX SDK's chain T Roff Rp Rpre R Rpost^-1 Rp^-1 Soff Sp S Sp^-1 and
    the model's geometric transform, against the same product composed here
    with scipy's Euler rotations (extrinsic 'xyz' is FBX's XYZ order)."""
    from scipy.spatial.transform import Rotation

    N = assets.FbxNode
    P = assets.fbx_p
    verts = np.array([0.3, -0.2, 0.5, 1.0, 0.1, 0.0, 0.2, 0.9, -0.4], np.float64)
    geom = N("Geometry", [10, "g\x00\x01Geometry", "Mesh"], [
        N("Vertices", [verts]), N("PolygonVertexIndex", [np.array([0, 1, -3], np.int32)])])
    props = dict(T=(1.0, -2.0, 0.5), Roff=(0.1, 0.2, 0.3), Rp=(1.0, 0.0, -1.0), Rpre=(-90.0, 0.0, 0.0),
                 R=(10.0, 20.0, 30.0), Rpost=(0.0, 15.0, 0.0), Soff=(0.0, 0.5, 0.0), Sp=(0.2, 0.2, 0.2),
                 S=(2.0, 1.0, 0.5), Gt=(0.0, 0.0, 1.0), Gr=(0.0, 0.0, 45.0), Gs=(1.0, 2.0, 1.0))
    model = N("Model", [21, "m\x00\x01Model", "Mesh"], [N("Properties70", [], [
        P("Lcl Translation", "Lcl Translation", *props["T"]), P("RotationOffset", "Vector3D", *props["Roff"]),
        P("RotationPivot", "Vector3D", *props["Rp"]), P("PreRotation", "Vector3D", *props["Rpre"]),
        P("Lcl Rotation", "Lcl Rotation", *props["R"]), P("RotationOrder", "enum", 5),
        P("PostRotation", "Vector3D", *props["Rpost"]), P("ScalingOffset", "Vector3D", *props["Soff"]),
        P("ScalingPivot", "Vector3D", *props["Sp"]), P("Lcl Scaling", "Lcl Scaling", *props["S"]),
        P("GeometricTranslation", "Vector3D", *props["Gt"]), P("GeometricRotation", "Vector3D", *props["Gr"]),
        P("GeometricScaling", "Vector3D", *props["Gs"])])])
    path = tmp_path / "chain.fbx"
    assets.write_fbx_tree(str(path), [N("Objects", [], [geom, model]), N("Connections", [], [
        N("C", ["OO", 21, 0]), N("C", ["OO", 10, 21])])], version=7500)
    d = assets.load_fbx(str(path))

    def tr(t):
        M = np.eye(4)
        M[:3, 3] = t
        return M

    def rot(deg, seq="xyz"):
        M = np.eye(4)
        angles = deg if seq == "xyz" else deg[::-1]  # 'zyx': z first, so pass (z, y, x)
        M[:3, :3] = Rotation.from_euler(seq, angles, degrees=True).as_matrix()
        return M

    def sc(s):
        return np.diag([*s, 1.0])

    inv = np.linalg.inv
    W = (tr(props["T"]) @ tr(props["Roff"]) @ tr(props["Rp"]) @ rot(props["Rpre"]) @ rot(props["R"], "zyx")
         @ inv(rot(props["Rpost"])) @ inv(tr(props["Rp"])) @ tr(props["Soff"]) @ tr(props["Sp"]) @ sc(props["S"])
         @ inv(tr(props["Sp"])) @ tr(props["Gt"]) @ rot(props["Gr"]) @ sc(props["Gs"]))
    expect = (np.c_[verts.reshape(-1, 3), np.ones(3)] @ W.T)[:, :3]
    got = np.asarray(d.positions, np.float64)[np.asarray(d.indices).reshape(-1)]
    np.testing.assert_allclose(got, expect, rtol=1e-5, atol=1e-5)


def test_load_model_dispatches_on_the_extension(tmp_path):
    desc, _ = scenes.textured_cornell_box()
    assets.save_obj(str(tmp_path / "box.obj"), desc)
    assets.save_fbx(str(tmp_path / "box.fbx"), desc)
    a = assets.load_model(str(tmp_path / "box.obj"), spec_usage=1)
    b = assets.load_model(str(tmp_path / "box.fbx"), spec_usage=1)
    ia, ib = np.asarray(a.indices).reshape(-1, 3), np.asarray(b.indices).reshape(-1, 3)
    assert np.asarray(a.positions)[ia].tobytes() == np.asarray(b.positions)[ib].tobytes()
    assert (a.materials["spec_usage"] == 1).all() and (b.materials["spec_usage"] == 1).all()
    with pytest.raises(ValueError):
        assets.load_model(str(tmp_path / "box.gltf"))


def test_fbx_embedded_texture(tmp_path):
    """A texture whose Video object embeds the PNG bytes is read from them
    (no file beside the FBX)."""
    N = assets.FbxNode
    rgba = (np.arange(4 * 3 * 4) * 7 % 256).astype(np.uint8).reshape(4, 3, 4)
    geom = N("Geometry", [10, "g\x00\x01Geometry", "Mesh"], [
        N("Vertices", [np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float64)]),
        N("PolygonVertexIndex", [np.array([0, 1, -3], np.int32)])])
    objs = [geom, N("Model", [20, "m\x00\x01Model", "Mesh"], [N("Properties70")]),
            N("Material", [30, "t\x00\x01Material", ""], [N("Properties70")]),
            N("Texture", [40, "tex\x00\x01Texture", ""], [N("RelativeFilename", ["missing.png"])]),
            N("Video", [50, "v\x00\x01Video", "Clip"], [N("Content", [assets.encode_png_rgba(rgba)])])]
    conns = [N("C", ["OO", 20, 0]), N("C", ["OO", 10, 20]), N("C", ["OO", 30, 20]),
             N("C", ["OP", 40, 30, "DiffuseColor"]), N("C", ["OO", 50, 40])]
    path = tmp_path / "emb.fbx"
    assets.write_fbx_tree(str(path), [N("Objects", [], objs), N("Connections", [], conns)])
    d = assets.load_fbx(str(path))
    assert d.material_textures.tolist() == [[0, -1, -1]]
    assert (d.textures[0] == rgba).all()
