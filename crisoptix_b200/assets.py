"""Scene files: Wavefront OBJ + MTL and FBX (binary and ASCII), with PNG textures.

The reference imports models with assimp (src/Model.cpp:9-207: triangulated,
normals generated where missing, optional uv flip) and reads textures with
stb_image as RGBA8 (src/Texture.cpp:8-30).  Neither library is part of this
package; this module reads the same inputs itself, for OBJ/MTL, FBX
(load_fbx, described with its section below) and 8-bit PNG:

* geometry: `v`, `vt`, `vn`, `f` (polygons fanned into triangles, negative
  indices relative), `usemtl`, `mtllib`; every distinct v/vt/vn corner is one
  vertex, as assimp's importer keeps them;
* faces without normals get their face normal (aiProcess_GenNormals);
* `flip_uv` replaces v by 1 - v (aiProcess_FlipUVs);
* materials as Model::LoadMaterials reads them (src/Model.cpp:209-373):
  `Kd` diffuse, `Ks` specular, `Ke` emissive, `Pr` roughness factor, with the
  reference's fallbacks when a key is absent (diffuse and specular 1,
  roughness 1, emissive 0); `map_Kd`, `map_Ks`, `map_Pr` (its
  aiTextureType_DIFFUSE_ROUGHNESS) give the three textures; `spec_usage`
  applies to every material of the model, as the reference's Model argument;
* faces of a material with a non-zero `Ke` also form one emitter per
  material (Emitter(mesh, transform, color), include/model/Emitter.h:57-71),
  since OBJ has no separate emitter list.

PNG: 8-bit greyscale, grey + alpha, RGB and RGBA, non-interlaced, all five
row filters; the result is RGBA8 as stbi_load(..., STBI_rgb_alpha) returns
it (missing alpha = 255, grey replicated).
"""
import os
import struct
import zlib
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import scenes

# ---- PNG ----------------------------------------------------------------------------

_SIG = b"\x89PNG\r\n\x1a\n"
_CHANNELS = {0: 1, 2: 3, 4: 2, 6: 4}  # colour type -> samples per pixel


def _paeth(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    p = a.astype(np.int16) + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c)).astype(np.uint8)


def _unfilter(raw: np.ndarray, h: int, stride: int, bpp: int) -> np.ndarray:
    out = np.zeros((h, stride), np.uint8)
    prev = np.zeros(stride, np.uint8)
    for y in range(h):
        ft, line = raw[y, 0], raw[y, 1:].astype(np.uint8)
        if ft == 0:
            cur = line.copy()
        elif ft == 2:
            cur = (line.astype(np.uint16) + prev).astype(np.uint8)
        elif ft == 1:
            # Sub: a running sum per channel, modulo 256
            cur = np.cumsum(line.reshape(-1, bpp), axis=0, dtype=np.uint8).reshape(-1)
        elif ft in (3, 4):
            cur = np.zeros(stride, np.uint8)
            for x in range(stride):  # left neighbour dependency: sequential
                a = int(cur[x - bpp]) if x >= bpp else 0
                b = int(prev[x])
                c = int(prev[x - bpp]) if x >= bpp else 0
                if ft == 3:
                    pred = (a + b) >> 1
                else:
                    p = a + b - c
                    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                    pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
                cur[x] = (int(line[x]) + pred) & 0xFF
        else:
            raise ValueError(f"PNG: unknown filter type {ft}")
        out[y] = cur
        prev = cur
    return out


def decode_png_rgba(data: bytes) -> np.ndarray:
    """(H, W, 4) uint8 RGBA of an 8-bit PNG (first row first)."""
    if data[:8] != _SIG:
        raise ValueError("not a PNG file")
    pos, idat = 8, []
    w = h = depth = color = interlace = None
    while pos + 12 <= len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        if zlib.crc32(kind + body) & 0xFFFFFFFF != crc:
            raise ValueError("PNG chunk CRC mismatch")
        if kind == b"IHDR":
            w, h, depth, color, _, _, interlace = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
        pos += 12 + n
    if w is None or depth != 8 or color not in _CHANNELS or interlace != 0:
        raise ValueError("only non-interlaced 8-bit grey, grey+alpha, RGB and RGBA PNG files are read")
    ch = _CHANNELS[color]
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8).reshape(h, 1 + w * ch)
    px = _unfilter(raw, h, w * ch, ch).reshape(h, w, ch)
    out = np.full((h, w, 4), 255, np.uint8)
    if ch in (1, 2):
        out[..., :3] = px[..., :1]
        if ch == 2:
            out[..., 3] = px[..., 1]
    else:
        out[..., :ch] = px
    return out


def encode_png_rgba(rgba: np.ndarray, filter_type: int = 0) -> bytes:
    """8-bit RGBA PNG of an (H, W, 4) uint8 array, every row with
    `filter_type` (0 none, 1 sub, 2 up, 3 average, 4 Paeth)."""
    a = np.ascontiguousarray(rgba, np.uint8)
    if a.ndim != 3 or a.shape[2] != 4:
        raise ValueError("expected an (H, W, 4) uint8 array")
    h, w, _ = a.shape
    rows = a.reshape(h, 4 * w).astype(np.int16)
    raw = np.zeros((h, 1 + 4 * w), np.uint8)
    raw[:, 0] = filter_type
    for y in range(h):
        cur = rows[y]
        prev = rows[y - 1] if y > 0 else np.zeros_like(cur)
        left = np.concatenate([np.zeros(4, np.int16), cur[:-4]])
        upleft = np.concatenate([np.zeros(4, np.int16), prev[:-4]])
        pred = {0: 0, 1: left, 2: prev, 3: (left + prev) >> 1,
                4: _paeth(left.astype(np.uint8), prev.astype(np.uint8), upleft.astype(np.uint8)).astype(np.int16)}
        raw[y, 1:] = ((cur - pred[filter_type]) & 0xFF).astype(np.uint8)

    def chunk(kind: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    return (_SIG + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
            chunk(b"IDAT", zlib.compress(raw.tobytes(), 6)) + chunk(b"IEND", b""))


# ---- OBJ / MTL ---------------------------------------------------------------------

def _floats(parts, n, default=0.0):
    v = [float(x) for x in parts[:n]]
    return v + [default] * (n - len(v))


def _read_mtl(path: str) -> Dict[str, dict]:
    mats: Dict[str, dict] = {}
    cur = None
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p or p[0].startswith("#"):
                continue
            key = p[0]
            if key == "newmtl":
                cur = mats.setdefault(" ".join(p[1:]), {})
            elif cur is None:
                continue
            elif key in ("Kd", "Ks", "Ke"):
                cur[key] = _floats(p[1:], 3)
            elif key == "Pr":
                cur[key] = float(p[1])
            elif key in ("map_Kd", "map_Ks", "map_Pr"):
                cur[key] = p[-1]  # the file name (options before it are ignored)
    return mats


def _index(tok: str, n: int) -> int:
    i = int(tok)
    return i - 1 if i > 0 else n + i


def load_obj(path: str, flip_uv: bool = False, spec_usage: int = 0) -> scenes.Scene:
    """Scene description of an OBJ file, its MTL libraries and PNG textures
    (paths relative to the OBJ's folder)."""
    base = os.path.dirname(os.path.abspath(path))
    vs: List[List[float]] = []
    vts: List[List[float]] = []
    vns: List[List[float]] = []
    mtl: Dict[str, dict] = {}
    mat_names: List[str] = []
    corners: Dict[Tuple[int, int, int], int] = {}
    pos: List[List[float]] = []
    nrm: List[List[float]] = []
    uv: List[List[float]] = []
    tris: List[List[int]] = []
    tri_mat: List[int] = []
    current = None

    def material_index(name):
        if name not in mat_names:
            mat_names.append(name)
        return mat_names.index(name)

    def corner(vi, ti, ni, face_n):
        key = (vi, ti, ni) if ni >= 0 else (vi, ti, -1 - len(pos))  # flat normal: own vertex
        if key not in corners:
            corners[key] = len(pos)
            pos.append(vs[vi])
            uv.append(vts[ti] if ti >= 0 else [0.0, 0.0])
            nrm.append(vns[ni] if ni >= 0 else face_n)
        return corners[key]

    with open(path) as f:
        for line in f:
            p = line.split()
            if not p or p[0].startswith("#"):
                continue
            key = p[0]
            if key == "v":
                vs.append(_floats(p[1:], 3))
            elif key == "vt":
                t = _floats(p[1:], 2)
                vts.append([t[0], 1.0 - t[1]] if flip_uv else t)
            elif key == "vn":
                vns.append(_floats(p[1:], 3))
            elif key == "mtllib":
                for name in p[1:]:
                    mtl.update(_read_mtl(os.path.join(base, name)))
            elif key == "usemtl":
                current = " ".join(p[1:])
            elif key == "f":
                refs = []
                for tok in p[1:]:
                    parts = tok.split("/")
                    vi = _index(parts[0], len(vs))
                    ti = _index(parts[1], len(vts)) if len(parts) > 1 and parts[1] else -1
                    ni = _index(parts[2], len(vns)) if len(parts) > 2 and parts[2] else -1
                    refs.append((vi, ti, ni))
                mi = material_index(current if current is not None else "")
                for k in range(1, len(refs) - 1):  # fan
                    tri = [refs[0], refs[k], refs[k + 1]]
                    a, b, c = (np.asarray(vs[r[0]], np.float64) for r in tri)
                    fn = np.cross(b - a, c - a)
                    ln = np.linalg.norm(fn)
                    fn = (fn / ln if ln > 0 else np.array([0.0, 0.0, 1.0])).tolist()
                    tris.append([corner(r[0], r[1], r[2], fn) for r in tri])
                    tri_mat.append(mi)
    textures: List[np.ndarray] = []
    tex_index: Dict[str, int] = {}

    def texture(name: Optional[str]) -> int:
        if name is None:
            return -1
        if name not in tex_index:
            with open(os.path.join(base, name), "rb") as tf:
                textures.append(decode_png_rgba(tf.read()))
            tex_index[name] = len(textures) - 1
        return tex_index[name]

    mats, mt, emitters, faces = [], [], [], []
    P = np.asarray(pos, np.float32).reshape(-1, 3)
    T = np.asarray(tris, np.uint32).reshape(-1, 3)
    TM = np.asarray(tri_mat, np.uint32)
    for i, name in enumerate(mat_names):
        d = mtl.get(name, {})
        m = np.zeros((), dtype=scenes.MATERIAL_DTYPE)
        m["diffuse"] = d.get("Kd", [1.0, 1.0, 1.0])
        m["specular"] = d.get("Ks", [1.0, 1.0, 1.0])
        m["emission"] = d.get("Ke", [0.0, 0.0, 0.0])
        m["roughness"] = d.get("Pr", 1.0)
        m["spec_usage"] = spec_usage
        mats.append(m)
        mt.append([texture(d.get("map_Kd")), texture(d.get("map_Ks")), texture(d.get("map_Pr"))])
        if any(v != 0.0 for v in d.get("Ke", [0.0, 0.0, 0.0])):
            sel = np.flatnonzero(TM == i)
            emitters.append((tuple(d["Ke"]), len(faces), len(sel)))
            faces.extend(P[T[sel]].reshape(-1, 9))
    if not tris:
        raise ValueError(f"{path}: no faces")
    mt_arr = np.asarray(mt, np.int32).reshape(-1, 3)
    return scenes.Scene(P, np.asarray(nrm, np.float32).reshape(-1, 3), T, TM, np.stack(mats),
                        np.zeros((0, 2), np.uint32), [], emitters,
                        np.asarray(faces, np.float32).reshape(-1, 9), name=os.path.basename(path),
                        uvs=np.asarray(uv, np.float32).reshape(-1, 2), textures=textures,
                        material_textures=mt_arr if (mt_arr >= 0).any() else None)


def _fmt(v) -> str:
    return " ".join(repr(float(x)) for x in v)


def save_obj(path: str, desc: scenes.Scene) -> None:
    """Write a non-instanced scene as OBJ + MTL (+ PNG textures) that
    load_obj reads back to the same triangles, vertices, materials and
    textures.  Emitter faces must be the faces of the emissive materials."""
    if desc.instances:
        raise ValueError("save_obj writes non-instanced scenes")
    base = os.path.dirname(os.path.abspath(path))
    stem = os.path.splitext(os.path.basename(path))[0]
    tex_names = []
    for i, t in enumerate(desc.textures):
        name = f"{stem}_tex{i}.png"
        with open(os.path.join(base, name), "wb") as f:
            f.write(encode_png_rgba(t, filter_type=i % 5))
        tex_names.append(name)
    with open(os.path.join(base, stem + ".mtl"), "w") as f:
        for i, m in enumerate(desc.materials):
            f.write(f"newmtl m{i}\nKd {_fmt(m['diffuse'])}\nKs {_fmt(m['specular'])}\n")
            f.write(f"Ke {_fmt(m['emission'])}\nPr {float(m['roughness'])!r}\n")
            if desc.material_textures is not None:
                for key, t in zip(("map_Kd", "map_Ks", "map_Pr"), desc.material_textures[i]):
                    if t >= 0:
                        f.write(f"{key} {tex_names[t]}\n")
    uvs = desc.uvs if desc.uvs is not None else np.zeros((len(desc.positions), 2), np.float32)
    with open(path, "w") as f:
        f.write(f"mtllib {stem}.mtl\n")
        for p in desc.positions:
            f.write(f"v {_fmt(p)}\n")
        for t in uvs:
            f.write(f"vt {_fmt(t)}\n")
        for n in desc.normals:
            f.write(f"vn {_fmt(n)}\n")
        cur = None
        for tri, mi in zip(desc.indices, desc.triangle_material):
            if mi != cur:
                f.write(f"usemtl m{int(mi)}\n")
                cur = mi
            f.write("f " + " ".join(f"{int(v) + 1}/{int(v) + 1}/{int(v) + 1}" for v in tri) + "\n")


# ---- FBX ----------------------------------------------------------------------------
# The reference reads FBX through assimp (src/Model.cpp:9-207).  This reader
# covers the binary format's node tree (FBX 7.x: 32-bit node records before
# version 7500, 64-bit from it; zlib-compressed arrays) and the parts of the
# scene graph the reference's Model uses, mapped as assimp's FBX importer maps
# them:
#
# * Geometry (Mesh): `Vertices`, `PolygonVertexIndex` (a negative index ends a
#   polygon: -(i + 1)); polygons fanned into triangles (aiProcess_Triangulate);
#   `LayerElementNormal` / `LayerElementUV` mapped ByPolygonVertex or
#   ByVertice, referenced Direct or IndexToDirect; `LayerElementMaterial`
#   AllSame or ByPolygon; polygons without normals get their face normal
#   (aiProcess_GenNormals); every polygon corner is its own vertex;
# * Model: the FBX SDK's transform chain -- translation, rotation offset and
#   pivot, pre-rotation, `Lcl Rotation` in the model's RotationOrder,
#   post-rotation, scaling offset and pivot, `Lcl Scaling` -- through the
#   parent chain (Connections "OO"), times the model's own geometric
#   translation / rotation / scaling, baked into the triangles (normals by
#   the inverse transpose);
# * Material: DiffuseColor, SpecularColor, EmissiveColor, each times its
#   ...Factor when present (assimp's factored colours), a Roughness or
#   RoughnessFactor property if the file has one, with the reference's
#   fallbacks otherwise (diffuse and specular 1, emission 0, roughness 1);
#   Texture objects connected ("OP") to DiffuseColor / SpecularColor /
#   Roughness (or 3ds Max's roughness_map) give the diffuse / specular /
#   roughness textures: embedded (a Video object's Content) or the file
#   (RelativeFilename, else FileName's base name, relative to the FBX's
#   folder); PNG;
# * faces of a material with non-zero emission form one emitter per material,
#   as in load_obj.
#
# The ASCII form (`Name: values { children }`, arrays as `*N { a: ... }`) is
# read into the same node tree; its embedded contents are not.

_FBX_MAGIC = b"Kaydara FBX Binary  \x00\x1a\x00"


class FbxNode:
    """One node of the FBX tree: name, property values, children."""

    def __init__(self, name: str, props=None, children=None):
        self.name = name
        self.props = list(props or [])
        self.children = list(children or [])

    def child(self, name: str) -> Optional["FbxNode"]:
        for c in self.children:
            if c.name == name:
                return c
        return None

    def all(self, name: str) -> List["FbxNode"]:
        return [c for c in self.children if c.name == name]


_ARRAY_DTYPE = {ord("f"): "<f4", ord("d"): "<f8", ord("l"): "<i8", ord("i"): "<i4", ord("b"): "u1"}


def _fbx_prop(buf: bytes, o: int):
    t = buf[o]
    o += 1
    if t == ord("Y"):
        return struct.unpack_from("<h", buf, o)[0], o + 2
    if t == ord("C"):
        return bool(buf[o]), o + 1
    if t == ord("I"):
        return struct.unpack_from("<i", buf, o)[0], o + 4
    if t == ord("F"):
        return struct.unpack_from("<f", buf, o)[0], o + 4
    if t == ord("D"):
        return struct.unpack_from("<d", buf, o)[0], o + 8
    if t == ord("L"):
        return struct.unpack_from("<q", buf, o)[0], o + 8
    if t in _ARRAY_DTYPE:
        n, enc, clen = struct.unpack_from("<III", buf, o)
        o += 12
        raw = buf[o:o + clen]
        if enc == 1:
            raw = zlib.decompress(raw)
        elif enc != 0:
            raise ValueError(f"FBX: array encoding {enc}")
        return np.frombuffer(raw, dtype=_ARRAY_DTYPE[t], count=n).copy(), o + clen
    if t in (ord("S"), ord("R")):
        n = struct.unpack_from("<I", buf, o)[0]
        o += 4
        v = bytes(buf[o:o + n])
        return (v.decode("utf-8", "replace") if t == ord("S") else v), o + n
    raise ValueError(f"FBX: property type {chr(t)!r} at byte {o - 1}")


def _fbx_node(buf: bytes, o: int, wide: bool):
    """(node or None for a null record, offset after it)."""
    hdr = "<QQQ" if wide else "<III"
    end, nprops, _plen = struct.unpack_from(hdr, buf, o)
    o += 24 if wide else 12
    nlen = buf[o]
    o += 1
    if end == 0:
        return None, o  # null record: the rest of it is zeros
    name = bytes(buf[o:o + nlen]).decode("ascii", "replace")
    o += nlen
    props = []
    for _ in range(nprops):
        v, o = _fbx_prop(buf, o)
        props.append(v)
    children = []
    while o < end:
        c, o2 = _fbx_node(buf, o, wide)
        if c is None:
            o = end
            break
        children.append(c)
        o = o2
    return FbxNode(name, props, children), end


_FBX_TOKEN = __import__("re").compile(
    r'\s+|;[^\n]*|(?P<name>[A-Za-z_][\w|]*):|(?P<str>"(?:[^"\\]|\\.)*")|(?P<count>\*\d+)'
    r'|(?P<num>[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?)|(?P<sym>[{},])|(?P<word>[A-Za-z_][\w|]*)')


def _fbx_ascii_tokens(text: str):
    toks = []
    for m in _FBX_TOKEN.finditer(text):
        k = m.lastgroup
        if k is None:
            continue  # white space, comment
        toks.append((k, m.group(k)))
    return toks


def _fbx_ascii_block(toks, i: int) -> Tuple[List[FbxNode], int]:
    nodes = []
    while i < len(toks) and toks[i] != ("sym", "}"):
        kind, name = toks[i]
        if kind != "name":
            raise ValueError(f"FBX (ASCII): expected a node name, got {name!r}")
        i += 1
        props: list = []
        children: List[FbxNode] = []
        while i < len(toks) and toks[i][0] in ("str", "num", "count", "word", "sym") and toks[i] != ("sym", "}"):
            kind, v = toks[i]
            if (kind, v) == ("sym", "{"):
                children, i = _fbx_ascii_block(toks, i + 1)
                i += 1  # the closing brace
                break
            if kind == "sym":  # a comma
                i += 1
            elif kind == "count":  # *N { a: values }
                if toks[i + 1] != ("sym", "{") or toks[i + 2] != ("name", "a"):
                    raise ValueError("FBX (ASCII): malformed array")
                i += 3
                vals = []
                while toks[i] != ("sym", "}"):
                    if toks[i][0] == "num":
                        vals.append(toks[i][1])
                    i += 1
                i += 1
                is_float = any(("." in x) or ("e" in x) or ("E" in x) for x in vals)
                props.append(np.array([float(x) for x in vals], np.float64) if is_float
                             else np.array([int(x) for x in vals], np.int64))
            elif kind == "num":
                props.append(float(v) if any(c in v for c in ".eE") else int(v))
                i += 1
            elif kind == "str":
                props.append(v[1:-1].replace("&quot;", '"'))
                i += 1
            else:
                props.append(v)
                i += 1
        nodes.append(FbxNode(name, props, children))
    return nodes, i


def _read_fbx_ascii(text: str) -> Tuple[int, List[FbxNode]]:
    nodes, _ = _fbx_ascii_block(_fbx_ascii_tokens(text), 0)
    version = 0
    for n in nodes:
        if n.name == "FBXHeaderExtension" and n.child("FBXVersion") is not None:
            version = int(n.child("FBXVersion").props[0])
    return version, nodes


def read_fbx_tree(data: bytes) -> Tuple[int, List[FbxNode]]:
    """(version, top-level nodes) of a binary or ASCII FBX file."""
    if not data.startswith(_FBX_MAGIC):
        text = data.decode("utf-8", "replace").lstrip("\ufeff")
        version, nodes = _read_fbx_ascii(text)
        if not any(n.name == "Objects" for n in nodes) and not any(n.name == "FBXHeaderExtension" for n in nodes):
            raise ValueError("not an FBX file")
        return version, nodes
    version = struct.unpack_from("<I", data, len(_FBX_MAGIC))[0]
    wide = version >= 7500
    o = len(_FBX_MAGIC) + 4
    nodes = []
    while o < len(data):
        if o + (25 if wide else 13) > len(data):
            break
        node, o = _fbx_node(data, o, wide)
        if node is None:
            break
        nodes.append(node)
    return version, nodes


def _p70(node: Optional[FbxNode]) -> Dict[str, list]:
    """An object's Properties70: property name -> its values (after the
    name, type, label and flags strings)."""
    out: Dict[str, list] = {}
    p = node.child("Properties70") if node is not None else None
    if p is not None:
        for q in p.all("P"):
            if q.props:
                out[str(q.props[0])] = list(q.props[4:])
    return out


# FBX's RotationOrder enum: the axes in the order they are applied
_ROT_ORDERS = ("xyz", "xzy", "yzx", "yxz", "zxy", "zyx")


def _euler(deg, order: int = 0) -> np.ndarray:
    """Rotation by Euler angles (degrees) applied in RotationOrder `order`
    (0, eEulerXYZ: about x first, then y, then z)."""
    a = np.radians(np.asarray(deg, np.float64)[:3])
    c, s = np.cos(a), np.sin(a)
    R = {"x": np.array([[1, 0, 0], [0, c[0], -s[0]], [0, s[0], c[0]]]),
         "y": np.array([[c[1], 0, s[1]], [0, 1, 0], [-s[1], 0, c[1]]]),
         "z": np.array([[c[2], -s[2], 0], [s[2], c[2], 0], [0, 0, 1]])}
    M = np.eye(3)
    for axis in _ROT_ORDERS[order if 0 <= order < 6 else 0]:
        M = R[axis] @ M
    return M


def _m4(R=None, t=None, s=None) -> np.ndarray:
    M = np.eye(4)
    if R is not None:
        M[:3, :3] = R
    if s is not None:
        M[:3, :3] = M[:3, :3] @ np.diag(np.asarray(s, np.float64)[:3])
    if t is not None:
        M[:3, 3] = np.asarray(t, np.float64)[:3]
    return M


def _fbx_local(props: Dict[str, list]) -> np.ndarray:
    """A model's local transform as the FBX SDK composes it:
    T * Roff * Rp * Rpre * R * Rpost^-1 * Rp^-1 * Soff * Sp * S * Sp^-1
    (pre- and post-rotations in XYZ order, R in the model's RotationOrder)."""
    def v(name, default):
        return props.get(name, default)[:3]

    order = int(props.get("RotationOrder", [0])[0])
    z3 = [0.0, 0.0, 0.0]
    Rp, Sp = _m4(t=v("RotationPivot", z3)), _m4(t=v("ScalingPivot", z3))
    Rpost = _m4(R=_euler(v("PostRotation", z3)))
    return (_m4(t=v("Lcl Translation", z3)) @ _m4(t=v("RotationOffset", z3)) @ Rp
            @ _m4(R=_euler(v("PreRotation", z3))) @ _m4(R=_euler(v("Lcl Rotation", z3), order))
            @ np.linalg.inv(Rpost) @ np.linalg.inv(Rp) @ _m4(t=v("ScalingOffset", z3)) @ Sp
            @ _m4(s=v("Lcl Scaling", [1.0, 1.0, 1.0])) @ np.linalg.inv(Sp))


def _fbx_geometric(props: Dict[str, list]) -> np.ndarray:
    """The geometric transform of a model's own geometry (not inherited)."""
    z3 = [0.0, 0.0, 0.0]
    return _m4(R=_euler(props.get("GeometricRotation", z3)[:3]), t=props.get("GeometricTranslation", z3)[:3],
               s=props.get("GeometricScaling", [1.0, 1.0, 1.0])[:3])


def _fbx_layer(geom: FbxNode, layer: str, data: str, index: str, width: int, corner_vertex: np.ndarray,
               corner_polygon: np.ndarray) -> Optional[np.ndarray]:
    """Per-corner values of the geometry's first `layer` (or None)."""
    el = geom.child(layer)
    if el is None or el.child(data) is None:
        return None
    mapping = str(el.child("MappingInformationType").props[0]) if el.child("MappingInformationType") else "ByVertice"
    ref = str(el.child("ReferenceInformationType").props[0]) if el.child("ReferenceInformationType") else "Direct"
    vals = np.asarray(el.child(data).props[0], np.float64).reshape(-1, width)
    n = len(corner_vertex)
    if mapping == "ByPolygonVertex":
        key = np.arange(n)
    elif mapping in ("ByVertice", "ByVertex", "ByControlPoint"):
        key = corner_vertex
    elif mapping == "ByPolygon":
        key = corner_polygon
    elif mapping == "AllSame":
        key = np.zeros(n, np.int64)
    else:
        raise ValueError(f"FBX {layer}: mapping {mapping}")
    if ref in ("IndexToDirect", "Index") and el.child(index) is not None:  # without indices: direct
        key = np.asarray(el.child(index).props[0], np.int64)[key]
    return vals[key]


def _factored(props: Dict[str, list], name: str, default) -> List[float]:
    """assimp's factored colour: <name>Color times <name>Factor when present
    (the old `<name>` key when there is no `<name>Color`)."""
    c = props.get(name + "Color", props.get(name))
    if c is None:
        return list(default)
    col = [float(x) for x in c[:3]]
    f = props.get(name + "Factor")
    return [x * float(f[0]) for x in col] if f else col


def load_fbx(path: str, flip_uv: bool = False, spec_usage: int = 0) -> scenes.Scene:
    """Scene description of an FBX file (binary or ASCII): every mesh model's polygons,
    triangulated and transformed to world space, its materials and their PNG
    textures (paths relative to the file's folder)."""
    base = os.path.dirname(os.path.abspath(path))
    with open(path, "rb") as f:
        _version, top = read_fbx_tree(f.read())
    find = {n.name: n for n in top}
    if "Objects" not in find:
        raise ValueError(f"{path}: no Objects")
    objects: Dict[int, FbxNode] = {int(n.props[0]): n for n in find["Objects"].children if n.props}
    oo, op = [], []
    for c in (find["Connections"].all("C") if "Connections" in find else []):
        if c.props[0] == "OO":
            oo.append((int(c.props[1]), int(c.props[2])))
        elif c.props[0] == "OP":
            op.append((int(c.props[1]), int(c.props[2]), str(c.props[3]) if len(c.props) > 3 else ""))

    def kind(i):
        n = objects.get(i)
        return n.name if n is not None else None

    parent = {c: p for c, p in oo if kind(c) == "Model" and kind(p) == "Model"}
    world_cache: Dict[int, np.ndarray] = {}

    def world(m: int) -> np.ndarray:
        if m not in world_cache:
            local = _fbx_local(_p70(objects[m]))
            world_cache[m] = world(parent[m]) @ local if m in parent else local
        return world_cache[m]

    mat_ids = [i for i, n in objects.items() if n.name == "Material"]
    model_mats: Dict[int, List[int]] = {}
    geom_models: Dict[int, List[int]] = {}
    for c, p in oo:
        if kind(c) == "Material" and kind(p) == "Model":
            model_mats.setdefault(p, []).append(mat_ids.index(c))
        elif kind(c) == "Geometry" and kind(p) == "Model":
            geom_models.setdefault(c, []).append(p)
    tex_of: Dict[Tuple[int, str], int] = {}
    for c, p, prop in op:
        if kind(c) == "Texture" and kind(p) == "Material":
            tex_of[(mat_ids.index(p), prop)] = c
    # embedded image bytes: a Video object connected to the texture
    video_of = {p: c for c, p in oo if kind(c) == "Video" and kind(p) == "Texture"}

    pos: List[np.ndarray] = []
    nrm: List[np.ndarray] = []
    uv: List[np.ndarray] = []
    tri_mat: List[np.ndarray] = []
    n_vert = 0
    extra_default = False  # polygons whose model has no material for their slot
    for gid, g in objects.items():
        if g.name != "Geometry" or g.child("Vertices") is None or g.child("PolygonVertexIndex") is None:
            continue
        V = np.asarray(g.child("Vertices").props[0], np.float64).reshape(-1, 3)
        pvi = np.asarray(g.child("PolygonVertexIndex").props[0], np.int64)
        ends = pvi < 0
        cv = np.where(ends, -pvi - 1, pvi)
        cp = np.concatenate([[0], np.cumsum(ends)[:-1]]).astype(np.int64)
        cn = _fbx_layer(g, "LayerElementNormal", "Normals", "NormalsIndex", 3, cv, cp)
        cu = _fbx_layer(g, "LayerElementUV", "UV", "UVIndex", 2, cv, cp)
        ml = g.child("LayerElementMaterial")
        starts = np.concatenate([[0], np.flatnonzero(ends)[:-1] + 1])
        npoly = len(starts)
        if ml is not None and ml.child("Materials") is not None:
            slots = np.asarray(ml.child("Materials").props[0], np.int64)
            mapping = str(ml.child("MappingInformationType").props[0]) if ml.child("MappingInformationType") \
                else "AllSame"
            poly_slot = slots[:npoly] if mapping == "ByPolygon" else np.full(npoly, slots[0] if len(slots) else 0)
        else:
            poly_slot = np.zeros(npoly, np.int64)
        # fan triangles: (first, k, k + 1) corners of each polygon
        tri_c, tri_p = [], []
        for p_i, (s, e) in enumerate(zip(starts, np.flatnonzero(ends))):
            for k in range(s + 1, e):
                tri_c.append((s, k, k + 1))
                tri_p.append(p_i)
        if not tri_c:
            continue
        tri_c = np.asarray(tri_c, np.int64)
        tri_p = np.asarray(tri_p, np.int64)
        for m in geom_models.get(gid, []):
            M = world(m) @ _fbx_geometric(_p70(objects[m]))
            A, t = M[:3, :3], M[:3, 3]
            ident = np.array_equal(M, np.eye(4))  # untransformed: values kept bit for bit
            P = V[cv[tri_c]] if ident else V[cv[tri_c]] @ A.T + t  # (T, 3, 3) per triangle corner
            if cn is not None:
                Nn = cn[tri_c]
                if not ident:
                    Nn = Nn @ np.linalg.inv(A)  # the inverse transpose
                    Nn = Nn / np.maximum(np.linalg.norm(Nn, axis=2, keepdims=True), 1e-30)
            else:
                fn = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
                ln = np.linalg.norm(fn, axis=1, keepdims=True)
                fn = np.where(ln > 0, fn / np.maximum(ln, 1e-30), np.array([[0.0, 0.0, 1.0]]))
                Nn = np.repeat(fn[:, None, :], 3, axis=1)
            U = cu[tri_c] if cu is not None else np.zeros((len(tri_c), 3, 2))
            if flip_uv:
                U = np.stack([U[..., 0], 1.0 - U[..., 1]], axis=-1)
            slots_m = model_mats.get(m, [])
            ts = poly_slot[tri_p]
            gm = np.array([slots_m[s] if 0 <= s < len(slots_m) else -1 for s in ts], np.int64)
            if (gm < 0).any():
                extra_default = True
                gm = np.where(gm < 0, len(mat_ids), gm)
            pos.append(P.reshape(-1, 3))
            nrm.append(Nn.reshape(-1, 3))
            uv.append(U.reshape(-1, 2))
            tri_mat.append(gm)
            n_vert += 3 * len(tri_c)
    if not pos:
        raise ValueError(f"{path}: no mesh polygons")
    textures: List[np.ndarray] = []
    tex_index: Dict[int, int] = {}

    def texture(tid: Optional[int]) -> int:
        if tid is None:
            return -1
        if tid not in tex_index:
            t = objects[tid]
            v = objects.get(video_of.get(tid, -1))
            content = v.child("Content") if v is not None else None
            if content is not None and content.props and isinstance(content.props[0], bytes) \
                    and content.props[0].startswith(_SIG):
                textures.append(decode_png_rgba(content.props[0]))
                tex_index[tid] = len(textures) - 1
                return tex_index[tid]
            name = None
            for key in ("RelativeFilename", "FileName"):
                if t.child(key) is not None and t.child(key).props and str(t.child(key).props[0]):
                    name = str(t.child(key).props[0]).replace("\\", "/")
                    break
            if name is None:
                return -1
            fp = os.path.join(base, name)
            if not os.path.exists(fp):
                fp = os.path.join(base, os.path.basename(name))
            with open(fp, "rb") as tf:
                textures.append(decode_png_rgba(tf.read()))
            tex_index[tid] = len(textures) - 1
        return tex_index[tid]

    mats, mt = [], []
    for i, mid in enumerate(mat_ids + ([None] if extra_default else [])):
        props = _p70(objects[mid]) if mid is not None else {}
        m = np.zeros((), dtype=scenes.MATERIAL_DTYPE)
        m["diffuse"] = _factored(props, "Diffuse", (1.0, 1.0, 1.0))
        m["specular"] = _factored(props, "Specular", (1.0, 1.0, 1.0))
        m["emission"] = _factored(props, "Emissive", (0.0, 0.0, 0.0))
        r = props.get("Roughness", props.get("RoughnessFactor"))
        m["roughness"] = float(r[0]) if r else 1.0
        m["spec_usage"] = spec_usage
        mats.append(m)
        rough_tex = tex_of.get((i, "Roughness"), tex_of.get((i, "3dsMax|Parameters|roughness_map")))
        mt.append([texture(tex_of.get((i, "DiffuseColor"))), texture(tex_of.get((i, "SpecularColor"))),
                   texture(rough_tex)])
    P = np.concatenate(pos).astype(np.float32)
    T = np.arange(len(P), dtype=np.uint32).reshape(-1, 3)
    TM = np.concatenate(tri_mat).astype(np.uint32)
    emitters, faces = [], []
    for i, m in enumerate(mats):
        e = [float(x) for x in m["emission"]]
        if any(v != 0.0 for v in e):
            sel = np.flatnonzero(TM == i)
            if len(sel):
                emitters.append((tuple(e), len(faces), len(sel)))
                faces.extend(P[T[sel]].reshape(-1, 9))
    mt_arr = np.asarray(mt, np.int32).reshape(-1, 3)
    return scenes.Scene(P, np.concatenate(nrm).astype(np.float32), T, TM, np.stack(mats),
                        np.zeros((0, 2), np.uint32), [], emitters,
                        np.asarray(faces, np.float32).reshape(-1, 9), name=os.path.basename(path),
                        uvs=np.concatenate(uv).astype(np.float32), textures=textures,
                        material_textures=mt_arr if (mt_arr >= 0).any() else None)


_ARRAY_CODE = {np.dtype("<f4"): b"f", np.dtype("<f8"): b"d", np.dtype("<i8"): b"l", np.dtype("<i4"): b"i",
               np.dtype("u1"): b"b"}


def _fbx_prop_bytes(v) -> bytes:
    if isinstance(v, (bool, np.bool_)):
        return b"C" + bytes([1 if v else 0])
    if isinstance(v, (int, np.integer)):
        return b"L" + struct.pack("<q", int(v))
    if isinstance(v, (float, np.floating)):
        return b"D" + struct.pack("<d", float(v))
    if isinstance(v, str):
        b = v.encode("utf-8")
        return b"S" + struct.pack("<I", len(b)) + b
    if isinstance(v, bytes):
        return b"R" + struct.pack("<I", len(v)) + v
    a = np.ascontiguousarray(v)
    dt = a.dtype.newbyteorder("<") if a.dtype.itemsize > 1 else np.dtype("u1")
    raw = a.astype(dt).tobytes()
    enc, data = (1, zlib.compress(raw)) if len(raw) > 64 else (0, raw)  # both encodings occur
    return _ARRAY_CODE[dt] + struct.pack("<III", a.size, enc, len(data)) + data


def _fbx_node_bytes(node: FbxNode, offset: int, wide: bool) -> bytes:
    name = node.name.encode("ascii")
    props = b"".join(_fbx_prop_bytes(v) for v in node.props)
    head_len = (25 if wide else 13) + len(name)
    body = b""
    if node.children:
        pos = offset + head_len + len(props)
        for c in node.children:
            cb = _fbx_node_bytes(c, pos, wide)
            body += cb
            pos += len(cb)
        body += b"\x00" * (25 if wide else 13)  # null record ends the child list
    end = offset + head_len + len(props) + len(body)
    head = struct.pack("<QQQ" if wide else "<III", end, len(node.props), len(props)) + bytes([len(name)]) + name
    return head + props + body


def write_fbx_tree(path: str, nodes: List[FbxNode], version: int = 7400) -> None:
    """Write top-level nodes as a binary FBX file of `version` (64-bit node
    records from 7500)."""
    wide = version >= 7500
    out = bytearray(_FBX_MAGIC + struct.pack("<I", version))
    for n in nodes:
        out += _fbx_node_bytes(n, len(out), wide)
    out += b"\x00" * (25 if wide else 13)
    with open(path, "wb") as f:
        f.write(bytes(out))


def _fbx_ascii_value(v) -> str:
    if isinstance(v, (bool, np.bool_)):
        return "T" if v else "F"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    if isinstance(v, bytes):
        return '""'  # embedded content is not written in the ASCII form
    s = str(v)
    if "\x00\x01" in s:  # binary "name\x00\x01Class" is "Class::name" in ASCII
        name, cls = s.split("\x00\x01", 1)
        s = f"{cls}::{name}"
    return '"' + s.replace('"', "&quot;") + '"'


def _fbx_ascii_lines(node: FbxNode, indent: str) -> List[str]:
    if len(node.props) == 1 and isinstance(node.props[0], np.ndarray):
        a = node.props[0].reshape(-1)
        vals = ",".join(repr(float(x)) if a.dtype.kind == "f" else str(int(x)) for x in a)
        return [f"{indent}{node.name}: *{a.size} {{", f"{indent}\ta: {vals}", f"{indent}}}"]
    head = f"{indent}{node.name}: " + ",".join(_fbx_ascii_value(v) for v in node.props)
    if not node.children:
        return [head]
    out = [head + " {"]
    for c in node.children:
        out.extend(_fbx_ascii_lines(c, indent + "\t"))
    return out + [f"{indent}}}"]


def write_fbx_ascii_tree(path: str, nodes: List[FbxNode]) -> None:
    """Write top-level nodes as an ASCII FBX file."""
    lines = ["; FBX 7.4.0 project file"]
    for n in nodes:
        lines.extend(_fbx_ascii_lines(n, ""))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def fbx_p(name: str, kind: str, *values) -> FbxNode:
    """A Properties70 entry."""
    return FbxNode("P", [name, kind, "", "A", *values])


def save_fbx(path: str, desc: scenes.Scene, version: int = 7400, ascii: bool = False) -> None:
    """Write a non-instanced scene as a binary (or ASCII) FBX that load_fbx
    reads back to the same triangles (every corner's position, normal and
    uv), materials, textures and emitters: one Geometry (normals and uvs by
    vertex, materials by polygon), one Model, one Material per material
    (textures connected to DiffuseColor, SpecularColor and Roughness)."""
    if desc.instances:
        raise ValueError("save_fbx writes non-instanced scenes")
    base = os.path.dirname(os.path.abspath(path))
    stem = os.path.splitext(os.path.basename(path))[0]
    tex_names = []
    for i, t in enumerate(desc.textures):
        name = f"{stem}_tex{i}.png"
        with open(os.path.join(base, name), "wb") as f:
            f.write(encode_png_rgba(t))
        tex_names.append(name)
    idx = np.asarray(desc.indices, np.int64).reshape(-1, 3).copy()
    idx[:, 2] = -idx[:, 2] - 1  # a negative index ends a polygon
    layers = [FbxNode("LayerElementNormal", [0], [
        FbxNode("MappingInformationType", ["ByVertice"]), FbxNode("ReferenceInformationType", ["Direct"]),
        FbxNode("Normals", [np.asarray(desc.normals, np.float64).reshape(-1)])])]
    if desc.uvs is not None:
        layers.append(FbxNode("LayerElementUV", [0], [
            FbxNode("MappingInformationType", ["ByVertice"]), FbxNode("ReferenceInformationType", ["Direct"]),
            FbxNode("UV", [np.asarray(desc.uvs, np.float64).reshape(-1)])]))
    layers.append(FbxNode("LayerElementMaterial", [0], [
        FbxNode("MappingInformationType", ["ByPolygon"]), FbxNode("ReferenceInformationType", ["IndexToDirect"]),
        FbxNode("Materials", [np.asarray(desc.triangle_material, np.int32)])]))
    objs = [FbxNode("Geometry", [1000, "geometry\x00\x01Geometry", "Mesh"], [
        FbxNode("Vertices", [np.asarray(desc.positions, np.float64).reshape(-1)]),
        FbxNode("PolygonVertexIndex", [idx.reshape(-1).astype(np.int32)])] + layers),
        FbxNode("Model", [2000, "model\x00\x01Model", "Mesh"], [FbxNode("Properties70")])]
    conns = [FbxNode("C", ["OO", 2000, 0]), FbxNode("C", ["OO", 1000, 2000])]
    for i, m in enumerate(desc.materials):
        objs.append(FbxNode("Material", [3000 + i, f"m{i}\x00\x01Material", ""], [FbxNode("Properties70", [], [
            fbx_p("DiffuseColor", "Color", *[float(x) for x in m["diffuse"]]),
            fbx_p("SpecularColor", "Color", *[float(x) for x in m["specular"]]),
            fbx_p("EmissiveColor", "Color", *[float(x) for x in m["emission"]]),
            fbx_p("Roughness", "Number", float(m["roughness"]))])]))
        conns.append(FbxNode("C", ["OO", 3000 + i, 2000]))
    mt = desc.material_textures
    for t, name in enumerate(tex_names):
        objs.append(FbxNode("Texture", [4000 + t, f"t{t}\x00\x01Texture", ""], [FbxNode("RelativeFilename", [name])]))
    if mt is not None:
        for i, row in enumerate(np.asarray(mt).reshape(-1, 3)):
            for slot, prop in enumerate(("DiffuseColor", "SpecularColor", "Roughness")):
                if row[slot] >= 0:
                    conns.append(FbxNode("C", ["OP", 4000 + int(row[slot]), 3000 + i, prop]))
    top = [FbxNode("FBXHeaderExtension", [], [FbxNode("FBXVersion", [version])]),
           FbxNode("Objects", [], objs), FbxNode("Connections", [], conns)]
    if ascii:
        write_fbx_ascii_tree(path, top)
    else:
        write_fbx_tree(path, top, version)


def load_model(path: str, flip_uv: bool = False, spec_usage: int = 0) -> scenes.Scene:
    """Model(path, flipUv, specTexUsage) (src/Model.cpp:9-44): the scene
    description of an OBJ or FBX file, by its extension."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".obj":
        return load_obj(path, flip_uv, spec_usage)
    if ext == ".fbx":
        return load_fbx(path, flip_uv, spec_usage)
    raise ValueError(f"{path}: only .obj and .fbx files are read")
