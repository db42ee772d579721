"""Scene files: Wavefront OBJ + MTL with PNG textures.

The reference imports models with assimp (src/Model.cpp:9-207: triangulated,
normals generated where missing, optional uv flip) and reads textures with
stb_image as RGBA8 (src/Texture.cpp:8-30).  Neither library is part of this
package; this module reads the same inputs itself, for OBJ/MTL and 8-bit PNG:

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
