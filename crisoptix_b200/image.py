"""Frame output without a display: sRGB tone mapping on the GPU and PNG / PFM
files on the host.

The reference tone-maps the HDR frame into an OpenGL pixel buffer and draws
it (src/main.cpp:110-135, src/kernel/tonemap.cu:23-39).  Here the same
tone-mapping kernel writes a device byte buffer, which the caller keeps or
writes to a file.  Row 0 of a frame buffer is the TOP row of the image: launch
row 0 maps to uv.y = -1, and the camera's V axis points down (Camera::GetData
negates the up vector, src/Camera.cpp:28), so that ray looks up.  The PNG
writer emits rows in order; the PFM writer, whose format stores the bottom row
first, emits them last to first.
"""
import struct
import zlib

import numpy as np

from ._abi import check, load


def tonemap(rgb, out=None, stream: int = 0):
    """sRGB bytes of a CUDA float32 tensor of shape (..., 3) through
    crisb_tonemap_srgb8: the sRGB transfer curve per channel, clamped to
    [0, 1], times 255, truncated.  Returns a uint8 tensor of the same shape."""
    import torch

    if not (isinstance(rgb, torch.Tensor) and rgb.is_cuda and rgb.dtype == torch.float32):
        raise TypeError("tonemap takes a CUDA float32 tensor")
    if rgb.shape[-1] != 3:
        raise ValueError("last dimension must be 3 (RGB)")
    rgb = rgb.contiguous()
    if out is None:
        out = torch.empty(rgb.shape, dtype=torch.uint8, device=rgb.device)
    elif out.shape != rgb.shape or out.dtype != torch.uint8 or not out.is_contiguous():
        raise ValueError("out must be a contiguous uint8 tensor of the input's shape")
    check(load().crisb_tonemap_srgb8(rgb.data_ptr(), out.data_ptr(), rgb.numel() // 3, stream))
    return out


def _chunk(kind: bytes, data: bytes) -> bytes:
    body = kind + data
    return struct.pack(">I", len(data)) + body + struct.pack(">I", zlib.crc32(body) & 0xFFFFFFFF)


def encode_png(srgb8: np.ndarray, bottom_up: bool = False) -> bytes:
    """8-bit RGB PNG of an (H, W, 3) uint8 array (filter 0 on every row)."""
    a = np.ascontiguousarray(srgb8)
    if a.dtype != np.uint8 or a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("expected an (H, W, 3) uint8 array")
    h, w, _ = a.shape
    rows = a[::-1] if bottom_up else a
    raw = np.zeros((h, 1 + 3 * w), np.uint8)
    raw[:, 1:] = rows.reshape(h, 3 * w)
    header = struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)
    return (b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", header) + _chunk(b"IDAT", zlib.compress(raw.tobytes(), 6)) +
            _chunk(b"IEND", b""))


def decode_png(data: bytes) -> np.ndarray:
    """(H, W, 3) uint8 array of an 8-bit RGB PNG written by encode_png (top row
    first, filter 0 rows only)."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG file")
    pos, idat = 8, b""
    w = h = 0
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if zlib.crc32(kind + body) & 0xFFFFFFFF != struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]:
            raise ValueError("PNG chunk CRC mismatch")
        if kind == b"IHDR":
            w, h, depth, color = struct.unpack(">IIBB", body[:10])
            if depth != 8 or color != 2:
                raise ValueError("only 8-bit RGB PNG files are read")
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    if raw[:, 0].any():
        raise ValueError("only filter-0 rows are read")
    return raw[:, 1:].reshape(h, w, 3).copy()


def write_png(path: str, srgb8: np.ndarray, bottom_up: bool = False) -> None:
    """Write an (H, W, 3) uint8 frame as PNG; `bottom_up` says row 0 is the
    bottom of the image (frame buffers have it at the top)."""
    with open(path, "wb") as f:
        f.write(encode_png(srgb8, bottom_up))


def write_pfm(path: str, rgb: np.ndarray) -> None:
    """Write an (H, W, 3) float frame (row 0 the top) as a little-endian PFM,
    which stores rows bottom to top."""
    a = np.ascontiguousarray(rgb, dtype="<f4")
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("expected an (H, W, 3) array")
    h, w, _ = a.shape
    with open(path, "wb") as f:
        f.write(f"PF\n{w} {h}\n-1.0\n".encode("ascii"))
        f.write(np.ascontiguousarray(a[::-1]).tobytes())


def read_pfm(path: str) -> np.ndarray:
    """(H, W, 3) float32 array of a colour PFM file, row 0 the top row."""
    with open(path, "rb") as f:
        if f.readline().strip() != b"PF":
            raise ValueError("not a colour PFM file")
        w, h = (int(v) for v in f.readline().split())
        scale = float(f.readline())
        a = np.frombuffer(f.read(w * h * 12), "<f4" if scale < 0 else ">f4")
    return np.ascontiguousarray(a.reshape(h, w, 3)[::-1]).astype(np.float32)


def save_frame(path: str, hdr, stream: int = 0) -> np.ndarray:
    """Tone-map a (H, W, 3) CUDA float32 frame on the GPU and write it as PNG.
    Returns the sRGB bytes."""
    import torch

    srgb = tonemap(hdr, stream=stream)
    if stream:
        torch.cuda.ExternalStream(stream).synchronize()
    host = srgb.cpu().numpy()
    write_png(path, host)
    return host
