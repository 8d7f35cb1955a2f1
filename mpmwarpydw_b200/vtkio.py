"""VTK XML files without the vtk package: PolyData (.vtp) particles and
ImageData (.vti) grids, as the reference's output and restart path writes and
reads them (utils/fs5PlotUtils.py:433-639 save_grid_and_particles_vti_vtp,
:253-431 load_restart_from_vtp).

Format (the VTK XML file format, version 0.1 / 1.0):
  * ``<VTKFile type=... byte_order="LittleEndian" header_type="UInt32|UInt64"
    compressor="vtkZLibDataCompressor">``;
  * each ``<DataArray type=... Name=... NumberOfComponents=... format=...>``
    holds its values ``ascii`` (text), ``binary`` (base64 inline) or
    ``appended`` (at ``offset`` in ``<AppendedData encoding="raw|base64">``
    after the ``_`` marker);
  * binary data is a header of header_type integers followed by the data.
    Uncompressed: [byte count].  Compressed: [number of blocks, uncompressed
    block size, uncompressed size of the last block, compressed size of each
    block], then the zlib blocks back to back.  Inline base64 encodes the
    header and the blocks as two separate base64 runs when compressed.

The writer produces inline binary, zlib-compressed, UInt32 headers (what
vtkXMLWriter and ParaView read), 32 KiB blocks.
"""
from __future__ import annotations

import base64
import re
import xml.etree.ElementTree as ET
import zlib

import numpy as np

VTK_TYPES = {
    "Int8": np.int8, "UInt8": np.uint8, "Int16": np.int16, "UInt16": np.uint16, "Int32": np.int32,
    "UInt32": np.uint32, "Int64": np.int64, "UInt64": np.uint64, "Float32": np.float32, "Float64": np.float64,
}
NP_TO_VTK = {np.dtype(v).str[1:]: k for k, v in VTK_TYPES.items()}
BLOCK = 32768


# ---------------------------------------------------------------------------
# reading
# ---------------------------------------------------------------------------
class _File:
    def __init__(self, path):
        raw = open(path, "rb").read()
        # an <AppendedData> section holds raw bytes that are not XML: cut it out
        # before parsing and keep it for the arrays that point into it
        self.appended = b""
        self.appended_encoding = None
        m = re.search(rb"<AppendedData[^>]*>", raw)
        if m:
            enc = re.search(rb'encoding="([^"]+)"', m.group(0))
            self.appended_encoding = enc.group(1).decode() if enc else "raw"
            start = raw.index(b"_", m.end()) + 1
            end = raw.rindex(b"</AppendedData>")
            self.appended = raw[start:end]
            if self.appended_encoding == "base64":
                self.appended = self.appended.strip()
            else:
                # raw data ends just before the closing tag's leading whitespace
                self.appended = self.appended.rstrip(b"\n\r\t ")
            raw = raw[:m.start()] + b"<AppendedData/>" + raw[end + len(b"</AppendedData>"):]
        self.root = ET.fromstring(raw)
        if self.root.tag != "VTKFile":
            raise ValueError(f"{path}: not a VTK XML file")
        if self.root.get("byte_order", "LittleEndian") != "LittleEndian":
            raise ValueError(f"{path}: big-endian VTK files are not supported")
        self.header = np.uint64 if self.root.get("header_type", "UInt32") == "UInt64" else np.uint32
        self.compressed = self.root.get("compressor") is not None
        comp = self.root.get("compressor")
        if comp is not None and comp != "vtkZLibDataCompressor":
            raise ValueError(f"{path}: compressor {comp} is not supported (zlib only)")

    # binary payload (header + data) starting at byte 0 of `buf`; returns (bytes, consumed)
    def _decode_binary(self, buf: bytes):
        hs = np.dtype(self.header).itemsize
        if not self.compressed:
            nbytes = int(np.frombuffer(buf[:hs], self.header)[0])
            return buf[hs:hs + nbytes], hs + nbytes
        nb = int(np.frombuffer(buf[:hs], self.header)[0])
        h = np.frombuffer(buf[:hs * (3 + nb)], self.header).astype(np.int64)
        sizes = h[3:]
        out, pos = [], hs * (3 + nb)
        for c in sizes:
            out.append(zlib.decompress(buf[pos:pos + int(c)]))
            pos += int(c)
        return b"".join(out), pos

    def _inline_base64(self, text: str):
        s = "".join(text.split())
        hs = np.dtype(self.header).itemsize
        if not self.compressed:
            return self._decode_binary(base64.b64decode(s))[0]
        # the header is its own base64 run: first read the block count
        first = base64.b64decode(s[:4 * ((hs + 2) // 3)])
        nb = int(np.frombuffer(first[:hs], self.header)[0])
        hlen = 4 * ((hs * (3 + nb) + 2) // 3)
        head = base64.b64decode(s[:hlen])
        body = base64.b64decode(s[hlen:])
        return self._decode_binary(head[:hs * (3 + nb)] + body)[0]

    def array(self, el):
        """numpy array of one DataArray element ((n,) or (n, components))."""
        dt = VTK_TYPES[el.get("type")]
        ncomp = int(el.get("NumberOfComponents", "1"))
        fmt = el.get("format", "ascii")
        if fmt == "ascii":
            a = np.array((el.text or "").split(), dtype=dt)
        elif fmt == "binary":
            a = np.frombuffer(self._inline_base64(el.text or ""), dtype=np.dtype(dt).newbyteorder("<")).copy()
        elif fmt == "appended":
            off = int(el.get("offset"))
            if self.appended_encoding == "base64":
                # each array is its own base64 run (or two, header and blocks) at its offset
                data = self._appended_base64(self.appended[off:].decode())
            else:
                data, _ = self._decode_binary(self.appended[off:])
            a = np.frombuffer(data, dtype=np.dtype(dt).newbyteorder("<")).copy()
        else:
            raise ValueError(f"DataArray format {fmt} is not supported")
        return a.reshape(-1, ncomp) if ncomp > 1 else a

    def _appended_base64(self, rest: str):
        hs = np.dtype(self.header).itemsize
        if not self.compressed:
            first = base64.b64decode(rest[:4 * ((hs + 2) // 3)])
            nbytes = int(np.frombuffer(first[:hs], self.header)[0])
            total = 4 * ((hs + nbytes + 2) // 3)
            return self._decode_binary(base64.b64decode(rest[:total]))[0]
        first = base64.b64decode(rest[:4 * ((hs + 2) // 3)])
        nb = int(np.frombuffer(first[:hs], self.header)[0])
        hlen = 4 * ((hs * (3 + nb) + 2) // 3)
        head = base64.b64decode(rest[:hlen])[:hs * (3 + nb)]
        sizes = np.frombuffer(head, self.header).astype(np.int64)[3:]
        blen = 4 * ((int(sizes.sum()) + 2) // 3)
        body = base64.b64decode(rest[hlen:hlen + blen])
        return self._decode_binary(head + body)[0]


def read_vtp(path):
    """Particles of a .vtp file: dict with ``points`` (n, 3), ``point_data``
    {name: array} and ``field_data`` {name: array}."""
    f = _File(path)
    piece = f.root.find("PolyData/Piece")
    if piece is None:
        raise ValueError(f"{path}: no PolyData piece")
    pts_el = piece.find("Points/DataArray")
    pts = f.array(pts_el).reshape(-1, 3) if pts_el is not None else np.zeros((0, 3))
    n = int(piece.get("NumberOfPoints", pts.shape[0]))
    if pts.shape[0] != n:
        raise ValueError(f"{path}: {pts.shape[0]} points, header says {n}")
    pd = {el.get("Name"): f.array(el) for el in piece.findall("PointData/DataArray")}
    fd = {el.get("Name"): f.array(el) for el in f.root.findall("PolyData/FieldData/DataArray")}
    return {"points": pts, "point_data": pd, "field_data": fd}


def read_vti(path):
    """Grid of a .vti file: dict with ``dims`` (nx, ny, nz), ``origin``,
    ``spacing`` and ``point_data`` {name: (nx, ny, nz[, c]) array in C order}."""
    f = _File(path)
    img = f.root.find("ImageData")
    ext = [int(v) for v in img.get("WholeExtent").split()]
    dims = (ext[1] - ext[0] + 1, ext[3] - ext[2] + 1, ext[5] - ext[4] + 1)
    out = {"dims": dims, "origin": np.array([float(v) for v in img.get("Origin").split()]),
           "spacing": np.array([float(v) for v in img.get("Spacing").split()]), "point_data": {}}
    for el in img.findall("Piece/PointData/DataArray"):
        a = f.array(el)
        c = a.shape[1] if a.ndim == 2 else None
        # VTK stores x fastest (Fortran order over (nx, ny, nz))
        shp = (dims[2], dims[1], dims[0]) + ((c,) if c else ())
        a = a.reshape(shp)
        out["point_data"][el.get("Name")] = np.ascontiguousarray(np.moveaxis(a, (0, 1, 2), (2, 1, 0)))
    return out


# ---------------------------------------------------------------------------
# writing
# ---------------------------------------------------------------------------
def _encode(a: np.ndarray) -> str:
    """Inline binary payload: UInt32 header of the zlib blocks, then the blocks,
    as two base64 runs."""
    raw = np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<"), copy=False).tobytes()
    blocks = [raw[i:i + BLOCK] for i in range(0, len(raw), BLOCK)] or [b""]
    comp = [zlib.compress(b) for b in blocks]
    last = len(blocks[-1]) if raw else 0
    head = np.array([len(blocks), BLOCK, last] + [len(c) for c in comp], dtype="<u4").tobytes()
    return base64.b64encode(head).decode() + base64.b64encode(b"".join(comp)).decode()


def _data_array(name, a, extra=""):
    a = np.asarray(a)
    if a.dtype == np.float16 or a.dtype.kind == "b":
        a = a.astype(np.float32 if a.dtype == np.float16 else np.uint8)
    ncomp = 1 if a.ndim == 1 else int(np.prod(a.shape[1:]))
    t = NP_TO_VTK[a.dtype.str[1:]]
    nc = f' NumberOfComponents="{ncomp}"' if ncomp > 1 else ""
    flat = a.reshape(a.shape[0], -1) if a.ndim > 1 else a
    return f'<DataArray type="{t}" Name="{name}"{nc} format="binary"{extra}>{_encode(flat)}</DataArray>'


def _header(kind):
    return (f'<?xml version="1.0"?>\n<VTKFile type="{kind}" version="1.0" byte_order="LittleEndian" '
            f'header_type="UInt32" compressor="vtkZLibDataCompressor">\n')


def write_vtp(path, points, point_data=None, field_data=None):
    """Particles as a .vtp file: one vertex per point, every point_data array
    (n,) or (n, c), field_data arrays (one tuple each, or more)."""
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    n = pts.shape[0]
    parts = [_header("PolyData"), "<PolyData>\n"]
    if field_data:
        parts.append("<FieldData>\n")
        for k, v in field_data.items():
            v = np.atleast_1d(np.asarray(v))
            parts.append(_data_array(k, v, f' NumberOfTuples="{v.shape[0]}"') + "\n")
        parts.append("</FieldData>\n")
    parts.append(f'<Piece NumberOfPoints="{n}" NumberOfVerts="{n}" NumberOfLines="0" NumberOfStrips="0" '
                 f'NumberOfPolys="0">\n<PointData>\n')
    for k, v in (point_data or {}).items():
        v = np.asarray(v)
        if v.shape[0] != n:
            raise ValueError(f"point array {k} has {v.shape[0]} entries for {n} points")
        parts.append(_data_array(k, v) + "\n")
    parts.append("</PointData>\n<Points>\n" + _data_array("Points", pts) + "\n</Points>\n<Verts>\n")
    parts.append(_data_array("connectivity", np.arange(n, dtype=np.int64)) + "\n")
    parts.append(_data_array("offsets", np.arange(1, n + 1, dtype=np.int64)) + "\n")
    parts.append("</Verts>\n</Piece>\n</PolyData>\n</VTKFile>\n")
    with open(path, "w") as fh:
        fh.write("".join(parts))


def write_vti(path, dims, origin, spacing, point_data):
    """A grid as a .vti file; each point_data array is (nx, ny, nz[, c]) in C order."""
    nx, ny, nz = (int(d) for d in dims)
    sp = [float(v) for v in np.broadcast_to(np.asarray(spacing, np.float64), (3,))]
    org = [float(v) for v in np.asarray(origin, np.float64).reshape(3)]
    parts = [_header("ImageData"),
             f'<ImageData WholeExtent="0 {nx - 1} 0 {ny - 1} 0 {nz - 1}" '
             f'Origin="{org[0]!r} {org[1]!r} {org[2]!r}" Spacing="{sp[0]!r} {sp[1]!r} {sp[2]!r}">\n',
             f'<Piece Extent="0 {nx - 1} 0 {ny - 1} 0 {nz - 1}">\n<PointData>\n']
    for k, v in point_data.items():
        v = np.asarray(v)
        c = v.shape[3] if v.ndim == 4 else None
        f = np.moveaxis(v, (0, 1, 2), (2, 1, 0)).reshape(nx * ny * nz, *((c,) if c else ()))  # x fastest
        parts.append(_data_array(k, f) + "\n")
    parts.append("</PointData>\n</Piece>\n</ImageData>\n</VTKFile>\n")
    with open(path, "w") as fh:
        fh.write("".join(parts))
