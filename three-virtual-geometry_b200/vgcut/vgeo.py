"""Baked geometry files (`.vgeo`): the reference's container for `VirtualMeshData` (src/core/io/serialize.ts).

Layout (little-endian), as the reference writes it:
    0   magic 'VGEO'
    4   u32 format version (1)
    8   u32 header byte length (UTF-8 JSON, space-padded to 4 bytes)
    12  u32 checksum of everything after this 16-byte prefix (serialize.ts:429-437)
    16  JSON header: {generator, keys (every top-level field in order), fields (typed arrays: name, type, length,
        encoding, [stride], [deflate], offset, byteLength), values (every other field; non-finite numbers as
        {"$number": "Infinity"})}
    ..  payload: one 4-byte aligned blob per typed-array field

Encodings: `raw` (the array's bytes), optionally `deflate` (raw deflate) on top; `meshlet-indices` (no bytes:
`indices` is rebuilt from meshletInfo / meshletVertices / meshletTriangles, serialize.ts:395-413); `meshopt-vertex`
(meshoptimizer's vertex codec over `stride`-byte elements, serialize.ts:338-343) and `meshlet-triangles` (u32 codec
length, meshoptimizer's index codec over the meshlet-vertex slots vertexOffset + local id, padded to 4 bytes, then
2-bit corner rotations per triangle; serialize.ts:264-300, :369-388). The codecs are in `vgcut.meshopt`; compressed
writing picks, per field, the smallest of raw and the codec candidates the reference tries (strides from its field
hints), deflates the best one where that is smaller, and keeps a candidate only if it decodes to the same bytes
(encodeField, serialize.ts:231-262).
"""
from __future__ import annotations

import json
import math
import zlib

import numpy as np

from . import build as B
from . import meshopt

MAGIC = 0x4F454756  # 'VGEO' as a little-endian u32
VG_FORMAT_VERSION = 1
PREFIX_BYTES = 16

# typed-array names of the reference <-> numpy
_TYPES = {"Int8Array": np.int8, "Uint8Array": np.uint8, "Uint8ClampedArray": np.uint8, "Int16Array": np.int16,
          "Uint16Array": np.uint16, "Int32Array": np.int32, "Uint32Array": np.uint32, "Float32Array": np.float32,
          "Float64Array": np.float64}
_NAME_OF = {np.dtype(np.int8): "Int8Array", np.dtype(np.uint8): "Uint8Array", np.dtype(np.int16): "Int16Array",
            np.dtype(np.uint16): "Uint16Array", np.dtype(np.int32): "Int32Array", np.dtype(np.uint32): "Uint32Array",
            np.dtype(np.float32): "Float32Array", np.dtype(np.float64): "Float64Array"}

# VirtualMeshData fields (buildVirtualMesh.ts:75-138) <-> this package's VirtualMeshData
_FIELDS = [("positions", "positions", np.float32), ("indices", "indices", np.uint32),
           ("meshletCount", "meshlet_count", None), ("meshletBounds", "meshlet_bounds", np.float32),
           ("meshletInfo", "meshlet_info", np.uint32), ("meshletVertices", "meshlet_vertices", np.uint32),
           ("meshletTriangles", "meshlet_triangles", np.uint32), ("levelRanges", "level_ranges", np.uint32),
           ("levelErrors", "level_errors", np.float32), ("levelGuardErrors", "level_guard_errors", np.float32),
           ("lodBoundsSphere", "lod_bounds_sphere", "sphere"), ("cullBoundsSphere", "cull_bounds_sphere", "sphere"),
           ("replacementGroup", "replacement_group", np.int32), ("replacementStart", "replacement_start", np.uint32),
           ("replacementIndices", "replacement_indices", np.uint32), ("boundingSphere", "bounding_sphere", "sphere"),
           ("stats", "stats", None)]
_KEY_ORDER = ["positions", "normals", "colors", "uvs", "indices", "meshletCount", "meshletBounds", "meshletInfo",
              "meshletVertices", "meshletTriangles", "levelRanges", "levelErrors", "levelGuardErrors",
              "lodBoundsSphere", "cullBoundsSphere", "replacementGroup", "replacementStart", "replacementIndices",
              "boundingSphere", "stats"]


class VirtualMeshFormatError(ValueError):
    """serialize.ts VirtualMeshFormatError: the bytes are not a readable geometry file."""

    def __init__(self, message: str):
        super().__init__(f"three-virtual-geometry: {message}")


def _align4(n: int) -> int:
    return (n + 3) & ~3


def checksum(data: bytes, start: int = PREFIX_BYTES) -> int:
    return int(B._lib().vgb_vgeo_checksum(data, len(data), start))


def _json_default(v):
    if isinstance(v, (np.integer,)):
        return int(v)
    if isinstance(v, (np.floating,)):
        return float(v)
    raise TypeError(type(v))


def _finite(v):
    """JSON has no Infinity / NaN: they go as {"$number": "..."} (serialize.ts jsonReplacer)."""
    if isinstance(v, float) and not math.isfinite(v):
        return {"$number": "Infinity" if v > 0 else ("-Infinity" if v < 0 else "NaN")}
    if isinstance(v, dict):
        return {k: _finite(x) for k, x in v.items()}
    if isinstance(v, (list, tuple)):
        return [_finite(x) for x in v]
    if isinstance(v, np.ndarray):
        raise VirtualMeshFormatError("typed array nested inside a field cannot be serialized; store it as a top-level field")
    return v


def _revive(v):
    if isinstance(v, dict):
        if list(v.keys()) == ["$number"]:
            return float(v["$number"])
        return {k: _revive(x) for k, x in v.items()}
    if isinstance(v, list):
        return [_revive(x) for x in v]
    return v


def to_record(data: B.VirtualMeshData) -> dict:
    """The reference's field names and types, in its key order (fields this package lacks come from `extra`)."""
    rec = {}
    ours = {ref: (name, kind) for ref, name, kind in _FIELDS}
    for key in _KEY_ORDER:
        if key in ours:
            name, kind = ours[key]
            v = getattr(data, name)
            if kind == "sphere":
                rec[key] = [float(x) for x in v]
            elif kind is None:
                rec[key] = v
            else:
                rec[key] = np.ascontiguousarray(v, kind)
        elif key in data.extra:
            rec[key] = data.extra[key]
    for key, v in data.extra.items():
        if key not in rec:
            rec[key] = v
    return rec


def from_record(rec: dict) -> B.VirtualMeshData:
    kw = {}
    for ref, name, kind in _FIELDS:
        if ref not in rec:
            raise VirtualMeshFormatError(f'geometry file lacks field "{ref}"')
        v = rec[ref]
        kw[name] = np.asarray(v, np.float32) if kind == "sphere" else v
    known = {ref for ref, _, _ in _FIELDS}
    return B.VirtualMeshData(**kw, extra={k: v for k, v in rec.items() if k not in known})


def rebuild_indices(length: int, info: np.ndarray, mverts: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """indices[firstIndex + 3t + k] = global vertex of corner k of the meshlet's triangle t (serialize.ts:395-413)."""
    info = np.asarray(info, np.uint32).reshape(-1, 4)
    out = np.zeros(length, np.uint32)
    for count, first, _, voff in info.tolist():
        if first + count * 3 > length or first // 3 + count > len(tris):
            raise VirtualMeshFormatError("geometry file is corrupt (meshlet range out of bounds)")
        p = np.asarray(tris[first // 3:first // 3 + count], np.uint32)
        local = np.stack([p & 255, (p >> 8) & 255, (p >> 16) & 255], axis=1).reshape(-1) + np.uint32(voff)
        if len(local) and int(local.max()) >= len(mverts):
            raise VirtualMeshFormatError("geometry file is corrupt (meshlet vertex out of bounds)")
        out[first:first + count * 3] = np.asarray(mverts, np.uint32)[local]
    return out


# per-field element strides the vertex codec is tried with (serialize.ts:92-100 FIELD_HINTS)
_STRIDES = {"positions": [12], "normals": [12], "colors": [12], "uvs": [8], "tangents": [16], "meshletBounds": [64],
            "meshletInfo": [16]}
_DEFLATE_RAW = {"meshletBounds"}


def _deflate(blob: bytes) -> bytes:
    z = zlib.compressobj(9, zlib.DEFLATED, -15)
    return z.compress(blob) + z.flush()


def encode_meshlet_triangles(tris: np.ndarray, info: np.ndarray) -> bytes | None:
    """encodeMeshletTriangles (serialize.ts:264-300): the triangles as an index-codec stream over meshlet-vertex
    slots plus each triangle's corner rotation; None when the meshlets do not cover every triangle exactly once or a
    triangle uses its top byte."""
    tris = np.asarray(tris, np.uint32).reshape(-1)
    info = np.asarray(info, np.uint32).reshape(-1, 4)
    slots = np.zeros(tris.size * 3, np.uint32)
    covered = np.zeros(tris.size, np.uint8)
    for count, first, _, voff in info.tolist():
        t0 = first // 3
        if t0 + count > tris.size:
            return None
        p = tris[t0:t0 + count]
        if covered[t0:t0 + count].any() or (p >> 24).any():
            return None
        covered[t0:t0 + count] = 1
        slots[t0 * 3:(t0 + count) * 3] = (np.stack([p & 255, (p >> 8) & 255, (p >> 16) & 255], 1) + voff).reshape(-1)
    if not covered.all():
        return None
    codec = meshopt.encode_index_buffer(slots)
    dec = meshopt.decode_index_buffer(codec, slots.size).reshape(-1, 3)
    s = slots.reshape(-1, 3)
    rot = np.full(tris.size, 3, np.uint8)
    rot[(s == dec).all(1)] = 0
    rot[(s[:, 0] == dec[:, 1]) & (s[:, 1] == dec[:, 2]) & (s[:, 2] == dec[:, 0]) & (rot == 3)] = 1
    rot[(s[:, 0] == dec[:, 2]) & (s[:, 1] == dec[:, 0]) & (s[:, 2] == dec[:, 1]) & (rot == 3)] = 2
    if (rot == 3).any():
        return None
    packed = np.zeros((tris.size + 3) // 4, np.uint8)
    np.bitwise_or.at(packed, np.arange(tris.size) >> 2, (rot << ((np.arange(tris.size) & 3) * 2)).astype(np.uint8))
    out = bytearray(4 + _align4(len(codec)))
    out[0:4] = len(codec).to_bytes(4, "little")
    out[4:4 + len(codec)] = codec
    return bytes(out) + packed.tobytes()


def decode_meshlet_triangles(length: int, blob: bytes, info: np.ndarray) -> np.ndarray:
    """decodeMeshletTriangles (serialize.ts:369-388)."""
    if len(blob) < 4:
        raise VirtualMeshFormatError("truncated triangle data")
    codec_len = int.from_bytes(blob[0:4], "little")
    rot_at = 4 + _align4(codec_len)
    if rot_at + (length + 3) // 4 > len(blob):
        raise VirtualMeshFormatError("truncated triangle data")
    slots = meshopt.decode_index_buffer(blob[4:4 + codec_len], length * 3).reshape(-1, 3)
    rot = np.frombuffer(blob[rot_at:rot_at + (length + 3) // 4], np.uint8)
    out = np.zeros(length, np.uint32)
    for count, first, _, voff in np.asarray(info, np.uint32).reshape(-1, 4).tolist():
        t0 = first // 3
        if t0 + count > length:
            raise VirtualMeshFormatError("meshlet range out of bounds")
        t = np.arange(t0, t0 + count)
        r = (rot[t >> 2] >> ((t & 3) * 2)) & 3
        xyz = slots[t0:t0 + count].astype(np.int64) - int(voff)
        a = np.where(r == 0, xyz[:, 0], np.where(r == 1, xyz[:, 1], xyz[:, 2]))
        b = np.where(r == 0, xyz[:, 1], np.where(r == 1, xyz[:, 2], xyz[:, 0]))
        c = np.where(r == 0, xyz[:, 2], np.where(r == 1, xyz[:, 0], xyz[:, 1]))
        if ((a | b | c) >> 8).any() or (np.minimum(np.minimum(a, b), c) < 0).any():
            raise VirtualMeshFormatError("meshlet-local vertex id out of range")
        out[t0:t0 + count] = (a | (b << 8) | (c << 16)).astype(np.uint32)
    return out


def _decode_field(f: dict, blob: bytes, dt: np.dtype, arrays: dict) -> np.ndarray:
    """decodeField (serialize.ts:328-361) after any inflate."""
    enc, nbytes = f["encoding"], f["length"] * dt.itemsize
    if enc == "raw":
        if len(blob) != nbytes:
            raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f["name"]}" has the wrong size)')
        return np.frombuffer(blob, dt).astype(dt.newbyteorder("="))
    if enc == "meshopt-vertex":
        stride = f.get("stride") or 0
        if stride <= 0 or stride % 4 or nbytes % stride:
            raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f["name"]}" stride)')
        raw = meshopt.decode_vertex_buffer(blob, nbytes // stride, stride) if nbytes else b""
        return np.frombuffer(raw, dt).astype(dt.newbyteorder("="))
    if enc == "meshlet-triangles":
        info = arrays.get("meshletInfo")
        if info is None:
            raise VirtualMeshFormatError(f'geometry file is corrupt ("{f["name"]}" needs "meshletInfo")')
        return decode_meshlet_triangles(f["length"], blob, info)
    if enc == "meshlet-indices":
        need = [arrays.get(k) for k in ("meshletInfo", "meshletVertices", "meshletTriangles")]
        if any(a is None for a in need):
            raise VirtualMeshFormatError(f'geometry file is corrupt ("{f["name"]}" needs the meshlet arrays)')
        return rebuild_indices(f["length"], *need)
    raise VirtualMeshFormatError(f'unknown encoding "{enc}" for field "{f["name"]}"')


def _encode_field(name: str, arr: np.ndarray, rec: dict, deflate: bool) -> tuple:
    """encodeField (serialize.ts:231-262): the smallest candidate that decodes back to the same bytes."""
    raw = arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()
    base = {"name": name, "type": _NAME_OF[arr.dtype], "length": int(arr.size)}
    raw_c = (dict(base, encoding="raw"), raw)
    cands = [raw_c]
    tri = encode_meshlet_triangles(arr, rec["meshletInfo"]) \
        if name == "meshletTriangles" and arr.dtype == np.uint32 and "meshletInfo" in rec else None
    if tri is not None:
        cands.append((dict(base, encoding="meshlet-triangles"), tri))
    elif len(raw) % 4 == 0 and len(raw) > 0:
        for stride in [s for s in _STRIDES.get(name, [max(4, arr.dtype.itemsize)])
                       if s % 4 == 0 and s <= 256 and len(raw) % s == 0]:
            cands.append((dict(base, encoding="meshopt-vertex", stride=stride),
                          meshopt.encode_vertex_buffer(raw, stride)))
    cands.sort(key=lambda c: len(c[1]))
    if deflate and len(raw) >= 64:
        todo = [cands[0], raw_c] if name in _DEFLATE_RAW and cands[0] is not raw_c else [cands[0]]
        cands += [(dict(e, deflate=True), _deflate(b)) for e, b in todo]
        cands.sort(key=lambda c: len(c[1]))
    dt = np.dtype(_TYPES[base["type"]]).newbyteorder("<")
    for entry, blob in cands:
        try:
            src = zlib.decompressobj(-15).decompress(blob) if entry.get("deflate") else blob
            if _decode_field(entry, src, dt, {"meshletInfo": rec.get("meshletInfo")}).astype(dt).tobytes() == raw:
                return entry, blob
        except (VirtualMeshFormatError, meshopt.CodecError):
            continue
    return raw_c


def encode(data, deflate: bool = True, keep_indices: bool = False, compress: bool = False) -> bytes:
    """A .vgeo file for `data` (VirtualMeshData or a record of the reference's fields); `indices` dropped and rebuilt
    on decode when the meshlet arrays reproduce it. compress=False: each array raw or, where smaller, raw-deflated.
    compress=True (the reference's default, encodeVirtualMesh): per array the smallest round-tripping candidate
    among raw, the meshoptimizer codecs and deflate over the best of them."""
    rec = to_record(data) if isinstance(data, B.VirtualMeshData) else dict(data)
    fields, blobs, values, offset = [], [], {}, 0
    keys = [k for k, v in rec.items()]
    for name in keys:
        value = rec[name]
        if not isinstance(value, np.ndarray):
            values[name] = _finite(value)
            continue
        if value.dtype not in _NAME_OF:
            raise VirtualMeshFormatError(f'cannot serialize field "{name}" of type {value.dtype}')
        arr = np.ascontiguousarray(value)
        entry = {"name": name, "type": _NAME_OF[arr.dtype], "length": int(arr.size)}
        blob = b""
        if name == "indices" and not keep_indices and _indices_match(rec):
            entry["encoding"] = "meshlet-indices"
        elif compress:
            entry, blob = _encode_field(name, arr, rec, deflate)
        else:
            raw = arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes()
            entry["encoding"], blob = "raw", raw
            if deflate and len(raw) >= 64:
                z = zlib.compressobj(9, zlib.DEFLATED, -15)
                packed = z.compress(raw) + z.flush()
                if len(packed) < len(raw):
                    entry["deflate"], blob = True, packed
        entry["offset"], entry["byteLength"] = offset, len(blob)
        fields.append(entry)
        blobs.append(blob)
        offset += _align4(len(blob))
    header = json.dumps({"generator": "three-virtual-geometry", "keys": keys, "fields": fields, "values": values},
                        separators=(",", ":"), default=_json_default).encode()
    hp = _align4(len(header))
    out = bytearray(PREFIX_BYTES + hp + offset)
    out[PREFIX_BYTES:PREFIX_BYTES + len(header)] = header
    out[PREFIX_BYTES + len(header):PREFIX_BYTES + hp] = b" " * (hp - len(header))
    base = PREFIX_BYTES + hp
    for f, blob in zip(fields, blobs):
        out[base + f["offset"]:base + f["offset"] + len(blob)] = blob
    out[0:4] = MAGIC.to_bytes(4, "little")
    out[4:8] = VG_FORMAT_VERSION.to_bytes(4, "little")
    out[8:12] = len(header).to_bytes(4, "little")
    out[12:16] = checksum(bytes(out)).to_bytes(4, "little")
    return bytes(out)


def _indices_match(rec: dict) -> bool:
    try:
        got = rebuild_indices(len(rec["indices"]), rec["meshletInfo"], rec["meshletVertices"], rec["meshletTriangles"])
    except (KeyError, VirtualMeshFormatError, IndexError):
        return False
    return np.array_equal(got, np.asarray(rec["indices"], np.uint32))


def decode_record(data: bytes) -> dict:
    """The reference's fields of a .vgeo file (decodeVirtualMesh, serialize.ts:159-208), with its checks."""
    b = bytes(data)
    if len(b) < PREFIX_BYTES or int.from_bytes(b[0:4], "little") != MAGIC:
        raise VirtualMeshFormatError("not a three-virtual-geometry geometry file (bad magic bytes)")
    version = int.from_bytes(b[4:8], "little")
    if version != VG_FORMAT_VERSION:
        raise VirtualMeshFormatError(f"unsupported geometry format version {version} (this build reads version "
                                     f"{VG_FORMAT_VERSION}); re-bake the file")
    hlen = int.from_bytes(b[8:12], "little")
    payload_start = PREFIX_BYTES + _align4(hlen)
    if payload_start > len(b) or len(b) % 4 != 0:
        raise VirtualMeshFormatError("geometry file is truncated")
    try:
        header = _revive(json.loads(b[PREFIX_BYTES:PREFIX_BYTES + hlen].decode()))
    except (UnicodeDecodeError, json.JSONDecodeError):
        raise VirtualMeshFormatError("geometry file is corrupt or truncated (unreadable header)") from None
    if not isinstance(header, dict) or not isinstance(header.get("fields"), list) or \
            not isinstance(header.get("keys"), list) or not isinstance(header.get("values"), dict):
        raise VirtualMeshFormatError("geometry file is corrupt (malformed header)")
    payload = b[payload_start:]
    rank = {"meshlet-triangles": 1, "meshlet-indices": 2}
    order = sorted(header["fields"], key=lambda f: rank.get(f.get("encoding"), 0))
    for f in order:
        if f.get("type") not in _TYPES or not isinstance(f.get("length"), int) or f["length"] < 0:
            raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f.get("name")}")')
        if f["offset"] % 4 != 0 or f["offset"] + f["byteLength"] > len(payload):
            raise VirtualMeshFormatError(f'geometry file is truncated (field "{f["name"]}")')
    if checksum(b) != int.from_bytes(b[12:16], "little"):
        raise VirtualMeshFormatError("geometry file is corrupt (checksum mismatch)")
    arrays = {}
    for f in order:
        dt = np.dtype(_TYPES[f["type"]]).newbyteorder("<")
        blob = payload[f["offset"]:f["offset"] + f["byteLength"]]
        try:
            if f.get("deflate"):
                blob = zlib.decompressobj(-15).decompress(blob)
        except zlib.error as e:
            raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f["name"]}": {e})') from None
        try:
            arrays[f["name"]] = _decode_field(f, blob, dt, arrays)
        except meshopt.CodecError as e:
            raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f["name"]}": {e})') from None
    return {k: (arrays[k] if k in arrays else header["values"].get(k)) for k in header["keys"]}


def decode(data: bytes) -> B.VirtualMeshData:
    return from_record(decode_record(data))


def load(path: str) -> B.VirtualMeshData:
    """loadVirtualMesh (serialize.ts:211-216) for a local file."""
    with open(path, "rb") as f:
        return decode(f.read())


def save(path: str, data: B.VirtualMeshData, **options) -> None:
    with open(path, "wb") as f:
        f.write(encode(data, **options))
