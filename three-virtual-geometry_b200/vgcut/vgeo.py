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
`indices` is rebuilt from meshletInfo / meshletVertices / meshletTriangles, serialize.ts:395-413). The reference's
compressed files also use meshoptimizer's vertex and index codecs (`meshopt-vertex`, `meshlet-triangles`);
meshoptimizer is an npm dependency that is not vendored with the reference, so this reader rejects those two
encodings with a VirtualMeshFormatError naming them, and the writer never produces them (files written with the
reference's `{compress: false}` read here, and files written here read in the reference).
"""
from __future__ import annotations

import json
import math
import zlib

import numpy as np

from . import build as B

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


def encode(data, deflate: bool = True, keep_indices: bool = False) -> bytes:
    """A .vgeo file for `data` (VirtualMeshData or a record of the reference's fields): each array raw or, where
    smaller, raw-deflated; `indices` dropped and rebuilt on decode when the meshlet arrays reproduce it."""
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
        enc = f["encoding"]
        if enc == "raw":
            if len(blob) != f["length"] * dt.itemsize:
                raise VirtualMeshFormatError(f'geometry file is corrupt (field "{f["name"]}" has the wrong size)')
            arrays[f["name"]] = np.frombuffer(blob, dt).astype(dt.newbyteorder("="))
        elif enc == "meshlet-indices":
            need = [arrays.get(k) for k in ("meshletInfo", "meshletVertices", "meshletTriangles")]
            if any(a is None for a in need):
                raise VirtualMeshFormatError(f'geometry file is corrupt ("{f["name"]}" needs the meshlet arrays)')
            arrays[f["name"]] = rebuild_indices(f["length"], *need)
        elif enc in ("meshopt-vertex", "meshlet-triangles"):
            raise VirtualMeshFormatError(f'field "{f["name"]}" uses the meshoptimizer codec "{enc}", which this reader '
                                         f"does not have (bake the file with compress: false)")
        else:
            raise VirtualMeshFormatError(f'unknown encoding "{enc}" for field "{f["name"]}"')
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
