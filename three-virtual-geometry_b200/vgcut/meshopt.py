"""meshoptimizer's vertex and index buffer codecs, from the host library (``vgb_vertex_*`` / ``vgb_index_*`` in
``include/vgbuild.h``): the two codecs of the reference's compressed ``.vgeo`` fields (src/core/io/serialize.ts:244
``encodeVertexBufferLevel(raw, count, stride, 2, 1)``, :290 ``encodeIndexBuffer(slots, count, 4)``).

The decoders read meshoptimizer's published stream formats (vertex codec versions 0 and 1, index codec versions 0
and 1); the encoders are this package's own. meshoptimizer itself is not vendored with the reference and no file it
wrote is available here, so the codecs are checked by round trips and hand-built streams, not against its output.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native


class CodecError(ValueError):
    """A stream the decoder cannot read: bad header or version (-1), truncated (-2), bytes left over (-3)."""


_REASON = {-1: "bad header or version", -2: "truncated", -3: "unread bytes at the end", -4: "bad arguments"}
_bound = False


def _lib() -> C.CDLL:
    global _bound
    lib = _native.load("libvgbuild.so")
    if not _bound:
        u8p, sz = C.POINTER(C.c_uint8), C.c_size_t
        lib.vgb_vertex_encode_bound.argtypes, lib.vgb_vertex_encode_bound.restype = [sz, sz], sz
        lib.vgb_vertex_encode.argtypes, lib.vgb_vertex_encode.restype = [u8p, sz, C.c_void_p, sz, sz, C.c_int], sz
        lib.vgb_vertex_decode.argtypes, lib.vgb_vertex_decode.restype = [C.c_void_p, sz, sz, u8p, sz], C.c_int
        lib.vgb_index_encode_bound.argtypes, lib.vgb_index_encode_bound.restype = [sz, sz], sz
        lib.vgb_index_encode.argtypes = [u8p, sz, C.POINTER(C.c_uint32), sz, C.c_int]
        lib.vgb_index_encode.restype = sz
        lib.vgb_index_decode.argtypes, lib.vgb_index_decode.restype = [C.POINTER(C.c_uint32), sz, u8p, sz], C.c_int
        _bound = True
    return lib


def _u8(buf) -> tuple:
    a = np.frombuffer(bytes(buf), np.uint8) if not isinstance(buf, np.ndarray) else np.ascontiguousarray(buf, np.uint8)
    if a.size == 0:
        a = np.zeros(1, np.uint8)[:0]
    return a, a.ctypes.data_as(C.POINTER(C.c_uint8))


def encode_vertex_buffer(data, stride: int, version: int = 1) -> bytes:
    """Vertex-codec stream of `data` (bytes or an array; its byte length a multiple of `stride`)."""
    raw = np.ascontiguousarray(np.frombuffer(memoryview(data).cast("B"), np.uint8))
    if stride <= 0 or stride % 4 or stride > 256 or raw.size % stride:
        raise CodecError(f"stride {stride} does not divide {raw.size} bytes into 4-byte multiples of at most 256")
    count = raw.size // stride
    lib = _lib()
    cap = lib.vgb_vertex_encode_bound(count, stride)
    out = np.empty(cap, np.uint8)
    n = lib.vgb_vertex_encode(out.ctypes.data_as(C.POINTER(C.c_uint8)), cap, raw.ctypes.data, count, stride, version)
    if n == 0:
        raise CodecError("vertex encode failed (bad arguments)")
    return out[:n].tobytes()


def decode_vertex_buffer(stream, count: int, stride: int) -> bytes:
    """`count` vertices of `stride` bytes from a vertex-codec stream."""
    src, p = _u8(stream)
    out = np.empty(max(1, count * stride), np.uint8)
    rc = _lib().vgb_vertex_decode(out.ctypes.data, count, stride, p, src.size)
    if rc:
        raise CodecError(f"vertex stream: {_REASON.get(rc, rc)}")
    return out[:count * stride].tobytes()


def encode_index_buffer(indices, version: int = 1) -> bytes:
    """Index-codec stream of a triangle list (32-bit indices, a multiple of 3)."""
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    if idx.size % 3:
        raise CodecError("index count is not a multiple of 3")
    lib = _lib()
    cap = lib.vgb_index_encode_bound(idx.size, int(idx.max()) + 1 if idx.size else 0)
    out = np.empty(cap, np.uint8)
    n = lib.vgb_index_encode(out.ctypes.data_as(C.POINTER(C.c_uint8)), cap,
                             idx.ctypes.data_as(C.POINTER(C.c_uint32)), idx.size, version)
    if n == 0:
        raise CodecError("index encode failed (bad arguments)")
    return out[:n].tobytes()


def decode_index_buffer(stream, count: int) -> np.ndarray:
    """`count` 32-bit indices (a triangle list) from an index-codec stream."""
    src, p = _u8(stream)
    out = np.empty(max(1, count), np.uint32)
    rc = _lib().vgb_index_decode(out.ctypes.data_as(C.POINTER(C.c_uint32)), count, p, src.size)
    if rc:
        raise CodecError(f"index stream: {_REASON.get(rc, rc)}")
    return out[:count]
