"""meshoptimizer's vertex and index codecs (the reference's compressed `.vgeo` fields, serialize.ts:244 / :290) and the
compressed container (the reference's default `compress: true`).

No file written by meshoptimizer is available here (it is an npm dependency the reference does not vendor), so the
decoders are pinned by streams built by hand from the published format description - each byte derived in the
comments - and by round trips through this package's own encoders; parity with meshoptimizer's own output is
unpinned."""
import json

import numpy as np
import pytest

from vgcut import meshopt, scenes, vgeo


# ---------------------------------------------------------------- vertex codec: hand-built streams
def test_vertex_v0_known_stream():
    # 16 vertices of 4 bytes, vertex i = (i, 0, 0, 0). Byte column 0: deltas from the previous vertex (the first,
    # (0, 0, 0, 0), before vertex 0) are 0, 1, 1, ..., zigzag-coded 0, 2, 2, ...; version 0 widths {0, 2, 4, 8}:
    # one group at 2 bits (header 0b01), values most significant first: 0,2,2,2 -> 0x2a, then 2,2,2,2 -> 0xaa x 3.
    # Columns 1-3 are zero: a 0-bit group each (header 0x00, no data). Tail: 32 bytes, the first vertex last.
    stream = bytes([0xa0, 0x01, 0x2a, 0xaa, 0xaa, 0xaa, 0x00, 0x00, 0x00]) + bytes(28) + bytes(4)
    got = np.frombuffer(meshopt.decode_vertex_buffer(stream, 16, 4), np.uint32)
    assert got.tolist() == list(range(16))


def test_vertex_v1_literal_zero_and_16bit_columns():
    # vertex i = 300 i as a u32, channel 1 (16-bit deltas): low word delta 300 (zigzag 600 = 0x0258) after vertex 0
    # (delta 0), high word 0. Column 0 (0x00, then 0x58 x 15) as literal bytes (control 3); column 1 (0, then 2 x 15)
    # in byte groups of control 0 (widths {0, 1, 2, 4}): 2 bits = header 0b10, packed 0x2a 0xaa 0xaa 0xaa;
    # columns 2, 3 all zero (control 2). Control byte: 3 | 0 << 2 | 2 << 4 | 2 << 6 = 0xa3. Tail: 19 zero bytes of
    # padding (24 - 5), the first vertex, channel byte 1.
    stream = bytes([0xa1, 0xa3, 0x00] + [0x58] * 15 + [0x02, 0x2a, 0xaa, 0xaa, 0xaa]) + bytes(19) + bytes(4) + b"\x01"
    got = np.frombuffer(meshopt.decode_vertex_buffer(stream, 16, 4), np.uint32)
    assert got.tolist() == [300 * i for i in range(16)]


def test_vertex_v1_one_bit_group_with_escapes():
    # byte 0 of vertex 3 is 5, everything else 0: column 0 deltas are +5 at vertex 3 and -5 at vertex 4 (zigzag 10, 9).
    # A 1-bit group (control 0, header 0b01): a set bit is the sentinel, bits least significant first -> bits 3, 4 of
    # byte 0 = 0x18, byte 1 = 0x00, then the escaped values 10, 9. Columns 1-3: control 2. Control byte
    # 0 | 2 << 2 | 2 << 4 | 2 << 6 = 0xa8. Tail: 19 zero bytes, first vertex, channel byte 0.
    stream = bytes([0xa1, 0xa8, 0x01, 0x18, 0x00, 0x0a, 0x09]) + bytes(19) + bytes(4) + b"\x00"
    got = np.frombuffer(meshopt.decode_vertex_buffer(stream, 16, 4), np.uint8).reshape(16, 4)
    want = np.zeros((16, 4), np.uint8)
    want[3, 0] = 5
    assert np.array_equal(got, want)


def test_vertex_decoder_rejects_bad_streams():
    good = meshopt.encode_vertex_buffer(np.arange(64, dtype=np.float32).tobytes(), 16)
    with pytest.raises(meshopt.CodecError, match="header"):
        meshopt.decode_vertex_buffer(b"\xb1" + good[1:], 16, 16)
    with pytest.raises(meshopt.CodecError, match="header"):
        meshopt.decode_vertex_buffer(b"\xa2" + good[1:], 16, 16)
    with pytest.raises(meshopt.CodecError, match="truncated"):
        meshopt.decode_vertex_buffer(good[:20], 16, 16)
    with pytest.raises(meshopt.CodecError):
        meshopt.decode_vertex_buffer(good + bytes(4), 16, 16)


# ---------------------------------------------------------------- vertex codec: round trips
@pytest.mark.parametrize("version", [0, 1])
@pytest.mark.parametrize("stride", [4, 8, 12, 16, 64, 256])
def test_vertex_round_trip(version, stride):
    rng = np.random.default_rng(stride * 3 + version)
    for count in (0, 1, 15, 16, 17, 255, 256, 257, 3001):
        noise = rng.integers(0, 256, count * stride, dtype=np.uint8).tobytes()
        assert meshopt.decode_vertex_buffer(meshopt.encode_vertex_buffer(noise, stride, version), count, stride) == noise
        smooth = np.cumsum(rng.integers(-3, 4, count * stride // 4), dtype=np.int64).astype(np.uint32).tobytes()
        enc = meshopt.encode_vertex_buffer(smooth, stride, version)
        assert meshopt.decode_vertex_buffer(enc, count, stride) == smooth
        if count >= 256:
            assert len(enc) < len(smooth) * 0.6, "slowly varying data compresses"


def test_vertex_round_trip_mesh_fields():
    m = scenes.icosphere_mesh(16)
    for arr, stride in ((m.positions, 12), (m.meshlet_bounds, 64), (m.meshlet_info, 16)):
        raw = np.ascontiguousarray(arr).tobytes()
        enc = meshopt.encode_vertex_buffer(raw, stride)
        assert meshopt.decode_vertex_buffer(enc, len(raw) // stride, stride) == raw
        assert len(enc) < len(raw)


# ---------------------------------------------------------------- index codec
def index_stream(codes, data):
    table = [0x00, 0x76, 0x87, 0x56, 0x67, 0x78, 0xa9, 0x86, 0x65, 0x89, 0x68, 0x98, 0x01, 0x69, 0, 0]
    return bytes([0xe1] + codes + data + table)


def test_index_known_streams():
    # (0, 1, 2): no edge in the FIFO, a = next (0): aux code 0x00 (b, c the next new vertices) is table entry 0 ->
    # code 0xf0. (2, 1, 3): its edge (2, 1) is FIFO entry 1 (pushed (1,0), (2,1), (0,2)); c = 3 = next -> 0x10.
    assert meshopt.decode_index_buffer(index_stream([0xf0, 0x10], []), 6).tolist() == [0, 1, 2, 2, 1, 3]
    # (5, 9, 7): no vertex is next (0) -> code 0xff, aux 0xff from the data, then three free indices as zigzag deltas
    # from the last one (0): +5 -> 10, +4 -> 8, -2 -> 3. (9, 5, 8): edge (9, 5) is FIFO entry 2; c = 8 = last + 1 ->
    # code 2 << 4 | 14 = 0x2e (version 1), no data.
    assert meshopt.decode_index_buffer(index_stream([0xff, 0x2e], [0xff, 0x0a, 0x08, 0x03]), 6).tolist() == \
        [5, 9, 7, 9, 5, 8]


def rotated_equal(a, b):
    a, b = np.asarray(a).reshape(-1, 3), np.asarray(b).reshape(-1, 3)
    return all(tuple(x) in {tuple(y), (y[1], y[2], y[0]), (y[2], y[0], y[1])} for x, y in zip(a, b))


@pytest.mark.parametrize("version", [0, 1])
def test_index_round_trip(version):
    m = scenes.icosphere_mesh(16)
    info = np.asarray(m.meshlet_info, np.uint32).reshape(-1, 4)
    tris = np.asarray(m.meshlet_triangles, np.uint32)
    slots = np.concatenate([(np.stack([tris[f // 3:f // 3 + c] & 255, (tris[f // 3:f // 3 + c] >> 8) & 255,
                                       (tris[f // 3:f // 3 + c] >> 16) & 255], 1) + v).reshape(-1)
                            for c, f, _, v in info.tolist()])
    rng = np.random.default_rng(version)
    cases = [slots, np.asarray(m.indices, np.uint32), rng.integers(0, 1 << 20, 3 * 500, dtype=np.uint32),
             np.array([0, 1, 2, 2, 1, 3, 0, 1, 2, 4, 5, 6, 0, 1, 2], np.uint32), np.zeros(0, np.uint32)]
    for idx in cases:
        enc = meshopt.encode_index_buffer(idx, version)
        dec = meshopt.decode_index_buffer(enc, idx.size)
        assert rotated_equal(dec, idx)
    assert len(meshopt.encode_index_buffer(slots, version)) < slots.size, "meshlet slots take under a byte per index"


def test_index_decoder_rejects_bad_streams():
    enc = meshopt.encode_index_buffer(np.arange(30, dtype=np.uint32))
    with pytest.raises(meshopt.CodecError, match="header"):
        meshopt.decode_index_buffer(b"\xd1" + enc[1:], 30)
    with pytest.raises(meshopt.CodecError, match="truncated"):
        meshopt.decode_index_buffer(enc[:10], 30)
    with pytest.raises(meshopt.CodecError, match="unread"):
        meshopt.decode_index_buffer(enc[:-16] + b"\0" + enc[-16:], 30)


# ---------------------------------------------------------------- compressed .vgeo
def test_compressed_file_round_trip_and_encodings():
    m = scenes.icosphere_mesh(16)
    plain = vgeo.encode(m)
    packed = vgeo.encode(m, compress=True)
    back = vgeo.decode(packed)
    ra, rb = vgeo.to_record(m), vgeo.to_record(back)
    for k in ra:
        if isinstance(ra[k], np.ndarray):
            assert ra[k].dtype == rb[k].dtype and ra[k].tobytes() == rb[k].tobytes(), k
    n = int.from_bytes(packed[8:12], "little")
    enc = {f["name"]: f["encoding"] for f in json.loads(packed[16:16 + n])["fields"]}
    assert enc["meshletTriangles"] == "meshlet-triangles"
    assert enc["indices"] == "meshlet-indices"
    assert "meshopt-vertex" in enc.values()
    assert len(packed) < len(plain), (len(packed), len(plain))


def test_meshlet_triangles_keep_corner_order():
    m = scenes.icosphere_mesh(8)
    blob = vgeo.encode_meshlet_triangles(m.meshlet_triangles, m.meshlet_info)
    assert blob is not None
    got = vgeo.decode_meshlet_triangles(len(m.meshlet_triangles), blob, m.meshlet_info)
    assert np.array_equal(got, np.asarray(m.meshlet_triangles, np.uint32))
    # a triangle using its top byte cannot be stored this way (serialize.ts:281)
    bad = np.array(m.meshlet_triangles, np.uint32)
    bad[0] |= 1 << 24
    assert vgeo.encode_meshlet_triangles(bad, m.meshlet_info) is None
