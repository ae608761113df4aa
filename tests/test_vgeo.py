""".vgeo files (the reference's baked geometry container, serialize.ts), after tests/serialize.test.ts: exact round
trips with and without deflate, indices dropped and rebuilt from the meshlet arrays or kept, the container's layout,
unknown fields (a typed array, null, an object holding Infinity) surviving, and the reference's rejections (empty,
foreign, newer version, flipped payload byte, truncation inside the payload and inside the header). Compressed files
(meshoptimizer's codecs, the reference's default) are covered in tests/test_meshopt.py; a codec field whose stream
is not one is rejected naming the field."""
import json

import numpy as np
import pytest

from vgcut import scenes, vgeo


@pytest.fixture(scope="module")
def mesh():
    return scenes.icosphere_mesh(12)


def same(a, b):
    ra, rb = vgeo.to_record(a), vgeo.to_record(b)
    assert list(ra.keys()) == list(rb.keys())
    for k in ra:
        x, y = ra[k], rb[k]
        if isinstance(x, np.ndarray):
            assert isinstance(y, np.ndarray) and x.dtype == y.dtype and x.tobytes() == y.tobytes(), k
        else:
            assert json.dumps(x, sort_keys=True) == json.dumps(y, sort_keys=True), k


def header_of(b):
    n = int.from_bytes(b[8:12], "little")
    return json.loads(b[16:16 + n])


@pytest.mark.parametrize("options", [{}, {"deflate": False}, {"keep_indices": True}])
def test_round_trip_is_exact(mesh, options):
    b = vgeo.encode(mesh, **options)
    back = vgeo.decode(b)
    same(mesh, back)
    f = next(f for f in header_of(b)["fields"] if f["name"] == "indices")
    if options.get("keep_indices"):
        assert f["encoding"] != "meshlet-indices"
    else:
        assert f["encoding"] == "meshlet-indices" and f["byteLength"] == 0, "indices dropped and rebuilt identically"


def test_container_layout(mesh, tmp_path):
    b = vgeo.encode(mesh)
    assert b[:4] == b"VGEO" and int.from_bytes(b[4:8], "little") == vgeo.VG_FORMAT_VERSION
    h = header_of(b)
    assert all(f["offset"] % 4 == 0 for f in h["fields"]) and len(b) % 4 == 0, "payload blobs are 4-byte aligned"
    assert h["keys"][0] == "positions" and "meshletBounds" in h["keys"]
    assert any(f.get("deflate") for f in h["fields"]), "deflate used where smaller"
    p = tmp_path / "m.vgeo"
    vgeo.save(str(p), mesh)
    same(mesh, vgeo.load(str(p)))


def test_unknown_fields_survive(mesh):
    ext = vgeo.from_record(vgeo.to_record(mesh))
    ext.extra = {"uvs": np.arange(len(mesh.positions) // 3 * 2, dtype=np.float32) * 0.25, "tangents": None,
                 "extra": {"scale": float("inf"), "tag": "x"}}
    back = vgeo.decode(vgeo.encode(ext))
    assert np.array_equal(back.extra["uvs"], ext.extra["uvs"]) and back.extra["uvs"].dtype == np.float32
    assert back.extra["tangents"] is None and back.extra["extra"] == {"scale": float("inf"), "tag": "x"}


def test_rejections(mesh):
    b = vgeo.encode(mesh)

    def patched(fn):
        c = bytearray(b)
        fn(c)
        return bytes(c)

    with pytest.raises(vgeo.VirtualMeshFormatError, match="not a three-virtual-geometry"):
        vgeo.decode(b"")
    with pytest.raises(vgeo.VirtualMeshFormatError, match="not a three-virtual-geometry"):
        vgeo.decode(b'{"glTF": "not this"}')
    with pytest.raises(vgeo.VirtualMeshFormatError, match="unsupported .*version"):
        vgeo.decode(patched(lambda c: c.__setitem__(slice(4, 8), (vgeo.VG_FORMAT_VERSION + 1).to_bytes(4, "little"))))
    with pytest.raises(vgeo.VirtualMeshFormatError, match="corrupt"):
        vgeo.decode(patched(lambda c: c.__setitem__(len(c) - 100, c[len(c) - 100] ^ 0x10)))
    with pytest.raises(vgeo.VirtualMeshFormatError, match="truncated"):
        vgeo.decode(b[:len(b) - 64])
    with pytest.raises(vgeo.VirtualMeshFormatError, match="truncated"):
        vgeo.decode(b[:40])


def test_bad_codec_stream_is_rejected_by_field(mesh):
    b = bytearray(vgeo.encode(mesh, deflate=False))
    n = int.from_bytes(b[8:12], "little")
    h = json.loads(b[16:16 + n])
    for f in h["fields"]:
        if f["name"] == "positions":
            f["encoding"], f["stride"] = "meshopt-vertex", 12
    text = json.dumps(h, separators=(",", ":")).encode()
    payload = bytes(b[16 + vgeo._align4(n):])
    pad = vgeo._align4(len(text)) - len(text)
    b = bytearray(16) + text + b" " * pad + payload
    b[0:8] = vgeo.MAGIC.to_bytes(4, "little") + vgeo.VG_FORMAT_VERSION.to_bytes(4, "little")
    b[8:12] = len(text).to_bytes(4, "little")
    b[12:16] = vgeo.checksum(bytes(b)).to_bytes(4, "little")
    with pytest.raises(vgeo.VirtualMeshFormatError, match='field "positions": vertex stream'):
        vgeo.decode(bytes(b))


def test_checksum_known_answer():
    # h = 0x811c9dc5 ^ 1; h = (h ^ 1) * 0x01000193 mod 2^32; h ^= h >> 15 (serialize.ts:429-437), by hand
    h = 0x811C9DC5 ^ 1
    h = ((h ^ 1) * 0x01000193) & 0xFFFFFFFF
    h ^= h >> 15
    assert vgeo.checksum(b"\0" * 16 + (1).to_bytes(4, "little")) == h
