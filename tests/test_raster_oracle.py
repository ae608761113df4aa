"""The oracle's occluder depth pass on hand-built triangles (known answers): depth of a plane at a known distance,
coverage of the pixel centres inside a triangle, back faces, triangles crossing the near plane (clipped: the part in
front is drawn with its plane's depth), and the entries it must skip (blended part 1, meshes that are not
occluders)."""
import numpy as np
import pytest

import oracle as O
from vgcut.camera import Camera, perspective

W, H = 64, 48


def run(positions, tris, entries, occluder=(1,), near=0.1, far=100.0):
    cam = Camera(view=np.eye(4).reshape(-1), proj=perspective(60.0, W / H, near, far), near=near, height=float(H),
                 width=float(W))
    m_info = np.array([[len(tris), 0, 0, 0]], np.uint32)
    m_tris = np.array([a | (b << 8) | (c << 16) for a, b, c in tris], np.uint32)
    m_verts = np.arange(len(positions), dtype=np.uint32)
    inst = np.eye(4, dtype=np.float32).reshape(1, 16)  # columns of the identity
    out = np.zeros((H, W), np.float32)
    e = np.ascontiguousarray(entries, np.uint32).reshape(-1, 4)
    O.lib().vgo_occluder_depth(O._u(e), len(e), O._f(inst), O._u(np.zeros(1, np.uint32)),
                               O._u(np.asarray(occluder, np.uint32)), O._u(m_info), O._u(m_tris), O._u(m_verts),
                               O._f(np.ascontiguousarray(positions, np.float32)),
                               np.ascontiguousarray(cam.view, np.float64).ctypes.data_as(O.C.POINTER(O.C.c_double)),
                               np.ascontiguousarray(cam.proj, np.float64).ctypes.data_as(O.C.POINTER(O.C.c_double)),
                               W, H, O._f(out))
    return out, cam


PART0 = (1 | (255 << 16))  # one triangle, fade range [0, 255]: drawn over every pixel


def test_plane_depth_and_coverage():
    z = -5.0
    # a big counter-clockwise (front-facing) triangle covering the view at distance 5
    pos = [(-20, -20, z), (20, -20, z), (0, 30, z)]
    out, cam = run(pos, [(0, 1, 2)], [(0, 0, 0, PART0)])
    p10, p14 = cam.proj[10], cam.proj[14]
    want = np.float32((p10 * z + p14) / -z)
    covered = out < 1.0
    assert covered.all(), "the triangle spans the whole view"
    assert np.allclose(out, want, rtol=0, atol=2e-6), (out.min(), out.max(), want)


def test_pixel_centres_inside_only():
    # NDC triangle (-0.5,-0.5), (0.5,-0.5), (0,0.5) at depth 5 (x, y scaled by 5 tan(fov/2) per axis)
    t = np.tan(np.radians(30.0))
    sx, sy = 5 * t * W / H, 5 * t
    pos = [(-0.5 * sx, -0.5 * sy, -5), (0.5 * sx, -0.5 * sy, -5), (0.0, 0.5 * sy, -5)]
    out, _ = run(pos, [(0, 1, 2)], [(0, 0, 0, PART0)])
    covered = out < 1.0
    # screen vertices (16, 36), (48, 36), (32, 12): pixel centres inside the three edges
    expect = np.zeros((H, W), bool)
    for py in range(H):
        for px in range(W):
            x, y = px + 0.5, py + 0.5
            e = [(48 - 16) * (y - 36) - (36 - 36) * (x - 16), (32 - 48) * (y - 36) - (12 - 36) * (x - 48),
                 (16 - 32) * (y - 12) - (36 - 12) * (x - 32)]
            expect[py, px] = all(v <= 0 for v in e) or all(v >= 0 for v in e)
    assert covered.sum() > 100
    assert abs(int(covered.sum()) - int(expect.sum())) <= 2 * (24 + 32), "coverage follows the pixel-centre rule"
    assert not covered[:11].any() and not covered[37:].any()


def test_back_faces_near_plane_and_skipped_entries():
    z = -5.0
    front = [(-20, -20, z), (20, -20, z), (0, 30, z)]
    back, _ = run(front, [(0, 2, 1)], [(0, 0, 0, PART0)])
    assert (back == 1.0).all(), "a clockwise (back-facing) triangle is not drawn"
    blended = 1 | (10 << 8) | (200 << 16)
    out, _ = run(front, [(0, 1, 2)], [(0, 0, 0, blended)])
    assert (out == 1.0).all(), "blended (part 1) meshlets are not occluders"
    out, _ = run(front, [(0, 1, 2)], [(0, 0, 0, PART0)], occluder=(0,))
    assert (out == 1.0).all(), "meshes that are not occluders are not drawn"


def test_blend_mask_known_values_and_tiling():
    """lodBlendMask (lodBlend.ts:36-45): the step of each pixel is floor(255 n), n the interleaved gradient noise at
    the pixel centre (float32 arithmetic, step by step); complementary ranges [0, k) and [k, 255) split every pixel
    between them, and a range keeps about its share of the pixels."""
    f = np.float32

    def step(px, py, frame):
        x = f(f(px) + f(0.5)) + f(f(frame) * f(5.588238))
        y = f(f(py) + f(0.5))
        a = f(f(x * f(0.06711056)) + f(y * f(0.00583715)))
        b = f(f(a - np.floor(a)) * f(52.9829189))
        return int(np.floor(f(f(b - np.floor(b)) * f(255.0))))

    for px, py, frame in [(0, 0, 0), (17, 3, 0), (1919, 1079, 0), (640, 360, 5), (3, 200, 7)]:
        s = step(px, py, frame)
        assert O.blend_keep(px, py, frame, s, s + 1) and not O.blend_keep(px, py, frame, s + 1, 255)
        assert not O.blend_keep(px, py, frame, 0, s)
    kept = 0
    for py in range(0, 48):
        for px in range(0, 64):
            a, b = O.blend_keep(px, py, 0, 0, 100), O.blend_keep(px, py, 0, 100, 255)
            assert a != b, "complementary ranges tile every pixel"
            kept += a
    assert abs(kept / (48 * 64) - 100 / 255) < 0.05


def test_visibility_oracle_single_triangle():
    """The oracle's visibility pass on one hand-built draw entry: a front-facing triangle covering the view at
    distance 5 is drawn where the pixel's blend step lies in the entry's range, with the entry's draw slot and the
    triangle's index in its meshlet; with a draw distance of 4 the instance (origin 5 away) shrinks to its origin and
    nothing is drawn."""
    from types import SimpleNamespace
    z = -5.0
    pos = np.array([(-20, -20, 0), (20, -20, 0), (0, 30, 0)], np.float32).reshape(-1)  # the instance sits at z
    mesh = SimpleNamespace(meshlet_info=np.array([1, 0, 0, 0], np.uint32), meshlet_triangles=np.array([0 | (1 << 8) | (2 << 16)], np.uint32),
                           meshlet_vertices=np.arange(3, dtype=np.uint32), positions=pos)
    cam = Camera(view=np.eye(4).reshape(-1), proj=perspective(60.0, W / H, 0.1, 100.0), near=0.1, height=float(H),
                 width=float(W))
    inst = np.eye(4, dtype=np.float32)
    inst[3, 2] = z  # columns: a translation to (0, 0, z)
    inst = inst.reshape(1, 16)
    draw_list = np.zeros((4, 4), np.uint32)
    draw_list[2] = (0, 0, 0, 1 | (40 << 8) | (200 << 16))  # draw slot 2: a blended entry, steps [40, 200)
    indices = np.array([(2 << 7) | 0, (2 << 7) | 1, (2 << 7) | 2], np.uint32)
    args = np.array([[3, 1, 0, 0, 0], [0, 1, 3, 0, 0]], np.uint32)
    out = O.visibility([mesh], [True], [float("inf")], inst, np.zeros(1, np.uint32), indices, draw_list, args, cam, W, H)
    drawn = out != np.uint64(0x3F800000FFFFFFFF)
    keep = np.array([[O.blend_keep(x, y, 0, 40, 200) for x in range(W)] for y in range(H)])
    assert np.array_equal(drawn, keep), "the triangle covers the view: the blend mask alone decides"
    assert (out[drawn] & np.uint64(0xFFFFFFFF) == np.uint64(2 << 7)).all()
    p10, p14 = cam.proj[10], cam.proj[14]
    depth = (out[drawn] >> np.uint64(32)).astype(np.uint32).view(np.float32)
    assert np.allclose(depth, (p10 * z + p14) / -z, rtol=0, atol=2e-6)
    gone = O.visibility([mesh], [True], [4.0], inst, np.zeros(1, np.uint32), indices, draw_list, args, cam, W, H)
    assert (gone == np.uint64(0x3F800000FFFFFFFF)).all(), "beyond its draw distance the instance shrinks to a point"


def plane_depth(cam, corners, px, py):
    """The NDC depth where pixel (px, py)'s centre ray meets the plane of `corners` (view space), and whether it hits
    the triangle in front of the near plane; double precision, from the ray-plane intersection."""
    P = np.asarray(cam.proj, float).reshape(4, 4).T
    a, b, c = (np.asarray(v, float) for v in corners)
    n = np.cross(b - a, c - a)
    x = (px + 0.5) / W * 2 - 1
    y = 1 - (py + 0.5) / H * 2
    d = np.array([x / P[0, 0], y / P[1, 1], -1.0])
    den = n @ d
    if abs(den) < 1e-12:
        return None, False
    t = (n @ a) / den
    q = t * d
    # barycentric inside test of q in (a, b, c)
    v0, v1, v2 = b - a, c - a, q - a
    d00, d01, d11, d20, d21 = v0 @ v0, v0 @ v1, v1 @ v1, v2 @ v0, v2 @ v1
    den2 = d00 * d11 - d01 * d01
    bb = (d11 * d20 - d01 * d21) / den2
    cc = (d00 * d21 - d01 * d20) / den2
    inside = bb >= 0 and cc >= 0 and bb + cc <= 1 and -q[2] >= cam.near
    z = q[2]
    return (P[2, 2] * z + P[2, 3]) / -z, inside


@pytest.mark.parametrize("corners", [
    [(-20, -20, -5.0), (20, -20, -5.0), (0, 30, 1.0)],   # two corners in front: a quad, two triangles
    [(-20, -20, 1.0), (20, -20, 1.0), (0, 30, -5.0)],    # one corner in front: one triangle
    [(-3, -4, -0.05), (3, -4, -0.05), (0, 4, -20.0)],    # two corners between the camera and the near plane
])
def test_near_plane_clipping(corners):
    out, cam = run(corners, [(0, 1, 2)], [(0, 0, 0, PART0)])
    covered = out < 1.0
    hits = err = edge = 0
    for py in range(H):
        for px in range(W):
            want, inside = plane_depth(cam, corners, px, py)
            if covered[py, px]:
                assert want is not None
                err = max(err, abs(float(out[py, px]) - want))
                hits += 1
                edge += not inside
            elif inside:
                edge += 1
    assert hits > 50, "the part in front of the near plane is drawn"
    assert err < 2e-5, f"depth off the triangle's plane by {err}"
    assert edge <= 2 * (W + H), "coverage follows the clipped triangle (up to its edge pixels)"
