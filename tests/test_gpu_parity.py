"""GPU cut vs the oracle, through the C ABI: bit-exact against the float mirror (same arithmetic order) on sets,
counters, draw args and controller state; against the double restatement of the reference outside the 1e-5
relative margin."""
import math

import numpy as np
import pytest

import oracle as O
from vgcut import engine, scenes
from vgcut.camera import Camera
from parity_util import Harness, MARGIN, key_set, small_ruins, d2h

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain():
    spec = scenes.plain_small(n=60, seed=1)
    h = Harness(spec)
    h.check_layout()
    return h


def cameras_around(n, radius, height, seed=5):
    r = np.random.default_rng(seed)
    out = []
    for k in range(n):
        a = r.uniform(0, 2 * math.pi)
        d = radius * r.uniform(0.3, 1.6)
        out.append(Camera.perspective_look_at((math.cos(a) * d, height * r.uniform(0.05, 1.5), math.sin(a) * d),
                                              (r.uniform(-3, 3), 0, r.uniform(-3, 3)), 60, 1920, 1080, 0.1, 1000))
    return out


@pytest.mark.parametrize("threshold", [0.5, 1.0, 2.0, 3.0])
def test_plain_small_bit_exact(plain, threshold):
    p = engine.ViewParams(error_threshold=threshold)
    for cam in plain.spec.cameras + cameras_around(6, 30, 10):
        plain.compare(cam, p)


def test_plain_small_levers(plain):
    cam = cameras_around(1, 25, 8, seed=9)[0]
    for p in [engine.ViewParams(frustum_culling=False), engine.ViewParams(min_pixel_radius=40.0),
              engine.ViewParams(lod_blend=1.0, error_threshold=2.0), engine.ViewParams(lod_blend=3.0, error_threshold=2.5)]:
        plain.compare(cam, p)


def test_untrimmed_mesh_without_sphere_containment():
    """A mesh whose LOD sphere does not hold its meshlets' spheres (data not from a conforming builder) gets no item
    trimming, and the cut still equals the oracle's."""
    import dataclasses
    spec = scenes.plain_small(n=24, seed=2)
    data = spec.meshes[0]
    shrunk = data.lod_bounds_sphere.copy()
    shrunk[3] *= 0.5
    spec.meshes[0] = dataclasses.replace(data, lod_bounds_sphere=shrunk)
    h = Harness(spec)
    for t, cam in zip([0.7, 1.5, 3.0], cameras_around(3, 22, 6, seed=4)):
        h.compare(cam, engine.ViewParams(error_threshold=t))


def test_gpu_vs_reference_semantics(plain):
    """Differences between the GPU selection and the double restatement are all decisions within the margin."""
    total = near = 0
    for cam in cameras_around(8, 30, 10, seed=21):
        p = engine.ViewParams(error_threshold=1.0)
        lists, _ = plain.compare(cam, p)
        entries, views = plain.reference(cam, p)
        g = key_set(lists[0], (0, 1, 3))
        o = key_set(entries[0], (0, 1, 2))
        total += len(o)
        for inst, m, _ in g ^ o:
            slack = O.explain(plain.scene, views[0], 0, inst, m)
            assert slack <= MARGIN, f"({inst}, {m}) differs with slack {slack}"
            near += 1
    assert total > 0
    print(f"margin decisions: {near} of {total}")


@pytest.fixture(scope="module")
def ruins_small():
    spec = small_ruins()
    flags = [dict(shadow=(i % 2 == 0), occlusion=True, max_draw_distance=(80.0 if i == 1 else float("inf")),
                  min_pixel_radius=(1.0 if i == 2 else 0.0)) for i in range(len(spec.meshes))]
    h = Harness(spec, flags)
    h.check_layout()
    return h


def test_ruins_small_with_shadow_and_occlusion(ruins_small):
    h = ruins_small
    vg = h.vg
    with_hzb = without = shadow = 0
    for k, cam in enumerate(h.spec.cameras):
        vg.build_hzb(k, h.spec.depth_images[k])
        hzb = O.hzb_build(h.spec.depth_images[k])
        p = engine.ViewParams(error_threshold=1.0, hzb=k, shadow_sweep=(30.0, -60.0, 10.0))
        lists, res = h.compare(cam, p, hzb_oracle=hzb)
        with_hzb += len(lists[0])
        shadow += len(lists[1])
        res_open, _ = h.oracle(cam, engine.ViewParams(error_threshold=1.0, shadow_sweep=(30.0, -60.0, 10.0)))
        without += len(res_open["entries"][0])
    assert shadow > 0, "the shadow cut is exercised"
    assert with_hzb < without, "occlusion removes instances or meshlets"


def test_hzb_mips_bit_exact(ruins_small):
    h = ruins_small
    img = h.spec.depth_images[0]
    h.vg.build_hzb(7, img)
    mips, levels, off, w, hh = O.hzb_build(img)
    info = h.vg.hzb_info(7)
    assert info["levels"] == levels and info["offset"][:levels] == off[:levels] and info["width"][:levels] == w[:levels]
    got = d2h(info["data"], len(mips), np.float32)
    assert np.array_equal(got, mips), "HZB mips differ from the oracle's max reduction"
    # from device memory too
    import torch
    d = torch.from_numpy(img).cuda()
    engine.check(engine.lib().vgc_hzb_build(h.vg.handle, 8, d.data_ptr(), img.shape[1], img.shape[0], 1, None))
    info = h.vg.hzb_info(8)
    assert np.array_equal(d2h(info["data"], len(mips), np.float32), mips)


@pytest.mark.parametrize("shape", [(611, 997), (1, 7), (9, 1), (130, 64), (1080, 1920), (67, 129), (300, 1004),
                                   (77, 100), (1, 4)])
def test_hzb_mips_odd_sizes(ruins_small, shape):
    """Edge clamping at every level: odd and tiny sizes through the host-copy, device and in-sequence builds (float4
    rows where the width is a multiple of 4 and the pointer aligned, with a partial tile at the right edge for 1004
    and 100; scalar loads otherwise)."""
    import torch
    h = ruins_small
    rng = np.random.default_rng(shape[0] * 7919 + shape[1])
    img = rng.random(shape, dtype=np.float32)
    mips = O.hzb_build(img)[0]
    h.vg.build_hzb(9, img)
    info = h.vg.hzb_info(9)
    assert np.array_equal(d2h(info["data"], len(mips), np.float32), mips)
    d = torch.from_numpy(img).cuda()
    # an unaligned device pointer takes the scalar-load path
    dd = torch.zeros(img.size + 1, dtype=torch.float32, device="cuda")
    dd[1:] = d.flatten()
    for ptr in (d.data_ptr(), dd.data_ptr() + 4):
        engine.check(engine.lib().vgc_hzb_build(h.vg.handle, 10, ptr, img.shape[1], img.shape[0], 1, None))
        assert np.array_equal(d2h(h.vg.hzb_info(10)["data"], len(mips), np.float32), mips)
    cam = h.spec.cameras[0]
    for ptr in (d.data_ptr(), dd.data_ptr() + 4):  # in the cut's tile stream: a tensor map, or plain loads
        v = engine.make_view(cam, engine.ViewParams(error_threshold=1.0, hzb=11), depth=(ptr, img.shape[1], img.shape[0]))
        h.vg.cut([v], first_slot=0)
        assert np.array_equal(d2h(h.vg.hzb_info(11)["data"], len(mips), np.float32), mips)
        assert h.vg.read_stats(0)["faults"] == 0


def test_hzb_stream_mixed_jobs(ruins_small):
    """One launch whose HZB builds differ in size and kind: 128 x 32 strips through tensor maps (widths a multiple of
    4, with partial strips at the right and bottom edges) and through plain loads (odd width, unaligned pointer,
    narrower than a strip) in one stream; every slot equals the oracle's max reduction, through the plain call and
    the captured graph."""
    import torch
    h = ruins_small
    shapes = [(1080, 1920), (77, 132), (611, 997), (130, 256), (40, 36), (300, 1004), (2160, 3840)]
    rng = np.random.default_rng(11)
    imgs = [rng.random(s, dtype=np.float32) for s in shapes]
    keep = []
    views = []
    for k, img in enumerate(imgs):
        d = torch.zeros(img.size + 4, dtype=torch.float32, device="cuda")
        off = 1 if k == 3 else 0  # job 3: a 4-byte offset pointer (no tensor map)
        d[off:off + img.size] = torch.from_numpy(img).flatten().cuda()
        keep.append(d)
        ptr = d.data_ptr() + 4 * off
        views.append(engine.make_view(h.spec.cameras[k % len(h.spec.cameras)],
                                      engine.ViewParams(error_threshold=1.0, hzb=40 + k, depth_as_mip0=(k % 2 == 1)),
                                      depth=(ptr, img.shape[1], img.shape[0])))
    for graph in (False, True):
        for k in range(len(shapes)):
            h.vg.build_hzb(40 + k, np.zeros((8, 8), np.float32))  # stale contents of another size
        h.vg.cut(views, first_slot=0, graph=graph)
        for k, img in enumerate(imgs):
            mips, levels, off, w, hh = O.hzb_build(img)
            data = d2h(h.vg.hzb_info(40 + k)["data"], len(mips), np.float32)
            lo = off[1] if k % 2 == 1 else 0  # mip 0 is not written when it is read from the depth image
            assert np.array_equal(data[lo:], mips[lo:]), (graph, shapes[k])
            assert h.vg.read_stats(k)["faults"] == 0


def test_capacity_retry_rounds():
    """An index buffer too small for the cut triggers the same-frame redo at a coarser threshold
    (GeometryPool.ts:1032) and the steer between frames; counters and controller state match the oracle round for
    round. (A draw list too small is not used here: the entries a GPU keeps past it follow its atomic order, and the
    controller's fill counts the kept entries' indices, so the retried rounds would follow that order too.)"""
    spec = scenes.plain_small(n=60, seed=2)
    h = Harness(spec, max_meshlets=1 << 16, max_triangles=40_000)
    cam = cameras_around(1, 12, 4, seed=3)[0]
    p = engine.ViewParams(error_threshold=0.5, state_slot=3)
    rounds = []
    for _ in range(3):  # state carries from frame to frame
        _, res = h.compare(cam, p)
        rounds.append(res["rounds"])
    assert h.order_dependent == 0 and rounds[0] >= 2, f"rounds {rounds}"


def test_batch_graph_equals_plain(plain):
    cams = cameras_around(5, 30, 10, seed=33)
    views = [engine.make_view(c, engine.ViewParams(error_threshold=t, state_slot=10 + i))
             for i, (c, t) in enumerate(zip(cams, [0.5, 1, 2, 3, 1]))]
    plain.vg.cut(views, first_slot=0, graph=False)
    a = [[plain.vg.draw_list(i, c) for c in (0, 1)] for i in range(5)]
    for _ in range(2):
        plain.vg.cut(views, first_slot=0, graph=True)
        b = [[plain.vg.draw_list(i, c) for c in (0, 1)] for i in range(5)]
        for i in range(5):
            for c in (0, 1):
                assert key_set(a[i][c], (0, 1, 3)) == key_set(b[i][c], (0, 1, 3))


def test_select_cut_matches_reference(terrain, park_miller):
    """GPU selectCut / selectBlendCut (cut.ts:26-77) vs the double oracle, margin decisions excepted."""
    vg = engine.VirtualGeometry()
    vg.create_mesh(terrain, np.eye(4, dtype=np.float32).reshape(1, 16))
    rand = park_miller(7)
    vms, cams = [], []
    for _ in range(12):
        eye = ((rand() - 0.5) * 300, 2 + rand() * 80, (rand() - 0.5) * 300)
        tgt = ((rand() - 0.5) * 200, 0, (rand() - 0.5) * 200)
        cams.append(Camera.perspective_look_at(eye, tgt, 60, 16, 9, 0.1, 5000))
    vm = np.array([c.view for c in cams])
    ps = np.array([c.proj[5] * 540 for c in cams])
    b = terrain.meshlet_bounds.reshape(-1, 16).astype(np.float64)
    for t, blend in [(0.5, 1), (1, 1), (3, 1), (1, 2), (2, 3)]:
        lo, hi = vg.select_cut(0, vm, ps, 0.1, 1.0, t, blend)
        for i, c in enumerate(cams):
            olo, ohi = O.select_blend_cut(terrain, c.view, ps[i], 0.1, t, blend)
            diff = np.nonzero((lo[i] != olo) | (hi[i] != ohi))[0]
            for m in diff:  # every difference sits within the margin of a threshold or a fade-step boundary
                V = np.asarray(c.view).reshape(4, 4).T
                def pe(cc, r, e):
                    p = V @ np.append(cc, 1.0)
                    return e * ps[i] / max(np.linalg.norm(p[:3]) - r, 0.1)
                own, par = pe(b[m, :3], b[m, 3], b[m, 8]), pe(b[m, 4:7], b[m, 7], b[m, 9])
                high = t * blend if blend > 1 else t
                close = [abs(own - high) / high, abs(par - t) / t]
                if blend > 1:
                    for e in (own, par):
                        x = math.log(max(e, 1e-30) / t) * 255 / math.log(blend)
                        close.append(abs(x - math.floor(x) - 0.5) / (255 / math.log(blend)))
                assert min(close) <= MARGIN, f"meshlet {m} differs beyond the margin"
            if blend == 1:
                sel = (hi[i] > 0).astype(np.uint8)
                assert len(O.verify_cut_coverage(terrain, sel)) == 0
                assert len(O.verify_cut_overlap(terrain, sel)) == 0
    vg.dispose()


def test_expand_writes_draw_slots(plain):
    cam = plain.spec.cameras[0]
    p = engine.ViewParams()
    lists, res = plain.compare(cam, p)
    import torch
    cap = 2_000_000 * 3
    buf = torch.full((cap,), 0xFFFFFFFF, dtype=torch.int64).to(torch.int32).cuda()
    engine.check(engine.lib().vgc_expand(plain.vg.handle, 0, 0, buf.data_ptr(), cap, None))
    torch.cuda.synchronize()
    idx = buf.cpu().numpy().view(np.uint32)
    e = lists[0]
    data = plain.spec.meshes[0]
    info = data.meshlet_info.reshape(-1, 4)
    counts = res["mesh_counts"]
    region = {0: 0, 1: int(counts[0, 0, 0])}
    for slot_in_list, (inst, m, first, packed) in enumerate(e[:200]):
        part = 0 if (packed & 0xFFFF00) == (255 << 16) else 1
        start = region[part] + first
        tri = packed & 255
        got = idx[start:start + 3 * tri]
        fi = info[m, 1] // 3
        tris = data.meshlet_triangles[fi:fi + tri]
        want = np.stack([tris & 255, (tris >> 8) & 255, (tris >> 16) & 255], 1).reshape(-1)
        assert np.array_equal(got & 127, want)
        assert np.all((got >> 7) == got[0] >> 7)


def test_instance_update_and_flags(plain):
    h = plain
    cam = h.spec.cameras[0]
    p = engine.ViewParams()
    before, _ = h.compare(cam, p)
    mesh = h.vg.meshes[0]
    mesh.visible = False
    stats, lists = h.gpu(cam, p)
    assert stats["visible_cells"] == 0 and len(lists[0]) == 0
    mesh.visible = True
    stats, lists = h.gpu(cam, p)
    assert key_set(lists[0], (0, 1, 3)) == key_set(before[0], (0, 1, 3))


def test_instance_updates_on_device():
    """setMatrixAt + commitInstances on a resident scene: only the moved matrices are uploaded and their cells are
    recomputed on the device; the device cells equal the host's and the oracle's computeCell bit for bit, and the cut
    equals the oracle's on the moved scene (the GPU order of the instances is kept)."""
    spec = scenes.plain_small(n=24, seed=6)
    h = Harness(spec)
    cam = cameras_around(1, 24, 7, seed=2)[0]
    h.compare(cam, engine.ViewParams())  # resident: the updates below take the device path
    rng = np.random.default_rng(5)
    mats = [np.array(m, np.float32).reshape(-1, 16) for m in spec.instances]
    mesh = h.vg.meshes[0]
    for i in rng.choice(len(mats[0]), 20, replace=False):
        m = mats[0][i].copy()
        m[12] += rng.uniform(-6, 6)
        m[14] += rng.uniform(-6, 6)
        m[[0, 5, 10]] *= rng.uniform(0.6, 1.6)
        mats[0][i] = m
        mesh.set_matrix_at(int(i), m)
    mesh.commit_instances()
    dev = h.vg.debug_cells_device()
    host, gpu_mats = h.vg.debug_scene()
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32)), "device cells differ from the host's"
    h.scene, h.mats, _ = O.scene_from_spec(spec.meshes, mats, h.flags, orders_in=h.orders)
    assert np.array_equal(gpu_mats, h.mats)
    ocells = np.asarray(h.scene.keep[-1]).reshape(-1, 8)
    assert np.array_equal(dev.view(np.uint32), ocells.view(np.uint32)), "device cells differ from the oracle's"
    for t in (0.8, 2.0):
        h.compare(cam, engine.ViewParams(error_threshold=t))


def test_hzb_built_in_cut_sequence(ruins_small):
    """A view that carries its depth image builds the HZB inside the cut's launches (plain and graph) with the same
    result as a separately built HZB."""
    import torch
    h = ruins_small
    for graph in (False, True):
        for k, cam in enumerate(h.spec.cameras[:3]):
            img = h.spec.depth_images[k]
            d = torch.from_numpy(img).cuda()
            p = engine.ViewParams(error_threshold=1.0, hzb=20 + k)
            v = engine.make_view(cam, p, depth=(d.data_ptr(), img.shape[1], img.shape[0]))
            h.vg.cut([v], first_slot=0, graph=graph)
            got = h.vg.draw_list(0, 0)
            res, _ = h.oracle(cam, p, hzb=O.hzb_build(img))
            assert key_set(got, (0, 1, 3)) == key_set(res["entries"][0], (0, 1, 2))
            info = h.vg.hzb_info(20 + k)
            mips = O.hzb_build(img)[0]
            assert np.array_equal(d2h(info["data"], len(mips), np.float32), mips)


def test_depth_as_mip0(ruins_small):
    """VGC_VIEW_DEPTH_AS_MIP0: the cut reads mip 0 from the view's depth image instead of a copy in the slot. Same
    draw sets and counters as the copying build (and as the oracle with the full HZB); the slot's mip 0 keeps what an
    earlier build left there while mips 1 and up are the new image's."""
    import torch
    h = ruins_small
    slot = 27
    first = h.spec.depth_images[0]
    for graph in (False, True):
        for k, cam in enumerate(h.spec.cameras[1:4], start=1):
            img = h.spec.depth_images[k]
            d = torch.from_numpy(img).cuda()
            got = {}
            for flag in (False, True):
                h.vg.build_hzb(slot, first)  # an earlier frame's HZB in the slot
                p = engine.ViewParams(error_threshold=1.0, hzb=slot, depth_as_mip0=flag)
                v = engine.make_view(cam, p, depth=(d.data_ptr(), img.shape[1], img.shape[0]))
                h.vg.cut([v], first_slot=0, graph=graph)
                got[flag] = (key_set(h.vg.draw_list(0, 0), (0, 1, 3)), h.vg.read_stats(0))
            assert got[True][0] == got[False][0], "the draw set differs with mip 0 read from the depth image"
            assert got[True][1] == got[False][1]
            res, _ = h.oracle(cam, engine.ViewParams(error_threshold=1.0, hzb=slot), hzb=O.hzb_build(img))
            assert got[True][0] == key_set(res["entries"][0], (0, 1, 2))
            info = h.vg.hzb_info(slot)
            mips, levels, off, w, hh = O.hzb_build(img)
            old = O.hzb_build(first)[0]
            data = d2h(info["data"], len(mips), np.float32)
            assert np.array_equal(data[:off[1]], old[:off[1]]), "mip 0 of the slot is not written"
            assert np.array_equal(data[off[1]:], mips[off[1]:]), "mips 1 and up are the new image's"


def test_bounded_wait_gives_up_and_context_stays_usable(ruins_small):
    """The mbarrier wait the HZB strip stream uses, on a barrier nothing completes: it gives up after its limit (not
    later than a few milliseconds past it) and reports that it did not complete; a cut with an HZB build afterwards
    is still exact and reports no fault."""
    import torch
    h = ruins_small
    for limit_us in (2000, 20000):
        done, ns = h.vg.wait_probe(limit_us)
        assert done == 0
        assert limit_us * 1000 <= ns < limit_us * 1000 + 50_000_000, ns
    img = h.spec.depth_images[0]
    d = torch.from_numpy(img).cuda()
    cam = h.spec.cameras[0]
    v = engine.make_view(cam, engine.ViewParams(error_threshold=1.0, hzb=12), depth=(d.data_ptr(), img.shape[1], img.shape[0]))
    h.vg.cut([v], first_slot=0)
    assert h.vg.read_stats(0)["faults"] == 0
    mips = O.hzb_build(img)[0]
    assert np.array_equal(d2h(h.vg.hzb_info(12)["data"], len(mips), np.float32), mips)
