"""The serving loop (vgc_server_*): requests against several resident scenes, submitted from two threads with
uneven timing, admitted by output slots and HBM budget, batched across scenes (one multi-scene launch) or per scene,
and overlapped on two streams. Every result must equal the same view cut alone (fresh controller state) on the same
scene - counters, chosen threshold, budget prediction and the drawn (instance, meshlet, fade) set of both cuts - and
the oracle's float mirror of that view."""
import random
import threading

import numpy as np
import pytest

import oracle as O
from parity_util import key_set
from vgcut import engine, scenes
from vgcut.camera import Camera

pytestmark = pytest.mark.gpu

COUNTERS = ("visible_cells", "occluded_instances", "selected", "drawn", "survived", "work", "requested_indices",
            "rounds", "effective_threshold", "predicted_triangles")


MAX_MESHLETS = 1 << 15
FRESH = [10000, 10000, 0, 0, 0, 0, 0, 0]


@pytest.fixture(scope="module")
def contexts():
    out = []
    for seed, n in ((1, 24), (2, 32), (3, 16)):
        spec = scenes.plain_small(n=n, seed=seed, grid=6 + seed)
        vg = engine.VirtualGeometry(max_meshlets=MAX_MESHLETS, output_slots=2)
        scenes.load_into(vg, spec, cast_shadow=(seed != 2))
        out.append((spec, vg))
    yield out
    for _, vg in out:
        vg.dispose()


@pytest.fixture(scope="module")
def oracle_scenes(contexts):
    out = []
    for k, (spec, _) in enumerate(contexts):
        scene, _, _ = O.scene_from_spec(spec.meshes, spec.instances, [dict(shadow=(k != 1)) for _ in spec.meshes])
        out.append(scene)
    return out


def random_request(rng, spec):
    eye = (rng.uniform(-30, 30), rng.uniform(2, 15), rng.uniform(-30, 30))
    width, height = rng.choice([(1280, 720), (1920, 1080), (3840, 2160)])
    cam = Camera.perspective_look_at(eye, (rng.uniform(-3, 3), 0.0, rng.uniform(-3, 3)), 60, width, height, 0.1, 1000)
    p = engine.ViewParams(error_threshold=rng.uniform(0.5, 2.0), shadow_sweep=(5.0, -20.0, 3.0))
    if rng.random() < 0.3:
        p.triangle_budget = rng.choice([5_000.0, 20_000.0, 80_000.0])
        p.threshold_range = (0.5, 3.0)
    return cam, p


def snapshot(vg, slot):
    s = vg.read_stats(slot)
    return {k: s[k] for k in COUNTERS}, [key_set(vg.draw_list(slot, c), (0, 1, 3)) for c in (0, 1)]


@pytest.mark.parametrize("cross_scene", [True, False])
def test_served_equals_alone_and_the_oracle(contexts, oracle_scenes, cross_scene):
    rng = random.Random(11)
    reqs = []
    for i in range(72):
        k = rng.randrange(len(contexts))
        cam, p = random_request(rng, contexts[k][0])
        reqs.append((k, cam, p))
    server = engine.Server([vg for _, vg in contexts], streams=2, max_batch=8, slots_per_scene=24,
                           cross_scene=cross_scene)
    tickets = [None] * len(reqs)

    def submit(idx):
        r = random.Random(idx)
        for i in idx_list[idx]:
            k, cam, p = reqs[i]
            tickets[i] = server.submit(k, engine.make_view(cam, p))
            if r.random() < 0.3:
                threading.Event().wait(r.uniform(0.0, 0.002))

    idx_list = [list(range(0, len(reqs), 2)), list(range(1, len(reqs), 2))]
    threads = [threading.Thread(target=submit, args=(j,)) for j in range(2)]
    try:
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        served = []
        for i, t in enumerate(tickets):
            res = server.wait(t)
            k = reqs[i][0]
            served.append((res, snapshot(contexts[k][1], res["slot"])))
            server.release(t)
        st = server.stats()
        assert st["completed"] == len(reqs) and st["batches"] >= len(reqs) // 8
        assert st["max_in_flight"] >= 1
        if cross_scene:
            assert st["multi_scene_batches"] > 0, "some batches mix scenes"
        else:
            assert st["multi_scene_batches"] == 0
    finally:
        server.close()
    if cross_scene:
        assert any(res["batch_scenes"] > 1 for res, _ in served)
    checked = 0
    for (k, cam, p), (res, (counters, sets)) in zip(reqs, served):
        assert res["status"] == 0 and res["done_us"] >= res["start_us"] >= res["submit_us"]
        # the oracle's float mirror of the same view; a round that overflowed the draw list makes what follows depend
        # on the GPU's atomic order (served and alone alike), so such a request is not compared
        o = O.cull_pass(oracle_scenes[k], O.make_view(cam, p, MAX_MESHLETS, (30_000_000, 12_000_000), state=FRESH),
                        "f32")
        c = o["counters"]
        assert counters["visible_cells"] == c[0]
        if any(m > MAX_MESHLETS for m in o["max_selected"]):
            continue
        checked += 1
        vg = contexts[k][1]
        alone = engine.ViewParams(**{**p.__dict__, "state_slot": 0, "fresh_state": True})
        vg.cut([engine.make_view(cam, alone)], first_slot=0)
        want_counters, want_sets = snapshot(vg, 0)
        assert counters == want_counters, f"served counters {counters} alone {want_counters}"
        assert {kk: res["stats"][kk] for kk in COUNTERS} == want_counters
        assert sets == want_sets
        assert counters["occluded_instances"] == c[1]
        for cut in (0, 1):
            assert [counters["selected"][cut], counters["survived"][cut], counters["work"][cut]] == \
                [c[2 + cut * 5], c[4 + cut * 5], c[5 + cut * 5]]
            if c[2 + cut * 5] <= MAX_MESHLETS:
                assert sets[cut] == key_set(o["entries"][cut], (0, 1, 2)), f"served cut {cut} differs from the oracle"
        if p.triangle_budget > 0:
            assert counters["predicted_triangles"] == o["predicted"]
            assert counters["effective_threshold"] == np.float32(o["threshold"])
    assert checked >= len(reqs) * 3 // 4, f"{checked} of {len(reqs)} served results compared with the oracle"
    assert any(len(s[1][1][0]) > 0 for s in served)


def test_admission_by_hbm_budget(contexts):
    vgs = [vg for _, vg in contexts]
    with pytest.raises(engine.VgcError, match="exceeds the budget"):
        engine.Server(vgs, hbm_budget_bytes=1)
    probe = engine.Server(vgs[:1], streams=1, max_batch=1, slots_per_scene=2)
    try:
        spec = contexts[0][0]
        t = probe.submit(0, engine.make_view(spec.cameras[0]))
        probe.wait(t)
        slot_bytes = probe.stats()["bytes_in_use"]
        probe.release(t)
    finally:
        probe.close()
    assert slot_bytes > 0
    # room for two unreleased requests: the rest wait until a release frees budget
    server = engine.Server(vgs[:1], streams=2, max_batch=4, slots_per_scene=8, hbm_budget_bytes=2 * slot_bytes)
    try:
        tickets = [server.submit(0, engine.make_view(contexts[0][0].cameras[0])) for _ in range(5)]
        server.wait(tickets[0])
        server.wait(tickets[1])
        with pytest.raises(engine.VgcError, match="timeout"):
            server.wait(tickets[2], timeout_ms=200)
        with pytest.raises(engine.VgcError, match="still queued"):
            server.release(tickets[2])
        for i in range(2, 5):
            server.release(tickets[i - 2])
            server.wait(tickets[i])
        server.release(tickets[3])
        server.release(tickets[4])
        st = server.stats()
        assert st["max_bytes_in_use"] <= 2 * slot_bytes and st["completed"] == 5
        with pytest.raises(engine.VgcError, match="unknown"):
            server.wait(tickets[0])
    finally:
        server.close()
