"""The oracle against hand-derived known-answer vectors (tests/golden/vectors.json, made by make_golden.py)."""
import json
import math
import os
from types import SimpleNamespace

import numpy as np
import pytest

import oracle as O

V = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "vectors.json")))


def tiny():
    t = V["tiny_dag"]
    return SimpleNamespace(
        meshlet_count=3, meshlet_bounds=np.array(t["bounds"], np.float32).reshape(-1),
        meshlet_info=np.array(t["info"], np.uint32).reshape(-1), level_ranges=np.array(t["level_ranges"], np.uint32),
        level_errors=np.array(t["level_errors"], np.float32), level_guard_errors=np.array(t["level_guard_errors"], np.float32),
        lod_bounds_sphere=np.array(t["lod_bounds_sphere"], np.float32),
        cull_bounds_sphere=np.array([0, 0, 0, 1], np.float32), bounding_sphere=np.array([0, 0, 0, 1], np.float32),
        meshlet_triangles=np.zeros(5, np.uint32),
        replacement_group=np.array(t["replacement_group"], np.int32),
        replacement_start=np.array(t["replacement_start"], np.uint32),
        replacement_indices=np.array(t["replacement_indices"], np.uint32), stats={"leafTriangles": 4}), t


@pytest.mark.parametrize("case", V["lod_fade_range"])
def test_lod_fade_range(case):
    parent = math.inf if case["parent"] == "inf" else case["parent"]
    got = O.lod_fade_range(case["own"], parent, case["t"], case["blend"])
    assert (list(got) if got else None) == case["expect"]


def test_tiny_dag_cut():
    d, t = tiny()
    for c in t["select"]:
        assert O.select_cut(d, t["view"], t["proj_scale"], t["near"], c["t"]).tolist() == c["expect"]
    for c in t["coverage"]:
        assert O.verify_cut_coverage(d, np.array(c["selected"], np.uint8)).tolist() == c["holes"]
    for c in t["overlap"]:
        assert O.verify_cut_overlap(d, np.array(c["selected"], np.uint8)).tolist() == c["overlaps"]
    for c in t["meshlet_range"]:
        assert list(O.instance_meshlet_range(d, t["view"], t["proj_scale"], t["near"], c["t"])) == c["expect"]
    for c in t["guaranteed_range"]:
        got = O.instance_guaranteed_range(d, t["view"], t["proj_scale"], t["near"], c["t"])
        assert (list(got) if got else None) == c["expect"]


@pytest.mark.parametrize("case", V["hzb"])
def test_hzb(case):
    mips, levels, off, w, h = O.hzb_build(np.array(case["depth"], np.float32).reshape(case["height"], case["width"]))
    assert levels == case["levels"]
    assert off[:levels] == case["offset"] and w[:levels] == case["widths"] and h[:levels] == case["heights"]
    assert np.array_equal(mips, np.array(case["mips"], np.float32))


def test_morton():
    m = V["morton"]
    mats = []
    for c in m["centres"]:
        e = np.eye(4, dtype=np.float32)
        e[:3, 3] = c
        mats.append(e.T.reshape(-1))
    assert O.morton_order(np.array(mats), m["sphere"]).tolist() == m["expect"]
    from vgcut import build as B
    assert B.morton_order(np.array(mats), np.array(m["sphere"], np.float32)).tolist() == m["expect"]


@pytest.mark.parametrize("case", V["frustum_planes"])
def test_frustum_planes(case):
    """three's Frustum.setFromProjectionMatrix(P * V, WebGPUCoordinateSystem), worked by hand."""
    got = O.frustum_planes(case["pv"])
    assert np.allclose(got, np.array(case["expect"]), rtol=0, atol=1e-12)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_pass_scene(precision):
    """The per-frame passes (cells, instances, selectLevels, fast path, meshlets, blend steps, HZB, shadow sweep) on
    the hand-built scene, both precisions of the oracle against the hand-derived answers."""
    from parity_util import check_golden_view, golden_pass_scene
    from vgcut import engine
    spec, flags, cam, names = golden_pass_scene(V)
    scene, _, _ = O.scene_from_spec(spec.meshes, spec.instances, flags)
    hzb = O.hzb_build(np.array(V["pass_scene"]["hzb"], np.float32))
    for view in V["pass_scene"]["views"]:
        p = engine.ViewParams(error_threshold=view["t"], lod_blend=view["blend"], shadow_sweep=tuple(view["sweep"]))
        v = O.make_view(cam, p, 1 << 10, (100_000, 100_000), hzb=hzb if view["hzb"] else None)
        r = O.cull_pass(scene, v, precision)
        c = r["counters"]
        check_golden_view(view, names, r["entries"],
                          dict(visible_cells=c[0], occluded_instances=c[1], work0=c[5]))
