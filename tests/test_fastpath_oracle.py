"""The reference's fast-path conservativeness test (tests/fastpath.test.ts:51-176) ported to the oracle."""
import math

import numpy as np

import oracle as O
from vgcut.camera import Camera, mat_mul


def model_matrix(t, s):
    m = np.eye(4) * s
    m[3, 3] = 1
    m[:3, 3] = t
    return m.T.reshape(-1)


def check(d, view, ps, near, t, s, counts):
    r = O.instance_guaranteed_range(d, view, ps, near, t, 1.0, s)
    if r is None:
        return
    start, end = r
    counts["fast"] += 1
    counts["single"] += end - start == 1
    if end <= start or end - start > 4:
        counts["bad"] += 1
    sel = O.select_cut(d, view, ps, near, t, s)
    idx = np.nonzero(sel)[0]
    if not (len(idx) == end - start and np.all((idx >= start) & (idx < end))):
        counts["bad"] += 1
    rb = O.instance_guaranteed_range(d, view, ps, near, t, 2.0, s)
    if rb is None:
        return
    counts["blend"] += 1
    lo, hi = O.select_blend_cut(d, view, ps, near, t, 2.0, s)
    inf = np.zeros(d.meshlet_count, bool)
    inf[rb[0]:rb[1]] = True
    if np.any(inf != (hi > 0)) or np.any(inf & ((lo != 0) | (hi != 255))):
        counts["bad"] += 1


def test_fast_path_is_conservative(terrain, park_miller):
    d = terrain
    rand = park_miller(11)
    counts = dict(fast=0, single=0, blend=0, bad=0)
    for k in range(40):
        direction = np.array([rand() - 0.5, 0.05 + rand() * 0.6, rand() - 0.5])
        direction /= np.linalg.norm(direction)
        dist = 10 ** (4.3 + rand() * 2) if k < 30 else 100 * 10 ** (rand() * 2)
        target = ((rand() - 0.5) * 200, 0, (rand() - 0.5) * 200)
        cam = Camera.perspective_look_at(direction * dist, target, 60, 16, 9, 0.1, 1e8)
        ps = cam.proj[5] * 540
        for j in range(5):
            s = [1, 0.5, 2, 3][j % 4] * (0.75 + rand() * 0.5)
            tr = ((rand() - 0.5) * 600, (rand() - 0.5) * 60, (rand() - 0.5) * 600)
            mv = mat_mul(cam.view, model_matrix(tr, s))
            for t in (0.5, 1, 3):
                check(d, mv, ps, 0.1, t, s, counts)
    # edge-of-band sweeps (fastpath.test.ts:112-171), every meshlet, own and parent bound
    b = d.meshlet_bounds.reshape(-1, 16).astype(np.float64)
    C = d.lod_bounds_sphere[:3].astype(np.float64)
    ps = Camera.perspective_look_at((0, 0, 1), (0, 0, 0), 60, 16, 9, 0.1, 1e8).proj[5] * 540
    for i in range(d.meshlet_count):
        for t in (0.5, 1, 3):
            for s in (1, 2.5):
                for mode in ("own", "parent"):
                    c, r, e = (b[i, 0:3], b[i, 3], b[i, 8]) if mode == "own" else (b[i, 4:7], b[i, 7], b[i, 9])
                    if not (0 < e < 1e29):
                        continue
                    off = float(np.linalg.norm(c - C))
                    u = c - C
                    u = u / np.linalg.norm(u) if np.dot(u, u) > 0 else np.array([0.3, 0.5, 0.81]) / 1.0
                    u = u / np.linalg.norm(u)
                    if mode == "parent":
                        u = -u
                    Dc = (e * s * ps) / t + s * (off + r) if mode == "own" else (e * s * ps) / t - s * (off - r)
                    if not Dc > 0:
                        continue
                    tr = np.array([(rand() - 0.5) * 600, (rand() - 0.5) * 60, (rand() - 0.5) * 600])
                    model = model_matrix(tr, s)
                    centre = C * s + tr
                    for k in range(0, 33, 4):
                        f = 0.996 + k * 0.00025
                        cam = Camera.perspective_look_at(centre + u * Dc * f, centre, 60, 16, 9, 0.1, 1e8)
                        check(d, mat_mul(cam.view, model), ps, 0.1, t, s, counts)
    assert counts["fast"] > 0 and counts["single"] > 0, "the fast path fires (test is not vacuous)"
    assert counts["blend"] > 0, "the fast path also fires with LOD blending"
    assert counts["bad"] == 0, "every fast-path range equals the per-meshlet LOD cut"
