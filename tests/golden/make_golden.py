"""Writes tests/golden/vectors.json: known-answer vectors for the cut path, derived by hand from the reference's
formulas (the reference ships no golden vectors, and its TypeScript cannot run in this repository's containers).

Each value below is worked out in the comment beside it from the formula it pins; nothing here calls the oracle or
the engine. Run: python tests/golden/make_golden.py
"""
import json
import math
import os

S2 = 255 / math.log(2)  # blend-step scale for lodBlend 2 (lodBlend.ts:56): 367.8887...

vectors = {
    # lodFadeRange(own, parent, threshold, blend) -> [lo, hi] or null (lodBlend.ts:52-61, Math.round halves up)
    "lod_fade_range": [
        # own 1 <= high 2, parent 4 > 1; lo = round(ln(1) * S2) = 0; hi = round(ln 4 * S2) = round(510.0) -> 255
        dict(own=1.0, parent=4.0, t=1.0, blend=2.0, expect=[0, 255]),
        # lo = round(ln 1.5 * S2) = round(149.17) = 149; hi = round(ln 3 * S2) = round(404.2) -> 255
        dict(own=1.5, parent=3.0, t=1.0, blend=2.0, expect=[149, 255]),
        # lo = round(ln 1.2 * S2) = round(67.07) = 67; hi = round(ln 1.6 * S2) = round(172.91) = 173
        dict(own=1.2, parent=1.6, t=1.0, blend=2.0, expect=[67, 173]),
        # own 3 > high 2: not in any cut of the band
        dict(own=3.0, parent=5.0, t=1.0, blend=2.0, expect=None),
        # parent 0.9 <= t: replaced everywhere in the band
        dict(own=0.5, parent=0.9, t=1.0, blend=2.0, expect=None),
        # blend 1 is the plain cut: own <= t < parent -> [0, 255]; own == t still drawn; parent == t not
        dict(own=0.5, parent=2.0, t=1.0, blend=1.0, expect=[0, 255]),
        dict(own=1.0, parent=2.0, t=1.0, blend=1.0, expect=[0, 255]),
        dict(own=0.5, parent=1.0, t=1.0, blend=1.0, expect=None),
        # leaf (own 0): lo = clamp(round(ln(1e-30) * S2)) = 0; hi = round(ln 1.05 * S2) = round(17.95) = 18
        dict(own=0.0, parent=1.05, t=1.0, blend=2.0, expect=[0, 18]),
        # root (parent infinite): hi = 255; lo = round(ln 1.99 * S2) = round(253.16) = 253
        dict(own=1.99, parent="inf", t=1.0, blend=2.0, expect=[253, 255]),
        # blend 3, t 2: scale 255 / ln 3 = 232.11; own 3 -> lo = round(ln 1.5 * 232.11) = round(94.11) = 94;
        # parent 5 -> hi = round(ln 2.5 * 232.11) = round(212.68) = 213
        dict(own=3.0, parent=5.0, t=2.0, blend=3.0, expect=[94, 213]),
    ],
    # A three-meshlet DAG: two leaves replaced by one root. Camera at (0, 0, 10) looking down -z
    # (viewMatrix = translation (0, 0, -10)), projScale 1000, near 0.1. Leaves' parent sphere and the root's own
    # sphere are (0, 0, 0, r = 1) with error 1: projected 1 * 1000 / (10 - 1) = 111.1 px.
    "tiny_dag": dict(
        bounds=[
            [-0.5, 0, 0, 0.5, 0, 0, 0, 1, 0.0, 1.0, 0, 0, -0.5, 0, 0, 0.5],
            [0.5, 0, 0, 0.5, 0, 0, 0, 1, 0.0, 1.0, 0, 0, 0.5, 0, 0, 0.5],
            [0, 0, 0, 1, 0, 0, 0, 0, 1.0, 1e30, 0, 0, 0, 0, 0, 1],
        ],
        info=[[2, 0, 0, 0], [2, 6, 0, 4], [1, 12, 1, 8]],
        level_ranges=[0, 2, 2, 1],
        level_errors=[0.0, 1.0, 1.0, 1e30],      # per level: min own, max parent
        level_guard_errors=[0.0, 1.0, 1.0, 1e30],  # per level: max own, min parent
        lod_bounds_sphere=[0, 0, 0, 1],
        replacement_group=[0, 0, -1],
        replacement_start=[0, 1],
        replacement_indices=[2],
        view=[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, -10, 1],
        proj_scale=1000.0,
        near=0.1,
        # selectCut: t = 100 -> leaves (parent 111.1 > 100, own 0 <= 100); t = 120 -> root (own 111.1 <= 120)
        select=[dict(t=100.0, expect=[1, 1, 0]), dict(t=120.0, expect=[0, 0, 1])],
        # verifyCutCoverage / verifyCutOverlap
        coverage=[dict(selected=[1, 1, 0], holes=[]), dict(selected=[0, 0, 1], holes=[]),
                  dict(selected=[1, 0, 0], holes=[1]), dict(selected=[0, 0, 0], holes=[0, 1])],
        overlap=[dict(selected=[1, 0, 1], overlaps=[0]), dict(selected=[1, 1, 0], overlaps=[])],
        # instanceMeshletRange: dMin = 10 - 1 = 9, dMax = 11, k = 1000. Level 0 possible iff 1000/9 = 111.1 > t;
        # level 1 possible iff 1000/11 = 90.9 <= t.
        meshlet_range=[dict(t=100.0, expect=[0, 3]), dict(t=50.0, expect=[0, 2]), dict(t=200.0, expect=[2, 3])],
        # instanceGuaranteedRange: t = 200: level 1 only, max own 1000/9 = 111.1 <= 199.8, parent infinite -> [2, 3];
        # t = 100: level 0 is possible but its min parent 1000/11 = 90.9 is not > 100.1 -> none
        guaranteed_range=[dict(t=200.0, expect=[2, 3]), dict(t=100.0, expect=None)],
    ),
    # HZB (OcclusionCulling.ts:284-350): max of 2 x 2, ceil halving, edge clamp
    "hzb": [
        dict(width=3, height=3, depth=[0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9],
             # mip 1 (2 x 2): (0,0) max(.1,.2,.4,.5) = .5; (1,0) x clamps to 2: max(.3,.6) = .6; (0,1) = max(.7,.8) = .8;
             # (1,1) = .9; mip 2 = .9
             levels=3, offset=[0, 9, 13], widths=[3, 2, 1], heights=[3, 2, 1],
             mips=[0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 0.5, 0.6, 0.8, 0.9, 0.9]),
        dict(width=5, height=2, depth=[1, 2, 3, 4, 5, 6, 7, 8, 9, 10],
             # mip 1 (3 x 1): max(1,2,6,7) = 7, max(3,4,8,9) = 9, x clamps to 4: max(5,10) = 10; mip 2 (2 x 1): 9, 10;
             # mip 3 (1 x 1): 10
             levels=4, offset=[0, 10, 13, 15], widths=[5, 3, 2, 1], heights=[2, 1, 1, 1],
             mips=[1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 7, 9, 10, 9, 10, 10]),
    ],
    # Morton order (GeometryPool.ts:1263-1311): centres (10,0,0), (0,0,0), (5,0,0), (0,10,0), unit spheres.
    # Box [0,10]^2 x {0}, extent 10: q = (1023,0,0), (0,0,0), (512,0,0), (0,1023,0); codes 0x09249249, 0,
    # 0x08000000, 0x12492492 -> order [1, 2, 0, 3]
    "morton": dict(centres=[[10, 0, 0], [0, 0, 0], [5, 0, 0], [0, 10, 0]], sphere=[0, 0, 0, 1], expect=[1, 2, 0, 3]),
}

out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vectors.json")
with open(out, "w") as f:
    json.dump(vectors, f, indent=1)
print("wrote", out)
