"""Writes tests/golden/vectors.json: known-answer vectors for the cut path, derived by hand from the reference's
formulas (the reference ships no golden vectors, and its TypeScript cannot run in this repository's containers).

Each value below is worked out in the comment beside it from the formula it pins; nothing here calls the oracle or
the engine. Run: python tests/golden/make_golden.py
"""
import json
import math
import os

S2 = 255 / math.log(2)  # blend-step scale for lodBlend 2 (lodBlend.ts:56): 367.8887...
H = math.sqrt(0.5)  # 1 / sqrt(2)
FULL = 255 << 16  # packed blend range of a meshlet drawn over every pixel (lo 0, hi 255)

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
    # three's Frustum.setFromProjectionMatrix(P * V, WebGPUCoordinateSystem) (VirtualGeometry.ts:429-437): planes
    # right = row3 - row0, left = row3 + row0, bottom = row3 + row1, top = row3 - row1, far = row3 - row2,
    # near = row2 (WebGPU depth in [0, 1]), each divided by the length of its normal.
    # P: fov 90 deg, aspect 1, near 1, far 100: rows (1,0,0,0), (0,1,0,0), (0,0,a,a), (0,0,-1,0), a = -100/99.
    "frustum_planes": [
        # V = identity: right (-1,0,-1,0)/sqrt2, left (1,0,-1,0)/sqrt2, bottom (0,1,-1,0)/sqrt2, top (0,-1,-1,0)/sqrt2,
        # far (0, 0, -1-a, -a) / (-1-a) = (0,0,1, a/(1+a)) = (0,0,1,100), near (0,0,a,a)/|a| = (0,0,-1,-1)
        dict(pv=[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -100 / 99, -1, 0, 0, -100 / 99, 0],
             expect=[[-H, 0, -H, 0], [H, 0, -H, 0], [0, H, -H, 0], [0, -H, -H, 0], [0, 0, 1, 100], [0, 0, -1, -1]]),
        # V = translation (0, 0, -10) (camera at z = 10): P * V has the constant column
        # (0, 0, -10a + a, 10): right/left constants 10/sqrt2, bottom/top 10/sqrt2,
        # far (0, 0, -1-a, 10 + 9a) / (-1-a) -> constant (10 + 9a)/(-1-a) = (10 - 900/99)/(1/99) = 90,
        # near (0, 0, a, -9a) / |a| = (0, 0, -1, 9)
        dict(pv=[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -100 / 99, -1, 0, 0, 900 / 99, 10],
             expect=[[-H, 0, -H, 10 * H], [H, 0, -H, 10 * H], [0, H, -H, 10 * H], [0, -H, -H, 10 * H], [0, 0, 1, 90],
                     [0, 0, -1, 9]]),
    ],
    # The per-frame passes on a hand-built scene: 23 meshes, each the tiny_dag above (two leaves of 2 triangles,
    # a root of 1; LOD, cull and bounding spheres (0, 0, 0, 1)) with ONE instance (translation + uniform scale s),
    # so instance k is mesh k and its cell holds it alone (cell radius r(1 + 1e-4) + 1e-3, max radius
    # r(1 + 1e-4) + 1e-4, GeometryPool.ts:519-545). Camera: V = identity (eye at the origin looking down -z), P as in
    # frustum_planes (fov 90, near 1, far 100), viewport 200 x 200 -> projScale = P[5] * 200 / 2 = 100. Global
    # minPixelRadius 0.7, shadowErrorScale 3, capacity scale 1. Meshlets are named by their index in the mesh (0, 1
    # leaves, 2 root); `packed` is triCount | lo << 8 | hi << 16 (full fade: lo 0, hi 255).
    # Formulas (GeometryPool.ts): cell cull (:740-758), instance tests (:870-898), pixelsAtMin/Max = s * 100 /
    # max(d -+ r, near) (:900-904), level possible / sure (:793-803, margin 1e-3), fast path (:817-823),
    # projectedError (:678-683), meshlet drawn + blend steps (:941-957), occludedSphere + occluded
    # (:701-705, OcclusionCulling.ts:119-170).
    "pass_scene": dict(
        instances=[
            # 0 "lod": d = 10, r = 1: pAtMin = 100/9 = 11.11, pAtMax = 100/11 = 9.09
            dict(name="lod", at=[0, 0, -10], s=1.0),
            # 1 "pe": s = 2, d = 10: pAtMin = 200/8 = 25 exactly, pAtMax = 200/12 = 16.67; the root's own error and
            # the leaves' parent error project to 1 * 2 / (10 - 2) * 100 = 25 exactly (float too)
            dict(name="pe", at=[0, 0, -10], s=2.0),
            # 2 "blend": d = 31: pAtMin = 100/30 = 3.333, pAtMax = 100/32 = 3.125
            dict(name="blend", at=[0, 0, -31], s=1.0),
            # frustum: distance to the plane of the centre (x, y, -10) is (10 - |x|)/sqrt2 for left/right and
            # (10 - |y|)/sqrt2 for bottom/top: 12 -> -1.414 < -1.0011 (cell culled); 10.6 -> -0.424 (kept, and the
            # leaf on the inner side, 0.5 closer, is drawn: its cull sphere reaches -0.424 + 0.354 > -0.5)
            dict(name="left_out", at=[-12, 0, -10], s=1.0), dict(name="left_in", at=[-10.6, 0, -10], s=1.0),
            dict(name="right_out", at=[12, 0, -10], s=1.0), dict(name="right_in", at=[10.6, 0, -10], s=1.0),
            dict(name="bottom_out", at=[0, -12, -10], s=1.0), dict(name="bottom_in", at=[0, -10.6, -10], s=1.0),
            dict(name="top_out", at=[0, 12, -10], s=1.0), dict(name="top_in", at=[0, 10.6, -10], s=1.0),
            # near (0,0,-1,-1): -z - 1: z = 0.5 -> -1.5 (culled); z = -0.6 -> -0.4 (kept; the leaves' cull spheres
            # reach -0.4 >= -0.5, drawn, parent error 1 * 100 / max(0.6 - 1, 1) = 100 > t)
            dict(name="near_out", at=[0, 0, 0.5], s=1.0), dict(name="near_in", at=[0, 0, -0.6], s=1.0),
            # far (0,0,1,100): z + 100: z = -102 -> -2 (culled); z = -100.5 -> -0.5 (kept; the root, own error
            # 100/99.5 = 1.005 px, is drawn through the meshlet pass since its cull sphere is not inside)
            dict(name="far_out", at=[0, 0, -102], s=1.0), dict(name="far_in", at=[0, 0, -100.5], s=1.0),
            # size (cell): d = 50, cell radius 0.50105, gap 49.49895, max radius 0.50015:
            # 0.50015 * 100 / 49.49895 = 1.0104 px < 2 -> culled; >= 1 -> kept, and the instance test
            # r * 100 / d = 0.5 * 100 / 50 = 1.0 is not < 1 -> kept (the limit itself draws)
            dict(name="small", at=[0, 0, -50], s=0.5, min_pixel_radius=2.0),
            dict(name="small_edge", at=[0, 0, -50], s=0.5, min_pixel_radius=1.0),
            # draw distance: cell gap 49.49895 > 49 -> culled; instance d - r = 49.5 < 50 -> kept
            dict(name="dist49", at=[0, 0, -50], s=0.5, max_draw_distance=49.0),
            dict(name="dist50", at=[0, 0, -50], s=0.5, max_draw_distance=50.0),
            dict(name="disabled", at=[0, 0, -10], s=1.0, enabled=False),
            # HZB: s = 0.5 at (-5, 5, -10) and (5, 5, -10); occludedSphere grows r by |z| * high / projScale =
            # 10 * 1 / 100 = 0.1 (t = 1) -> R = 0.6, nearDepth 9.4, farDepth 10.6.
            # x/depth in [-5.6/9.4, -4.4/10.6] = [-0.595745, -0.415094] -> texels floor((0.5 + x/2) * 4) = 0..1;
            # y/depth in [0.415094, 0.595745] -> rows floor((0.5 - y/2) * 4) = 0..1 (row 0 at the top): extent 2 ->
            # mip 1, one texel (0, 0) = max of the top-left 2 x 2 of mip 0. minZ = P14/9.4 - P10 =
            # (100/99)(1 - 1/9.4) = 0.902643; top-left 0.5 -> hidden; the mirror image at x = +5 reads the
            # top-right 0.95 > 0.902643 -> visible
            dict(name="occluded", at=[-5, 5, -10], s=0.5, occlusion=True),
            dict(name="unoccluded", at=[5, 5, -10], s=0.5, occlusion=True),
            # shadow: left of the frustum (-1.414 on the left plane); the swept test adds max(dot(n, sweep), 0):
            # sweep (5, 0, 0) -> +3.536 on the left plane -> min over planes 2.12 >= 1 (kept, cull sphere inside the
            # swept frustum); sweep (-5, 0, 0) -> +0 -> culled
            dict(name="shadow", at=[-12, 0, -10], s=1.0, shadow=True),
        ],
        hzb=[[0.5, 0.5, 0.95, 0.95], [0.5, 0.5, 0.95, 0.95], [0.95, 0.95, 0.95, 0.95], [0.95, 0.95, 0.95, 0.95]],
        views=[
            # A: t = 5, lodBlend 1 (no band: low = high = 5).
            #  lod: level 0 possible (11.11 > 5), sure (0 <= 4.995, 9.09 > 5.005); level 1 not (9.09 > 5);
            #       2 meshlets <= 4, cull sphere inside -> fast path, leaves.
            #  pe: level 0 possible (25 > 5), sure (16.67 > 5.005); level 1 not (16.67 > 5) -> fast path, leaves.
            #  blend: level 0 not (3.33 <= 5); level 1 possible, sure (3.33 <= 4.995) -> fast path, root.
            #  *_in: kept, their cull spheres cross a plane -> no fast path: one work item each (6 items).
            #  small_edge, dist50: pAtMin = 50/49.5 = 1.0101: level 1 only, sure -> fast path, root.
            #  occluded/unoccluded (no HZB in this view): pAtMin = 50/11.747 = 4.256 -> level 1, sure -> root.
            #  Cells kept: lod, pe, blend, 6 *_in, small_edge, dist50, occluded, unoccluded = 13; fast-path meshlets
            #  2 + 2 + 1 + 1 + 1 + 1 + 1 = 9. Shadow cut: the only shadow mesh is culled without a sweep.
            dict(name="A", t=5.0, blend=1.0, sweep=[0, 0, 0], hzb=False,
                 expect=dict(visible_cells=13, work0=6, fast_emitted=9, occluded_instances=0, cut1=[],
                             cut0={"lod": [[0, 2 | FULL], [1, 2 | FULL]], "pe": [[0, 2 | FULL], [1, 2 | FULL]],
                                   "blend": [[2, 1 | FULL]], "small_edge": [[2, 1 | FULL]],
                                   "dist50": [[2, 1 | FULL]], "occluded": [[2, 1 | FULL]],
                                   "unoccluded": [[2, 1 | FULL]]},
                             present0=["left_in", "right_in", "bottom_in", "top_in", "near_in", "far_in"])),
            # B: pe at t = 24.99: level 0 possible (25 > 24.99) but not sure (16.67 < 25.01); level 1 possible ->
            # item [0, 3): leaves own 0, parent 25 > 24.99 -> drawn; root own 25 > 24.99 -> not.
            dict(name="B1", t=24.99, blend=1.0, sweep=[0, 0, 0], hzb=False,
                 expect=dict(only="pe", cut0={"pe": [[0, 2 | FULL], [1, 2 | FULL]]})),
            # t = 25: level 0 not possible (25 > 25 false); level 1 possible (16.67 <= 25), not sure (25 > 24.975)
            # -> item [2, 3): root own 25 <= 25 -> drawn (the leaves' parent 25 > 25 fails).
            dict(name="B2", t=25.0, blend=1.0, sweep=[0, 0, 0], hzb=False,
                 expect=dict(only="pe", cut0={"pe": [[2, 1 | FULL]]})),
            # C: t = 2.5, lodBlend 2: width = 1 + smoothstep(1.25, 2.5, 2.5) = 2 -> low 2.5, high 5, steps
            # 255 / ln 2. blend: level 0 possible (3.33 > 2.5), not sure (3.125 < 5.005); level 1 possible
            # (3.125 <= 5), not sure (3.33 > 2.4975) -> item. Leaves: own 0 -> lo 0; parent 1 * 100/30 = 3.333 ->
            # hi = round(ln(3.333/2.5) * 367.889) = round(105.84) = 106. Root: own 3.333 -> lo 106; parent infinite
            # -> hi 255.
            dict(name="C", t=2.5, blend=2.0, sweep=[0, 0, 0], hzb=False,
                 expect=dict(only="blend", cut0={"blend": [[0, 2 | 106 << 16], [1, 2 | 106 << 16],
                                                           [2, 1 | 106 << 8 | 255 << 16]]})),
            # D: t = 1, HZB above: occluded hidden (1 instance counted), unoccluded drawn: level 0 possible
            # (4.256 > 1), sure (3.92 > 1.001) -> fast path, leaves.
            dict(name="D", t=1.0, blend=2.0, sweep=[0, 0, 0], hzb=True,
                 expect=dict(occluded_instances=1, absent0=["occluded"],
                             cut0={"unoccluded": [[0, 2 | FULL], [1, 2 | FULL]]})),
            # E: shadow cut threshold 5 * 3 = 15: d = 15.62, pAtMin = 100/14.62 = 6.84 -> level 1 only, sure
            # (6.84 <= 14.985), cull sphere inside the swept frustum -> fast path, root.
            dict(name="E1", t=5.0, blend=1.0, sweep=[5, 0, 0], hzb=False,
                 expect=dict(cut1=[["shadow", 2, 1 | FULL]], absent0=["shadow"])),
            dict(name="E2", t=5.0, blend=1.0, sweep=[-5, 0, 0], hzb=False, expect=dict(cut1=[], absent0=["shadow"])),
        ],
    ),
}

out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "vectors.json")
with open(out, "w") as f:
    json.dump(vectors, f, indent=1)
print("wrote", out)
