"""A second, independent restatement of the reference's ray tracer, in
numpy float32 scalars, against the oracle's trace of the same octree: the
camera ray (compute.wgsl:4590-4594, rt_main 4651-4685, with the per-scene
eye offsets and rotationMatrix 4524-4587 of scenes 0, 3, 4, 5), slab test
(4059-4070), the traversal state machine with its per-node 2x2x2 march
(4189-4403: descend, leave through the far side, a leaf ends the ray),
darkening, the movement colour of stale leaves, normals (stored, or by
finite differences 4143-4184), normal visualisation, the non-cinematic
colour of get_color_single (4481-4516) and the gamma curve (4643-4645).
Depth and normals are compared bit for bit; colours bit for bit before the
gamma curve, which is checked to 2 ulp (the oracle's pow is its own).

The octree is rebuilt from the oracle's cells (children of (l, ix, iy, iz)
are (l + 1, 2 ix + i, 2 iy + j, 2 iz + k) at child index i + 2 j + 4 k).
Where the reference reads past an empty stack (peak() returning its failure
index) the ray ends on the next pass whatever it read, so that read is not
modelled.  No device needed."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from temporalsetinversion_b200 import api, scenes

f32 = np.float32
ONE, ZERO, HALF = f32(1), f32(0), f32(0.5)
EPS = f32(0.0001)  # compute.wgsl:4141


def mn(a, b):  # minimumNumber: NaN loses, -0 < +0
    if a != a:
        return b
    if b != b or a < b:
        return a
    if b < a:
        return b
    return a if np.signbit(a) else b


def mx(a, b):
    if a != a:
        return b
    if b != b or a > b:
        return a
    if b > a:
        return b
    return b if np.signbit(a) else a


def length(v):
    return np.sqrt(f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2]))


def slabs(p0, p1, ro, inv):  # efficient_slabs, 4059-4070
    t0 = [f32((p0[a] - ro[a]) * inv[a]) for a in range(3)]
    t1 = [f32((p1[a] - ro[a]) * inv[a]) for a in range(3)]
    d1 = mx(mn(t0[0], t1[0]), mx(mn(t0[1], t1[1]), mn(t0[2], t1[2])))
    d2 = mn(mx(t0[0], t1[0]), mn(mx(t0[1], t1[1]), mx(t0[2], t1[2])))
    return (d1 <= d2 and d2 >= 0), mx(d1, ZERO), mx(d2, ZERO)


def sign(x):
    return ONE if x > 0 else (f32(-1) if x < 0 else ZERO)


class Octree:
    def __init__(self, cells):
        self.c = {(int(c["level"]), int(c["ix"]), int(c["iy"]), int(c["iz"])): c for c in cells}

    def box(self, k, pad=ZERO):
        c = self.c[k]
        return ([f32(c[a][0] - pad) for a in "xyz"], [f32(c[a][1] + pad) for a in "xyz"])

    def child(self, k, ci):
        l, x, y, z = k
        return (l + 1, 2 * x + (ci & 1), 2 * y + ((ci >> 1) & 1), 2 * z + (ci >> 2))


def field_normal(tape, p, t):  # finite_diff_normal, 4143-4184, with the scene's own f
    h = f32(0.01)
    ks = [(1, -1, -1), (-1, -1, 1), (-1, 1, -1), (1, 1, 1)]  # k.xyy, k.yyx, k.yxy, k.xxx
    boxes = np.zeros((4, 8), f32)
    for q, k in enumerate(ks):
        for a in range(3):
            boxes[q, 2 * a: 2 * a + 2] = f32(p[a] + f32(f32(k[a]) * h))
        boxes[q, 6:8] = t
    f = oracle.eval_boxes(tape, boxes, reverse=False)[:, 0].astype(f32)
    v = [f32(ks[0][a]) * f[0] for a in range(3)]
    for q in range(1, 4):
        v = [f32(v[a] + f32(f32(ks[q][a]) * f[q])) for a in range(3)]
    n = length(v)
    return [f32(v[a] / n) for a in range(3)]


def trace(tree, tape, prm, ro, rd, time):
    """trace(), 4189-4403, non-cinematic: (colour, distance, normal)."""
    inv = [f32(ONE / rd[a]) for a in range(3)]
    stack = [(0, 0, 0, 0)]
    c = [ONE, ONE, ONE]
    normal = [ZERO, ZERO, ZERO]
    ro2 = list(ro)
    p0, p1 = tree.box(stack[-1])
    hit = slabs(p0, p1, ro2, inv)
    if not hit[0]:
        return c, f32(-1), normal
    intersected = False
    for _ in range(5000):
        if intersected:
            break
        if not stack:
            return c, f32(-1), normal
        region = stack.pop()
        if not hit[0]:  # missed: back to the enclosing node
            if stack:
                p0, p1 = tree.box(stack[-1])
                hit = slabs(p0, p1, ro2, inv)
            continue
        ext = [f32(p1[a] - p0[a]) for a in range(3)]
        rol = [f32(f32(f32(f32(ro2[a] + f32(f32(hit[1] + EPS) * rd[a])) - p0[a]) * f32(2)) / ext[a])
               for a in range(3)]
        rdl = [f32(rd[a] * f32(f32(2) / ext[a])) for a in range(3)]
        mp = [int(math.floor(rol[a])) for a in range(3)]
        dd = [f32(ONE / abs(rdl[a])) for a in range(3)]
        sg = [sign(rdl[a]) for a in range(3)]
        sd = [f32(f32(f32(f32(sg[a] * f32(f32(mp[a]) - rol[a])) + f32(sg[a] * HALF)) + HALF) * dd[a])
              for a in range(3)]
        mask = [ZERO, ZERO, ZERO]
        old = list(ro2)
        for _i in range(32):
            if not prm.normal_viz and mx(ext[0], mx(ext[1], ext[2])) < ONE:
                c = [f32(v * f32(prm.octree_darken_factor)) for v in c]
            t = f32(f32(f32(length([f32(mask[a] * f32(sd[a] - dd[a])) for a in range(3)]) + hit[1]) + EPS) + ZERO)
            ro2 = [f32(old[a] + f32(t * rd[a])) for a in range(3)]
            if t >= f32(hit[2] - EPS):  # left this node through its far side
                ro2 = [f32(old[a] + f32(hit[2] * rd[a])) for a in range(3)]
                if stack:
                    p0, p1 = tree.box(stack[-1])
                    hit = slabs(p0, p1, ro2, inv)
                break
            ci = mp[0] + 2 * mp[1] + 4 * mp[2]
            if ci < 0 or ci >= 8:
                break
            child = tree.child(region, ci)
            cv = tree.c[child]
            if cv["f"] <= 0:
                tp0, tp1 = tree.box(child, EPS)
                th = slabs(tp0, tp1, ro2, inv)
                if th[0]:
                    if cv["has_children"]:
                        stack += [region, child]
                        p0, p1, hit = tp0, tp1, th
                        ext = [f32(p1[a] - p0[a]) for a in range(3)]
                        break
                    intersected = True
                    normal = [f32(cv["dx"]), f32(cv["dy"]), f32(cv["dz"])]
                    if prm.fast_normals:
                        normal = field_normal(tape, ro2, tree.c[region]["t"] if prm.swept_volume else time)
                    if prm.normal_viz:
                        n = length(normal)
                        c = [f32(f32(f32(normal[a] / n) * HALF) + HALF) for a in range(3)]
                    else:
                        tt = mn(mx(f32(f32(time - cv["t"]) * f32(60)), ZERO), ONE)  # mylerp's clamp
                        a_, b_ = [ZERO, ONE, ONE], [ZERO, ZERO, ZERO]  # 1 - movement, 1 - base
                        c = [f32(c[a] - f32(f32(a_[a] * f32(ONE - tt)) + f32(b_[a] * tt))) for a in range(3)]
                    break
            m = [sd[0] <= mn(sd[1], sd[2]), sd[1] <= mn(sd[2], sd[0]), sd[2] <= mn(sd[0], sd[1])]
            mask = [ONE if v else ZERO for v in m]
            sd = [f32(sd[a] + f32(mask[a] * dd[a])) for a in range(3)]
            mp = [mp[a] + int(m[a]) * int(sg[a]) for a in range(3)]
    c = [mx(mn(v, ONE), ZERO) for v in c]
    dist = abs(length([f32(ro2[a] - ro[a]) for a in range(3)])) if intersected else f32(-1)
    return c, dist, normal


PI = f32(math.pi)  # compute.wgsl:2476


def rotation(axis, angle):  # rotationMatrix, 4524-4587: columns, each 4 floats
    n = length(axis)
    ax = [f32(axis[a] / n) for a in range(3)]
    s_, c_ = f32(math.sin(float(angle))), f32(math.cos(float(angle)))
    oc = f32(ONE - c_)
    x, y, z = ax

    def t(a, b):
        return f32(f32(oc * a) * b)
    return [[f32(t(x, x) + c_), f32(t(x, y) - f32(z * s_)), f32(t(z, x) + f32(y * s_)), ZERO],
            [f32(t(x, y) + f32(z * s_)), f32(t(y, y) + c_), f32(t(y, z) - f32(x * s_)), ZERO],
            [f32(t(z, x) - f32(y * s_)), f32(t(y, z) + f32(x * s_)), f32(t(z, z) + c_), ZERO],
            [ZERO, ZERO, ZERO, ONE]]


def matmul(a, b):  # a * b, both as lists of columns; each sum in index order
    out = []
    for col in range(4):
        out.append([f32(f32(f32(f32(a[0][r] * b[col][0]) + f32(a[1][r] * b[col][1])) + f32(a[2][r] * b[col][2]))
                        + f32(a[3][r] * b[col][3])) for r in range(4)])
    return out


def scene_camera(view, scene_id, h):
    """rt_main 4660-4683: the eye (view column 3) and view after the scene's
    offset and rotation, and the pixel row shift of scene 0."""
    cols = [[f32(view[4 * c + r]) for r in range(4)] for c in range(4)]
    eye = cols[3][:3]
    if scene_id == 3:
        eye = [f32(eye[a] + f32(v)) for a, v in enumerate((7.7, -2.21, 7.7))]
        cols = matmul(rotation((ZERO, ONE, ZERO), f32(f32(PI / f32(4)) * f32(3))), cols)
    elif scene_id == 4:
        eye = [f32(eye[a] + f32(v)) for a, v in enumerate((0.0, -0.78, -7.0))]
    elif scene_id == 5:
        eye = [f32(eye[a] + f32(v)) for a, v in enumerate((7.13, 2.14, -5.6))]
        cols = matmul(rotation((ZERO, ONE, ZERO), f32(PI / f32(4))), cols)
        cols = matmul(rotation((f32(-1), ZERO, f32(-1)), f32(f32(PI / f32(4)) * f32(0.45))), cols)
    shift = f32(f32(h) * f32(0.32)) if scene_id == 0 else ZERO
    return eye, [v for c in cols for v in c], shift


def camera_rays(view, w, h, shift=ZERO):  # ray_direction 4590-4594 and view * vec4(d, 0), fov 90
    m = [f32(v) for v in view]
    rad = f32(f32(90) * f32(math.pi / 180))
    z = f32(f32(h) / f32(math.tan(float(f32(rad / f32(2))))))
    for py in range(h):
        for px in range(w):
            pyf = f32(f32(py) - shift)
            d = [f32(f32(f32(px) - f32(f32(w) / f32(2))) + HALF), f32(-f32(f32(pyf - f32(f32(h) / f32(2))) + HALF)),
                 f32(-z)]
            n = length(d)
            d = [f32(d[a] / n) for a in range(3)]
            g = [f32(f32(f32(f32(m[r] * d[0]) + f32(m[4 + r] * d[1])) + f32(m[8 + r] * d[2])) + f32(m[12 + r] * ZERO))
                 for r in range(3)]
            yield px, py, g


CASES = {
    "spheres16": (scenes.spheres16(0), (0.5, 0.5, 1.3)),
    "csg24": (scenes.csg(24, 3, 0.9), (1.2, 0.8, 1.4)),
}


@pytest.mark.parametrize("shading", ["stored_normals", "field_normals", "normal_viz"])
@pytest.mark.parametrize("scene", sorted(CASES))
def test_trace_matches_restatement(scene, shading):
    """A 40x24 image of a localsubdiv-7 octree after frames at t = 0 and
    1/60, traced at t = 1.75/60 so that every hit leaf is coloured by its
    age (the movement colour's lerp at a fraction), per pixel."""
    oracle.build()
    text, eye = CASES[scene]
    tape = api.IR.new(text).gpu_instructions
    prm = api.default_params(localsubdiv=7, delta=0.01, lipschitz_corrected=1, fast_normals=int(shading == "field_normals"),
                             normal_viz=int(shading == "normal_viz"))
    S = oracle.Scene(tape, prm)
    S.invert(0.0)
    S.invert(1.0 / 60.0)
    time = f32(1.75 / 60.0)
    tree = Octree(S.cells())
    w, h = 40, 24
    view = scenes.camera_look_at(eye)
    u = api.make_uniforms(view, (w, h), float(time))
    got = S.trace(u)
    ro = [f32(view[12]), f32(view[13]), f32(view[14])]
    hits = aged = 0
    with np.errstate(all="ignore"):
        for px, py, rd in camera_rays(view, w, h):
            c, d, n = trace(tree, tape, prm, ro, rd, time)
            alpha = ONE
            if prm.normal_viz and d < 0:
                c, alpha = [f32(10)] * 3, ZERO
            where = "pixel (%d, %d)" % (px, py)
            assert got["depth"][py, px].view(np.uint32) == d.view(np.uint32), (where, got["depth"][py, px], d)
            assert np.array_equal(got["normal"][py, px], np.array(n, f32), equal_nan=True), (where, got["normal"][py, px], n)
            assert got["rgba"][py, px, 3] == alpha, where
            want = np.array([f32(float(v) ** 0.45) if v == v else np.nan for v in c], f32)
            ulps = np.abs(got["rgba"][py, px, :3].view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
            same_nan = np.isnan(want) & np.isnan(got["rgba"][py, px, :3])
            assert np.all((ulps <= 2) | same_nan), (where, got["rgba"][py, px], c)
            hits += int(d >= 0)
            aged += int(d >= 0 and not prm.normal_viz and ZERO < c[1] < c[0])  # red, partly faded to white
    assert hits > 100, hits
    assert prm.normal_viz or aged > 50, aged


# per scene id: the eye the shader should end up with
SCENE_EYES = {0: (0.5, 0.9, 1.3), 3: (0.6, 0.5, 1.2), 4: (0.4, 0.6, 1.4), 5: (0.7, 0.4, 1.1)}
OFFSETS = {0: (0, 0, 0), 3: (7.7, -2.21, 7.7), 4: (0.0, -0.78, -7.0), 5: (7.13, 2.14, -5.6)}


def _base_view(scene_id):
    """A uniforms.view whose scene-adjusted camera looks at the origin from
    SCENE_EYES: rotation undone in float64, eye minus the scene's offset."""
    want = np.asarray(scenes.camera_look_at(SCENE_EYES[scene_id]), np.float64).reshape(4, 4)  # rows = columns
    rot = np.eye(4)
    if scene_id == 3:
        rot = np.asarray(rotation((ZERO, ONE, ZERO), f32(f32(PI / f32(4)) * f32(3))), np.float64)
    elif scene_id == 5:
        r1 = np.asarray(rotation((ZERO, ONE, ZERO), f32(PI / f32(4))), np.float64)
        r2 = np.asarray(rotation((f32(-1), ZERO, f32(-1)), f32(f32(PI / f32(4)) * f32(0.45))), np.float64)
        rot = (r2.T @ r1.T).T  # column lists: the product r2 * r1 as columns
    base = want.copy()
    base[:3] = (np.linalg.inv(rot.T) @ want[:3].T).T  # undo view' = R * view on the direction columns
    base[3, :3] = np.asarray(SCENE_EYES[scene_id]) - np.asarray(OFFSETS[scene_id])
    return [float(v) for v in base.reshape(-1)]


@pytest.mark.parametrize("scene_id", sorted(SCENE_EYES))
def test_scene_cameras_match_restatement(scene_id):
    """The per-scene cameras of rt_main (eye offsets, view rotations, scene
    0's row shift) on a 40x24 image of a localsubdiv-7 octree, per pixel."""
    oracle.build()
    tape = api.IR.new(scenes.spheres16(0)).gpu_instructions
    prm = api.default_params(localsubdiv=7, delta=0.01, scene_id=scene_id)
    S = oracle.Scene(tape, prm)
    S.invert(0.0)
    tree = Octree(S.cells())
    w, h = 40, 24
    view = _base_view(scene_id)
    got = S.trace(api.make_uniforms(view, (w, h), 0.0))
    eye, m, shift = scene_camera(view, scene_id, h)
    hits = 0
    with np.errstate(all="ignore"):
        for px, py, rd in camera_rays(m, w, h, shift):
            c, d, n = trace(tree, tape, prm, eye, rd, f32(0))
            where = "scene %d pixel (%d, %d)" % (scene_id, px, py)
            assert got["depth"][py, px].view(np.uint32) == d.view(np.uint32), (where, got["depth"][py, px], d)
            assert np.array_equal(got["normal"][py, px], np.array(n, f32)), where
            want = np.array([f32(float(v) ** 0.45) for v in c], f32)
            ulps = np.abs(got["rgba"][py, px, :3].view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
            assert np.all(ulps <= 2), (where, got["rgba"][py, px], c)
            hits += int(d >= 0)
    assert hits > 30, hits


def test_swept_volume_field_normals_match_restatement():
    """Swept volume with finite-difference normals: the normal is taken at
    the time of the hit leaf's parent (compute.wgsl:4337-4342), not at the
    frame's time (traced here at t = 0.6 after sweeps up to 0.5), per pixel."""
    oracle.build()
    tape = api.IR.new(scenes.swept(8, 4)).gpu_instructions
    prm = api.default_params(localsubdiv=6, pointsample=0, swept_volume=1, fast_normals=1)
    S = oracle.Scene(tape, prm)
    S.invert(0.25, 0.0)
    S.invert(0.5, 0.25)
    tree = Octree(S.cells())
    w, h = 40, 24
    view = scenes.camera_look_at((0.4, 0.6, 1.6))
    time = f32(0.6)
    got = S.trace(api.make_uniforms(view, (w, h), float(time)))
    ro = [f32(view[12]), f32(view[13]), f32(view[14])]
    hits = 0
    with np.errstate(all="ignore"):
        for px, py, rd in camera_rays(view, w, h):
            c, d, n = trace(tree, tape, prm, ro, rd, time)
            where = "pixel (%d, %d)" % (px, py)
            assert got["depth"][py, px].view(np.uint32) == d.view(np.uint32), where
            assert np.array_equal(got["normal"][py, px], np.array(n, f32), equal_nan=True), where
            hits += int(d >= 0)
    assert hits > 50, hits
