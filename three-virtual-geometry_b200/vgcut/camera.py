"""Camera matrices in three.js conventions (column-major ``Matrix4.elements``, WebGPU [0, 1] depth).

The cut reads ``camera.matrixWorldInverse`` and ``camera.projectionMatrix`` (VirtualGeometry.ts:414-427); these
helpers build them from a position / target / field of view the way three's ``PerspectiveCamera`` and
``Object3D.lookAt`` do, in double precision.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def perspective(fov_deg: float, aspect: float, near: float, far: float) -> np.ndarray:
    """PerspectiveCamera.updateProjectionMatrix with the WebGPU coordinate system (depth in [0, 1])."""
    top = near * math.tan(math.radians(0.5 * fov_deg))
    height = 2 * top
    width = aspect * height
    left = -0.5 * width
    right, bottom = left + width, top - height
    x = 2 * near / (right - left)
    y = 2 * near / (top - bottom)
    a = (right + left) / (right - left)
    b = (top + bottom) / (top - bottom)
    c = -far / (far - near)
    d = -far * near / (far - near)
    m = np.zeros(16)
    m[0], m[8] = x, a
    m[5], m[9] = y, b
    m[10], m[14] = c, d
    m[11] = -1.0
    return m


def orthographic(left: float, right: float, top: float, bottom: float, near: float, far: float) -> np.ndarray:
    """OrthographicCamera projection, WebGPU depth range [0, 1]."""
    w, h, p = 1.0 / (right - left), 1.0 / (top - bottom), 1.0 / (far - near)
    m = np.zeros(16)
    m[0], m[12] = 2 * w, -(right + left) * w
    m[5], m[13] = 2 * h, -(top + bottom) * h
    m[10], m[14] = -p, -near * p
    m[15] = 1.0
    return m


def look_at_world(eye, target, up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """Camera world matrix looking from ``eye`` toward ``target`` (three's Matrix4.lookAt for cameras: -z forward)."""
    eye = np.asarray(eye, float)
    z = eye - np.asarray(target, float)
    if np.dot(z, z) == 0:
        z = np.array([0.0, 0.0, 1.0])
    z /= np.linalg.norm(z)
    x = np.cross(np.asarray(up, float), z)
    if np.dot(x, x) == 0:
        z2 = z + np.array([1e-4, 0, 0]) if abs(up[2]) == 1 else z + np.array([0, 0, 1e-4])
        z2 /= np.linalg.norm(z2)
        x = np.cross(np.asarray(up, float), z2)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = x, y, z, eye
    return m.T.reshape(-1)  # column-major elements


def invert_rigid(world: np.ndarray) -> np.ndarray:
    """Inverse of a rigid column-major matrix (camera.matrixWorldInverse)."""
    m = np.asarray(world, float).reshape(4, 4).T
    r, t = m[:3, :3], m[:3, 3]
    inv = np.eye(4)
    inv[:3, :3] = r.T
    inv[:3, 3] = -r.T @ t
    return inv.T.reshape(-1)


def mat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Column-major a * b."""
    A = np.asarray(a, float).reshape(4, 4).T
    B = np.asarray(b, float).reshape(4, 4).T
    return (A @ B).T.reshape(-1)


def compose(position, yaw: float = 0.0, scale: float = 1.0) -> np.ndarray:
    """Instance matrix: translation * rotation about y * uniform scale, column-major 16 floats."""
    c, s = math.cos(yaw), math.sin(yaw)
    m = np.array([c * scale, 0, -s * scale, 0, 0, scale, 0, 0, s * scale, 0, c * scale, 0,
                  position[0], position[1], position[2], 1.0])
    return m


@dataclass
class Camera:
    """What the cut needs from a three.js camera: view matrix, projection, near, drawing-buffer CSS height."""
    view: np.ndarray
    proj: np.ndarray
    near: float
    height: float = 1080.0
    width: float = 1920.0
    extra: dict = field(default_factory=dict)

    @property
    def proj_scale(self) -> float:
        """projection[1][1] * viewportHeight / 2 (VirtualGeometry.ts:425)."""
        return float(self.proj[5] * self.height * 0.5)

    @staticmethod
    def perspective_look_at(eye, target, fov: float = 60.0, width: float = 1920, height: float = 1080,
                            near: float = 0.1, far: float = 5000.0) -> "Camera":
        world = look_at_world(eye, target)
        return Camera(view=invert_rigid(world), proj=perspective(fov, width / height, near, far), near=near,
                      height=float(height), width=float(width), extra={"eye": np.asarray(eye, float)})


def cascade_clips(camera, light_dir, splits, caster_reach: float = 200.0) -> list:
    """World -> clip matrices of orthographic shadow cascades for `camera` (cascaded shadow maps): cascade i bounds
    the slice [splits[i], splits[i+1]] of the camera frustum in light space, its near plane pulled `caster_reach`
    toward the light so casters outside the slice that shade it stay inside. `light_dir` points from the light into
    the scene."""
    d = np.asarray(light_dir, float)
    d = d / np.linalg.norm(d)
    cam_world = invert_rigid(camera.view)
    W = np.asarray(cam_world, float).reshape(4, 4).T
    P = np.asarray(camera.proj, float).reshape(4, 4).T
    tan_y = 1.0 / P[1, 1]
    tan_x = 1.0 / P[0, 0]
    out = []
    for a, b in zip(splits[:-1], splits[1:]):
        corners = []
        for z in (a, b):
            for sx in (-1, 1):
                for sy in (-1, 1):
                    corners.append(W @ np.array([sx * tan_x * z, sy * tan_y * z, -z, 1.0]))
        corners = np.array(corners)[:, :3]
        centre = corners.mean(axis=0)
        up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.99 else (0.0, 0.0, 1.0)
        light_view = invert_rigid(look_at_world(centre - d, centre, up))
        L = np.asarray(light_view, float).reshape(4, 4).T
        ls = (L[:3, :3] @ corners.T).T + L[:3, 3]
        lo, hi = ls.min(axis=0), ls.max(axis=0)
        # light looks down -z: near = -max z (pulled toward the light), far = -min z
        proj = orthographic(lo[0], hi[0], hi[1], lo[1], -hi[2] - caster_reach, -lo[2])
        out.append(mat_mul(proj, light_view))
    return out
