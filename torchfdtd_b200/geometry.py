"""Analytic solid membership for staircase voxelization.

Restates reference ``torchfdtd/geometry.py``: ``axis_rotation`` :9-15,
``rotation_matrix`` :18-25, ``radii`` :28-30, the even-odd polygon test
``_polygon_parity``/``polygon_contains`` :88-106, ``contains`` :106-133 and
``object_bounds`` :136-148. Membership decides which cells receive a
material's permittivity, so the boundary conventions (closed inequalities,
contour edges count as material) follow the reference exactly.
"""
import math

import numpy as np


def axis_rotation(axis, angle):
    if axis == 'none':
        return np.eye(3)
    angle %= 360
    exact = {0: (1., 0.), 90: (0., 1.), 180: (-1., 0.), 270: (0., -1.)}
    c, s = exact.get(angle, (math.cos(math.radians(angle)), math.sin(math.radians(angle))))
    a = 'xyz'.index(axis)
    b, d = (a + 1) % 3, (a + 2) % 3
    r = np.eye(3)
    r[b, b] = r[d, d] = c
    r[b, d], r[d, b] = -s, s
    return r


def rotation_matrix(obj):
    """Local to world: the legacy z rotation first, then the three fixed-axis rotations in order."""
    angle = math.radians(obj.rotation)
    c, s = math.cos(angle), math.sin(angle)
    r = np.array([[c, -s, 0.], [s, c, 0.], [0., 0., 1.]])
    for axis, a in zip(obj.rotation_axes, obj.rotation_angles):
        r = axis_rotation(axis, a) @ r
    return r


def radii(obj):
    return (obj.radius, obj.radius_2 if obj.make_ellipsoid else obj.radius,
            obj.radius_3 if obj.make_ellipsoid else obj.radius)


def _contour_parity(x, y, vertices):
    shape = np.broadcast_shapes(np.shape(x), np.shape(y))
    inside = np.zeros(shape, bool)
    boundary = np.zeros(shape, bool)
    v = np.asarray(vertices)
    span = np.ptp(v, axis=0).max()
    tol = 64 * np.finfo(float).eps * max(span, 1e-300)
    for (ax, ay), (bx, by) in zip(v, np.roll(v, -1, axis=0)):
        cross = (bx - ax) * (y - ay) - (by - ay) * (x - ax)
        boundary |= ((abs(cross) <= tol * max(abs(bx - ax), abs(by - ay))) & (x >= min(ax, bx) - tol) & (x <= max(ax, bx) + tol)
                     & (y >= min(ay, by) - tol) & (y <= max(ay, by) + tol))
        if by != ay:
            inside ^= ((ay > y) != (by > y)) & (x < (bx - ax) * (y - ay) / (by - ay) + ax)
    return inside, boundary


def polygon_contains(x, y, vertices, holes=()):
    inside, boundary = _contour_parity(x, y, vertices)
    for hole in holes:
        parity, edge = _contour_parity(x, y, hole)
        inside ^= parity
        boundary |= edge
    return inside | boundary


def contains(obj, x, y, z):
    delta = [x - obj.center[0], y - obj.center[1], z - obj.center[2]]
    only_z = all(axis in ('none', 'z') or angle % 360 == 0 for axis, angle in zip(obj.rotation_axes, obj.rotation_angles))
    isotropic = not obj.make_ellipsoid
    invariant = ((obj.kind == 'sphere' and isotropic)
                 or (obj.kind in ('circle', 'ring') and isotropic and only_z and (obj.kind != 'ring' or obj.angular_span == 360)))
    if invariant or (obj.rotation == 0 and not any(obj.rotation_angles)):
        u, v, w = delta
    elif not any(obj.rotation_angles):
        a = math.radians(obj.rotation)
        c, s = math.cos(a), math.sin(a)
        u, v, w = c * delta[0] + s * delta[1], -s * delta[0] + c * delta[1], delta[2]
    else:
        m = rotation_matrix(obj)
        u, v, w = [sum(m[a, b] * delta[a] for a in range(3) if m[a, b] != 0) for b in range(3)]
    if obj.kind == 'rectangle':
        return (abs(u) <= obj.size[0] / 2) & (abs(v) <= obj.size[1] / 2) & (abs(w) <= obj.size[2] / 2)
    if obj.kind == 'polygon':
        return polygon_contains(u, v, obj.vertices, obj.holes) & (abs(w) <= obj.size[2] / 2)
    rx, ry, rz = radii(obj)
    if obj.kind == 'sphere':
        return (u / rx)**2 + (v / ry)**2 + (w / rz)**2 <= 1 if obj.make_ellipsoid else u * u + v * v + w * w <= rx * rx
    mask = ((u / rx)**2 + (v / ry)**2 <= 1 if obj.make_ellipsoid else u * u + v * v <= rx * rx) & (abs(w) <= obj.size[2] / 2)
    if obj.kind == 'ring':
        if obj.inner_radius > 0:
            if obj.make_ellipsoid:
                mask &= (u / obj.inner_radius)**2 + (v / obj.inner_radius_2)**2 >= 1
            else:
                mask &= u * u + v * v >= obj.inner_radius**2
        if obj.angular_span < 360:
            angle = (np.degrees(np.arctan2(v, u)) - obj.theta_start) % 360
            mask &= (angle <= obj.angular_span + 1e-12) | ((u == 0) & (v == 0))
    return mask


def object_bounds(obj):
    """Centre and full span of a conservative axis-aligned support box."""
    r = rotation_matrix(obj)
    center = np.asarray(obj.center)
    if obj.kind == 'polygon':
        points = np.array([[x, y, z] for x, y in obj.vertices for z in (-obj.size[2] / 2, obj.size[2] / 2)]) @ r.T + center
        low, high = points.min(axis=0), points.max(axis=0)
        return tuple((low + high) / 2), tuple(high - low)
    if obj.kind == 'rectangle':
        half = np.abs(r) @ (np.array(obj.size) / 2)
    elif obj.kind == 'sphere':
        half = np.sqrt((r * r) @ (np.array(radii(obj))**2))
    else:
        rx, ry, _ = radii(obj)
        half = np.sqrt((r[:, 0] * rx)**2 + (r[:, 1] * ry)**2) + abs(r[:, 2]) * obj.size[2] / 2
    return tuple(center), tuple(2 * half)
