"""Analytic obstacle signed distance functions, restated in float64 NumPy.

Test infrastructure only (see ``oracle/__init__.py``).

Follows the WGSL shape library ``src/js/30-wgsl-sim.js:40-114`` and its JS mirror
``src/js/10-scene.js:125-171`` (shape ids and parameter packing: ``10-scene.js:143-157``,
object packing: ``src/js/50-sim.js:165-211``). Every arithmetic step is written out in the
order the CUDA path evaluates it (plain IEEE float64 +,-,*,/,sqrt, no fused multiply-add),
so lattice values and face fractions agree bit for bit with the device.

An object is a dict with keys
  type   0 round box, 1 sphere, 2 cylinder, 3 cone, 4 torus, 5 cup, 6 container, 7 gutter
         (obstacles, flag 1) or 9 drain cylinder (flag 2)
  pos    centre (3,) in solver coordinates (y up)
  rot    3x3 world-from-local rotation R (``m3.euler``, ``src/js/00-util.js:22-30``)
  dims   (4,) shape parameters as packed by ``shapeParams`` (``10-scene.js:143-157``)
  lin, ang  linear / angular velocity of the solid (3,) each
  bound  bounding radius (``boundRadius`` ``10-scene.js:177-188`` + 0.002)
  flag   1 obstacle, 2 drain
"""
import math
import numpy as np

BIG = 1e9


def euler_deg(rx, ry, rz):
    """R = Rz·Ry·Rx from degrees (``src/js/00-util.js:22-30``)."""
    d = math.pi / 180.0
    cx, sx, cy, sy, cz, sz = (math.cos(rx * d), math.sin(rx * d), math.cos(ry * d),
                              math.sin(ry * d), math.cos(rz * d), math.sin(rz * d))
    return np.array([[cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx],
                     [sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx],
                     [-sy, cy * sx, cy * cx]])


def shape_params(shape, dims):
    """(type, d0..d3) of an obstacle from its editor dims (``10-scene.js:143-157``)."""
    d = dims
    if shape == 'box':
        return 0, [d['w'] / 2, d['h'] / 2, d['d'] / 2, min(0.003, d['w'] / 4, d['h'] / 4, d['d'] / 4)]
    if shape == 'plate':
        return 0, [d['w'] / 2, d['t'] / 2, d['d'] / 2, min(0.002, d['t'] / 4)]
    if shape == 'sphere':
        return 1, [d['r'], 0.0, 0.0, 0.0]
    if shape == 'cylinder':
        return 2, [d['r'], d['h'] / 2, 0.0, 0.0]
    if shape == 'cone':
        return 3, [d['r'], d['h'] / 2, 0.0, 0.0]
    if shape == 'torus':
        return 4, [d['R'], d['r'], 0.0, 0.0]
    if shape == 'cup':
        return 5, [d['r'], d['h'] / 2, min(d['t'], d['r'] * 0.8), 0.0]
    if shape == 'container':
        return 6, [d['w'] / 2, d['h'] / 2, d['d'] / 2, min(d['t'], d['w'] / 3, d['d'] / 3, d['h'] * 0.8)]
    if shape == 'gutter':
        return 7, [d['len'] / 2, d['r'], d['t'], 0.0]
    return 0, [0.05, 0.05, 0.05, 0.0]


def bound_radius(t, a, b, c, e):
    """``boundRadius`` (``10-scene.js:177-188``)."""
    if t == 0 or t == 6:
        return math.sqrt(a * a + b * b + c * c)
    if t == 1:
        return a
    if t in (2, 3, 5):
        return math.sqrt(a * a + b * b)
    if t == 4:
        return a + b
    if t == 7:
        return math.sqrt(a * a + (b + c) * (b + c))
    return 0.1


def make_obstacle(shape, pos, rot_deg=(0.0, 0.0, 0.0), lin=(0, 0, 0), ang=(0, 0, 0), **dims):
    t, d = shape_params(shape, dims)
    return dict(type=t, pos=np.array(pos, float), rot=euler_deg(*rot_deg), dims=np.array(d, float),
                lin=np.array(lin, float), ang=np.array(ang, float),
                bound=bound_radius(t, *d) + 0.002, flag=1)


def make_drain(pos, r, rot_deg=(0.0, 0.0, 0.0)):
    """Drain cylinder of radius r and half height 0.012 (``50-sim.js:181``)."""
    return dict(type=9, pos=np.array(pos, float), rot=euler_deg(*rot_deg), dims=np.array([r, 0.012, 0, 0], float),
                lin=np.zeros(3), ang=np.zeros(3), bound=r + 0.02, flag=2)


# ---------------------------------------------------------------- vectorised shape functions (p: (N,3))
def _len3(x, y, z):
    return np.sqrt(x * x + y * y + z * z)


def _len2(x, y):
    return np.sqrt(x * x + y * y)


def to_local(o, p):
    """q = Rᵀ (p - pos), each component dot(column, d) summed left to right (``30-wgsl-sim.js:42``)."""
    d = p - o['pos']
    R = o['rot']
    dx, dy, dz = d[:, 0], d[:, 1], d[:, 2]
    return np.stack([R[0, 0] * dx + R[1, 0] * dy + R[2, 0] * dz,
                     R[0, 1] * dx + R[1, 1] * dy + R[2, 1] * dz,
                     R[0, 2] * dx + R[1, 2] * dy + R[2, 2] * dz], 1)


def sd_round_box(q, bx, by, bz, r):
    """``sdRoundBox`` (``30-wgsl-sim.js:43-46``)."""
    qx = np.abs(q[:, 0]) - bx + r
    qy = np.abs(q[:, 1]) - by + r
    qz = np.abs(q[:, 2]) - bz + r
    out = _len3(np.maximum(qx, 0.0), np.maximum(qy, 0.0), np.maximum(qz, 0.0))
    return out + np.minimum(np.maximum(qx, np.maximum(qy, qz)), 0.0) - r


def sd_cyl(q, r, hh):
    """``sdCyl`` (``30-wgsl-sim.js:47-50``)."""
    dx = _len2(q[:, 0], q[:, 2]) - r
    dy = np.abs(q[:, 1]) - hh
    return np.minimum(np.maximum(dx, dy), 0.0) + _len2(np.maximum(dx, 0.0), np.maximum(dy, 0.0))


def sd_cone(q, r, hh):
    """``sdCone`` (``30-wgsl-sim.js:51-59``)."""
    qx = _len2(q[:, 0], q[:, 2])
    qy = q[:, 1]
    k2x, k2y = -r, 2.0 * hh
    cax = qx - np.minimum(qx, np.where(qy < 0.0, r, 0.0))
    cay = np.abs(qy) - hh
    t = np.clip(((0.0 - qx) * k2x + (hh - qy) * k2y) / (k2x * k2x + k2y * k2y), 0.0, 1.0)
    cbx = qx - 0.0 + k2x * t
    cby = qy - hh + k2y * t
    s = np.where((cbx < 0.0) & (cay < 0.0), -1.0, 1.0)
    return s * np.sqrt(np.minimum(cax * cax + cay * cay, cbx * cbx + cby * cby))


def shape_sdf(o, p):
    """``shapeSdf`` (``30-wgsl-sim.js:60-77``)."""
    q = to_local(o, p)
    d = o['dims']
    t = o['type']
    if t == 0:
        return sd_round_box(q, d[0], d[1], d[2], d[3])
    if t == 1:
        return _len3(q[:, 0], q[:, 1], q[:, 2]) - d[0]
    if t == 2:
        return sd_cyl(q, d[0], d[1])
    if t == 3:
        return sd_cone(q, d[0], d[1])
    if t == 4:
        return _len2(_len2(q[:, 0], q[:, 2]) - d[0], q[:, 1]) - d[1]
    if t == 5:
        q2 = q.copy()
        q2[:, 1] = q[:, 1] - d[2]
        return np.maximum(sd_cyl(q, d[0], d[1]), -sd_cyl(q2, d[0] - d[2], d[1]))
    if t == 6:
        q2 = q.copy()
        q2[:, 1] = q[:, 1] - d[3]
        return np.maximum(sd_round_box(q, d[0], d[1], d[2], 0.002),
                          -sd_round_box(q2, d[0] - d[3], d[1], d[2] - d[3], 0.001))
    if t == 7:
        a = np.abs(_len2(q[:, 1], q[:, 2]) - d[1]) - 0.5 * d[2]
        return np.maximum(np.maximum(a, q[:, 1]), np.abs(q[:, 0]) - d[0])
    return np.full(len(p), BIG)


def scene_sdf(objs, p, cull=False):
    """Minimum over obstacles (flag 1) of the shape distance (``sceneSdf`` ``30-wgsl-sim.js:78-87``).

    cull=True is the WGSL loop exactly: an object whose bounding sphere is farther than the running
    minimum is skipped (``:83``). For most shapes that never changes the result, but the gutter's distance
    can be smaller than the distance to its bounding sphere, so the web version's value differs from the
    true minimum there. cull=False is the true minimum (what a mesh distance lattice holds)."""
    best = np.full(len(p), BIG)
    for o in objs:
        if o['flag'] != 1:
            continue
        d = shape_sdf(o, p)
        if cull:
            c = _len3(p[:, 0] - o['pos'][0], p[:, 1] - o['pos'][1], p[:, 2] - o['pos'][2]) - o['bound']
            d = np.where(c > best, best, d)
        best = np.minimum(best, d)
    return best


def in_drain_analytic(objs, p):
    """``inDrain`` (``30-wgsl-sim.js:107-114``): inside any drain cylinder."""
    out = np.zeros(len(p), bool)
    for o in objs:
        if o['flag'] != 2:
            continue
        out |= sd_cyl(to_local(o, p), o['dims'][0], o['dims'][1]) < 0.0
    return out


def lattice(objs, origin, h, shape, cull=False):
    """Obstacle distances on the half-cell lattice origin + h/2·index (``solver.py:103-110``).

    shape = (2nx+1, 2nyl+1, 2nz+1). Returns float64 of that shape (BIG where no obstacle). cull: the web
    version's culled minimum (see scene_sdf)."""
    hh = h / 2
    axes = [origin[a] + hh * np.arange(shape[a]) for a in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing='ij')
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    return scene_sdf(objs, pts, cull).reshape(shape)


def drains_for_solver(objs):
    """Drains in the reference solver's form (Rt, c, r, half height) (``solver.py:50-52``, ``:167-174``)."""
    out = []
    for o in objs:
        if o['flag'] == 2:
            out.append((o['rot'].T.copy(), o['pos'].copy(), float(o['dims'][0]), float(o['dims'][1])))
    return out
