"""Liquid surface mesh of the per-frame export: distance field of the particle spheres on a half-cell lattice,
smoothed, meshed with surface nets; lone particles as small icospheres; pool vertices settled onto the top-view
height map; the liquid's velocity at every vertex.

Test infrastructure only (see ``oracle/__init__.py``).

Follows ``blender_addon/suiri_lab/meshing.py``: ``surface`` (``:52-111``), ``_surface_nets`` (``:114-174``),
``settle_on_top`` (``:177-199``), the icosphere (``:26-49``), the separable blur (``:8-23``), and the vertex
velocity of ``bake.py:231-235`` (``Solver._sample``, ``solver.py:251-266``). The float32 arrays of the reference
are kept float32 with their rounding points made explicit: the distance field is float32, each blur tap is
added in float64 and rounded back to float32, the crossing parameter fa / (fa - fb) is a float32 division.

``weights`` (the normalised blur kernel) may be given: the reference forms it with NumPy's ``exp``, whose
vectorised form may differ from the C library's in the last bit, so a comparison with another implementation
passes the weights that implementation used.
"""
import math
import numpy as np


def blur_weights(sigma):
    """Normalised Gaussian taps, radius max(1, ceil(2.5σ)) (``meshing.py:9-11``)."""
    r = max(1, int(math.ceil(2.5 * sigma)))
    k = np.exp(-0.5 * (np.arange(-r, r + 1) / sigma) ** 2)
    return k / k.sum()


def smooth3(f, w):
    """Separable blur along x, y, z of a float32 lattice, edge values held (``meshing.py:8-23``)."""
    r = len(w) // 2
    f = np.asarray(f, np.float32)
    for ax in range(3):
        n = f.shape[ax]
        idx = np.arange(n)
        acc = np.zeros_like(f)
        for t, wt in enumerate(w):
            src = np.take(f, np.clip(idx + t - r, 0, n - 1), axis=ax)
            acc = (acc.astype(np.float64) + np.float64(wt) * src.astype(np.float64)).astype(np.float32)
        f = acc
    return f


def icosphere():
    """Unit icosahedron subdivided once (42 vertices, 80 faces), vertices numbered as created: the 12 corners,
    then each edge midpoint the first time a face asks for it, faces visited in order, each split into its three
    corner triangles and the middle one (``meshing.py:26-49``)."""
    p = (1 + math.sqrt(5)) / 2
    base = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
                     [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], float)
    base /= np.linalg.norm(base, axis=1)[:, None]
    faces20 = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
               (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
               (8, 6, 7), (9, 8, 1)]
    verts = list(base)
    cache = {}

    def midpoint(a, b):
        key = (a, b) if a < b else (b, a)
        if key not in cache:
            m = verts[a] + verts[b]
            cache[key] = len(verts)
            verts.append(m / np.linalg.norm(m))
        return cache[key]

    tris = []
    for a, b, c in faces20:
        ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
        tris.extend([(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)])
    return np.array(verts), np.array(tris, np.int64)


ICO_V, ICO_F = icosphere()


def lone_mask(t):
    """Particles drawn as their own spheres: those with at most 6 particles in the 3×3×3 cells around theirs
    (counted at the frame end, outside the grid none) (``meshing.py:60-73``)."""
    g = (t.pos - t.origin) / t.h
    c = np.floor(g).astype(np.int64)
    ing = np.all((g >= 0) & (g < [t.nx, t.ny, t.nz]), axis=1)
    P = np.pad(t.count, 1)
    nx, ny, nz = t.count.shape
    box = sum(P[1 + dx:1 + dx + nx, 1 + dy:1 + dy + ny, 1 + dz:1 + dz + nz]
              for dx in (-1, 0, 1) for dy in (-1, 0, 1) for dz in (-1, 0, 1))
    near = np.zeros(len(t.pos), np.int64)
    ci = c[ing]
    near[ing] = box[ci[:, 0], ci[:, 1], ci[:, 2]]
    return near <= 6


def body_field(body, h, r):
    """Distance to the union of spheres of radius r on a lattice of spacing h/2 around the body particles, far
    value 2·spacing, clipped to [-r, far] (``meshing.py:76-93``). Returns (lo, phi float32 [x][y][z])."""
    sp = h / 2
    pad = r + 4 * sp
    lo = body.min(0) - pad
    hi = body.max(0) + pad
    n = np.ceil((hi - lo) / sp).astype(np.int64) + 1
    far = 2 * sp
    phi = np.full(int(n.prod()), far, np.float32)
    q = (body - lo) / sp
    base = np.floor(q).astype(np.int64)
    for ox in (-1, 0, 1, 2):
        for oy in (-1, 0, 1, 2):
            for oz in (-1, 0, 1, 2):
                node = base + (ox, oy, oz)
                e = (node - q) * sp
                d = np.sqrt(e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1] + e[:, 2] * e[:, 2]) - r
                ok = np.all((node >= 0) & (node < n), axis=1) & (d < far)
                flat = (node[ok, 0] * n[1] + node[ok, 1]) * n[2] + node[ok, 2]
                np.minimum.at(phi, flat, d[ok].astype(np.float32))
    phi = np.clip(phi.reshape(n), np.float32(-r), np.float32(far))
    return lo, phi


_CORNERS = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
_EDGES = [(p, q) for p in _CORNERS for q in _CORNERS if sum(abs(u - v) for u, v in zip(p, q)) == 1 and p < q]


def surface_nets(phi):
    """Surface nets on lattice values phi (inside < 0): a vertex in every cell whose 8 corners are neither all
    inside nor all outside, at the mean of the crossings on its sign-changing edges; a quad around every
    sign-changing lattice edge whose four cells all exist, turned to face outwards. Vertices numbered in cell
    order (x slowest), quads by edge axis x, y, z, each in edge order (``meshing.py:114-174``).
    Returns vertices in lattice units and quads (Q, 4)."""
    X, Y, Z = phi.shape
    inside = phi < 0
    n_in = np.zeros((X - 1, Y - 1, Z - 1), np.int8)
    for a, b, c in _CORNERS:
        n_in += inside[a:X - 1 + a, b:Y - 1 + b, c:Z - 1 + c]
    mixed = (n_in > 0) & (n_in < 8)
    cells = np.argwhere(mixed)
    if len(cells) == 0:
        return np.zeros((0, 3)), np.zeros((0, 4), np.int64)
    vid = np.full(mixed.shape, -1, np.int64)
    vid[mixed] = np.arange(len(cells))
    acc = np.zeros((len(cells), 3))
    cnt = np.zeros(len(cells))
    for pa, pb in _EDGES:
        fa = phi[cells[:, 0] + pa[0], cells[:, 1] + pa[1], cells[:, 2] + pa[2]]
        fb = phi[cells[:, 0] + pb[0], cells[:, 1] + pb[1], cells[:, 2] + pb[2]]
        cross = (fa < 0) != (fb < 0)
        den = np.where(cross, fa - fb, np.float32(1))
        tpar = np.where(cross, fa / den, np.float32(0)).astype(np.float64)
        ax = [u != v for u, v in zip(pa, pb)].index(True)
        pt = np.tile(np.array(pa, float), (len(cells), 1))
        pt[:, ax] += tpar
        acc[cross] += pt[cross]
        cnt[cross] += 1
    verts = cells + acc / np.maximum(cnt, 1)[:, None]
    out = []
    for ax in range(3):
        a1, a2 = [a for a in range(3) if a != ax]
        lo_in = np.take(inside, np.arange(phi.shape[ax] - 1), axis=ax)
        hi_in = np.take(inside, np.arange(1, phi.shape[ax]), axis=ax)
        crossing = lo_in != hi_in
        for a in (a1, a2):       # the four cells need 1 <= index <= shape - 2 on both other axes
            sl = [slice(None)] * 3
            sl[a] = 0
            crossing[tuple(sl)] = False
            sl[a] = phi.shape[a] - 1
            crossing[tuple(sl)] = False
        e = np.argwhere(crossing)
        if len(e) == 0:
            continue

        def around(o1, o2):
            c = e.copy()
            c[:, a1] -= o1
            c[:, a2] -= o2
            return vid[c[:, 0], c[:, 1], c[:, 2]]

        q = np.stack([around(1, 1), around(0, 1), around(0, 0), around(1, 0)], 1)
        outward = lo_in[e[:, 0], e[:, 1], e[:, 2]]
        rev = outward if ax == 1 else ~outward
        q[rev] = q[rev][:, ::-1]
        out.append(q)
    quads = np.concatenate(out) if out else np.zeros((0, 4), np.int64)
    return verts, quads[np.all(quads >= 0, axis=1)]


def surface(t, smooth=0.8, weights=None):
    """(verts (V, 3), quads (Q, 4), tris (T, 3)) of the liquid of oracle tank `t` (``meshing.py:52-111``): the
    body's surface-nets mesh, its vertices held inside the glass and above the floor where they lie in the tank,
    then 42 vertices and 80 triangles per lone particle, in particle order."""
    pos, h = t.pos, t.h
    r = t.radius                       # 0.5·h·1.05 (solver.py:74)
    if len(pos) == 0:
        return np.zeros((0, 3)), np.zeros((0, 4), np.int64), np.zeros((0, 3), np.int64)
    lone = lone_mask(t)
    body = pos[~lone]
    verts = np.zeros((0, 3))
    quads = np.zeros((0, 4), np.int64)
    if len(body):
        sp = h / 2
        lo, phi = body_field(body, h, r)
        phi = smooth3(phi, blur_weights(smooth) if weights is None else np.asarray(weights, float))
        v, quads = surface_nets(phi)
        verts = lo + v * sp
        x0, z0 = t.origin[0], t.origin[2]
        x1, z1 = x0 + t.nx * h, z0 + t.nz * h
        m = 0.0005
        held = ((verts[:, 0] > x0 - sp) & (verts[:, 0] < x1 + sp) & (verts[:, 2] > z0 - sp) & (verts[:, 2] < z1 + sp)
                & (verts[:, 1] < t.rim))
        verts[held, 0] = np.clip(verts[held, 0], x0 + m, x1 - m)
        verts[held, 2] = np.clip(verts[held, 2], z0 + m, z1 - m)
        verts[held, 1] = np.maximum(verts[held, 1], m)
    drops = pos[lone]
    tris = np.zeros((0, 3), np.int64)
    if len(drops):
        first = len(verts) + np.arange(len(drops)) * len(ICO_V)
        tris = (ICO_F[None] + first[:, None, None]).reshape(-1, 3)
        verts = np.concatenate([verts, (drops[:, None, :] + ICO_V[None] * r).reshape(-1, 3)])
    return verts, quads, tris


def settle_on_top(t, verts, top=None):
    """Vertices within 0.6h of the wet top-view height map (bilinear at texel centres, all four taps wet) take
    its height, in place (``meshing.py:177-199``)."""
    H = t.top if top is None else top
    W = H.shape[0]
    if len(verts) == 0:
        return
    lo = t.origin[[0, 2]]
    size = np.array([t.nx, t.nz]) * t.h
    u = (verts[:, [0, 2]] - lo) / size * W - 0.5
    sel = np.nonzero(np.all((u >= 0) & (u <= W - 1), axis=1))[0]
    if len(sel) == 0:
        return
    us = u[sel]
    b = np.minimum(np.floor(us).astype(np.int64), W - 2)
    f = us - b
    h00, h10 = H[b[:, 1], b[:, 0]], H[b[:, 1], b[:, 0] + 1]
    h01, h11 = H[b[:, 1] + 1, b[:, 0]], H[b[:, 1] + 1, b[:, 0] + 1]
    wet = (h00 >= 0) & (h10 >= 0) & (h01 >= 0) & (h11 >= 0)
    level = (h00 * (1 - f[:, 0]) + h10 * f[:, 0]) * (1 - f[:, 1]) + (h01 * (1 - f[:, 0]) + h11 * f[:, 0]) * f[:, 1]
    y = verts[sel, 1]
    take = wet & (y > level - 0.6 * t.h) & (y < level + 0.6 * t.h)
    verts[sel[take], 1] = level[take]


def vertex_velocity(t, verts, velg=None):
    """The liquid's velocity at each vertex: trilinear in each face-velocity component with clamped taps, zero
    outside the grid (``bake.py:231-235``, ``Solver._sample`` ``solver.py:251-266``)."""
    out = np.zeros((len(verts), 3))
    if len(verts) == 0:
        return out
    V = t.velg if velg is None else velg
    g = (verts - t.origin) / t.h
    for comp in range(3):
        off = np.full(3, 0.5)
        off[comp] = 0.0
        q = g - off
        b = np.floor(q).astype(np.int64)
        f = q - b
        F = V[comp]
        hi = np.array(F.shape) - 1
        s = np.zeros(len(g))
        for dx in (0, 1):
            wx = f[:, 0] if dx else 1 - f[:, 0]
            for dy in (0, 1):
                wy = f[:, 1] if dy else 1 - f[:, 1]
                for dz in (0, 1):
                    wz = f[:, 2] if dz else 1 - f[:, 2]
                    c = np.clip(b + (dx, dy, dz), 0, hi)
                    s += wx * wy * wz * F[c[:, 0], c[:, 1], c[:, 2]]
        out[:, comp] = s
    ing = np.all((g >= 0) & (g < [t.nx, t.ny, t.nz]), axis=1)
    out[~ing] = 0.0
    return out
