"""One tank of the FLIP/PIC liquid: the reference CPU solver's sub-step, restated in NumPy.

Test infrastructure only (see ``oracle/__init__.py``).

Follows ``blender_addon/suiri_lab/solver.py`` (the reference's NumPy port of its WGSL kernels):
float64 everywhere except the red-black SOR, which runs in float32 in the same operation order as
``solver.py:473-509`` (so pressures can be compared bit for bit). Grid arrays are indexed [i, j, k]
with shapes (nx+1, ny+1, nz+1) for faces ("nodes") and (nx, ny, nz) for cells, y up, origin at the
minimum corner (``solver.py:58-100``).

Differences from ``solver.py`` that the test harness needs, none of which changes the arithmetic:
  * particles carry an integer id (``pid``) so that sets can be compared after re-ordering;
  * the grid can be given explicitly (nx, ny, nz, h) instead of derived from a quality preset;
  * obstacles are either the reference's lattice (``Solids.sdf``, trilinear, ``solver.py:116-140``)
    or the web version's analytic shapes (``30-wgsl-sim.js:78-106``) — ``sdf_mode``;
  * the ripple grid may be rectangular (Rx, Rz); Rx = Rz is the reference's square layer;
  * spawning randomness is either the reference's PCG64 stream (``rng_mode='numpy'``, consumed in
    the reference's order) or the GPU path's integer hash (``rng_mode='hash'``).
"""
import math
import numpy as np

from . import sdf as sdfm
from . import hashrng

RHO = 998.0
SIGMA_RHO = 0.0728 / 998.0
OFF = (np.array([0.0, 0.5, 0.5]), np.array([0.5, 0.0, 0.5]), np.array([0.5, 0.5, 0.0]))   # solver.py:234


class Tank:
    def __init__(self, nx, ny, nz, h, *, origin=None, extra_height=0.0, flip=0.96, omega=1.6, iters=40,
                 g=9.81, ppc=8.0, drift=6.0, friction=0.03, ww_rate=7.0, whitewater=True, ww_cap=140000,
                 ripple=(128, 128), wmap=256, seed=1, rng_mode='numpy', sdf_mode='lattice', advect='euler',
                 drop_d=None):
        self.nx, self.ny, self.nz, self.h = int(nx), int(ny), int(nz), float(h)
        h = self.h
        self.origin = np.array([-self.nx * h / 2, 0.0, -self.nz * h / 2]) if origin is None else np.array(origin, float)
        self.rim = self.ny * h                                              # solver.py:68
        self.nyl = self.ny + max(0, int(math.ceil(extra_height / h)))      # solver.py:70
        self.ns = (self.nx + 1, self.ny + 1, self.nz + 1)
        self.FLIP, self.OMEGA, self.iters, self.G = flip, omega, iters, g
        self.PPC, self.DRIFT, self.FRICTION, self.WW_RATE = ppc, drift, friction, ww_rate
        self.whitewater, self.ww_cap = whitewater, ww_cap
        self.vp = (h / 2) ** 3
        self.radius = 0.5 * h * 1.05
        self.rng = np.random.default_rng(seed)
        self.rng_mode, self.sdf_mode = rng_mode, sdf_mode
        if advect not in ('euler', 'rk2'):
            raise ValueError('advect is euler or rk2')
        self.advect = advect
        # (median, sigma_log): sub-grid drops get their own lognormal diameters (hashrng.drop_diameter);
        # None: every drop has the particle mass, as the reference
        self.drop_d = drop_d
        self.time, self.frame, self.vmax, self.impacts = 0.0, 0, 1.0, 0
        self.pos = np.zeros((0, 3)); self.vel = np.zeros((0, 3)); self.air = np.zeros(0)
        self.pid = np.zeros(0, np.int64)
        self.wpos = np.zeros((0, 3)); self.wvel = np.zeros((0, 3)); self.wlife = np.zeros(0); self.wkind = np.zeros(0)
        self.velg = np.zeros((3,) + self.ns); self.velold = np.zeros((3,) + self.ns)
        self.mask = np.zeros((3,) + self.ns, bool)
        self.count = np.zeros((self.nx, self.ny, self.nz), np.int64)
        self.pres = np.zeros((self.nx, self.ny, self.nz))
        self.div = np.zeros((self.nx, self.ny, self.nz))
        self.objs = []
        self.lat = None          # obstacle lattice (2nx+1, 2nyl+1, 2nz+1) or None
        self.oid = None
        self.Rx, self.Rz = ripple
        self.rsrc = np.zeros((self.Rz + 1, self.Rx + 1))
        self.wmap = wmap
        self.geom()

    # ------------------------------------------------------------------ particles in / out
    def add_particles(self, pos, vel=None, air=None, pid=None):
        pos = np.asarray(pos, np.float64).reshape(-1, 3)
        n = len(pos)
        vel = np.zeros((n, 3)) if vel is None else np.asarray(vel, np.float64).reshape(-1, 3)
        air = np.zeros(n) if air is None else np.asarray(air, np.float64).reshape(-1)
        start = int(self.pid.max()) + 1 if len(self.pid) else 0
        pid = np.arange(start, start + n) if pid is None else np.asarray(pid, np.int64)
        self.pos = np.concatenate([self.pos, pos]); self.vel = np.concatenate([self.vel, vel])
        self.air = np.concatenate([self.air, air]); self.pid = np.concatenate([self.pid, pid])

    # ------------------------------------------------------------------ obstacles
    def lattice_shape(self):
        return (2 * self.nx + 1, 2 * self.nyl + 1, 2 * self.nz + 1)      # solver.py:103-104

    def set_objects(self, objs, lattice=None):
        """Obstacles and drains. In lattice mode the lattice is the analytic SDF sampled at the
        half-cell points (what the Blender host computes from meshes, ``bake.py:83-119``) unless given."""
        self.objs = list(objs)
        obst = [o for o in self.objs if o['flag'] == 1]
        if obst:
            # analytic mode: the face fractions sample the web version's culled sceneSdf (30-wgsl-sim.js:127-129)
            self.lat = (sdfm.lattice(obst, self.origin, self.h, self.lattice_shape(), cull=self.sdf_mode == 'analytic')
                        if lattice is None else lattice)
            # nearest obstacle per lattice point, for solid velocities (solver.py:153-165)
            hh = self.h / 2
            s = self.lattice_shape()
            axes = [self.origin[a] + hh * np.arange(s[a]) for a in range(3)]
            X, Y, Z = np.meshgrid(*axes, indexing='ij')
            pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
            ds = np.stack([sdfm.shape_sdf(o, pts) for o in obst], 0)
            self.oid = np.argmin(ds, 0).reshape(s)
        else:
            self.lat = None
            self.oid = None
        self.geom()

    def _obstacles(self):
        return [o for o in self.objs if o['flag'] == 1]

    def sdf_at(self, p):
        """Distance to the nearest obstacle (``solver.py:116-140``; analytic: ``30-wgsl-sim.js:78-87``)."""
        n = len(p)
        obst = self._obstacles()
        if not obst or n == 0:
            return np.full(n, 1e9)
        if self.sdf_mode == 'analytic':
            return sdfm.scene_sdf(obst, p, cull=True)
        lat = self.lat
        g = (p - self.origin) / (self.h / 2)
        s = np.array(lat.shape)
        inside = np.all((g >= 0) & (g <= s - 1), axis=1)
        out = np.full(n, 1e9)
        if not inside.any():
            return out
        gi = g[inside]
        b = np.minimum(np.floor(gi).astype(np.int64), s - 2)
        f = gi - b
        acc = np.zeros(len(gi))
        for dx in (0, 1):
            wx = f[:, 0] if dx else 1 - f[:, 0]
            for dy in (0, 1):
                wy = f[:, 1] if dy else 1 - f[:, 1]
                for dz in (0, 1):
                    wz = f[:, 2] if dz else 1 - f[:, 2]
                    acc += wx * wy * wz * lat[b[:, 0] + dx, b[:, 1] + dy, b[:, 2] + dz]
        out[inside] = acc
        return out

    def sdf_normal(self, p):
        """Central differences with e = 6e-4 (``solver.py:142-151``, ``30-wgsl-sim.js:88-95``)."""
        e = 0.0006
        ex, ey, ez = np.array([e, 0, 0]), np.array([0, e, 0]), np.array([0, 0, e])
        n = np.stack([self.sdf_at(p + ex) - self.sdf_at(p - ex),
                      self.sdf_at(p + ey) - self.sdf_at(p - ey),
                      self.sdf_at(p + ez) - self.sdf_at(p - ez)], axis=1)
        ln = np.linalg.norm(n, axis=1)
        ok = ln > 1e-9
        out = np.tile([0.0, 1.0, 0.0], (len(p), 1))
        out[ok] = n[ok] / ln[ok, None]
        return out

    def solid_vel(self, p):
        """Velocity of the nearest obstacle (``solver.py:153-165``; analytic ``30-wgsl-sim.js:96-106``)."""
        v = np.zeros((len(p), 3))
        obst = self._obstacles()
        if not obst or len(p) == 0:
            return v
        if self.sdf_mode == 'analytic':
            # solidVelAt (30-wgsl-sim.js:96-106): culled like sceneSdf, the first strict minimum wins
            best = np.full(len(p), 1e9)
            ids = np.full(len(p), -1)
            for k, o in enumerate(obst):
                c = np.linalg.norm(p - o['pos'], axis=1) - o['bound']
                d = sdfm.shape_sdf(o, p)
                take = ~(c > best) & (d < best)
                best = np.where(take, d, best)
                ids = np.where(take, k, ids)
        else:
            g = np.rint((p - self.origin) / (self.h / 2)).astype(np.int64)
            g = np.clip(g, 0, np.array(self.oid.shape) - 1)
            ids = self.oid[g[:, 0], g[:, 1], g[:, 2]]
        for k, o in enumerate(obst):
            m = ids == k
            if m.any():
                v[m] = o['lin'] + np.cross(o['ang'], p[m] - o['pos'])
        return v

    def in_drain(self, p):
        """``solver.py:167-174`` / ``30-wgsl-sim.js:107-114``."""
        out = np.zeros(len(p), bool)
        for o in self.objs:
            if o['flag'] != 2:
                continue
            q = (p - o['pos']) @ o['rot']          # = (Rᵀ (p - c)) row-wise
            out |= (np.sqrt(q[:, 0] ** 2 + q[:, 2] ** 2) < o['dims'][0]) & (np.abs(q[:, 1]) < o['dims'][1])
        return out

    def geom(self):
        """Open fraction of every face and the solid velocity there (``solver.py:176-207``,
        ``30-wgsl-sim.js:118-157``): the 4 face corners and twice the face centre, all on the lattice."""
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        self.frac = np.zeros((3,) + self.ns)
        self.svel = np.zeros((3,) + self.ns)
        obst = self._obstacles()

        def open_frac(s0, s1, s2, s3, sc):
            pos = np.maximum(s0, 0) + np.maximum(s1, 0) + np.maximum(s2, 0) + np.maximum(s3, 0) + 2 * np.maximum(sc, 0)
            tot = np.abs(s0) + np.abs(s1) + np.abs(s2) + np.abs(s3) + 2 * np.abs(sc)
            return np.where(tot < 1e-12, 1.0, np.clip(pos / np.maximum(tot, 1e-30), 0, 1))

        if obst:
            L = self.lat[:, :2 * ny + 1, :]
            ev = lambda a, b: slice(a, b, 2)
            # x faces at (i, j+1/2, k+1/2), 0 < i < nx
            I = ev(2, 2 * nx - 1)
            self.frac[0, 1:nx, :ny, :nz] = open_frac(L[I, ev(0, 2 * ny - 1), ev(0, 2 * nz - 1)],
                                                     L[I, ev(2, 2 * ny + 1), ev(0, 2 * nz - 1)],
                                                     L[I, ev(2, 2 * ny + 1), ev(2, 2 * nz + 1)],
                                                     L[I, ev(0, 2 * ny - 1), ev(2, 2 * nz + 1)],
                                                     L[I, ev(1, 2 * ny), ev(1, 2 * nz)])
            J = ev(2, 2 * ny - 1)
            self.frac[1, :nx, 1:ny, :nz] = open_frac(L[ev(0, 2 * nx - 1), J, ev(0, 2 * nz - 1)],
                                                     L[ev(2, 2 * nx + 1), J, ev(0, 2 * nz - 1)],
                                                     L[ev(2, 2 * nx + 1), J, ev(2, 2 * nz + 1)],
                                                     L[ev(0, 2 * nx - 1), J, ev(2, 2 * nz + 1)],
                                                     L[ev(1, 2 * nx), J, ev(1, 2 * nz)])
            K = ev(2, 2 * nz - 1)
            self.frac[2, :nx, :ny, 1:nz] = open_frac(L[ev(0, 2 * nx - 1), ev(0, 2 * ny - 1), K],
                                                     L[ev(2, 2 * nx + 1), ev(0, 2 * ny - 1), K],
                                                     L[ev(2, 2 * nx + 1), ev(2, 2 * ny + 1), K],
                                                     L[ev(0, 2 * nx - 1), ev(2, 2 * ny + 1), K],
                                                     L[ev(1, 2 * nx), ev(1, 2 * ny), K])
        else:
            self.frac[0, 1:nx, :ny, :nz] = 1
            self.frac[1, :nx, 1:ny, :nz] = 1
            self.frac[2, :nx, :ny, 1:nz] = 1
        self.frac[1, :nx, ny, :nz] = 1.0                                   # open air above the grid
        if obst and any(np.any(o['lin']) or np.any(o['ang']) for o in obst):
            for a, sl in ((0, (slice(1, nx), slice(0, ny), slice(0, nz))), (1, (slice(0, nx), slice(1, ny), slice(0, nz))),
                          (2, (slice(0, nx), slice(0, ny), slice(1, nz)))):
                ii, jj, kk = np.meshgrid(np.arange(self.ns[0])[sl[0]], np.arange(self.ns[1])[sl[1]],
                                         np.arange(self.ns[2])[sl[2]], indexing='ij')
                off = np.full(3, 0.5); off[a] = 0.0
                p = self.origin + h * (np.stack([ii, jj, kk], -1).reshape(-1, 3) + off)
                self.svel[a][sl] = self.solid_vel(p)[:, a].reshape(ii.shape)

    # ------------------------------------------------------------------ lattice helpers
    def grid_pos(self, x):
        return (x - self.origin) / self.h

    def in_grid(self, g):
        return np.all((g >= 0) & (g < [self.nx, self.ny, self.nz]), axis=1)

    def corners(self, q):
        """8 nodes around q: flat node index, existence, trilinear weight (``solver.py:216-232``)."""
        b = np.floor(q).astype(np.int64)
        f = q - b
        s0, s1, s2 = self.ns
        bx, by, bz = b[:, 0], b[:, 1], b[:, 2]
        vx = ((bx >= 0) & (bx < s0), (bx >= -1) & (bx < s0 - 1))
        vy = ((by >= 0) & (by < s1), (by >= -1) & (by < s1 - 1))
        vz = ((bz >= 0) & (bz < s2), (bz >= -1) & (bz < s2 - 1))
        wx = (1 - f[:, 0], f[:, 0]); wy = (1 - f[:, 1], f[:, 1]); wz = (1 - f[:, 2], f[:, 2])
        base = (bx * s1 + by) * s2 + bz
        for dx in (0, 1):
            for dy in (0, 1):
                vxy = vx[dx] & vy[dy]
                wxy = wx[dx] * wy[dy]
                for dz in (0, 1):
                    yield base + ((dx * s1 + dy) * s2 + dz), vxy & vz[dz], wxy * wz[dz]

    def transfer(self, g, comp, vp):
        """PIC and FLIP velocity from faces that took weight this step (``solver.py:236-249``,
        ``31-wgsl-sim2.js:9-36``)."""
        q = g - OFF[comp]
        sn = np.zeros(len(g)); so = np.zeros(len(g)); sw = np.zeros(len(g))
        vn = self.velg[comp].ravel(); vo = self.velold[comp].ravel(); mk = self.mask[comp].ravel()
        for idx, ok, w in self.corners(q):
            idx = np.where(ok, idx, 0)
            use = ok & mk[idx]
            ww = np.where(use, w, 0.0)
            sn += ww * vn[idx]; so += ww * vo[idx]; sw += ww
        good = sw >= 1e-6
        pic = np.where(good, sn / np.maximum(sw, 1e-30), vp)
        flip = np.where(good, vp + (sn - so) / np.maximum(sw, 1e-30), vp)
        return pic, flip

    def sample(self, g, comp):
        """Clamped trilinear sample of the new velocity (``solver.py:251-266``, ``31-wgsl-sim2.js:39-56``)."""
        q = g - OFF[comp]
        b = np.floor(q).astype(np.int64)
        f = q - b
        vn = self.velg[comp]
        s = np.zeros(len(g))
        hi = np.array(self.ns) - 1
        for dx in (0, 1):
            wx = f[:, 0] if dx else 1 - f[:, 0]
            for dy in (0, 1):
                wy = f[:, 1] if dy else 1 - f[:, 1]
                for dz in (0, 1):
                    wz = f[:, 2] if dz else 1 - f[:, 2]
                    c = np.clip(b + (dx, dy, dz), 0, hi)
                    s += wx * wy * wz * vn[c[:, 0], c[:, 1], c[:, 2]]
        return s

    def count_at(self, c):
        """Particles in cells c; above and outside the grid: 0 (``solver.py:268-274``)."""
        ok = np.all(c >= 0, axis=1) & (c[:, 0] < self.nx) & (c[:, 1] < self.ny) & (c[:, 2] < self.nz)
        out = np.zeros(len(c), np.int64)
        cc = c[ok]
        out[ok] = self.count[cc[:, 0], cc[:, 1], cc[:, 2]]
        return out

    def air_at(self, c):
        """``solver.py:276-279`` / ``31-wgsl-sim2.js:97-101``."""
        above = c[:, 1] >= self.ny
        outside = np.any(c < 0, axis=1) | (c[:, 0] >= self.nx) | (c[:, 2] >= self.nz)
        return above | (~outside & (self.count_at(c) == 0))

    # ------------------------------------------------------------------ tank walls
    def footprint(self):
        lo = self.origin[[0, 2]]
        return lo, lo + np.array([self.nx, self.nz]) * self.h

    def in_footprint(self, x):
        lo, hi = self.footprint()
        return (x[:, 0] > lo[0]) & (x[:, 0] < hi[0]) & (x[:, 2] > lo[1]) & (x[:, 2] < hi[1])

    def tank_clamp(self, x0, x, v, r):
        """Glass walls below the rim, the floor, and re-entry from outside (``solver.py:290-301``,
        ``31-wgsl-sim2.js:66-80``)."""
        lo, hi = self.footprint()
        was = self.in_footprint(x0)
        m = was & (x[:, 1] < self.rim)
        for a, (l, u) in ((0, (lo[0], hi[0])), (2, (lo[1], hi[1]))):
            low = m & (x[:, a] < l + r); x[low, a] = l + r; v[low, a] = np.maximum(v[low, a], 0)
            high = m & (x[:, a] > u - r); x[high, a] = u - r; v[high, a] = np.minimum(v[high, a], 0)
        fl = was & (x[:, 1] < self.origin[1] + r)
        x[fl, 1] = self.origin[1] + r; v[fl, 1] = np.maximum(v[fl, 1], 0)
        back = ~was & (x[:, 1] < self.rim) & self.in_footprint(x)
        x[back, 0] = x0[back, 0]; x[back, 2] = x0[back, 2]
        v[back, 0] *= -0.2; v[back, 2] *= -0.2

    # ------------------------------------------------------------------ the sub-step, phase by phase
    def count_cells(self):
        """Cell binning (``solver.py:430-436``): count per cell of particles inside the grid."""
        g = self.grid_pos(self.pos)
        ing = self.in_grid(g)
        c = g[ing].astype(np.int64)
        flat = (c[:, 0] * self.ny + c[:, 1]) * self.nz + c[:, 2]
        self.count = np.bincount(flat, minlength=self.nx * self.ny * self.nz).reshape(self.nx, self.ny, self.nz)
        return g, ing

    def p2g(self, g, ing):
        """Trilinear splat at the staggered offsets, velocity clamped to ±30 (``solver.py:443-460``)."""
        size = int(np.prod(self.ns))
        vclamp = np.clip(self.vel, -30, 30)
        gi = g[ing]
        self.mom = np.zeros((3, size)); self.wt = np.zeros((3, size))
        for comp in range(3):
            q = gi - OFF[comp]
            mom = np.zeros(size); wt = np.zeros(size)
            vals = vclamp[ing, comp]
            for idx, ok, w in self.corners(q):
                use = ok & (w > 0)
                idx = idx[use]
                mom += np.bincount(idx, w[use] * vals[use], size)
                wt += np.bincount(idx, w[use], size)
            self.mom[comp], self.wt[comp] = mom, wt
            m = wt > 4e-6
            v = np.where(m, mom / np.maximum(wt, 1e-30), 0.0).reshape(self.ns)
            self.velg[comp] = v
            self.velold[comp] = v
            self.mask[comp] = m.reshape(self.ns)

    def forces_and_divergence(self, dt):
        """Gravity, solid faces, cut-cell divergence with drift correction (``solver.py:461-472``)."""
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        fluid = self.count > 0
        self.velg[1] -= self.G * dt
        for a in range(3):
            solid = self.frac[a] <= 0
            self.velg[a][solid] = self.svel[a][solid]
        F = [self.frac[a] * self.velg[a] + (1 - self.frac[a]) * self.svel[a] for a in range(3)]
        div = (F[0][1:nx + 1, :ny, :nz] - F[0][:nx, :ny, :nz] + F[1][:nx, 1:ny + 1, :nz] - F[1][:nx, :ny, :nz]
               + F[2][:nx, :ny, 1:nz + 1] - F[2][:nx, :ny, :nz]) / h
        div -= self.DRIFT * np.maximum(self.count / self.PPC - 1, 0)
        div[~fluid] = 0
        self.div = div
        return fluid

    def sor_operands(self, div, fluid):
        """Float32 operands of the SOR exactly as ``solver.py:478-491`` forms them, on the whole grid:
        C (6 coefficients per cell: x-, x+, y-, y+, z-, z+), inv, rhs and the per-colour relaxation U."""
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        f32 = np.float32
        fx, fy, fz = (self.frac[a].astype(f32) for a in range(3))
        C = [np.ascontiguousarray(a) for a in (fx[0:nx, :ny, :nz], fx[1:nx + 1, :ny, :nz],
                                               fy[:nx, 0:ny, :nz], fy[:nx, 1:ny + 1, :nz],
                                               fz[:nx, :ny, 0:nz], fz[:nx, :ny, 1:nz + 1])]
        den = C[0] + C[1] + C[2] + C[3] + C[4] + C[5]
        inv = np.where(den > 0, 1.0 / np.maximum(den, 1e-30), 0.0).astype(f32)
        ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing='ij', sparse=True)
        color = (ii + jj + kk) & 1
        U = [(fluid & (den > 0) & (color == c)).astype(f32) * f32(self.OMEGA) for c in (0, 1)]
        rhs = (h * h * div).astype(f32)
        return C, inv, U, rhs

    def sor(self, fluid, p_init=None, iters=None):
        """Red-black SOR in float32, parity 0 first, in the operation order of ``solver.py:494-505``.

        Non-liquid cells hold zero pressure, the outside of the grid reads as zero (its wall faces have
        coefficient 0, the open top has coefficient 1: Dirichlet p = 0). Equivalent to the reference's
        bounding-box form, whose extra margin only ever touches non-liquid cells."""
        C, inv, U, rhs = self.sor_operands(self.div, fluid)
        p0 = np.where(fluid, self.pres, 0.0) if p_init is None else p_init
        p = sor_f32(C, inv, U, rhs, p0, self.iters if iters is None else iters)
        p[~fluid] = 0
        self.pres = p
        return p

    def project(self, fluid):
        """Subtract the pressure gradient on faces touching liquid; closed faces take the solid
        velocity (``solver.py:510-523``, ``30-wgsl-sim.js:299-341``)."""
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        p = self.pres
        pp = np.zeros((nx + 2, ny + 2, nz + 2)); pp[1:-1, 1:-1, 1:-1] = p
        ff = np.zeros((nx + 2, ny + 2, nz + 2), bool); ff[1:-1, 1:-1, 1:-1] = fluid
        for a in range(3):
            sl = [slice(0, nx), slice(0, ny), slice(0, nz)]
            sl[a] = slice(0, self.ns[a])
            hi_ = [slice(1, nx + 1), slice(1, ny + 1), slice(1, nz + 1)]; lo_ = list(hi_)
            hi_[a] = slice(1, self.ns[a] + 1); lo_[a] = slice(0, self.ns[a])
            grad = (pp[tuple(hi_)] - pp[tuple(lo_)]) / h
            touch = ff[tuple(hi_)] | ff[tuple(lo_)]
            fa = self.frac[a][tuple(sl)]
            va = self.velg[a][tuple(sl)]
            sa = self.svel[a][tuple(sl)]
            va[:] = np.where(fa <= 0, sa, np.where(touch, va - grad, va))

    def substep(self, dt):
        """One sub-step without emission (``solver.py:438-525``)."""
        g, ing = self.count_cells()
        self.p2g(g, ing)
        fluid = self.forces_and_divergence(dt)
        self.sor(fluid)
        self.project(fluid)
        self.g2p(dt)
        self.time += dt

    # ------------------------------------------------------------------ grid -> particles
    def g2p(self, dt):
        """FLIP/PIC blend, explicit Euler advection, obstacle collision with friction, tank walls,
        drains, sub-grid drops and whitewater spawning (``solver.py:527-630``, ``31-wgsl-sim2.js:149-251``).

        ``advect='rk2'`` is not in the reference: in-grid particles move by the midpoint rule through the
        interpolated grid velocity u (the PIC transfer, which falls back to the particle's blended velocity
        where no face took weight): u0 = u(x0), xm = x0 + u0·(dt/2), x = x0 + u(xm)·dt, with u(xm) falling
        back to u0; a particle whose midpoint leaves the grid, and every particle outside it, moves by
        explicit Euler with its blended velocity. The stored velocity is the blended one either way."""
        h = self.h
        N = len(self.pos)
        self.spawned = 0
        if N == 0:
            return
        x0 = self.pos
        v = self.vel.copy()
        g = self.grid_pos(x0)
        ing = self.in_grid(g)
        u0 = None
        if ing.any():
            gi = g[ing]; vi = v[ing]
            new = np.empty_like(vi)
            u0 = np.empty_like(vi)
            for comp in range(3):
                pic, flip = self.transfer(gi, comp, vi[:, comp])
                new[:, comp] = pic + self.FLIP * (flip - pic)
                u0[:, comp] = pic
            v[ing] = new
        v[~ing, 1] -= self.G * dt
        x = x0 + v * dt
        if self.advect == 'rk2' and u0 is not None:
            xm = x0[ing] + u0 * (0.5 * dt)
            gm = self.grid_pos(xm)
            ok = self.in_grid(gm)
            u1 = u0.copy()
            for comp in range(3):
                pic, _ = self.transfer(gm[ok], comp, u0[ok, comp])
                u1[ok, comp] = pic
            xi = x[ing]
            xi[ok] = x0[ing][ok] + u1[ok] * dt
            x[ing] = xi
        rc = 0.32 * h
        d = self.sdf_at(x)
        hit = d < rc
        if hit.any():
            xs = x[hit]
            nrm = self.sdf_normal(xs)
            xs += nrm * (rc - d[hit])[:, None]
            vs = self.solid_vel(xs)
            rel = v[hit] - vs
            vn = np.sum(rel * nrm, axis=1)
            neg = vn < 0
            vh = v[hit]
            vh[neg] = vs[neg] + (rel[neg] - nrm[neg] * vn[neg, None]) * (1 - self.FRICTION)
            v[hit] = vh
            x[hit] = xs
        self.tank_clamp(x0, x, v, rc)
        alive = ~self.in_drain(x)
        alive &= ~(~self.in_footprint(x) & (x[:, 1] < 0.002))
        alive &= ~(np.any(np.abs(x[:, [0, 2]]) > 20, axis=1) | (x[:, 1] < -1) | (x[:, 1] > 30))
        # sub-grid drops: free-flying mark (solver.py:565-583)
        c0 = np.floor(g).astype(np.int64)
        air = self.air.copy()
        if ing.any():
            idx = np.nonzero(ing)[0]
            cc = c0[idx]
            n0 = self.count_at(cc)
            air[idx[n0 >= 4]] = 0.0
            cand = (n0 <= 2) & (cc[:, 1] + 2 < self.ny)
            if cand.any():
                ci = cc[cand]
                around = np.zeros(len(ci), np.int64); above = np.zeros(len(ci), np.int64)
                for dz in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        for dy in (-1, 0, 1):
                            around += self.count_at(ci + (dx, dy, dz))
                        above += self.count_at(ci + (dx, 1, dz)) + self.count_at(ci + (dx, 2, dz))
                sel = idx[cand][(around <= 4) & (above == 0)]
                air[sel] = 1.0
        # merging with the pool: ripple impulse and crown splash (solver.py:584-606)
        g1 = self.grid_pos(x)
        c1 = np.floor(g1).astype(np.int64)
        cand = (air > 0.5) & (self.vel[:, 1] < -0.3) & self.in_grid(g1)
        self.merged = np.zeros(0, np.int64)
        if cand.any():
            ids = np.nonzero(cand)[0]
            others = self.count_at(c1[ids]) - np.all(c1[ids] == c0[ids], axis=1)
            ids = ids[others >= 3]
            if len(ids):
                gl = g1[ids]
                vl = np.stack([self.transfer(gl, a, v[ids, a])[0] for a in range(3)], 1)
                dv = vl[:, 1] - self.vel[ids, 1]
                ok = dv > 0.3
                ids, vl, dv = ids[ok], vl[ok], dv[ok]
                if len(ids):
                    v[ids] = vl
                    air[ids] = 0.0
                    self.impacts += len(ids)
                    self.merged = self.pid[ids].copy()
                    m = np.full(len(ids), RHO * (0.5 * h) ** 3)
                    if self.drop_d is not None:
                        D = hashrng.drop_diameter(self.pid[ids], *self.drop_d)
                        m = RHO * (math.pi / 6.0) * D * D * D
                    self.ripple_deposit(x[ids], 2.0 * m * np.minimum(dv, 8.0), 2e-3)
                    cnt = self.count_at(c1[ids])
                    level = self.origin[1] + (c1[ids, 1] + np.minimum(cnt / self.PPC, 1.0)) * h
                    for k in range(len(ids)):
                        self.crown(np.array([x[ids[k], 0], level[k] + 0.25 * h, x[ids[k], 2]]), -self.vel[ids[k], 1],
                                   float(m[k]), int(self.pid[ids[k]]))
        if ing.any():
            sp = np.linalg.norm(v[ing], axis=1)
            self.vmax = float(min(sp.max(), 60.0)) if len(sp) else 0.0
        if self.whitewater and ing.any():
            self.spawn_whitewater(x, v, c0, ing, dt)
        self.pos = x[alive]; self.vel = v[alive]; self.air = air[alive]; self.pid = self.pid[alive]

    def spawn_whitewater(self, x, v, c0, ing, dt):
        """Fast particles next to air spawn spray with probability rate·e²·dt (``solver.py:610-629``,
        ``31-wgsl-sim2.js:233-249``)."""
        h = self.h
        idx = np.nonzero(ing)[0]
        sp = np.linalg.norm(v[idx], axis=1)
        fast = sp > 0.75
        if not fast.any():
            return
        fi = idx[fast]
        cc = c0[fi]
        near = np.zeros(len(fi), bool)
        for a in range(3):
            for sgn in (-1, 1):
                o = np.zeros(3, np.int64); o[a] = sgn
                near |= self.air_at(cc + o)
        fi = fi[near]
        e = np.clip((np.linalg.norm(v[fi], axis=1) - 0.75) / 1.6, 0, 1)
        if self.rng_mode == 'numpy':
            born = self.rng.random(len(fi)) < self.WW_RATE * e * e * dt
            fi = fi[born]
            if len(fi):
                j = self.rng.random((len(fi), 3)) - 0.5
                self.ww_add(x[fi] + j * h * 0.6, v[fi] * (0.8 + 0.35 * self.rng.random(len(fi)))[:, None] + j * 0.35,
                            1.0 + 2.5 * self.rng.random(len(fi)), np.zeros(len(fi)))
                self.spawned = len(fi)
        else:
            st = hashrng.Stream(hashrng.seed_ww(self.pid[fi], self.frame))
            born = st.rnd() < self.WW_RATE * e * e * dt
            j = np.stack([st.rnd(), st.rnd(), st.rnd()], 1) - 0.5
            life = 1.0 + 2.5 * st.rnd()
            f = 0.8 + 0.35 * st.rnd()
            fi, j, life, f = fi[born], j[born], life[born], f[born]
            self.spawned_ids = self.pid[fi].copy()
            if len(fi):
                self.ww_add(x[fi] + j * h * 0.6, v[fi] * f[:, None] + j * 0.35, life, np.zeros(len(fi)))
            self.spawned = len(fi)

    def crown(self, x, U, m, pid):
        """Crown splash above K = We·Oh^-0.4 (``solver.py:632-657``, ``31-wgsl-sim2.js:119-148``)."""
        if not self.whitewater:
            return
        D = (6 * m / (math.pi * RHO)) ** (1 / 3)
        We = RHO * U * U * D / 0.0728
        Oh = 0.001 / math.sqrt(RHO * 0.0728 * D)
        K = We * Oh ** -0.4
        n = int(min(max(round(4 * (K / 2100 - 1)), 0), 24))
        nj = (2 if K > 2100 else 1) if K > 700 else 0
        if n + nj == 0:
            return
        if self.rng_mode == 'numpy':
            rnd = self.rng.random
        else:
            st = hashrng.Stream(hashrng.seed_crown(pid, self.frame))
            rnd = lambda: float(st.rnd())
        P, V, L = [], [], []
        r0 = 0.6 * D
        ph0 = rnd() * 2 * math.pi
        for i in range(n):
            ph = ph0 + 2 * math.pi * (i + 0.3 * rnd()) / n
            el = 0.9 + 0.45 * rnd()
            sp = U * (0.15 + 0.2 * rnd())
            d = np.array([math.cos(ph), 0.0, math.sin(ph)])
            P.append(x + d * r0); V.append(d * math.cos(el) * sp + np.array([0, math.sin(el) * sp, 0])); L.append(0.5 + 0.4 * rnd())
        for j in range(nj):
            sp = U * (0.22 + 0.04 * j) * (0.9 + 0.2 * rnd())
            P.append(x + np.array([0, 0.001 * j, 0])); V.append(np.array([(rnd() - 0.5) * 0.05, sp, (rnd() - 0.5) * 0.05])); L.append(0.7)
        self.ww_add(np.array(P), np.array(V), np.array(L), np.zeros(len(P)))

    def ww_add(self, p, v, life, kind):
        room = self.ww_cap - len(self.wpos)
        if room <= 0:
            return
        p, v, life, kind = p[:room], v[:room], life[:room], kind[:room]
        self.wpos = np.concatenate([self.wpos, p]); self.wvel = np.concatenate([self.wvel, v])
        self.wlife = np.concatenate([self.wlife, life]); self.wkind = np.concatenate([self.wkind, kind])

    def ripple_deposit(self, x, impulse, cap):
        """Nearest ripple vertex gets the clamped impulse (``solver.py:667-672``, ``31-wgsl-sim2.js:110-114``)."""
        lo, hi = self.footprint()
        uv = (x[:, [0, 2]] - lo) / (hi - lo)
        i = np.clip(np.rint(uv[:, 0] * self.Rx), 0, self.Rx).astype(np.int64)
        j = np.clip(np.rint(uv[:, 1] * self.Rz), 0, self.Rz).astype(np.int64)
        np.add.at(self.rsrc, (j, i), np.clip(impulse, 0, cap))

    # ------------------------------------------------------------------ whitewater (once per frame)
    def advance_whitewater(self, dt):
        """Spray falls, foam rides the surface, bubbles rise (``solver.py:675-713``, ``31-wgsl-sim2.js:361-409``)."""
        if len(self.wpos) == 0:
            return
        x = self.wpos; v = self.wvel.copy(); life = self.wlife.copy()
        g = self.grid_pos(x)
        ing = self.in_grid(g)
        kind = np.zeros(len(x))
        if ing.any():
            idx = np.nonzero(ing)[0]
            c = g[idx].astype(np.int64)
            n = self.count[c[:, 0], c[:, 1], c[:, 2]]
            up = self.count_at(c + (0, 1, 0))
            k = np.where(n > 0, np.where(up > 0, 2.0, np.where(g[idx, 1] - c[:, 1] < np.minimum(n / self.PPC, 1.0), 1.0, 0.0)), 0.0)
            kind[idx] = k
        land = (self.wkind < 0.5) & (kind > 0.5) & (self.wvel[:, 1] < -0.3)
        if land.any():
            self.ripple_deposit(x[land], 4.2e-6 * -self.wvel[land, 1], 1e-4)
        spray = kind == 0
        v[spray, 1] -= self.G * dt
        v[spray] *= 1.0 / (1.0 + 0.6 * dt)
        life[spray] -= dt * 0.7
        wet = ~spray
        if wet.any():
            gw = g[wet]
            vf = np.stack([self.sample(gw, a) for a in range(3)], 1)
            foam = kind[wet] == 1
            vw = np.where(foam[:, None], vf * [1, 0.2, 1], vf + [0, 0.16, 0])
            v[wet] = vw
            life[wet] -= dt * np.where(foam, 0.5, 0.3)
        x0 = x
        x = x0 + v * dt
        d = self.sdf_at(x)
        inside = d < 0
        if inside.any():
            x[inside] -= self.sdf_normal(x[inside]) * d[inside][:, None]
        self.tank_clamp(x0, x, v, 0.001)
        outside = ~self.in_footprint(x) & (x[:, 1] < 0.001)
        keep = (life > 0) & ~outside & (x[:, 1] > -0.5) & ~self.in_drain(x)
        self.wpos, self.wvel, self.wlife, self.wkind = x[keep], v[keep], life[keep], kind[keep]

    # ------------------------------------------------------------------ one frame
    def substeps_for(self, frame_dt):
        """CFL sub-step count (``solver.py:717-719``, ``50-sim.js:302-305``)."""
        vmax = max(self.vmax, 0.4)
        return int(min(max(math.ceil(frame_dt / (1.4 * self.h / vmax)), 1), 6))

    def step(self, frame_dt, ripple_layer=None, ripple_depth=0.0):
        """A frame: CFL sub-steps, then whitewater, top height and ripples (``solver.py:716-728``). A
        ripple_depth > 0 fixes the dispersion depth (the build's extension for a stated depth); otherwise it is
        the mean liquid depth, as the reference."""
        n = self.substeps_for(frame_dt)
        dt = frame_dt / n
        for _ in range(n):
            self.frame += 1
            self.substep(dt)
        self.frame_end(frame_dt, ripple_layer, ripple_depth)
        return n

    def frame_end(self, frame_dt, ripple_layer=None, ripple_depth=0.0):
        """The frame's tail after its sub-steps: counts, whitewater, top height, ripples (``solver.py:720-728``)."""
        self.count_cells()
        self.advance_whitewater(frame_dt)
        if ripple_layer is not None:
            from . import ripple as rp
            self.top = rp.top_height(self)
            mean_depth = min(max(len(self.pos) * self.vp / (self.nx * self.nz * self.h * self.h), 0.003), self.rim)
            ripple_layer.frame(frame_dt, ripple_depth if ripple_depth > 0 else mean_depth, self.rsrc, rp.ripple_mask(self))
            self.rsrc[:] = 0

    @property
    def liters(self):
        return len(self.pos) * self.vp * 1000

    def kinetic_energy(self):
        """Σ ½ m |v|² over liquid particles, m = ρ·(h/2)³."""
        return 0.5 * RHO * self.vp * float(np.sum(self.vel * self.vel))

    def max_divergence(self):
        """Post-projection max |div| over liquid cells (faces as the projection left them)."""
        nx, ny, nz, h = self.nx, self.ny, self.nz, self.h
        F = [self.frac[a] * self.velg[a] + (1 - self.frac[a]) * self.svel[a] for a in range(3)]
        div = (F[0][1:nx + 1, :ny, :nz] - F[0][:nx, :ny, :nz] + F[1][:nx, 1:ny + 1, :nz] - F[1][:nx, :ny, :nz]
               + F[2][:nx, :ny, 1:nz + 1] - F[2][:nx, :ny, :nz]) / h
        fl = self.count > 0
        return float(np.abs(div[fl]).max()) if fl.any() else 0.0


def sor_f32(C, inv, U, rhs, p_init, iters):
    """The float32 red-black loop of ``solver.py:489-506`` on the whole grid: C the 6 coefficient arrays
    (x-, x+, y-, y+, z-, z+), inv = 1/ΣC, U = (ω on active cells of colour 0, of colour 1), rhs = h²·div."""
    f32 = np.float32
    nx, ny, nz = rhs.shape
    P = np.zeros((nx + 2, ny + 2, nz + 2), f32)
    Pi = P[1:-1, 1:-1, 1:-1]
    Pi[...] = p_init
    nbr = (P[:-2, 1:-1, 1:-1], P[2:, 1:-1, 1:-1], P[1:-1, :-2, 1:-1], P[1:-1, 2:, 1:-1], P[1:-1, 1:-1, :-2], P[1:-1, 1:-1, 2:])
    num = np.empty((nx, ny, nz), f32); tmp = np.empty((nx, ny, nz), f32)
    for _ in range(iters):
        for Uc in U:
            np.multiply(C[0], nbr[0], out=num)
            for d in range(1, 6):
                np.multiply(C[d], nbr[d], out=tmp)
                num += tmp
            num -= rhs
            num *= inv
            num -= Pi
            num *= Uc
            Pi += num
    return Pi.astype(np.float64)


def sor_operands_from(frac32, rhs32, fluid, omega):
    """SOR operands from float32 face fractions (3, nx+1, ny+1, nz+1) and a float32 right-hand side, formed
    as ``solver.py:478-487`` does."""
    f32 = np.float32
    nx, ny, nz = rhs32.shape
    fx, fy, fz = (np.asarray(frac32[a], f32) for a in range(3))
    C = [np.ascontiguousarray(a) for a in (fx[0:nx, :ny, :nz], fx[1:nx + 1, :ny, :nz], fy[:nx, 0:ny, :nz],
                                           fy[:nx, 1:ny + 1, :nz], fz[:nx, :ny, 0:nz], fz[:nx, :ny, 1:nz + 1])]
    den = C[0] + C[1] + C[2] + C[3] + C[4] + C[5]
    inv = np.where(den > 0, 1.0 / np.maximum(den, 1e-30), 0.0).astype(f32)
    ii, jj, kk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing='ij', sparse=True)
    color = (ii + jj + kk) & 1
    U = [(fluid & (den > 0) & (color == c)).astype(f32) * f32(omega) for c in (0, 1)]
    return C, inv, U, np.asarray(rhs32, f32)


def residual_f64(C, rhs, fluid, p):
    """FP64 residual max |h²·div − A p| over active cells, A the cut-cell Laplacian of the SOR:
    (Σ C_d p_nb − rhs) − den·p, evaluated in float64 from the float32 operands."""
    nx, ny, nz = p.shape
    P = np.zeros((nx + 2, ny + 2, nz + 2)); P[1:-1, 1:-1, 1:-1] = np.where(fluid, p, 0.0)
    nbr = (P[:-2, 1:-1, 1:-1], P[2:, 1:-1, 1:-1], P[1:-1, :-2, 1:-1], P[1:-1, 2:, 1:-1], P[1:-1, 1:-1, :-2], P[1:-1, 1:-1, 2:])
    Cd = [c.astype(np.float64) for c in C]
    den = sum(Cd)
    r = sum(c * n for c, n in zip(Cd, nbr)) - rhs.astype(np.float64) - den * P[1:-1, 1:-1, 1:-1]
    act = fluid & (den > 0)
    return float(np.abs(r[act]).max()) if act.any() else 0.0
