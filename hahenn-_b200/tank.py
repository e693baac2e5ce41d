"""Python host API over libsuiri_cuda.so, mirroring the reference's two front-ends for the liquid step:

* the web version's ``FluidSim`` (``src/js/50-sim.js:28-376``): construction from a scene, ``set_objects``,
  ``step(frame_dt)``, ``clear_water``, ``save_water``/``restore_water``, ``stats``, ``water_liters``;
* the Blender add-on's ``Solver`` (``blender_addon/suiri_lab/solver.py:58-794``): ``emit_block``, ``step``,
  ``set_solids`` (a distance lattice), and ``pos``/``vel``/``air`` arrays, ``liters``.

Every call goes through the C ABI; all state lives on the GPU.
"""
import ctypes as C
import json

import numpy as np

from . import native as N


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Tank:
    """One tank on the GPU (the plain drop-in path)."""

    def __init__(self, scene=None, *, nx=0, ny=0, nz=0, h=0.0, quality='standard', clamp_tank=True,
                 extra_height=0.0, flip=0.96, omega=1.6, iters=0, gravity=9.81, friction=0.03, ppc=8.0, drift=6.0,
                 ww_rate=7.0, whitewater=True, capacity=0, ww_capacity=0, ripple=(0, 0), wmap=0, sdf_mode='analytic',
                 device=0, seed=1, ripple_sigma=0.0728, ripple_rho=998.0, ripple_depth=0.0, advect='euler',
                 drop_d=None, sor_mode=0, watchdog_polls=None):
        L = N.lib()
        p = N.Params()
        N.check(L.suiri_params_default(C.byref(p)))
        p.nx, p.ny, p.nz, p.h = int(nx), int(ny), int(nz), float(h)
        self._quality = quality.encode()
        p.quality = self._quality
        p.clamp_tank = 1 if clamp_tank else 0
        p.extra_height = float(extra_height)
        p.flip, p.omega, p.iters, p.gravity, p.friction = float(flip), float(omega), int(iters), float(gravity), float(friction)
        p.ppc, p.drift, p.ww_rate, p.whitewater = float(ppc), float(drift), float(ww_rate), 1 if whitewater else 0
        p.capacity, p.ww_capacity = int(capacity), int(ww_capacity)
        if ripple is None:
            p.ripple_rx = p.ripple_rz = -1
        else:
            p.ripple_rx, p.ripple_rz = int(ripple[0]), int(ripple[1])
        p.wmap = int(wmap)
        p.sdf_mode = {'analytic': 0, 'lattice': 1}[sdf_mode]
        p.device, p.seed = int(device), int(seed)
        p.ripple_sigma, p.ripple_rho, p.ripple_depth = float(ripple_sigma), float(ripple_rho), float(ripple_depth)
        p.advect = {'euler': 0, 'rk2': 1}[advect]
        if drop_d is not None:          # (median [m], sigma_log): lognormal sub-grid drop diameters
            p.drop_d_median, p.drop_d_sigma_log = float(drop_d[0]), float(drop_d[1])
        p.sor_mode = int(sor_mode)
        if watchdog_polls is not None:
            p.watchdog_polls = int(watchdog_polls)
        if scene is not None and not isinstance(scene, (str, bytes)):
            scene = json.dumps(scene)
        h_ = C.c_void_p()
        N.check(L.suiri_create(scene.encode() if isinstance(scene, str) else scene, C.byref(p), C.byref(h_)))
        self._h = h_
        st = self.stats()
        self.nx, self.ny, self.nz, self.h = st['nx'], st['ny'], st['nz'], st['h']
        self.origin = np.array(st['origin'])
        self.ns = (self.nx + 1, self.ny + 1, self.nz + 1)

    # ------------------------------------------------------------------ lifecycle
    def close(self):
        if getattr(self, '_h', None):
            N.lib().suiri_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        return N.check(rc, self._h)

    @property
    def handle(self):
        return self._h

    # ------------------------------------------------------------------ scene
    def set_objects(self, items, dt_move=0.0):
        """setObjects (``50-sim.js:165-211``): obstacles and drains from scene items; returns 'moving'."""
        mv = C.c_int32()
        self._c(N.lib().suiri_set_objects(self._h, json.dumps(items).encode(), float(dt_move), C.byref(mv)))
        return bool(mv.value)

    def set_obstacles(self, objs):
        """Binary obstacle records: dicts with type, flag, pos, rot (3x3), dims (4), lin, ang."""
        arr = (N.Object * max(1, len(objs)))()
        for i, o in enumerate(objs):
            r = arr[i]
            r.type, r.flag = int(o['type']), int(o['flag'])
            r.pos[:] = [float(v) for v in o['pos']]
            r.rot[:] = [float(v) for v in np.asarray(o['rot'], float).ravel()]
            r.dims[:] = [float(v) for v in o['dims']]
            r.lin[:] = [float(v) for v in o.get('lin', (0, 0, 0))]
            r.ang[:] = [float(v) for v in o.get('ang', (0, 0, 0))]
        self._c(N.lib().suiri_set_obstacles(self._h, arr, len(objs)))

    def set_lattice(self, sdf, oid=None):
        """Solids lattice [i, j, k] (``solver.py:47-56``) — switches to lattice mode."""
        sdf = np.asarray(sdf, np.float64)
        lx, ly, lz = sdf.shape
        s = np.ascontiguousarray(sdf.transpose(2, 1, 0))
        o = None if oid is None else np.ascontiguousarray(np.asarray(oid, np.int32).transpose(2, 1, 0))
        self._c(N.lib().suiri_set_lattice(self._h, _ptr(s), _ptr(o), lx, ly, lz))

    def eval_sdf(self, pts):
        """Distance to the nearest obstacle at points (N,3), as the step sees it (analytic or lattice)."""
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        out = np.empty(len(p))
        self._c(N.lib().suiri_eval_sdf(self._h, _ptr(p), len(p), _ptr(out)))
        return out

    # ------------------------------------------------------------------ water
    def add_particles(self, pos, vel=None, air=None):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32).reshape(-1, 3)
        air = None if air is None else np.ascontiguousarray(air, np.float32).reshape(-1)
        first = C.c_uint32()
        self._c(N.lib().suiri_add_particles(self._h, _ptr(pos), _ptr(vel), _ptr(air), len(pos), C.byref(first)))
        return first.value

    def set_emitters(self, emitters):
        """Fixed-rate device emitters: dicts with shape ('disc' | 'rain'), pos, dir, radius, speed,
        count (particles per sub-step) and airborne."""
        arr = (N.Emitter * max(1, len(emitters)))()
        for i, e in enumerate(emitters):
            r = arr[i]
            r.shape = {'disc': 0, 'rain': 3}[e.get('shape', 'disc')]
            r.airborne = 1 if e.get('airborne', False) else 0
            r.pos[:] = [float(v) for v in e['pos']]
            r.dir[:] = [float(v) for v in e.get('dir', (0.0, -1.0, 0.0))]
            r.radius, r.speed, r.per_substep = float(e['radius']), float(e['speed']), float(e['count'])
            r.radius_z = float(e.get('radius_z', 0.0))
        self._c(N.lib().suiri_set_emitters(self._h, arr, len(emitters)))

    def emit_block(self, lo, hi, fill=False):
        lo_ = (C.c_double * 3)(*[float(v) for v in lo])
        hi_ = (C.c_double * 3)(*[float(v) for v in hi])
        self._c(N.lib().suiri_emit_block(self._h, lo_, hi_, 1 if fill else 0))

    def reset(self):
        self._c(N.lib().suiri_reset(self._h))

    def clear_water(self):
        self._c(N.lib().suiri_clear(self._h))

    def save_water(self):
        i = C.c_int32()
        self._c(N.lib().suiri_snapshot(self._h, C.byref(i)))
        return i.value

    def save_state(self):
        """The tank's state in its one water-copy slot (for rolling back, e.g. after tuning)."""
        return self.save_water()

    def restore_state(self, copy_id):
        if not self.restore_water(copy_id):
            raise RuntimeError('the saved state was already restored or replaced')

    def restore_water(self, copy_id):
        try:
            self._c(N.lib().suiri_restore(self._h, int(copy_id)))
            return True
        except N.SuiriError as e:
            if e.code == -6:
                return False
            raise

    # ------------------------------------------------------------------ time stepping
    def substep(self, dt):
        self._c(N.lib().suiri_substep(self._h, float(dt)))

    def step(self, frame_dt):
        n = C.c_int32()
        self._c(N.lib().suiri_step(self._h, float(frame_dt), C.byref(n)))
        return n.value

    def frame_end(self, frame_dt):
        """The end of a frame after sub-steps taken with `substep` (counts, whitewater, top height, ripples)."""
        self._c(N.lib().suiri_frame_end(self._h, float(frame_dt)))

    def sync(self):
        self._c(N.lib().suiri_sync(self._h))

    def use_graphs(self, on=True):
        self._c(N.lib().suiri_use_graphs(self._h, 1 if on else 0))

    def time_substeps(self, dt, steps):
        ms = C.c_double()
        self._c(N.lib().suiri_time_substeps(self._h, float(dt), int(steps), C.byref(ms)))
        return ms.value

    def time_sor(self, iters):
        ms = C.c_double()
        self._c(N.lib().suiri_time_sor(self._h, int(iters), C.byref(ms)))
        return ms.value

    def stream(self):
        s = C.c_void_p()
        self._c(N.lib().suiri_stream(self._h, C.byref(s)))
        return s.value

    def profile(self, on=True):
        self._c(N.lib().suiri_profile(self._h, 1 if on else 0))

    def tune(self, blocks_per_sm=4, sor_mode=0):
        """sor_mode: 0 one launch per colour sweep, 1 one cooperative launch, 2/3 temporal blocking (2/4 sweeps),
        4 the whole solve held in one thread-block cluster's shared memory."""
        self._c(N.lib().suiri_tune(self._h, int(blocks_per_sm), int(sor_mode)))

    def tune_piece(self, piece_kb=0):
        """Shared memory per CTA of the cluster-resident solve, KiB (0: the device maximum)."""
        self._c(N.lib().suiri_tune_piece(self._h, int(piece_kb)))

    def tune_g2p(self, form=0):
        """Grid-to-particle pass: 0 grid-stride walk, 1 per brick with its faces in shared memory."""
        self._c(N.lib().suiri_tune_g2p(self._h, int(form)))

    def residual(self, on=True):
        """Evaluate every solve's FP64 residual on the device (stats: residual_max, residual_rms, rhs_max)."""
        self._c(N.lib().suiri_residual(self._h, 1 if on else 0))

    def sor_phase_ms(self):
        ms = C.c_double()
        self._c(N.lib().suiri_sor_phase_ms(self._h, C.byref(ms)))
        return ms.value

    def phase_ms(self):
        """Device ms of each phase of the last sub-step (profiling on), keyed by native.PHASES."""
        ms = (C.c_double * len(N.PHASES))()
        self._c(N.lib().suiri_phase_ms(self._h, ms))
        return dict(zip(N.PHASES, list(ms)))

    # ------------------------------------------------------------------ read-back
    def particles4(self, out=None):
        """Liquid particles as the C ABI gives them: (pos4 (N,4) x, y, z, airborne; vel4 (N,4) vx, vy, vz, id
        bits). One read: the arrays are sized from the stats' upper bound (or `out`, a pair of (M,4) float32
        arrays to fill), then trimmed to the particles alive."""
        if out is None:
            m = self.stats()['count']
            out = (np.empty((m, 4), np.float32), np.empty((m, 4), np.float32))
        P, V = out
        n = C.c_int64()
        self._c(N.lib().suiri_read_particles(self._h, _ptr(P), _ptr(V), len(P), C.byref(n)))
        if n.value > len(P):               # more than the bound allows cannot happen; read again to be safe
            return self.particles4((np.empty((n.value, 4), np.float32), np.empty((n.value, 4), np.float32)))
        return P[:n.value], V[:n.value]

    def particles(self):
        """(pos (N,3), vel (N,3), air (N,), id (N,) uint32) of the liquid particles."""
        P, V = self.particles4()
        return P[:, :3].copy(), V[:, :3].copy(), P[:, 3].copy(), V[:, 3].copy().view(np.uint32)

    @property
    def pos(self):
        return self.particles()[0].astype(np.float64)

    @property
    def vel(self):
        return self.particles()[1].astype(np.float64)

    @property
    def air(self):
        return self.particles()[2].astype(np.float64)

    def whitewater(self):
        n = C.c_int64()
        self._c(N.lib().suiri_read_whitewater(self._h, None, None, 0, C.byref(n)))
        P = np.empty((n.value, 4), np.float32)
        V = np.empty((n.value, 4), np.float32)
        self._c(N.lib().suiri_read_whitewater(self._h, _ptr(P), _ptr(V), n.value, C.byref(n)))
        return P, V

    def add_whitewater(self, pos, vel, life, kind):
        """Append whitewater particles: pos, vel (N,3), life, kind (N,) (0 spray, 1 foam, 2 bubble)."""
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        P = np.empty((len(pos), 4), np.float32)
        V = np.empty((len(pos), 4), np.float32)
        P[:, :3], P[:, 3] = pos, np.asarray(life, np.float32).reshape(-1)
        V[:, :3], V[:, 3] = np.asarray(vel, np.float32).reshape(-1, 3), np.asarray(kind, np.float32).reshape(-1)
        self._c(N.lib().suiri_add_whitewater(self._h, _ptr(P), _ptr(V), len(P)))

    def grid(self, field):
        """A grid field as the oracle indexes it: faces (3, nx+1, ny+1, nz+1), cells (nx, ny, nz)."""
        nx, ny, nz = self.nx, self.ny, self.nz
        L = N.lib()
        if field in (N.FIELD_CELL_COUNT, N.FIELD_PRES, N.FIELD_RHS):
            out = np.empty((nz, ny, nx), np.int32 if field == N.FIELD_CELL_COUNT else np.float32)
            self._c(L.suiri_read_grid(self._h, field, _ptr(out), out.nbytes))
            return out.transpose(2, 1, 0)
        if field in (N.FIELD_FRAC, N.FIELD_VEL, N.FIELD_VELOLD, N.FIELD_MASK):
            out = np.empty((3, nz + 1, ny + 1, nx + 1), np.uint8 if field == N.FIELD_MASK else np.float32)
            self._c(L.suiri_read_grid(self._h, field, _ptr(out), out.nbytes))
            out = out.transpose(0, 3, 2, 1)
            return out.astype(bool) if field == N.FIELD_MASK else out
        raise ValueError('use ripple_field / top_height for ripple fields')

    def ripple_field(self, field, shape, dtype):
        out = np.empty(shape, dtype)
        self._c(N.lib().suiri_read_grid(self._h, field, _ptr(out), out.nbytes))
        return out

    def frame_maps(self, sun, out=None, read=True):
        """The maps the bake writes per frame (``bake.py:241-249``) from the last frame: float32 (W, W, 4) =
        top height (-1 dry), ripple slope d/dx, d/dz at texel centres, floor light (``Solver.caustics``,
        ``solver.py:796-846``) for the sun direction `sun`. `out` may be a reused (W, W, 4) float32 array."""
        s = np.ascontiguousarray(sun, np.float64)
        if s.shape != (3,):
            raise ValueError('sun is a 3-vector')
        if not read:                      # built on the device only (timing)
            self._c(N.lib().suiri_frame_maps(self._h, _ptr(s), None, 0))
            return None
        W = self.stats()['wmap']
        if out is None:
            out = np.empty((W, W, 4), np.float32)
        if out.dtype != np.float32 or out.shape != (W, W, 4) or not out.flags.c_contiguous:
            raise ValueError(f'out must be a C-contiguous float32 array of shape {(W, W, 4)}')
        self._c(N.lib().suiri_frame_maps(self._h, _ptr(s), _ptr(out), out.nbytes))
        return out

    def surface_mesh(self, smooth=0.8):
        """The liquid's surface mesh as the frame export writes it (``meshing.surface`` + ``settle_on_top`` +
        the vertex velocity, ``meshing.py:52-199``, ``bake.py:228-235``): dict of verts (V, 3) float32, vel
        (V, 3) float32, quads (Q, 4) int32, tris (T, 3) int32, and the build's info (lattice, blur weights)."""
        info = N.MeshInfo()
        self._c(N.lib().suiri_surface_mesh(self._h, float(smooth), C.byref(info)))
        V, Q, T = info.verts, info.quads, info.tris
        verts = np.empty((V, 3), np.float32); vel = np.empty((V, 3), np.float32)
        quads = np.empty((Q, 4), np.int32); tris = np.empty((T, 3), np.int32)
        self._c(N.lib().suiri_surface_mesh_read(self._h, _ptr(verts), _ptr(vel), _ptr(quads), _ptr(tris), V, Q, T))
        return dict(verts=verts, vel=vel, quads=quads, tris=tris, body_verts=info.body_verts, lone=info.lone,
                    lattice=tuple(info.lattice), lo=tuple(info.lo), spacing=info.spacing,
                    weights=np.array(info.weights[:info.taps]),
                    phase_ms=dict(zip(N.MESH_PHASES, info.phase_ms)))

    def caustics(self, sun):
        """Floor light relative to plain sunlight, (W, W) float32 (``Solver.caustics``)."""
        return self.frame_maps(sun)[..., 3].copy()

    @staticmethod
    def _stats_dict(s):
        return dict(count=s.count, ww_count=s.ww_count, impacts=s.impacts, vmax=s.vmax, time=s.time, liters=s.liters,
                    full=bool(s.full), frame=s.frame, errors=s.errors, nx=s.nx, ny=s.ny, nz=s.nz, h=s.h, origin=tuple(s.origin),
                    active_cells=s.active_cells, residual_max=s.residual_max, residual_rms=s.residual_rms,
                    rhs_max=s.rhs_max, ripple=(s.ripple_rx, s.ripple_rz), wmap=s.wmap)

    def stats(self):
        s = N.Stats()
        self._c(N.lib().suiri_get_stats(self._h, C.byref(s)))
        return self._stats_dict(s)

    def poll_stats(self):
        """Non-blocking (FluidSim.pollStats): the stats of the read the previous call started, or None if it
        has not finished; every call starts a new read behind the work enqueued so far."""
        s, fresh = N.Stats(), C.c_int32(0)
        self._c(N.lib().suiri_poll_stats(self._h, C.byref(s), C.byref(fresh)))
        return self._stats_dict(s) if fresh.value else None

    @property
    def water_liters(self):
        return self.stats()['liters']

    liters = water_liters


def balanced_lanes(cells, particles, k):
    """Lane per tank for `k` lanes of tanks contiguous in size (cells), each lane with about the same number of
    particles: small tanks stay together (their latency-bound sweeps do not wait for large tanks' kernels) and
    no lane holds most of the work. Tanks of the same size share a lane."""
    cells, particles = np.asarray(cells), np.asarray(particles, np.float64)
    order = np.argsort(cells, kind='stable')
    cum = np.cumsum(particles[order])
    tot = cum[-1] if len(cum) else 0.0
    lane = np.empty(len(cells), np.int32)
    for rank, i in enumerate(order):
        before = cum[rank] - particles[i]
        lane[i] = min(k - 1, int(k * (before + 0.5 * particles[i]) / max(tot, 1.0)))
    for rank in range(1, len(order)):
        a, b = order[rank - 1], order[rank]
        if cells[a] == cells[b]:
            lane[b] = lane[a]
    return lane


class Batch:
    """Many tanks stepped by shared launches (one descriptor table, one CUDA graph per sub-step)."""

    def __init__(self, tanks, lanes=None):
        """`lanes`: None for the size lanes (under 2^16 cells, under 2^19, larger), or a lane index 0..7 per
        tank (see `balanced_lanes`)."""
        self.tanks = list(tanks)
        arr = (C.c_void_p * len(self.tanks))(*[t.handle.value for t in self.tanks])
        h = C.c_void_p()
        if lanes is None:
            N.check(N.lib().suiri_batch_create(arr, len(self.tanks), C.byref(h)))
        else:
            lo = np.ascontiguousarray(lanes, np.int32)
            if lo.shape != (len(self.tanks),):
                raise ValueError('one lane per tank')
            N.check(N.lib().suiri_batch_create_lanes(arr, len(self.tanks), _ptr(lo), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, '_h', None):
            N.lib().suiri_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def substep(self, dt):
        N.check(N.lib().suiri_batch_substep(self._h, float(dt)))

    def save_state(self):
        """Every tank's state in its water-copy slot."""
        self.sync()
        return [t.save_water() for t in self.tanks]

    def restore_state(self, ids):
        self.sync()
        for t, i in zip(self.tanks, ids):
            t.restore_state(i)

    def sync(self):
        N.check(N.lib().suiri_batch_sync(self._h))

    def tune(self, blocks_per_sm=4, sor_mode=0):
        N.check(N.lib().suiri_batch_tune(self._h, int(blocks_per_sm), int(sor_mode)))

    def tune_piece(self, piece_kb=0):
        N.check(N.lib().suiri_batch_tune_piece(self._h, int(piece_kb)))

    def tune_g2p(self, form=0):
        N.check(N.lib().suiri_batch_tune_g2p(self._h, int(form)))

    def tune_lane(self, lane, blocks_per_sm=4, sor_mode=0, piece_kb=0, g2p_form=0):
        N.check(N.lib().suiri_batch_tune_lane(self._h, int(lane), int(blocks_per_sm), int(sor_mode), int(piece_kb),
                                              int(g2p_form)))

    def lane(self, k):
        """A tuning target for lane k alone (the autotuner's interface); timing covers the whole batch."""
        return _LaneTarget(self, k)

    def residual(self, on=True):
        N.check(N.lib().suiri_batch_residual(self._h, 1 if on else 0))

    def lanes(self):
        n = C.c_int32()
        N.check(N.lib().suiri_batch_lanes(self._h, C.byref(n)))
        return n.value

    def phase_ms(self, lane):
        ms = (C.c_double * len(N.PHASES))()
        N.check(N.lib().suiri_batch_phase_ms(self._h, int(lane), ms))
        return dict(zip(N.PHASES, list(ms)))

    def profile(self, on=True):
        N.check(N.lib().suiri_batch_profile(self._h, 1 if on else 0))

    def sor_phase_ms(self):
        ms = C.c_double()
        N.check(N.lib().suiri_batch_sor_phase_ms(self._h, C.byref(ms)))
        return ms.value

    def time_substeps(self, dt, steps):
        ms = C.c_double()
        N.check(N.lib().suiri_batch_time_substeps(self._h, float(dt), int(steps), C.byref(ms)))
        return ms.value

    def stream(self):
        s = C.c_void_p()
        N.check(N.lib().suiri_batch_stream(self._h, C.byref(s)))
        return s.value


class _LaneTarget:
    """One size lane of a batch as an autotuner target: its knobs are set through suiri_batch_tune_lane, the
    other lanes keep theirs; sub-steps and saved states are the whole batch's."""

    def __init__(self, batch, lane, knobs=(4, 0, 0, 0)):
        self.batch, self.k = batch, int(lane)
        self.knobs = list(knobs)

    def _apply(self):
        self.batch.tune_lane(self.k, *self.knobs)

    def tune(self, blocks_per_sm=4, sor_mode=0):
        self.knobs[0], self.knobs[1] = int(blocks_per_sm), int(sor_mode)
        self._apply()

    def tune_piece(self, piece_kb=0):
        self.knobs[2] = int(piece_kb)

    def tune_g2p(self, form=0):
        self.knobs[3] = int(form)
        self._apply()

    def time_substeps(self, dt, steps):
        return self.batch.time_substeps(dt, steps)
