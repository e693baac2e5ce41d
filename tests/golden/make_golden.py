"""Generate the golden fixtures by running the reference's own CPU solver.

Runs ``blender_addon/suiri_lab/solver.py`` from the read-only reference checkout (it imports only math and
numpy) on seeded inputs and stores inputs and outputs as small ``.npz`` files in this folder. The oracle
(``oracle/``) is pinned against these files by ``tests/test_oracle_golden.py``; the CUDA path is compared
with the oracle and, where shapes allow, with these files directly.

Usage, with REF the root of a checkout of the reference (given as the argument or in SUIRI_REFERENCE):
    python tests/golden/make_golden.py REF [scenario ...]

Obstacle lattices are the analytic shapes of ``oracle/sdf.py`` sampled at the solver's lattice points
(``solver.py:106-110``) — the role the Blender host's mesh distance queries play (``bake.py:83-119``).
"""
import importlib.util
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import sdf as sdfm            # noqa: E402


def load_solver(ref):
    path = os.path.join(ref, 'blender_addon', 'suiri_lab', 'solver.py')
    spec = importlib.util.spec_from_file_location('ref_solver_%d' % np.random.randint(1 << 30), path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


MESHING = None                          # the reference's meshing module (main loads it)


def load_meshing(ref):
    path = os.path.join(ref, 'blender_addon', 'suiri_lab', 'meshing.py')
    spec = importlib.util.spec_from_file_location('ref_meshing', path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make(S, nx, ny, nz, h, *, flip, omega, iters, g=9.81, whitewater=False, seed=1, ripple=16, wmap=32, ww=4000):
    S.FLIP, S.OMEGA, S.G = flip, omega, g
    S.QUALITY['GOLD'] = dict(h=h, cap=10_000_000, ww=ww, iters=iters, ripple=ripple, wmap=wmap)
    sv = S.Solver(nx * h, ny * h, nz * h, 'GOLD', whitewater=whitewater, seed=seed)
    assert (sv.nx, sv.ny, sv.nz) == (nx, ny, nz), (sv.nx, sv.ny, sv.nz)
    return sv


def jitter_cells(rng, cells, h, origin, ppc):
    u = rng.random((len(cells), ppc, 3))
    return (origin + (cells[:, None, :] + u) * h).reshape(-1, 3).astype(np.float32).astype(np.float64)


def cells_where(nx, ny, nz, pred):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing='ij')
    m = pred(i, j, k)
    return np.stack([i[m], j[m], k[m]], 1)


def set_objects(S, sv, objs):
    obst = [o for o in objs if o['flag'] == 1]
    lat = sdfm.lattice(obst, sv.origin, sv.h, sv.lattice_shape()) if obst else np.full(sv.lattice_shape(), 1e9)
    oid = np.full(sv.lattice_shape(), -1, np.int32)
    motions = [(o['lin'], o['ang'], o['pos']) for o in obst]
    sv.set_solids(S.Solids(lat, oid if not obst else np.zeros(sv.lattice_shape(), np.int32), motions,
                           sdfm.drains_for_solver(objs)))
    return lat


def snap(sv):
    return dict(count=sv.count.astype(np.int32), velold=sv.velold.copy(), mask=sv.mask.copy(), velg=sv.velg.copy(),
                pres=sv.pres.copy(), frac=sv.frac.copy())


def scenario_dam(S):
    """16³ dam break, two sub-steps, no whitewater."""
    nx = ny = nz = 16
    h = 1.0 / 16
    sv = make(S, nx, ny, nz, h, flip=0.95, omega=1.7, iters=30)
    rng = np.random.default_rng(11)
    cells = cells_where(nx, ny, nz, lambda i, j, k: (i < 6) & (j < 8))
    pos = jitter_cells(rng, cells, h, sv.origin, 8)
    vel = (rng.random(pos.shape) - 0.5) * 0.2
    sv.pos, sv.vel, sv.air = pos.copy(), vel.copy(), np.zeros(len(pos))
    out = dict(nx=nx, ny=ny, nz=nz, h=h, origin=sv.origin, flip=0.95, omega=1.7, iters=30, g=9.81, dt=1 / 240,
               pos0=pos, vel0=vel)
    sv._substep(1 / 240, ())
    for k, v in snap(sv).items():
        out['s1_' + k] = v
    out['s1_pos'], out['s1_vel'], out['s1_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
    sv._substep(1 / 240, ())
    for k, v in snap(sv).items():
        out['s2_' + k] = v
    out['s2_pos'], out['s2_vel'], out['s2_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
    return out


def scenario_obstacles(S):
    """20×12×16 tank with a sphere, a turned box, a cone and a drain; particles thrown at the obstacles."""
    nx, ny, nz = 20, 12, 16
    h = 1.0 / 20
    sv = make(S, nx, ny, nz, h, flip=0.95, omega=1.8, iters=40)
    objs = [sdfm.make_obstacle('sphere', [0.15, 0.18, 0.0], r=0.09),
            sdfm.make_obstacle('box', [-0.25, 0.1, 0.12], rot_deg=(0, 30, 0), w=0.16, h=0.1, d=0.12),
            sdfm.make_obstacle('cone', [-0.05, 0.1, -0.2], rot_deg=(10, 0, 20), r=0.08, h=0.14),
            sdfm.make_drain([0.38, 0.0, -0.28], 0.06)]
    lat = set_objects(S, sv, objs)
    rng = np.random.default_rng(12)
    cells = cells_where(nx, ny, nz, lambda i, j, k: (j < 5))
    pos = jitter_cells(rng, cells, h, sv.origin, 8)
    keep = sv.sdf_at(pos) >= 0
    pos = pos[keep]
    vel = np.zeros_like(pos)
    vel[:, 0] = 0.8 * np.sin(pos[:, 2] * 9.0)
    vel[:, 1] = -0.6
    vel[:, 2] = 0.5 * np.cos(pos[:, 0] * 7.0)
    sv.pos, sv.vel, sv.air = pos.copy(), vel.copy(), np.zeros(len(pos))
    out = dict(nx=nx, ny=ny, nz=nz, h=h, origin=sv.origin, flip=0.95, omega=1.8, iters=40, g=9.81, dt=1 / 240,
               pos0=pos, vel0=vel, lattice=lat, frac=sv.frac.copy())
    sv._substep(1 / 240, ())
    for k, v in snap(sv).items():
        out['s1_' + k] = v
    out['s1_pos'], out['s1_vel'], out['s1_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
    sv._substep(1 / 240, ())
    out['s2_pres'] = sv.pres.copy()
    out['s2_pos'], out['s2_vel'], out['s2_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
    return out


def scenario_drops(S):
    """Airborne drops falling into a pool: the free-flight mark, merging, ripple impulses, crowns and
    whitewater spawning (reference PCG64 stream, seed 5)."""
    nx, ny, nz = 16, 16, 16
    h = 1.0 / 16
    sv = make(S, nx, ny, nz, h, flip=0.96, omega=1.6, iters=20, whitewater=True, seed=5, ripple=16, wmap=32)
    rng = np.random.default_rng(13)
    pool = jitter_cells(rng, cells_where(nx, ny, nz, lambda i, j, k: j < 5), h, sv.origin, 8)
    # single drops just above the surface falling fast, flagged airborne
    nd = 40
    dx = sv.origin[0] + (rng.random(nd) * 0.8 + 0.1) * nx * h
    dz = sv.origin[2] + (rng.random(nd) * 0.8 + 0.1) * nz * h
    dy = 5 * h + 0.004 + rng.random(nd) * 0.01
    drops = np.stack([dx, dy, dz], 1).astype(np.float32).astype(np.float64)
    pos = np.concatenate([pool, drops])
    vel = np.zeros_like(pos)
    vel[:len(pool)] = (rng.random((len(pool), 3)) - 0.5) * 2.5          # lively pool, spawns whitewater
    vel[len(pool):, 1] = -3.0 - 2.0 * rng.random(nd)
    air = np.zeros(len(pos)); air[len(pool):] = 1.0
    sv.pos, sv.vel, sv.air = pos.copy(), vel.copy(), air.copy()
    out = dict(nx=nx, ny=ny, nz=nz, h=h, origin=sv.origin, flip=0.96, omega=1.6, iters=20, g=9.81, dt=1 / 120,
               pos0=pos, vel0=vel, air0=air, seed=5, ripple=16)
    sv._substep(1 / 120, ())
    out['s1_pos'], out['s1_vel'], out['s1_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
    out['s1_rsrc'], out['s1_impacts'] = sv.rsrc.copy(), sv.impacts
    out['s1_wpos'], out['s1_wvel'], out['s1_wlife'] = sv.wpos.copy(), sv.wvel.copy(), sv.wlife.copy()
    return out


SUN = (0.35, 0.85, 0.25)      # a low sun from +x, +z: refracted rays leave the texel they enter


def scenario_frame(S):
    """A whole frame (CFL sub-steps, whitewater advance, top height, ripple mask and ripple step) with
    obstacles, then a second frame."""
    nx, ny, nz = 16, 12, 16
    h = 1.0 / 16
    sv = make(S, nx, ny, nz, h, flip=0.96, omega=1.6, iters=20, whitewater=True, seed=7, ripple=16, wmap=32)
    objs = [sdfm.make_obstacle('cylinder', [0.1, 0.15, -0.1], r=0.08, h=0.3),
            sdfm.make_obstacle('torus', [-0.2, 0.15, 0.15], R=0.1, r=0.03)]
    lat = set_objects(S, sv, objs)
    rng = np.random.default_rng(14)
    pos = jitter_cells(rng, cells_where(nx, ny, nz, lambda i, j, k: (j < 4) | ((i < 4) & (j < 9))), h, sv.origin, 8)
    pos = pos[sv.sdf_at(pos) >= 0]
    vel = (rng.random(pos.shape) - 0.5) * 1.6
    drops = np.stack([rng.uniform(-0.3, 0.3, 12), rng.uniform(0.4, 0.6, 12), rng.uniform(-0.3, 0.3, 12)], 1)
    pos = np.concatenate([pos, drops.astype(np.float32).astype(np.float64)])
    vel = np.concatenate([vel, np.tile([0.0, -4.0, 0.0], (12, 1))])
    air = np.zeros(len(pos)); air[-12:] = 1
    wp = np.stack([rng.uniform(-0.4, 0.4, 300), rng.uniform(0.0, 0.5, 300), rng.uniform(-0.4, 0.4, 300)], 1)
    wv = (rng.random((300, 3)) - 0.5) * 2.0
    wl = rng.uniform(0.2, 2.0, 300)
    wk = np.floor(rng.random(300) * 3.0)
    sv.pos, sv.vel, sv.air = pos.copy(), vel.copy(), air.copy()
    sv.wpos, sv.wvel, sv.wlife, sv.wkind = wp.copy(), wv.copy(), wl.copy(), wk.copy()
    out = dict(nx=nx, ny=ny, nz=nz, h=h, origin=sv.origin, flip=0.96, omega=1.6, iters=20, g=9.81,
               pos0=pos, vel0=vel, air0=air, wpos0=wp, wvel0=wv, wlife0=wl, wkind0=wk, lattice=lat, seed=7,
               ripple=16, wmap=32, frame_dt=1 / 60)
    for f in (1, 2):
        sv.step(1 / 60)
        out[f'f{f}_pos'], out[f'f{f}_vel'], out[f'f{f}_air'] = sv.pos.copy(), sv.vel.copy(), sv.air.copy()
        out[f'f{f}_wpos'], out[f'f{f}_wvel'], out[f'f{f}_wlife'] = sv.wpos.copy(), sv.wvel.copy(), sv.wlife.copy()
        out[f'f{f}_top'], out[f'f{f}_field'], out[f'f{f}_S'] = sv.top.copy(), sv.ripple.field.copy(), sv.ripple.S.copy()
        out[f'f{f}_frame'], out[f'f{f}_time'], out[f'f{f}_vmax'] = sv.frame, sv.time, sv.vmax
        out[f'f{f}_caustics'] = sv.caustics(SUN)
        # the frame's mesh export (bake.py:228-235)
        v, q, tr = MESHING.surface(sv)
        MESHING.settle_on_top(sv, v)
        g = (v - sv.origin) / sv.h
        vel = np.stack([sv._sample(g, a) for a in range(3)], 1) if len(v) else np.zeros((0, 3))
        if len(v):
            vel[~sv._in_grid(g)] = 0.0
        out[f'f{f}_mesh_v'], out[f'f{f}_mesh_q'], out[f'f{f}_mesh_t'], out[f'f{f}_mesh_vel'] = v, q, tr, vel
        out[f'f{f}_count'] = sv.count.copy()
    out['sun'] = np.array(SUN)
    return out


def scenario_ripple(S):
    """The ripple layer alone: two frames with an impulse source and a mask (R = 32)."""
    R = 32
    rl = S.RippleLayer(R, 0.6, 0.4)
    rng = np.random.default_rng(15)
    src = np.zeros((R + 1, R + 1))
    src[rng.integers(0, R + 1, 20), rng.integers(0, R + 1, 20)] = rng.random(20) * 2e-3
    mask = np.clip(rng.random((R + 1, R + 1)) * 1.5, 0, 1)
    out = dict(R=R, Lx=0.6, Lz=0.4, src=src, mask=mask, depth=0.05, dt=1 / 60)
    rl.frame(1 / 60, 0.05, src, mask)
    out['f1_S'], out['f1_field'] = rl.S.copy(), rl.field.copy()
    rl.frame(1 / 60, 0.05, np.zeros_like(src), mask)
    out['f2_S'], out['f2_field'] = rl.S.copy(), rl.field.copy()
    return out


def scenario_dam32(S):
    """The 32³ dam-break workload (53,248 particles), one sub-step: binning, P2G and pressure."""
    sys.path.insert(0, os.path.join(ROOT, 'hahenn-_b200'))
    import workloads
    w = workloads.dam_break()
    sv = make(S, 32, 32, 32, w['h'], flip=0.95, omega=1.7, iters=60)
    assert np.allclose(sv.origin, w['origin'])
    pos = w['pos'].astype(np.float64)
    sv.pos, sv.vel, sv.air = pos.copy(), np.zeros_like(pos), np.zeros(len(pos))
    sv._substep(1 / 240, ())
    return dict(count=sv.count.astype(np.int16), velold=sv.velold.astype(np.float32), pres=sv.pres.astype(np.float32),
                mask=sv.mask, n=len(pos), pos_sum=sv.pos.sum(0), vel_sum=sv.vel.sum(0),
                vel_absmax=np.abs(sv.vel).max(0))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('SUIRI_REFERENCE')
    if not ref:
        sys.exit('usage: make_golden.py REF (the reference checkout; or set SUIRI_REFERENCE)')
    only = set(sys.argv[2:])                 # scenario names to regenerate (all when none given)
    global MESHING
    MESHING = load_meshing(ref)
    for name, fn in (('dam16', scenario_dam), ('obstacles', scenario_obstacles), ('drops', scenario_drops),
                     ('frame', scenario_frame), ('ripple', scenario_ripple), ('dam32', scenario_dam32)):
        if only and name not in only:
            continue
        S = load_solver(ref)
        out = fn(S)
        path = os.path.join(HERE, f'{name}.npz')
        np.savez_compressed(path, **out)
        print(name, os.path.getsize(path) // 1024, 'KiB')


if __name__ == '__main__':
    main()
