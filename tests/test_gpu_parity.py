"""CUDA path against the oracle (and the reference's own fixtures) on identical seeded inputs.

Every test goes through the C ABI (libsuiri_cuda.so via ctypes). Tolerances are in tests/parity.py."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import flip as of
from oracle import ripple as orp
from parity import (assert_close_field, assert_mesh_matches_oracle, assert_particles, f32, gpu_from, obstacle_items, oracle_from,
                    sync_oracle_particles)

pytestmark = pytest.mark.gpu


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz'), allow_pickle=False))


def grid_fields(pkg, gpu):
    N = pkg.native
    return dict(count=gpu.grid(N.FIELD_CELL_COUNT), mask=gpu.grid(N.FIELD_MASK), velold=gpu.grid(N.FIELD_VELOLD),
                pres=gpu.grid(N.FIELD_PRES), vel=gpu.grid(N.FIELD_VEL), frac=gpu.grid(N.FIELD_FRAC),
                rhs=gpu.grid(N.FIELD_RHS))


def compare_substep(pkg, gpu, ora, what):
    g = grid_fields(pkg, gpu)
    np.testing.assert_array_equal(g['count'], ora.count, err_msg=f'{what}: cell counts')
    np.testing.assert_array_equal(g['mask'], ora.mask, err_msg=f'{what}: valid-face masks')
    assert_close_field(g['velold'], ora.velold, what=f'{what}: P2G velocity')
    assert_close_field(g['pres'], ora.pres, what=f'{what}: pressure')
    assert_close_field(g['vel'], ora.velg, what=f'{what}: projected velocity')
    assert_particles(gpu, ora, what)
    return g


def test_dam16_two_substeps(pkg):
    d = load('dam16')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']))
    gpu = gpu_from(pkg, nx, ny, nz, h, **kw)
    ora = oracle_from(nx, ny, nz, h, d['origin'], **kw)
    np.testing.assert_array_equal(gpu.origin, d['origin'])
    pos, vel = f32(d['pos0']), f32(d['vel0'])
    gpu.add_particles(pos, vel)
    ora.add_particles(pos, vel)
    for s in (1, 2):
        gpu.substep(float(d['dt']))
        ora.frame = s
        ora.substep(float(d['dt']))
        g = compare_substep(pkg, gpu, ora, f'sub-step {s}')
        if s == 1:   # the reference solver itself, same particle positions
            np.testing.assert_array_equal(g['count'], d['s1_count'])
            np.testing.assert_array_equal(g['mask'], d['s1_mask'])
            assert_close_field(g['pres'], d['s1_pres'], what='pressure vs reference')
        sync_oracle_particles(gpu, ora)
    gpu.close()


def test_rk2_advection_matches_oracle(pkg):
    """The midpoint (RK2) advection option, which the reference does not have, against the oracle's
    statement of it on the dam break: grids exactly as in Euler mode, particles within tolerance, and the
    positions measurably different from explicit Euler."""
    d = load('dam16')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']))
    pos, vel = f32(d['pos0']), f32(d['vel0'])
    gpu = gpu_from(pkg, nx, ny, nz, h, advect='rk2', **kw)
    eul = gpu_from(pkg, nx, ny, nz, h, **kw)
    ora = oracle_from(nx, ny, nz, h, d['origin'], advect='rk2', **kw)
    for t in (gpu, eul, ora):
        t.add_particles(pos, vel)
    for s in (1, 2, 3):
        gpu.substep(float(d['dt']))
        eul.substep(float(d['dt']))
        ora.frame = s
        ora.substep(float(d['dt']))
        compare_substep(pkg, gpu, ora, f'RK2 sub-step {s}')
        sync_oracle_particles(gpu, ora)
    pr, _, _, ir = gpu.particles()
    pe, _, _, ie = eul.particles()
    dx = np.abs(pr[np.argsort(ir)] - pe[np.argsort(ie)]).max()
    assert dx > 1e-5, f'RK2 positions differ from Euler by only {dx:.2e} m'
    gpu.close()
    eul.close()


@pytest.mark.parametrize('sor_mode', [0, 2, 3, 4])
def test_sor_bit_exact_with_reference_operation_order(pkg, sor_mode):
    """Given the GPU's own float32 operands, the reference's float32 SOR loop reproduces its pressure bit for
    bit, for one launch per sweep, temporal blocking and the cluster-resident solve. The device's FP64
    residual of the solve equals the host's FP64 residual of the same operands, and is stated."""
    d = load('dam16')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    gpu = gpu_from(pkg, nx, ny, nz, h, flip=0.95, omega=1.7, iters=30)
    gpu.tune(4, sor_mode)
    gpu.residual(True)
    gpu.add_particles(f32(d['pos0']), f32(d['vel0']))
    gpu.substep(1 / 240)
    g = grid_fields(pkg, gpu)
    fluid = g['count'] > 0
    C, inv, U, rhs = of.sor_operands_from(g['frac'], g['rhs'], fluid, 1.7)
    p = of.sor_f32(C, inv, U, rhs, np.zeros(rhs.shape), 30)
    p[~fluid] = 0
    np.testing.assert_array_equal(g['pres'].astype(np.float64), p)
    r30 = of.residual_f64(C, rhs, fluid, p)
    r0 = of.residual_f64(C, rhs, fluid, np.zeros_like(p))
    assert r30 < r0
    st = gpu.stats()
    act = fluid & (sum(C) > 0)
    assert st['active_cells'] == int(act.sum())
    assert abs(st['residual_max'] - r30) <= 1e-12 * r30, (st['residual_max'], r30)
    assert st['rhs_max'] == float(np.abs(rhs.astype(np.float64)[act]).max())
    print(f"FP64 residual after 30 iterations: max {st['residual_max']:.3e} (rms {st['residual_rms']:.3e}), "
          f"{st['residual_max'] / st['rhs_max']:.3e} of max |h²·div|; before the solve {r0:.3e}")
    gpu.close()


@pytest.mark.parametrize('mode', ['analytic', 'lattice'])
def test_obstacles_face_fractions_and_substep(pkg, mode):
    d = load('obstacles')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']))
    items, objs = obstacle_items()
    gpu = gpu_from(pkg, nx, ny, nz, h, sdf_mode=mode, **kw)
    gpu.set_objects(items)
    if mode == 'lattice':
        gpu.set_lattice(d['lattice'])
    ora = oracle_from(nx, ny, nz, h, d['origin'], sdf_mode=mode, **kw)
    ora.set_objects(objs)
    np.testing.assert_array_equal(ora.frac, d['frac'])
    pos, vel = f32(d['pos0']), f32(d['vel0'])
    gpu.add_particles(pos, vel)
    ora.add_particles(pos, vel)
    gpu.substep(float(d['dt']))
    ora.frame = 1
    ora.substep(float(d['dt']))
    g = compare_substep(pkg, gpu, ora, f'obstacles ({mode})')
    # face fractions: float32 of the same float64 value as the reference's
    np.testing.assert_array_equal(g['frac'], d['frac'].astype(np.float32))
    np.testing.assert_array_equal(g['count'], d['s1_count'])
    if mode == 'lattice':
        assert_close_field(g['pres'], d['s1_pres'], what='pressure vs reference')
    sync_oracle_particles(gpu, ora)
    gpu.substep(float(d['dt']))
    ora.frame = 2
    ora.substep(float(d['dt']))
    compare_substep(pkg, gpu, ora, f'obstacles ({mode}) sub-step 2')
    gpu.close()


ALL_SHAPES = [
    dict(kind='obstacle', shape='box', pos=[-0.2, 0.1, -0.1], rot=[10, 30, 0], dims=dict(w=0.1, h=0.06, d=0.08)),
    dict(kind='obstacle', shape='plate', pos=[0.0, 0.25, 0.1], rot=[0, 0, 15], dims=dict(w=0.22, d=0.1, t=0.012)),
    dict(kind='obstacle', shape='sphere', pos=[0.2, 0.1, 0.1], rot=[0, 0, 0], dims=dict(r=0.05)),
    dict(kind='obstacle', shape='cylinder', pos=[0.1, 0.08, -0.15], rot=[0, 0, 20], dims=dict(r=0.03, h=0.12)),
    dict(kind='obstacle', shape='cone', pos=[-0.15, 0.05, 0.15], rot=[0, 45, 0], dims=dict(r=0.04, h=0.08)),
    dict(kind='obstacle', shape='torus', pos=[0.05, 0.18, -0.02], rot=[30, 0, 0], dims=dict(R=0.05, r=0.014)),
    dict(kind='obstacle', shape='cup', pos=[-0.05, 0.06, 0.0], rot=[0, 0, 0], dims=dict(r=0.04, h=0.1, t=0.006)),
    dict(kind='obstacle', shape='container', pos=[0.2, 0.04, -0.1], rot=[0, 20, 0], dims=dict(w=0.14, h=0.06, d=0.1, t=0.008)),
    dict(kind='obstacle', shape='gutter', pos=[-0.1, 0.2, -0.05], rot=[0, 0, -14], dims=dict(len=0.28, r=0.03, t=0.006))]


@pytest.mark.parametrize('mode', ['analytic', 'lattice'])
def test_obstacle_distances_every_shape(pkg, mode):
    """The device's distances equal the oracle's bit for bit: the analytic shape library (all eight shapes,
    turned) and the trilinear lattice."""
    from parity import objs_from_items
    nx, ny, nz, h = 24, 12, 16, 1 / 40
    t = pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, whitewater=False, ripple=None, capacity=1024, sdf_mode=mode)
    t.set_objects(ALL_SHAPES)
    ora = oracle_from(nx, ny, nz, h, t.origin, flip=0.96, omega=1.6, iters=1, sdf_mode=mode)
    ora.set_objects(objs_from_items(ALL_SHAPES))
    if mode == 'lattice':
        t.set_lattice(ora.lat)
    rng = np.random.default_rng(9)
    pts = t.origin + rng.random((20000, 3)) * np.array([nx, ny, nz]) * h
    np.testing.assert_array_equal(t.eval_sdf(pts), ora.sdf_at(pts))
    t.substep(1 / 240)                     # face fractions are computed at the first sub-step
    np.testing.assert_array_equal(t.grid(pkg.native.FIELD_FRAC), ora.frac.astype(np.float32))
    t.close()


def test_collisions_near_every_shape(pkg):
    """Particles within a few collision radii of all eight shapes (turned) and others anywhere in the tank,
    one sub-step in analytic mode: they equal the oracle's, which tests every particle against the scene
    distance, so the device's culls (the bounding sphere, then a box in the obstacle's frame) skip no
    collision."""
    from parity import objs_from_items
    nx, ny, nz, h = 24, 12, 16, 1 / 40
    kw = dict(flip=0.96, omega=1.6, iters=20)
    gpu = gpu_from(pkg, nx, ny, nz, h, **kw)
    gpu.set_objects(ALL_SHAPES)
    ora = oracle_from(nx, ny, nz, h, gpu.origin, **kw)
    ora.set_objects(objs_from_items(ALL_SHAPES))
    rng = np.random.default_rng(21)
    pts = gpu.origin + rng.random((400000, 3)) * np.array([nx, ny, nz]) * h
    d = ora.sdf_at(pts)
    rc = 0.32 * h
    near = pts[(d > -rc) & (d < 3 * rc)][:8000]
    pos = f32(np.concatenate([near, pts[-4000:]]))
    vel = f32(rng.uniform(-0.6, 0.6, pos.shape))
    assert len(near) == 8000
    gpu.add_particles(pos, vel)
    ora.add_particles(pos, vel)
    gpu.substep(1 / 240)
    ora.frame = 1
    ora.substep(1 / 240)
    assert_particles(gpu, ora, 'collisions near every shape')
    gpu.close()


def test_drops_merge_ripple_impulse_crown_and_spawn(pkg):
    d = load('drops')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']), whitewater=True)
    R = int(d['ripple'])
    gpu = gpu_from(pkg, nx, ny, nz, h, ripple=(R, R), ww_capacity=4000, **kw)
    ora = oracle_from(nx, ny, nz, h, d['origin'], ripple=(R, R), ww_cap=4000, rng_mode='hash', **kw)
    pos, vel, air = f32(d['pos0']), f32(d['vel0']), d['air0']
    gpu.add_particles(pos, vel, air)
    ora.add_particles(pos, vel, air)
    gpu.substep(float(d['dt']))
    ora.frame = 1
    ora.substep(float(d['dt']))
    assert_particles(gpu, ora, 'drops')
    st = gpu.stats()
    assert st['impacts'] == ora.impacts and ora.impacts > 0
    src = gpu.ripple_field(pkg.native.FIELD_RIPPLE_SRC, (R + 1, R + 1), np.float64)
    assert_close_field(src, ora.rsrc, rtol=1e-9, what='ripple impulses')
    wp, wv = gpu.whitewater()
    assert len(wp) == len(ora.wpos) and len(wp) > 0
    # whitewater order follows atomics: compare as sets keyed by position
    o1 = np.lexsort(wp[:, :3].T.astype(np.float64))
    o2 = np.lexsort(ora.wpos.T)
    np.testing.assert_allclose(wp[o1, :3], ora.wpos[o2], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(wp[o1, 3], ora.wlife[o2], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(wv[o1, :3], ora.wvel[o2], rtol=1e-4, atol=1e-5)
    gpu.close()


def test_frame_step_whitewater_top_height_and_ripples(pkg):
    d = load('frame')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    R, W = int(d['ripple']), int(d['wmap'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']), whitewater=True)
    gpu = gpu_from(pkg, nx, ny, nz, h, ripple=(R, R), wmap=W, ww_capacity=4000, sdf_mode='lattice', **kw)
    ora = oracle_from(nx, ny, nz, h, d['origin'], ripple=(R, R), wmap=W, ww_cap=4000, rng_mode='hash', sdf_mode='lattice', **kw)
    from oracle import sdf as sdfm
    objs = [sdfm.make_obstacle('cylinder', [0.1, 0.15, -0.1], r=0.08, h=0.3),
            sdfm.make_obstacle('torus', [-0.2, 0.15, 0.15], R=0.1, r=0.03)]
    ora.set_objects(objs)
    gpu.set_objects([dict(kind='obstacle', shape='cylinder', pos=[0.1, 0.15, -0.1], rot=[0, 0, 0], dims=dict(r=0.08, h=0.3)),
                     dict(kind='obstacle', shape='torus', pos=[-0.2, 0.15, 0.15], rot=[0, 0, 0], dims=dict(R=0.1, r=0.03))])
    gpu.set_lattice(d['lattice'])
    pos, vel, air = f32(d['pos0']), f32(d['vel0']), d['air0']
    gpu.add_particles(pos, vel, air)
    ora.add_particles(pos, vel, air)
    layer = orp.RippleLayer(R, R, nx * h, nz * h)
    n_gpu = gpu.step(float(d['frame_dt']))
    n_ora = ora.step(float(d['frame_dt']), layer)
    assert n_gpu == n_ora
    assert_particles(gpu, ora, 'frame')
    top = gpu.ripple_field(pkg.native.FIELD_TOP, (W, W), np.float32)
    assert_close_field(top, ora.top, what='top height')
    mask = gpu.ripple_field(pkg.native.FIELD_RIPPLE_MASK, (R + 1, R + 1), np.float32)
    assert_close_field(mask, orp.ripple_mask(ora), what='ripple mask')
    fld = gpu.ripple_field(pkg.native.FIELD_RIPPLE, (R + 1, R + 1, 3), np.float32)
    for c in range(3):     # heights in m, slopes: float32 FFT round-off floor 1e-12
        assert_close_field(fld[..., c], layer.field[..., c], rtol=1e-4, atol=1e-12, what=f'ripple field {c}')
    # floor light of the frame: from the GPU's own maps as the oracle forms it, and against the oracle's frame
    sun = d['sun']
    maps = gpu.frame_maps(sun)
    top64 = gpu.ripple_field(pkg.native.FIELD_TOP64, (W, W), np.float64)
    _check_frame_maps(maps, top64, fld, nx * h, nz * h, sun)
    assert_close_field(maps[..., 3], orp.caustics(ora.top, layer.field, nx * h, nz * h, sun), rtol=1e-4,
                       what='floor light against the oracle frame')
    # the frame's surface mesh: pool, obstacle walls and the lone drops in flight
    m = assert_mesh_matches_oracle(pkg, gpu, ora)
    assert m['quads'].shape[0] > 1000 and m['lone'] > 0
    gpu.close()


def _check_frame_maps(maps, top64, fld, Lx, Lz, sun):
    """The frame maps against the oracle evaluated on the same height map and ripple field: top height
    exactly (float32 of the float64 map), ripple slopes at texel centres and floor light within float32
    rounding (both sides float64 on identical inputs; the light's fixed-point sums add 2^-32 per tap)."""
    W = top64.shape[0]
    np.testing.assert_array_equal(maps[..., 0], top64.astype(np.float32))
    f64 = fld.astype(np.float64)
    ii, jj = np.meshgrid(np.arange(W), np.arange(W))
    sx, sz = orp.slope_at(f64, Lx, Lz, (ii + 0.5) * (Lx / W), (jj + 0.5) * (Lz / W))
    np.testing.assert_allclose(maps[..., 1], sx, rtol=1e-6, atol=1e-9 * max(np.abs(sx).max(), 1e-30))
    np.testing.assert_allclose(maps[..., 2], sz, rtol=1e-6, atol=1e-9 * max(np.abs(sz).max(), 1e-30))
    light = orp.caustics(top64, f64, Lx, Lz, sun)
    np.testing.assert_allclose(maps[..., 3], light, rtol=1e-6, atol=1e-7)


def test_surface_mesh_under_rain(pkg):
    """The surface mesh of the full scene's shape at a quarter of each axis after rain frames: a pool with
    ripples and drops in flight (lone spheres), with the reference's blur (σ 0.8, 5 taps) and a wider one
    (σ 1.6, 9 taps), each against the oracle on the GPU's state; then the mesh of an empty tank."""
    w = pkg.workloads.full_scene(scale=4)
    nx, ny, nz, h = w['nx'], w['ny'], w['nz'], w['h']
    prm = w['params']
    gpu = pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, ripple=w['ripple'], wmap=128, capacity=len(w['pos']) + 20000,
                   ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'], drop_d=prm['drop_d'],
                   flip=prm['flip'], omega=prm['omega'], iters=40)
    ora = oracle_from(nx, ny, nz, h, w['origin'], ripple=w['ripple'], wmap=128, flip=prm['flip'], omega=prm['omega'],
                      iters=40)
    gpu.add_particles(w['pos'])
    rng = np.random.default_rng(8)
    for f in range(2):
        n = 300
        drops = np.stack([rng.uniform(-0.45 * nx * h, 0.45 * nx * h, n), rng.uniform(0.5, 0.9, n) * ny * h,
                          rng.uniform(-0.45 * nz * h, 0.45 * nz * h, n)], 1)
        dv = np.zeros((n, 3)); dv[:, 1] = -2.0
        gpu.add_particles(f32(drops), f32(dv), np.ones(n))
        for _ in range(3):
            gpu.step(1 / 60)
    for smooth in (0.8, 1.6):
        m = assert_mesh_matches_oracle(pkg, gpu, ora, smooth)
        assert len(m['weights']) == 2 * max(1, int(np.ceil(2.5 * smooth))) + 1
        assert m['quads'].shape[0] > 10000 and m['lone'] > 10
    gpu.clear_water()
    m = gpu.surface_mesh()
    assert m['verts'].shape == (0, 3) and m['quads'].shape == (0, 4) and m['tris'].shape == (0, 3)
    gpu.close()


def test_frame_maps_floor_light_under_rain(pkg):
    """The per-frame light and surface maps of the full scene's shape at a quarter of each axis (128² map,
    256×128 ripple layer) after three frames of rain: ripples from the merged drops and the liquid's own
    slope bend the light. Three suns (overhead, oblique, low from -x), each against the oracle on the GPU's
    height map and ripple field."""
    w = pkg.workloads.full_scene(scale=4)
    nx, ny, nz, h = w['nx'], w['ny'], w['nz'], w['h']
    Rx, Rz = w['ripple']
    prm = w['params']
    W = 128
    gpu = pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, ripple=(Rx, Rz), wmap=W, capacity=len(w['pos']) + 20000,
                   ww_capacity=20000, ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'],
                   drop_d=prm['drop_d'], flip=prm['flip'], omega=prm['omega'], iters=40)
    gpu.add_particles(w['pos'])
    rng = np.random.default_rng(5)
    for f in range(3):
        n = 200
        drops = np.stack([rng.uniform(-0.45 * nx * h, 0.45 * nx * h, n), rng.uniform(0.3, 0.45, n) * ny * h,
                          rng.uniform(-0.45 * nz * h, 0.45 * nz * h, n)], 1)
        dv = np.zeros((n, 3)); dv[:, 1] = -4.0
        gpu.add_particles(f32(drops), f32(dv), np.ones(n))
        for _ in range(4):
            gpu.step(1 / 60)
    assert gpu.stats()['impacts'] > 0
    top64 = gpu.ripple_field(pkg.native.FIELD_TOP64, (W, W), np.float64)
    fld = gpu.ripple_field(pkg.native.FIELD_RIPPLE, (Rz + 1, Rx + 1, 3), np.float32)
    assert np.abs(fld[..., 1]).max() > 0
    out = np.empty((W, W, 4), np.float32)
    for sun in ((0.0, 1.0, 0.0), (0.35, 0.85, 0.25), (-0.8, 0.45, 0.1)):
        maps = gpu.frame_maps(sun, out)
        assert maps is out
        _check_frame_maps(maps, top64, fld, nx * h, nz * h, sun)
        assert maps[..., 3].max() > maps[..., 3].min() + 1e-3          # the surface bends the light
    with pytest.raises(pkg.native.SuiriError):
        gpu.frame_maps((0.0, 0.0, 0.0))
    gpu.close()


@pytest.mark.parametrize('depth', [0.0, 0.05])
def test_ripple_layer_spectral_update(pkg, depth):
    """Two ripple frames with impulses from merging drops, at the mean liquid depth (0) and at a stated depth
    (the per-mode update then computed once and reused on the second frame)."""
    R = 32
    gpu = pkg.Tank(nx=24, ny=8, nz=16, h=0.025, iters=4, whitewater=False, ripple=(R, R), wmap=32, capacity=16384,
                   ripple_depth=depth)
    # drops landing put impulses into the source grid; here: add a few airborne particles that merge
    rng = np.random.default_rng(3)
    pool = gpu.origin + (np.stack(np.meshgrid(np.arange(24), np.arange(3), np.arange(16), indexing='ij'), -1).reshape(-1, 3)
                         + 0.5) * 0.025
    pool = np.repeat(pool, 8, 0) + (rng.random((len(pool) * 8, 3)) - 0.5) * 0.02
    drops = np.stack([rng.uniform(-0.2, 0.2, 30), np.full(30, 3 * 0.025 + 0.003), rng.uniform(-0.15, 0.15, 30)], 1)
    pos = np.concatenate([pool, drops])
    vel = np.zeros_like(pos)
    vel[len(pool):, 1] = -4.0
    air = np.zeros(len(pos)); air[len(pool):] = 1
    ora = oracle_from(24, 8, 16, 0.025, gpu.origin, flip=0.96, omega=1.6, iters=4, ripple=(R, R), wmap=32)
    gpu.add_particles(f32(pos), f32(vel), air)
    ora.add_particles(f32(pos), f32(vel), air)
    layer = orp.RippleLayer(R, R, 24 * 0.025, 16 * 0.025)
    for f in range(2):
        gpu.step(1 / 60)
        ora.step(1 / 60, layer, ripple_depth=depth)
    S = gpu.ripple_field(pkg.native.FIELD_RIPPLE_STATE, (2 * R, 2 * R, 2), np.float32)
    assert np.abs(layer.S).max() > 0
    assert_close_field(S[..., 0], layer.S.real, rtol=1e-4, what='ripple state (height)')
    assert_close_field(S[..., 1], layer.S.imag, rtol=1e-4, what='ripple state (velocity)')
    gpu.close()


def test_sor_bit_exact_when_the_sweep_grid_is_capped(pkg):
    """A tank with more active cells of one colour than the GPU has resident sweep threads (256×64×64, the
    lower 7/8 liquid: ≈458k cells a colour against 148 SMs × 2048), with a sphere, a turned box and a tilted
    cone cutting cells: the sweep grid is capped at what is resident and each thread also relaxes the cells one
    grid further on, cut cells among them. Pressures equal the reference's float32 loop bit for bit."""
    nx, ny, nz, h = 256, 64, 64, 1.0 / 64
    cells = pkg.workloads.block_cells(nx, ny, nz, lambda i, j, k: j < 56)
    pos = pkg.workloads.fill_cells(cells, h, pkg.workloads.grid_origin(nx, nz, h), 1, 7)
    gpu = gpu_from(pkg, nx, ny, nz, h, flip=0.95, omega=1.7, iters=8, capacity=len(pos) + 1024)
    gpu.set_objects(obstacle_items()[0][:3])
    gpu.add_particles(f32(pos))
    gpu.substep(1 / 240)
    assert gpu.stats()['errors'] == 0
    g = grid_fields(pkg, gpu)
    fluid = g['count'] > 0
    assert fluid.sum() // 2 > 148 * 2048
    C, inv, U, rhs = of.sor_operands_from(g['frac'], g['rhs'], fluid, 1.7)
    p = of.sor_f32(C, inv, U, rhs, np.zeros(rhs.shape), 8)
    p[~fluid] = 0
    np.testing.assert_array_equal(g['pres'].astype(np.float64), p)
    gpu.close()


@pytest.mark.parametrize('axes,seeds,lanes', [((16, 24, 32), (1, 2, 3), None), ((16, 48), (1, 2, 16), None),
                                              ((16, 24, 32), (1, 2, 3), (2, 0, 5))])
def test_batch_equals_solo_bit_for_bit(pkg, axes, seeds, lanes):
    """Tanks of uneven sizes stepped in one batch give exactly the particles they give alone; with the 48³
    tank (seed 16) the batch spans two size lanes (its own stream and graph each, forked and joined every
    sub-step); with lanes given explicitly, each tank in a lane of its own."""
    specs = [pkg.workloads.random_tank(s, axes=axes) for s in seeds]
    if axes == (16, 48):
        sizes = [w['nx'] * w['ny'] * w['nz'] for w in specs]
        assert min(sizes) < 1 << 16 <= max(sizes), sizes

    def make():
        out = []
        for w in specs:
            t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.7, iters=20,
                         whitewater=True, ripple=None, capacity=len(w['pos']) * 2)
            t.set_objects(w['objects'])
            t.add_particles(w['pos'])
            out.append(t)
        return out

    solo, batched = make(), make()
    b = pkg.Batch(batched, lanes)
    for _ in range(6):
        for t in solo:
            t.substep(1 / 240)
        b.substep(1 / 240)
    b.sync()
    for a, c in zip(solo, batched):
        pa, va, aa, ia = a.particles()
        pc, vc, ac, ic = c.particles()
        oa, oc = np.argsort(ia), np.argsort(ic)
        np.testing.assert_array_equal(ia[oa], ic[oc])
        np.testing.assert_array_equal(pa[oa], pc[oc])
        np.testing.assert_array_equal(va[oa], vc[oc])
    b.close()
    for t in solo + batched:
        t.close()


def _run_form(pkg, w, mode, iters, steps=3, piece_kb=0):
    t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.8, iters=iters, whitewater=True,
                 ripple=None, capacity=len(w['pos']) * 2)
    t.set_objects(w['objects'])
    t.add_particles(w['pos'])
    if piece_kb:
        t.tune_piece(piece_kb)
    t.tune(4, mode)
    for _ in range(steps):
        t.substep(1 / 240)
    assert t.stats()['errors'] == 0
    pos, vel, air, ids = t.particles()
    o = np.argsort(ids)
    out = (t.grid(pkg.native.FIELD_PRES), pos[o], vel[o])
    t.close()
    return out


@pytest.mark.parametrize('mode,piece_kb', [(1, 0), (1, 2), (2, 0), (3, 0), (4, 0)])
def test_solve_forms_equal_per_sweep_launches(pkg, mode, piece_kb):
    """The cooperative whole-solve launch (1; with 2 KB of shared memory a block most of its cells are read
    from the lists each sweep instead of held), the temporal-blocked launches (2: two sweeps each, 3: four)
    and the cluster-resident solve (4) relax the same colours in the same order as one launch per sweep (0):
    identical pressures and particles, bit for bit."""
    w = pkg.workloads.obstacles_inflow(scale=4)
    for a, b in zip(_run_form(pkg, w, 0, 40), _run_form(pkg, w, mode, 40, piece_kb=piece_kb)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('piece_kb', [12, 24, 54])
def test_cluster_solve_pieces_across_ctas(pkg, piece_kb):
    """The cluster-resident solve with less shared memory per CTA, so the 32×16×16 tank is cut into pieces
    of 1 z plane (16 CTAs: every plane's z neighbours are ghost planes pushed by the next CTAs), 3 planes (six
    pieces, the last of one plane) and 8 planes (two): bit for bit the per-sweep launches."""
    w = pkg.workloads.obstacles_inflow(scale=4)
    assert (w['nx'], w['ny'], w['nz']) == (32, 16, 16)
    for a, b in zip(_run_form(pkg, w, 0, 40), _run_form(pkg, w, 4, 40, piece_kb=piece_kb)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('mode', [2, 3, 4])
@pytest.mark.parametrize('iters', [6, 7, 1, 3])
def test_temporal_blocking_edges(pkg, iters, mode):
    """Temporal blocking on a grid that is no multiple of the tile (odd x). Four sweeps a launch: an odd
    number of launches (6 iterations: 3 launches, the result copied back), a short last launch (7:
    4+4+4+2 sweeps), a single launch of two sweeps (1). Two sweeps a launch: odd counts (1, 3, 7)."""
    w = pkg.workloads.random_tank(5, axes=(21, 37, 19))
    for a, b in zip(_run_form(pkg, w, 0, iters), _run_form(pkg, w, mode, iters)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('mode', [1, 2, 3, 4])
def test_temporal_blocking_batch_uneven_iterations(pkg, mode):
    """In a batch the tile launches (and the cluster solve's sweeps) run to the largest iteration count;
    tanks with fewer iterations stop relaxing but keep their pressures (carried between the two buffers by
    the tile forms; held in shared memory by the cluster form, where small tanks share a cluster): every
    tank equals its solo run."""
    specs = [(pkg.workloads.random_tank(s, axes=(16, 24, 40)), it) for s, it in ((11, 5), (12, 12), (13, 9))]

    def make(mode):
        out = []
        for w, it in specs:
            t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.7, iters=it,
                         whitewater=True, ripple=None, capacity=len(w['pos']) * 2)
            t.set_objects(w['objects'])
            t.add_particles(w['pos'])
            if mode is not None:
                t.tune(4, mode)
            out.append(t)
        return out

    solo, batched = make(0), make(None)
    b = pkg.Batch(batched)
    b.tune(4, mode)
    for _ in range(4):
        for t in solo:
            t.substep(1 / 240)
        b.substep(1 / 240)
    b.sync()
    for a, c in zip(solo, batched):
        np.testing.assert_array_equal(a.grid(pkg.native.FIELD_PRES), c.grid(pkg.native.FIELD_PRES))
        pa, va, aa, ia = a.particles()
        pc, vc, ac, ic = c.particles()
        oa, oc = np.argsort(ia), np.argsort(ic)
        np.testing.assert_array_equal(pa[oa], pc[oc])
        np.testing.assert_array_equal(va[oa], vc[oc])
    b.close()
    for t in solo + batched:
        t.close()


def test_snapshot_restore(pkg):
    w = pkg.workloads.dam_break(16)
    t = pkg.Tank(nx=16, ny=16, nz=16, h=w['h'], flip=0.95, omega=1.7, iters=20, whitewater=False, ripple=None,
                 capacity=len(w['pos']) * 2)
    t.add_particles(w['pos'])
    for _ in range(3):
        t.substep(1 / 240)
    p0 = t.particles()
    sid = t.save_water()
    for _ in range(3):
        t.substep(1 / 240)
    assert not np.array_equal(t.particles()[0], p0[0])
    assert t.restore_water(sid)
    p1 = t.particles()
    for a, b in zip(p0, p1):
        np.testing.assert_array_equal(a, b)
    assert not t.restore_water(sid)      # one copy, restored once
    t.close()


def _match_sets(a, b, tol):
    """Pair the rows of a and b (N, k) one to one by nearest position (first 3 columns); the order of
    whitewater particles follows atomics, so they are compared as sets."""
    from scipy.spatial import cKDTree
    assert len(a) == len(b), f'{len(a)} against {len(b)}'
    if not len(a):
        return np.zeros(0, np.int64)
    d, j = cKDTree(b[:, :3]).query(a[:, :3])
    assert np.all(d <= tol), f'unpaired rows, worst distance {d.max():.3e}'
    assert len(np.unique(j)) == len(j), 'two rows paired with one'
    return j


def test_whitewater_advance_two_frames(pkg):
    """Spray, foam and bubbles seeded from the frame fixture's whitewater state (wpos0, wvel0, wlife0, wkind0,
    arrays of the reference's own solver) advance over two frames with the liquid: the GPU's whitewater equals
    the oracle's after each frame (spawns by the hash stream in both, landing spray into ripple impulses):
    same count, positions and life within the particle tolerance, velocities within 1e-4, same kind."""
    d = load('frame')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    R, W = int(d['ripple']), int(d['wmap'])
    kw = dict(flip=float(d['flip']), omega=float(d['omega']), iters=int(d['iters']), whitewater=True)
    gpu = gpu_from(pkg, nx, ny, nz, h, ripple=(R, R), wmap=W, ww_capacity=4000, sdf_mode='lattice', **kw)
    ora = oracle_from(nx, ny, nz, h, d['origin'], ripple=(R, R), wmap=W, ww_cap=4000, rng_mode='hash', sdf_mode='lattice', **kw)
    from oracle import sdf as sdfm
    ora.set_objects([sdfm.make_obstacle('cylinder', [0.1, 0.15, -0.1], r=0.08, h=0.3),
                     sdfm.make_obstacle('torus', [-0.2, 0.15, 0.15], R=0.1, r=0.03)])
    gpu.set_objects([dict(kind='obstacle', shape='cylinder', pos=[0.1, 0.15, -0.1], rot=[0, 0, 0], dims=dict(r=0.08, h=0.3)),
                     dict(kind='obstacle', shape='torus', pos=[-0.2, 0.15, 0.15], rot=[0, 0, 0], dims=dict(R=0.1, r=0.03))])
    gpu.set_lattice(d['lattice'])
    pos, vel, air = f32(d['pos0']), f32(d['vel0']), d['air0']
    gpu.add_particles(pos, vel, air)
    ora.add_particles(pos, vel, air)
    wp, wv, wl, wk = f32(d['wpos0']), f32(d['wvel0']), f32(d['wlife0']), d['wkind0'].astype(np.float64)
    gpu.add_whitewater(wp, wv, wl, wk)
    ora.wpos, ora.wvel, ora.wlife, ora.wkind = wp.copy(), wv.copy(), wl.copy(), wk.copy()
    P0, V0 = gpu.whitewater()
    np.testing.assert_array_equal(P0[:, :3], wp.astype(np.float32))
    layer = orp.RippleLayer(R, R, nx * h, nz * h)
    for f in (1, 2):
        n_gpu = gpu.step(float(d['frame_dt']))
        n_ora = ora.step(float(d['frame_dt']), layer)
        assert n_gpu == n_ora
        assert_particles(gpu, ora, f'frame {f}')
        P, V = gpu.whitewater()
        assert len(P) == len(ora.wpos) > 0, (len(P), len(ora.wpos))
        ref = np.concatenate([ora.wpos, ora.wlife[:, None]], 1)
        j = _match_sets(P.astype(np.float64), ref, 1e-5)
        err = np.abs(P[:, :3] - ora.wpos[j])
        assert np.all(err <= 1e-6 + 1e-6 * np.abs(ora.wpos[j])), f'frame {f}: whitewater position err {err.max():.3e}'
        np.testing.assert_allclose(P[:, 3], ora.wlife[j], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(V[:, :3], ora.wvel[j], rtol=1e-4, atol=1e-5)
        np.testing.assert_array_equal(V[:, 3], ora.wkind[j])
        src = gpu.ripple_field(pkg.native.FIELD_RIPPLE_STATE, (2 * R, 2 * R, 2), np.float32)
        # near zero here (no drop lands): compared down to the float32 FFT's round-off floor, as the field is
        assert_close_field(src[..., 0], layer.S.real, rtol=1e-4, atol=1e-11, what=f'frame {f}: ripple state')
        sync_oracle_particles(gpu, ora)       # the next frame starts from the GPU's float32 liquid
    gpu.close()


def test_rectangular_ripple_layer_full_scene_quarter(pkg):
    """The full scene's shape at a quarter of each axis: 64×32×32 cells, bottom 8 layers of liquid, a
    rectangular ripple layer of 256×128 cells (mirrored FFT 512×256: an odd power-of-two exponent on x, so
    the radix-4 passes end with one radix-2 pass on that axis only), σ = 0.072 N/m, ρ = 1000 kg/m³ at the
    stated depth 0.1 m, and rain: sub-grid drops of lognormal diameter (median 2 mm, σ_log 0.4) added on
    the host at 4 m/s. Over two frames: particles, impacts, top height, ripple mask, spectral state and
    field against the oracle."""
    w = pkg.workloads.full_scene(scale=4)
    nx, ny, nz, h = w['nx'], w['ny'], w['nz'], w['h']
    Rx, Rz = w['ripple']
    assert (nx, ny, nz, Rx, Rz) == (64, 32, 32, 256, 128)
    prm = w['params']
    kw = dict(flip=prm['flip'], omega=prm['omega'], iters=40, whitewater=True)
    gpu = pkg.Tank(nx=nx, ny=ny, nz=nz, h=h, ripple=(Rx, Rz), wmap=128, capacity=len(w['pos']) + 20000,
                   ww_capacity=20000, ripple_sigma=prm['sigma'], ripple_rho=prm['rho'], ripple_depth=prm['depth'],
                   drop_d=prm['drop_d'], **kw)
    ora = oracle_from(nx, ny, nz, h, w['origin'], ripple=(Rx, Rz), wmap=128, ww_cap=20000, rng_mode='hash', **kw)
    ora.drop_d = prm['drop_d']
    layer = orp.RippleLayer(Rx, Rz, nx * h, nz * h, sigma_rho=prm['sigma'] / prm['rho'], rho=prm['rho'])
    gpu.add_particles(w['pos'])
    ora.add_particles(f32(w['pos']))
    rng = np.random.default_rng(11)
    W_, D_ = nx * h, nz * h
    impacts = 0
    for f in (1, 2):
        n = 60                                 # a burst of rain per frame, so that drops land in both frames
        drops = np.stack([rng.uniform(-0.45 * W_, 0.45 * W_, n), rng.uniform(0.3, 0.45, n) * ny * h,
                          rng.uniform(-0.45 * D_, 0.45 * D_, n)], 1)
        dv = np.zeros((n, 3)); dv[:, 1] = -4.0
        gpu.add_particles(f32(drops), f32(dv), np.ones(n))
        ora.add_particles(f32(drops), f32(dv), np.ones(n))
        for _ in range(6):                    # the drops fall to the pool, then one frame is compared
            # each sub-step compared and the oracle continued from the GPU's particles: at 131k particles a few
            # lie within the float32/float64 difference of a cell face after an unsynchronised sub-step, and
            # the discrete cell counts (liquid cells, drift) then differ between the two
            n = ora.substeps_for(1 / 60)
            for _ in range(n):
                gpu.substep(1 / 60 / n)
                ora.frame += 1
                ora.substep(1 / 60 / n)
                # velocities within 1e-4: around landing drops the corner sums of faces with little total
                # weight lose digits in float32 (the reference GPU path's own arithmetic), against float64 in
                # the oracle; the vertical velocity of particles on the floor clamp is a tie (assert_particles)
                assert_particles(gpu, ora, f'burst {f}', vel_rtol=1e-4, floor_y=float(np.float32(0.32 * h)))
                sync_oracle_particles(gpu, ora)
            gpu.frame_end(1 / 60)
            ora.frame_end(1 / 60, layer, ripple_depth=prm['depth'])
        st = gpu.stats()
        assert st['impacts'] == ora.impacts
        assert ora.impacts > impacts, 'no drop merged in this burst'
        impacts = ora.impacts
        # crowns of the drops' own diameters (and spray of fast particles): the same whitewater
        P, V = gpu.whitewater()
        assert st['ww_count'] == len(ora.wpos) > 0
        j = _match_sets(P.astype(np.float64), np.concatenate([ora.wpos, ora.wlife[:, None]], 1), 1e-4)
        np.testing.assert_allclose(P[:, 3], ora.wlife[j], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(V[:, :3], ora.wvel[j], rtol=1e-3, atol=1e-4)
        top = gpu.ripple_field(pkg.native.FIELD_TOP, (128, 128), np.float32)
        assert_close_field(top, ora.top, what=f'burst {f}: top height')
        S = gpu.ripple_field(pkg.native.FIELD_RIPPLE_STATE, (2 * Rz, 2 * Rx, 2), np.float32)
        assert np.abs(layer.S).max() > 0
        assert_close_field(S[..., 0], layer.S.real, rtol=1e-4, what=f'burst {f}: ripple state (height)')
        assert_close_field(S[..., 1], layer.S.imag, rtol=1e-4, what=f'burst {f}: ripple state (velocity)')
        # the field is the inverse FFT of the state: errors at 1e-4 of the state's largest mode add up over the
        # 512×256 modes to a few 1e-4 of the field's largest value at single vertices
        fld = gpu.ripple_field(pkg.native.FIELD_RIPPLE, (Rz + 1, Rx + 1, 3), np.float32)
        for c in range(3):
            assert_close_field(fld[..., c], layer.field[..., c], rtol=1e-3, atol=1e-12, what=f'burst {f}: field {c}')
    gpu.close()


def test_full_size_obstacles_inflow_substeps(pkg):
    """Two sub-steps of the obstacles-and-inflow workload at its full size: 128×64×64 cells at h = 1/64 m,
    1.70M particles, the sphere, the turned box and the cylinder (analytic shapes), the floor drain, and the
    faucet's particles of each sub-step generated on the host and added to both; 100 SOR iterations at
    ω = 1.8. Cell counts and valid-face masks bit-exact; P2G velocity, pressure, projected velocity and
    particles within the parity tolerances; the post-projection divergence equal to the oracle's."""
    import bench
    from parity import gpu_max_divergence, objs_from_items
    w = pkg.workloads.obstacles_inflow()
    prm = w['params']
    nx, ny, nz, h = w['nx'], w['ny'], w['nz'], w['h']
    kw = dict(flip=prm['flip'], omega=prm['omega'], iters=prm['iters'], whitewater=True)
    gpu = gpu_from(pkg, nx, ny, nz, h, capacity=int(len(w['pos']) * 1.1), **kw)
    gpu.set_objects(w['objects'])
    ora = oracle_from(nx, ny, nz, h, w['origin'], **kw)
    ora.set_objects(objs_from_items(w['objects']))
    gpu.add_particles(w['pos'])
    ora.add_particles(f32(w['pos']))
    rng = np.random.default_rng(5)
    for s in (1, 2):
        p, v = bench.faucet_particles(w['emitters'][0], prm['dt'], rng)
        gpu.add_particles(p, v)
        ora.add_particles(f32(p), f32(v))
        gpu.substep(prm['dt'])
        ora.frame = s
        ora.substep(prm['dt'])
        compare_substep(pkg, gpu, ora, f'full-size sub-step {s}')
        dg, do = gpu_max_divergence(pkg, gpu), ora.max_divergence()
        assert abs(dg - do) <= 1e-3 * do, (dg, do)
        sync_oracle_particles(gpu, ora)
    gpu.close()


def test_full_batch_of_64_tanks_one_substep(pkg):
    """The batching workload at its full size: the 64 uneven tanks (11.7M particles, 80 SOR iterations,
    0-3 analytic obstacles each) advanced one sub-step as one batch in its size lanes; every 8th tank (sizes
    across both lanes) against the oracle run on that tank alone: counts and masks bit-exact, P2G velocity,
    pressure, projected velocity and particles within the parity tolerances."""
    from parity import objs_from_items
    specs = pkg.workloads.batch_tanks(64)
    tanks = []
    for w in specs:
        prm = w['params']
        t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=prm['flip'], omega=prm['omega'],
                     iters=prm['iters'], gravity=prm['g'], whitewater=True, ripple=None,
                     capacity=int(len(w['pos']) * 1.2) + 1000, ww_capacity=20000, sdf_mode='analytic')
        t.set_objects(w['objects'])
        t.add_particles(w['pos'])
        tanks.append(t)
    b = pkg.Batch(tanks)
    assert b.lanes() >= 2
    dt = 1 / 240
    b.substep(dt)
    b.sync()
    for i in range(0, 64, 8):
        w = specs[i]
        prm = w['params']
        ora = oracle_from(w['nx'], w['ny'], w['nz'], w['h'], w['origin'], flip=prm['flip'], omega=prm['omega'],
                          iters=prm['iters'], g=prm['g'], whitewater=True, ww_cap=20000)
        ora.set_objects(objs_from_items(w['objects']))
        ora.add_particles(f32(w['pos']))
        ora.frame = 1
        ora.substep(dt)
        compare_substep(pkg, tanks[i], ora, f'batch tank {i} ({w["nx"]}x{w["ny"]}x{w["nz"]})')
    b.close()
    for t in tanks:
        t.close()


@pytest.mark.parametrize('form', [1, 2])
@pytest.mark.parametrize('advect', ['euler', 'rk2'])
def test_g2p_brick_form_equals_the_walk(pkg, advect, form):
    """The per-brick grid-to-particle form (1: faces staged in shared memory, one block per 8×8×8 brick and
    one for the particles outside the grid) and the split form (2: the common path, with the particles that
    need obstacles, the free-flight test, merging or a whitewater spawn deferred to a second pass) give the
    particles of the grid-stride walk bit for bit: a tank with obstacles and an odd size, a pool with airborne
    drops falling into it, and particles above the rim (outside the grid), with Euler and RK2 advection;
    whitewater counts, impacts and the speed maximum agree."""
    w = pkg.workloads.random_tank(5, axes=(21, 37, 19))
    rng = np.random.default_rng(4)
    hi = np.array([w['nx'], w['ny'], w['nz']]) * w['h'] + w['origin']
    n_air = 300
    drops = w['origin'] + rng.random((n_air, 3)) * (hi - w['origin'])
    drops[:, 1] = rng.uniform(0.7, 1.3, n_air) * hi[1]              # some above the rim, outside the grid
    pos = np.concatenate([w['pos'], drops.astype(np.float32)])
    vel = np.zeros_like(pos); vel[len(w['pos']):, 1] = -3.0
    air = np.zeros(len(pos)); air[len(w['pos']):] = 1

    def run(form):
        t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.7, iters=20, whitewater=True,
                     ripple=(16, 16), capacity=len(pos) * 2, advect=advect)
        t.set_objects(w['objects'])
        t.add_particles(pos, vel, air)
        t.tune_g2p(form)
        for _ in range(5):
            t.substep(1 / 240)
        st = t.stats()
        p, v, a, ids = t.particles()
        o = np.argsort(ids)
        out = (p[o], v[o], a[o], ids[o], st['ww_count'], st['vmax'], st['impacts'])
        t.close()
        return out

    walk, brick = run(0), run(form)
    for x, y in zip(walk[:4], brick[:4]):
        np.testing.assert_array_equal(x, y)
    assert walk[4:] == brick[4:]


def test_moving_obstacles_solid_velocity_and_collisions(pkg):
    """A sphere moving at 0.4 m/s along x and a turned box spinning at 3 rad/s about the vertical axis (the
    solid velocity that setObjects gives moving obstacles, src/js/30-wgsl-sim.js:96-106, solver.py:153-165),
    analytic shapes, in a pool stirred at random: face fractions bit-exact; P2G velocity, the projected
    velocity (closed faces take the nearest obstacle's velocity, and the cut faces' fluxes carry it into the
    divergence), pressure and particles (collisions rebound relative to the moving surface) within the parity
    tolerances, over two sub-steps."""
    from oracle import sdf as sdfm
    nx, ny, nz, h = 32, 16, 24, 1 / 32
    objs = [sdfm.make_obstacle('sphere', [0.1, 0.2, 0.0], lin=(0.4, 0.0, 0.0), r=0.08),
            sdfm.make_obstacle('box', [-0.22, 0.12, 0.1], (0, 20, 0), ang=(0.0, 3.0, 0.0), w=0.12, h=0.1, d=0.08)]
    gpu = gpu_from(pkg, nx, ny, nz, h, flip=0.95, omega=1.7, iters=30)
    gpu.set_obstacles([dict(type=o['type'], flag=1, pos=o['pos'], rot=o['rot'], dims=o['dims'], lin=o['lin'],
                            ang=o['ang']) for o in objs])
    ora = oracle_from(nx, ny, nz, h, gpu.origin, flip=0.95, omega=1.7, iters=30)
    ora.set_objects(objs)
    cells = pkg.workloads.block_cells(nx, ny, nz, lambda i, j, k: j < 10)
    pos = pkg.workloads.fill_cells(cells, h, gpu.origin, 8, 3)
    pos = pos[ora.sdf_at(pos.astype(np.float64)) > 0.3 * h]          # particles outside the obstacles
    vel = (np.random.default_rng(8).random(pos.shape) - 0.5).astype(np.float32)
    gpu.add_particles(pos, vel)
    ora.add_particles(f32(pos), f32(vel))
    for s in (1, 2):
        gpu.substep(1 / 240)
        ora.frame = s
        ora.substep(1 / 240)
        g = compare_substep(pkg, gpu, ora, f'moving obstacles, sub-step {s}')
        np.testing.assert_array_equal(g['frac'], ora.frac.astype(np.float32))
        closed = ora.frac <= 0
        assert np.abs(ora.svel[closed]).max() > 0.1                  # the solids' velocity reaches the faces
        sync_oracle_particles(gpu, ora)
    gpu.close()
