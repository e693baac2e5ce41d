"""CUDA path against the oracle (and the reference's own fixtures) on identical seeded inputs.

Every test goes through the C ABI (libsuiri_cuda.so via ctypes). Tolerances are in tests/parity.py."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import flip as of
from oracle import ripple as orp
from parity import (assert_close_field, assert_particles, f32, gpu_from, obstacle_items, oracle_from,
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


@pytest.mark.parametrize('sor_mode', [0, 2, 3])
def test_sor_bit_exact_with_reference_operation_order(pkg, sor_mode):
    """Given the GPU's own float32 operands, the reference's float32 SOR loop reproduces its pressure bit for
    bit, for one launch per sweep and for temporal blocking; the FP64 residual of the solve is stated."""
    d = load('dam16')
    nx, ny, nz, h = int(d['nx']), int(d['ny']), int(d['nz']), float(d['h'])
    gpu = gpu_from(pkg, nx, ny, nz, h, flip=0.95, omega=1.7, iters=30)
    gpu.tune(4, sor_mode)
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
    lower 7/8 liquid: ≈458k cells a colour against 148 SMs × 2048): the sweep grid is capped at what is
    resident and each thread also relaxes the cells one grid further on. Pressures equal the reference's
    float32 loop bit for bit."""
    nx, ny, nz, h = 256, 64, 64, 1.0 / 64
    cells = pkg.workloads.block_cells(nx, ny, nz, lambda i, j, k: j < 56)
    pos = pkg.workloads.fill_cells(cells, h, pkg.workloads.grid_origin(nx, nz, h), 1, 7)
    gpu = gpu_from(pkg, nx, ny, nz, h, flip=0.95, omega=1.7, iters=8, capacity=len(pos) + 1024)
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


@pytest.mark.parametrize('axes,seeds', [((16, 24, 32), (1, 2, 3)), ((16, 48), (1, 2, 16))])
def test_batch_equals_solo_bit_for_bit(pkg, axes, seeds):
    """Tanks of uneven sizes stepped in one batch give exactly the particles they give alone; with the 48³
    tank (seed 16) the batch spans two size lanes (its own stream and graph each, forked and joined every
    sub-step)."""
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
    b = pkg.Batch(batched)
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


def _run_form(pkg, w, mode, iters, steps=3):
    t = pkg.Tank(nx=w['nx'], ny=w['ny'], nz=w['nz'], h=w['h'], flip=0.95, omega=1.8, iters=iters, whitewater=True,
                 ripple=None, capacity=len(w['pos']) * 2)
    t.set_objects(w['objects'])
    t.add_particles(w['pos'])
    t.tune(4, mode)
    for _ in range(steps):
        t.substep(1 / 240)
    assert t.stats()['errors'] == 0
    pos, vel, air, ids = t.particles()
    o = np.argsort(ids)
    out = (t.grid(pkg.native.FIELD_PRES), pos[o], vel[o])
    t.close()
    return out


@pytest.mark.parametrize('mode', [1, 2, 3])
def test_solve_forms_equal_per_sweep_launches(pkg, mode):
    """The cooperative whole-solve launch (1) and the temporal-blocked launches (2: two sweeps each, 3:
    four) relax the same colours in the same order as one launch per sweep (0): identical pressures and
    particles, bit for bit."""
    w = pkg.workloads.obstacles_inflow(scale=4)
    for a, b in zip(_run_form(pkg, w, 0, 40), _run_form(pkg, w, mode, 40)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('mode', [2, 3])
@pytest.mark.parametrize('iters', [6, 7, 1, 3])
def test_temporal_blocking_edges(pkg, iters, mode):
    """Temporal blocking on a grid that is no multiple of the tile (odd x). Four sweeps a launch: an odd
    number of launches (6 iterations: 3 launches, the result copied back), a short last launch (7:
    4+4+4+2 sweeps), a single launch of two sweeps (1). Two sweeps a launch: odd counts (1, 3, 7)."""
    w = pkg.workloads.random_tank(5, axes=(21, 37, 19))
    for a, b in zip(_run_form(pkg, w, 0, iters), _run_form(pkg, w, mode, iters)):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize('mode', [2, 3])
def test_temporal_blocking_batch_uneven_iterations(pkg, mode):
    """In a batch the tile launches run to the largest iteration count; tanks with fewer iterations stop
    relaxing but keep being carried between the two pressure buffers: every tank equals its solo run."""
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
