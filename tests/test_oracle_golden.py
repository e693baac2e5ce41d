"""Pins the CPU oracle against fixtures produced by the reference's own solver (tests/golden/make_golden.py).

Binning, counts, masks and the float32 SOR pressures must agree bit for bit; float64 phases that sum in
the same order also agree exactly; everything else within 1e-12 relative.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import flip as of
from oracle import meshing as om
from oracle import ripple as orp
from oracle import sdf as sdfm


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + '.npz'), allow_pickle=False))


def tank_from(d, **kw):
    t = of.Tank(int(d['nx']), int(d['ny']), int(d['nz']), float(d['h']), origin=d['origin'], flip=float(d['flip']),
                omega=float(d['omega']), iters=int(d['iters']), g=float(d['g']), **kw)
    return t


def close(a, b, rtol=1e-12, atol=1e-13):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    err = np.abs(a - b)
    lim = atol + rtol * np.abs(b)
    assert np.all(err <= lim), f'max err {err.max()} at {np.unravel_index(np.argmax(err - lim), err.shape)}'


def test_dam16_two_substeps_bit_exact():
    d = load('dam16')
    t = tank_from(d, whitewater=False)
    t.add_particles(d['pos0'], d['vel0'])
    for s in (1, 2):
        t.substep(float(d['dt']))
        np.testing.assert_array_equal(t.count, d[f's{s}_count'])
        np.testing.assert_array_equal(t.mask, d[f's{s}_mask'])
        np.testing.assert_array_equal(t.velold, d[f's{s}_velold'])
        np.testing.assert_array_equal(t.pres, d[f's{s}_pres'])        # float32 SOR, same operation order
        np.testing.assert_array_equal(t.velg, d[f's{s}_velg'])
        np.testing.assert_array_equal(t.pos, d[f's{s}_pos'])
        np.testing.assert_array_equal(t.vel, d[f's{s}_vel'])
        np.testing.assert_array_equal(t.air, d[f's{s}_air'])


def test_obstacles_lattice_mode():
    d = load('obstacles')
    t = tank_from(d, whitewater=False)
    objs = [sdfm.make_obstacle('sphere', [0.15, 0.18, 0.0], r=0.09),
            sdfm.make_obstacle('box', [-0.25, 0.1, 0.12], rot_deg=(0, 30, 0), w=0.16, h=0.1, d=0.12),
            sdfm.make_obstacle('cone', [-0.05, 0.1, -0.2], rot_deg=(10, 0, 20), r=0.08, h=0.14),
            sdfm.make_drain([0.38, 0.0, -0.28], 0.06)]
    t.set_objects(objs)
    np.testing.assert_array_equal(t.lat, d['lattice'])
    np.testing.assert_array_equal(t.frac, d['frac'])
    t.add_particles(d['pos0'], d['vel0'])
    t.substep(float(d['dt']))
    for k in ('count', 'mask', 'velold', 'pres', 'velg'):
        np.testing.assert_array_equal(getattr(t, k), d['s1_' + k], err_msg=k)
    np.testing.assert_array_equal(t.pos, d['s1_pos'])
    np.testing.assert_array_equal(t.vel, d['s1_vel'])
    t.substep(float(d['dt']))
    np.testing.assert_array_equal(t.pres, d['s2_pres'])
    np.testing.assert_array_equal(t.pos, d['s2_pos'])
    np.testing.assert_array_equal(t.vel, d['s2_vel'])
    np.testing.assert_array_equal(t.air, d['s2_air'])


def test_drops_merge_crown_whitewater_pcg64():
    d = load('drops')
    t = tank_from(d, whitewater=True, seed=int(d['seed']), ripple=(int(d['ripple']),) * 2, ww_cap=4000)
    t.add_particles(d['pos0'], d['vel0'], d['air0'])
    t.frame = 1                                   # the reference counts sub-steps inside step() only
    t.substep(float(d['dt']))
    np.testing.assert_array_equal(t.pos, d['s1_pos'])
    np.testing.assert_array_equal(t.vel, d['s1_vel'])
    np.testing.assert_array_equal(t.air, d['s1_air'])
    assert t.impacts == int(d['s1_impacts']) and t.impacts > 0
    close(t.rsrc, d['s1_rsrc'])
    assert len(t.wpos) == len(d['s1_wpos']) and len(t.wpos) > 0
    np.testing.assert_array_equal(t.wpos, d['s1_wpos'])
    np.testing.assert_array_equal(t.wvel, d['s1_wvel'])
    np.testing.assert_array_equal(t.wlife, d['s1_wlife'])


def test_frame_step_whitewater_top_height_ripple():
    d = load('frame')
    R = int(d['ripple'])
    t = tank_from(d, whitewater=True, seed=int(d['seed']), ripple=(R, R), wmap=int(d['wmap']), ww_cap=4000)
    objs = [sdfm.make_obstacle('cylinder', [0.1, 0.15, -0.1], r=0.08, h=0.3),
            sdfm.make_obstacle('torus', [-0.2, 0.15, 0.15], R=0.1, r=0.03)]
    t.set_objects(objs)
    np.testing.assert_array_equal(t.lat, d['lattice'])
    t.add_particles(d['pos0'], d['vel0'], d['air0'])
    t.wpos, t.wvel, t.wlife, t.wkind = d['wpos0'].copy(), d['wvel0'].copy(), d['wlife0'].copy(), d['wkind0'].copy()
    layer = orp.RippleLayer(R, R, t.nx * t.h, t.nz * t.h)
    for f in (1, 2):
        t.step(float(d['frame_dt']), layer)
        assert t.frame == int(d[f'f{f}_frame'])
        np.testing.assert_array_equal(t.pos, d[f'f{f}_pos'])
        np.testing.assert_array_equal(t.vel, d[f'f{f}_vel'])
        np.testing.assert_array_equal(t.wpos, d[f'f{f}_wpos'])
        np.testing.assert_array_equal(t.wlife, d[f'f{f}_wlife'])
        np.testing.assert_array_equal(t.top, d[f'f{f}_top'])
        close(layer.field, d[f'f{f}_field'], 1e-9, 1e-15)
        close(layer.S, d[f'f{f}_S'], 1e-9, 1e-15)
        close(orp.caustics(t.top, layer.field, t.nx * t.h, t.nz * t.h, d['sun']), d[f'f{f}_caustics'], 1e-12, 1e-13)
        np.testing.assert_array_equal(t.count, d[f'f{f}_count'])
        v, q, tr = om.surface(t)
        om.settle_on_top(t, v)
        np.testing.assert_array_equal(v, d[f'f{f}_mesh_v'])
        np.testing.assert_array_equal(q, d[f'f{f}_mesh_q'])
        np.testing.assert_array_equal(tr, d[f'f{f}_mesh_t'])
        np.testing.assert_array_equal(om.vertex_velocity(t, v), d[f'f{f}_mesh_vel'])


def test_caustics_of_the_reference_frames():
    """Floor light from the reference's own height map and ripple field after each fixture frame."""
    d = load('frame')
    h = float(d['h'])
    for f in (1, 2):
        light = orp.caustics(d[f'f{f}_top'], d[f'f{f}_field'], int(d['nx']) * h, int(d['nz']) * h, d['sun'])
        close(light, d[f'f{f}_caustics'], 1e-12, 1e-13)
        assert light.max() > 1.5 and light.min() < 0.5          # the surface focuses and shadows light


@pytest.mark.parametrize('sun', [(0.0, 1.0, 0.0), (0.35, 0.85, 0.25), (-0.6, 0.5, 0.1)])
def test_caustics_under_flat_water(sun):
    """Flat water of any depth maps every texel onto itself: away from the edges (whose outer samples land
    off the map) the light is the transmitted fraction 1 - Fresnel(cos θ_sun); dry floor takes it all."""
    W, L = 24, 0.48
    field = np.zeros((17, 17, 3))
    s = np.asarray(sun) / np.linalg.norm(sun)
    for depth in (0.0, 0.05, 0.2):
        light = orp.caustics(np.full((W, W), depth), field, L, L, sun)
        np.testing.assert_allclose(light[2:-2, 2:-2], 1 - orp.fresnel_w(s[1]), rtol=1e-12)
    dry = orp.caustics(np.full((W, W), -1.0), field, L, L, sun)
    np.testing.assert_allclose(dry[2:-2, 2:-2], 1.0, rtol=1e-12)


def test_ripple_layer_alone():
    d = load('ripple')
    R = int(d['R'])
    layer = orp.RippleLayer(R, R, float(d['Lx']), float(d['Lz']))
    layer.frame(float(d['dt']), float(d['depth']), d['src'], d['mask'])
    np.testing.assert_array_equal(layer.S, d['f1_S'])
    np.testing.assert_array_equal(layer.field, d['f1_field'])
    layer.frame(float(d['dt']), float(d['depth']), np.zeros_like(d['src']), d['mask'])
    np.testing.assert_array_equal(layer.S, d['f2_S'])


def test_dam32_workload_one_substep(pkg):
    d = load('dam32')
    w = pkg.workloads.dam_break()
    t = of.Tank(32, 32, 32, w['h'], origin=w['origin'], flip=0.95, omega=1.7, iters=60, whitewater=False)
    t.add_particles(w['pos'].astype(np.float64))
    assert len(t.pos) == int(d['n']) == 53248
    t.substep(1 / 240)
    np.testing.assert_array_equal(t.count, d['count'])
    np.testing.assert_array_equal(t.mask, d['mask'])
    np.testing.assert_array_equal(t.velold.astype(np.float32), d['velold'])
    np.testing.assert_array_equal(t.pres.astype(np.float32), d['pres'])
    np.testing.assert_array_equal(t.pos.sum(0), d['pos_sum'])
    np.testing.assert_array_equal(t.vel.sum(0), d['vel_sum'])


def test_sor_residual_checker_decreases():
    """The FP64 residual of the SOR operands falls as iterations are added (used to state the error)."""
    d = load('dam16')
    t = tank_from(d, whitewater=False)
    t.add_particles(d['pos0'], d['vel0'])
    g, ing = t.count_cells()
    t.p2g(g, ing)
    fluid = t.forces_and_divergence(float(d['dt']))
    C, inv, U, rhs = t.sor_operands(t.div, fluid)
    r = []
    for it in (5, 20, 80):
        t.pres[:] = 0
        p = t.sor(fluid, p_init=np.zeros_like(t.pres), iters=it)
        r.append(of.residual_f64(C, rhs, fluid, p))
    assert r[0] > r[1] > r[2]


def test_drop_diameters_are_lognormal_and_fixed_by_the_id():
    """The build's sub-grid drop sizes (the reference gives every drop the particle mass): median 2 mm and
    log-standard-deviation 0.4 over many ids, a pure function of the id, |z| clamped to 4."""
    from oracle import hashrng
    ids = np.arange(400000)
    D = hashrng.drop_diameter(ids, 0.002, 0.4)
    z = np.log(D / 0.002) / 0.4
    assert abs(np.median(D) / 0.002 - 1) < 0.01
    assert abs(z.std() - 1) < 0.01 and abs(z.mean()) < 0.01
    assert np.abs(z).max() <= 4 + 1e-12
    np.testing.assert_array_equal(hashrng.drop_diameter(ids[::-1], 0.002, 0.4), D[::-1])
    # the particle-mass rule is the default
    t = of.Tank(8, 8, 8, 1 / 16, rng_mode='hash')
    assert t.drop_d is None
